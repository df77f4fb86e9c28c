// Split-BF16x3 form of the coherent sum on a 128 x 128 coarse grid, on the 5th-generation tensor cores
// (tcgen05.mma, accumulators in tensor memory).  Same result as coherent_fft.cu -- the |fft2(.)|^2
// accumulation of CalculateAbbeImage (CalculateAerialImage.py:76-92) and CalculateAerialImage_SOCS
// (CalculateAerialImage_SOCS.py:5-10) -- with the band-to-coarse transform written as two dense DFT
// contractions:
//   E^T[sc][sr] = sum_ir sum_ic Cr[sr][ir] A[ir][ic] Cc[sc][ic],   A = P[z][k] .* band[b][c]  (<= 64 x 64),
//   Cc[sc][ic] = exp(-2 pi i (m0c+ic) sc / 128),  Cr[sr][ir] = exp(-2 pi i (m0r+ir) sr / 128).
// Stage 1 (M = sc, N = ir, K = ic):  H^T = Cc A^T     -- A operand Cc (shared memory, constant),
//                                                        B operand A (shared memory, built per field);
// Stage 2 (M = sc, N = sr, K = ir):  E^T = H^T Cr^T   -- A operand H^T (tensor memory, converted from the
//                                                        stage-1 accumulator), B operand Cr (constant).
// Complex products are four real ones; the minus sign of the imaginary-times-imaginary term is the
// instruction's negate-B bit.  Every real operand x is split x = hi + lo with hi = bf16(x), lo = bf16(x - hi)
// and a product is hi*hi + hi*lo + lo*hi with FP32 accumulation (the lo*lo term, ~2^-16 relative, is
// dropped): about 16 mantissa bits, against 24 for the FP32 forms.
//
// Work: the images' fields form one list of tasks t = (b*nz + z)*F + f, F = nk*nch, cut into equal
// contiguous ranges, one per CTA (one CTA per SM: the CTA holds all 512 tensor-memory columns).  A CTA
// accumulates w |E|^2 of its fields in registers and writes one partial coarse image per image it touches,
// to slot (CTA - first CTA of that image); the first CTA of an image zero-fills the slots no CTA owns, so
// the partial sums fold in a fixed order (deterministic).
//
// Pipeline per task i: [tensor] stage 2 of i, then stage 1 of i+1 | [CUDA cores] build the B operand of
// i+1 while stage 2 of i runs, then read and accumulate |E|^2 of i while stage 1 of i+1 runs, then convert
// the stage-1 accumulator of i+1 into the stage-2 A operand.
//
// Waits on the MMA-completion barriers are bounded (2 s of %globaltimer); on expiry the CTA records a
// status (oi_device_status), waits a bounded time for its outstanding MMAs, frees tensor memory and exits.
#include <cuda_bf16.h>
#include <cstdint>
#include "oi_common.cuh"

namespace oi {

__device__ int g_device_status = 0;

namespace tc {

constexpr int T = 256;              // threads per CTA (8 warps: two per tensor-memory lane quarter)
constexpr int MC = 128, MR = 128;   // coarse grid
constexpr int BMAX = 64;            // band rows / columns (padded)
// shared memory (offsets from a 1024-byte aligned base); every operand is K-major, 128-byte swizzled:
// element (row, k) of a [rows][64] bf16 matrix at row*128 + (((k/8) ^ (row%8)) * 16) + (k%8)*2
constexpr uint32_t MAT128 = 128 * 128;                  // bytes of one 128-row operand
constexpr uint32_t MAT64 = 64 * 128;                    // bytes of one 64-row operand
constexpr uint32_t OFF_CC = 0;                          // Cc: re hi, re lo, im hi, im lo
constexpr uint32_t OFF_CR = OFF_CC + 4 * MAT128;        // Cr: re hi, re lo, im hi, im lo
constexpr uint32_t OFF_B1 = OFF_CR + 4 * MAT128;        // two buffers of A: re hi, re lo, im hi, im lo
constexpr uint32_t B1_BYTES = 4 * MAT64;
constexpr uint32_t OFF_MISC = OFF_B1 + 2 * B1_BYTES;    // barriers, tensor-memory base
constexpr uint32_t SMEM_BYTES = OFF_MISC + 64 + 1024;   // + alignment slack
// tensor memory columns (128 lanes x 512 columns of 32 bits)
constexpr uint32_t COL_D2 = 0;      // E^T: re [0,128), im [128,256)
constexpr uint32_t COL_D1 = 256;    // H^T: re [256,320), im [320,384)
constexpr uint32_t COL_A2H = 384;   // H^T as bf16 pairs, hi: [Hr | Hi] along K (64 columns)
constexpr uint32_t COL_A2L = 448;   // lo
constexpr uint32_t NCOLS = 512;
constexpr unsigned long long WAIT_NS = 2000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// K-major, 128-byte swizzle, 8-row groups 1024 bytes apart, descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t sdesc(uint32_t addr) {
  const uint32_t lo = ((addr >> 4) & 0x3FFFu) | (1u << 16);
  const uint32_t hi = (1024u >> 4) | (1u << 14) | (2u << 29);
  return ((uint64_t)hi << 32) | lo;
}
// kind::f16, bf16 x bf16 -> f32, both K-major, M = 128.
__host__ __device__ constexpr uint32_t idesc(int n, bool neg_b) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (neg_b ? (1u << 14) : 0u) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(128 >> 4) << 24);
}
__device__ __forceinline__ void mma_ss(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(id), "r"(acc));
}
__device__ __forceinline__ void mma_ts(uint32_t d, uint32_t a_tmem, uint64_t b, uint32_t id, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(d),
      "r"(a_tmem), "l"(b), "r"(id), "r"(acc));
}
__device__ __forceinline__ void commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}
__device__ __forceinline__ bool try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the barrier phase of the given parity; false on expiry.
__device__ __forceinline__ bool wait_bar(uint32_t bar, uint32_t parity) {
  if (try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer();
  while (!try_wait(bar, parity))
    if (globaltimer() - t0 > WAIT_NS) return false;
  return true;
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Two 32-lane x 16-column loads and their completion wait in one asm statement: the destination registers are
// written asynchronously, so no use of them may be scheduled before tcgen05.wait::ld.
__device__ __forceinline__ void tmem_ld16x2(uint32_t addr_a, uint32_t addr_b, float (&va)[16], float (&vb)[16]) {
  uint32_t a[16], b[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%32];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%33];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3]), "=r"(a[4]), "=r"(a[5]), "=r"(a[6]), "=r"(a[7]),
        "=r"(a[8]), "=r"(a[9]), "=r"(a[10]), "=r"(a[11]), "=r"(a[12]), "=r"(a[13]), "=r"(a[14]), "=r"(a[15]),
        "=r"(b[0]), "=r"(b[1]), "=r"(b[2]), "=r"(b[3]), "=r"(b[4]), "=r"(b[5]), "=r"(b[6]), "=r"(b[7]),
        "=r"(b[8]), "=r"(b[9]), "=r"(b[10]), "=r"(b[11]), "=r"(b[12]), "=r"(b[13]), "=r"(b[14]), "=r"(b[15])
      : "r"(addr_a), "r"(addr_b)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    va[i] = __uint_as_float(a[i]);
    vb[i] = __uint_as_float(b[i]);
  }
}
__device__ __forceinline__ void tmem_st16(uint32_t addr, const uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::
          "r"(addr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
      "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
      : "memory");
}
__device__ __forceinline__ void wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ uint32_t bf16x2_bits(__nv_bfloat162 h) {
  return (uint32_t)__bfloat16_as_ushort(h.x) | ((uint32_t)__bfloat16_as_ushort(h.y) << 16);
}
// (a, b) -> packed bf16 pairs hi = bf16(a, b), lo = bf16((a, b) - hi)
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  const float2 hf = __bfloat1622float2(h);
  hi = bf16x2_bits(h);
  lo = bf16x2_bits(__floats2bfloat162_rn(a - hf.x, b - hf.y));
}
__device__ __forceinline__ uint32_t swz(int row, int chunk) {
  return (uint32_t)(row * 128 + ((chunk ^ (row & 7)) << 4));
}
__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d)
               : "memory");
}

// The DFT matrix exp(-2 pi i (m0+i) s / 128), rows s < 128, columns i < 64, split into hi/lo re/im operands.
__device__ void build_dft(uint32_t base, const float2* __restrict__ w, int m0, int tid) {
  for (int chunk = tid; chunk < 128 * 8; chunk += T) {
    const int s = chunk >> 3, g = chunk & 7;
    uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int i0 = 8 * g + 2 * e;
      const float2 t0 = __ldg(w + (((m0 + i0) * s) & (MC - 1)));
      const float2 t1 = __ldg(w + (((m0 + i0 + 1) * s) & (MC - 1)));
      split2(t0.x, t1.x, rh[e], rl[e]);
      split2(-t0.y, -t1.y, ih[e], il[e]);  // conj: w holds exp(+2 pi i j / 128)
    }
    const uint32_t o = base + swz(s, g);
    st_shared_v4(o, rh[0], rh[1], rh[2], rh[3]);
    st_shared_v4(o + MAT128, rl[0], rl[1], rl[2], rl[3]);
    st_shared_v4(o + 2 * MAT128, ih[0], ih[1], ih[2], ih[3]);
    st_shared_v4(o + 3 * MAT128, il[0], il[1], il[2], il[3]);
  }
}

struct Args {
  const float2* band;         // [batch][nch][br][bc]
  long long band_img_stride;  // nch * br * bc
  int nch, br, bc, m0r, m0c;
  const float2* pupil;        // [batch?][nz][nk][br][bc]
  long long pupil_batch_stride;
  const float* weight;        // [nz][nk]
  int nz, nk;
  long long images;           // batch * nz
  long long tasks;            // images * nk * nch
  int nparts;
  const float2* wr;           // exp(+2 pi i j / 128)
  const float2* wc;
  float* coarse;              // [nparts][images][128][128]
};

// CTA owning task t when `tasks` are cut into gridDim.x ranges [floor(i T / G), floor((i+1) T / G)).
__host__ __device__ __forceinline__ long long cta_of(long long t, long long tasks, long long g) {
  return ((t + 1) * g - 1) / tasks;
}

// A = P .* band for task t, zero-padded to 64 x 64, as hi/lo re/im operands (64 rows ir, K = ic).
__device__ __forceinline__ void build_field(const Args& a, long long t, uint32_t base, int tid) {
  const int F = a.nk * a.nch;
  const long long q = t / F;
  const int f = (int)(t - q * F), k = f / a.nch, c = f - k * a.nch;
  const long long b = q / a.nz;
  const int z = (int)(q - b * a.nz);
  const int plane = a.br * a.bc;
  const float2* pk = a.pupil + b * a.pupil_batch_stride + ((long long)z * a.nk + k) * plane;
  const float2* hc = a.band + b * a.band_img_stride + (long long)c * plane;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const int chunk = tid + T * j, ir = chunk >> 3, g = chunk & 7;
    uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      float2 v[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int ic = 8 * g + 2 * e + h;
        v[h] = make_float2(0.f, 0.f);
        if (ir < a.br && ic < a.bc) {
          const int o = ir * a.bc + ic;
          v[h] = cmul(__ldg(pk + o), __ldg(hc + o));
        }
      }
      split2(v[0].x, v[1].x, rh[e], rl[e]);
      split2(v[0].y, v[1].y, ih[e], il[e]);
    }
    const uint32_t o = base + swz(ir, g);
    st_shared_v4(o, rh[0], rh[1], rh[2], rh[3]);
    st_shared_v4(o + MAT64, rl[0], rl[1], rl[2], rl[3]);
    st_shared_v4(o + 2 * MAT64, ih[0], ih[1], ih[2], ih[3]);
    st_shared_v4(o + 3 * MAT64, il[0], il[1], il[2], il[3]);
  }
}

// Stage 1: D1 = Cc A^T  (re: Ccr Ar - Cci Ai, im: Ccr Ai + Cci Ar), 48 MMAs of 128 x 64 x 16.
__device__ __forceinline__ void issue_stage1(uint32_t tmem, uint32_t cc, uint32_t b1) {
  constexpr uint32_t ID = idesc(64, false), IDN = idesc(64, true);
#pragma unroll
  for (int out = 0; out < 2; ++out) {
    const uint32_t d = tmem + COL_D1 + 64 * out;
    uint32_t acc = 0;
#pragma unroll
    for (int term = 0; term < 2; ++term) {
      const uint32_t x = cc + (term ? 2 * MAT128 : 0);                         // Ccr / Cci
      const uint32_t y = b1 + ((out ^ term) ? 2 * MAT64 : 0);                  // Ar / Ai
      const uint32_t id = (out == 0 && term == 1) ? IDN : ID;
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        const uint32_t ko = 32 * ks;
        mma_ss(d, sdesc(x + ko), sdesc(y + ko), id, acc);                      // hi hi
        acc = 1;
        mma_ss(d, sdesc(x + ko), sdesc(y + MAT64 + ko), id, 1);                // hi lo
        mma_ss(d, sdesc(x + MAT128 + ko), sdesc(y + ko), id, 1);               // lo hi
      }
    }
  }
}

// Stage 2: D2 = A2 Cr^T with A2 = [Hr | Hi] along K (re: Hr Crr - Hi Cri, im: Hr Cri + Hi Crr),
// 48 MMAs of 128 x 128 x 16.
__device__ __forceinline__ void issue_stage2(uint32_t tmem, uint32_t cr) {
  constexpr uint32_t ID = idesc(128, false), IDN = idesc(128, true);
#pragma unroll
  for (int out = 0; out < 2; ++out) {
    const uint32_t d = tmem + COL_D2 + 128 * out;
#pragma unroll
    for (int ks = 0; ks < 8; ++ks) {
      const int part = ks >> 2;
      const uint32_t bm = cr + ((out ^ part) ? 2 * MAT128 : 0) + 32 * (ks & 3);  // Crr / Cri
      const uint32_t id = (out == 0 && part == 1) ? IDN : ID;
      const uint32_t ah = tmem + COL_A2H + 8 * ks, al = tmem + COL_A2L + 8 * ks;
      mma_ts(d, ah, sdesc(bm), id, ks == 0 ? 0u : 1u);                         // hi hi
      mma_ts(d, ah, sdesc(bm + MAT128), id, 1);                                  // hi lo
      mma_ts(d, al, sdesc(bm), id, 1);                                           // lo hi
    }
  }
}

__global__ void __launch_bounds__(T, 1) coherent_tc_kernel(Args a) {
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char* gbase = smem_raw + (base - raw);
  const uint32_t bar1 = base + OFF_MISC, bar2 = base + OFF_MISC + 8;
  volatile uint32_t* tmem_slot = (volatile uint32_t*)(gbase + OFF_MISC + 16);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long G = gridDim.x;
  const long long t0 = (long long)blockIdx.x * a.tasks / G, t1 = ((long long)blockIdx.x + 1) * a.tasks / G;
  const int F = a.nk * a.nch;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(base + OFF_MISC + 16),
                 "r"(NCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar1) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar2) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  build_dft(base + OFF_CC, a.wc, a.m0c, tid);
  build_dft(base + OFF_CR, a.wr, a.m0r, tid);
  if (t0 < t1) build_field(a, t0, base + OFF_B1, tid);
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;  // this warp's tensor-memory lane quarter
  const int half = warp >> 2;                                    // column half this warp reads
  const int sc = 32 * (warp & 3) + lane;                         // coarse column = accumulator row
  uint32_t ph1 = 0, ph2 = 0;
  int pending1 = 0, pending2 = 0;
  bool failed = false;

  if (t0 < t1 && tid == 0) {
    issue_stage1(tmem, base + OFF_CC, base + OFF_B1);
    commit(bar1);
  }
  pending1 = (t0 < t1);

  float acc[64];
#pragma unroll
  for (int j = 0; j < 64; ++j) acc[j] = 0.f;
  float wprev = 0.f;

  for (long long t = t0; t < t1; ++t) {
    const long long i = t - t0;
    // (1) |E|^2 of task t-1 (overlaps stage 1 of t on the tensor pipe)
    if (i > 0) {
      const bool ok = wait_bar(bar2, ph2);
      if (__syncthreads_or(!ok)) { failed = true; break; }
      ph2 ^= 1;
      pending2 = 0;
      fence_after();
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        float re[16], im[16];
        tmem_ld16x2(tmem + lane_base + COL_D2 + 64 * half + 16 * p, tmem + lane_base + COL_D2 + 128 + 64 * half + 16 * p,
                    re, im);
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[16 * p + j] = fmaf(wprev, fmaf(re[j], re[j], im[j] * im[j]), acc[16 * p + j]);
      }
      // flush when task t-1 was the last of its image in this range
      const long long qp = (t - 1) / F;
      if (t / F != qp) {
        const long long slot = blockIdx.x - cta_of(qp * F, a.tasks, G);
        float* out = a.coarse + (slot * a.images + qp) * (long long)(MR * MC) + sc;
#pragma unroll
        for (int j = 0; j < 64; ++j) {
          out[(64 * half + j) * MC] = acc[j];
          acc[j] = 0.f;
        }
      }
    }
    // (2) stage-1 accumulator of t -> stage-2 A operand (bf16 hi/lo pairs)
    {
      const bool ok = wait_bar(bar1, ph1);
      if (__syncthreads_or(!ok)) { failed = true; break; }
      ph1 ^= 1;
      pending1 = 0;
      fence_after();
#pragma unroll
      for (int p = 0; p < 2; ++p) {
        float h[16], h2[16];
        tmem_ld16x2(tmem + lane_base + COL_D1 + 64 * half + 32 * p, tmem + lane_base + COL_D1 + 64 * half + 32 * p + 16,
                    h, h2);
        uint32_t hi[16], lo[16];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          split2(h[2 * j], h[2 * j + 1], hi[j], lo[j]);
          split2(h2[2 * j], h2[2 * j + 1], hi[8 + j], lo[8 + j]);
        }
        tmem_st16(tmem + lane_base + COL_A2H + 32 * half + 16 * p, hi);
        tmem_st16(tmem + lane_base + COL_A2L + 32 * half + 16 * p, lo);
      }
      wait_st();
    }
    {
      const int f = (int)(t % F), k = f / a.nch;
      wprev = __ldg(a.weight + (long long)((t / F) % a.nz) * a.nk + k);
    }
    // zero-fill the partial slots of this image that no CTA owns (done by the image's first CTA)
    if (t % F == 0) {
      const long long q = t / F;
      const long long first = cta_of(q * F, a.tasks, G), last = cta_of(q * F + F - 1, a.tasks, G);
      for (long long slot = last - first + 1; slot < a.nparts; ++slot) {
        float* out = a.coarse + (slot * a.images + q) * (long long)(MR * MC);
        for (int e = tid; e < MR * MC / 4; e += T) ((float4*)out)[e] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
    fence_before();
    __syncthreads();
    if (tid == 0) {
      fence_after();
      issue_stage2(tmem, base + OFF_CR);
      commit(bar2);
    }
    pending2 = 1;
    // (3) B operand of t+1 (overlaps stage 2 of t), then stage 1 of t+1
    if (t + 1 < t1) {
      build_field(a, t + 1, base + OFF_B1 + (uint32_t)((i + 1) & 1) * B1_BYTES, tid);
      fence_async_smem();
      __syncthreads();
      if (tid == 0) {
        fence_after();
        issue_stage1(tmem, base + OFF_CC, base + OFF_B1 + (uint32_t)((i + 1) & 1) * B1_BYTES);
        commit(bar1);
      }
      pending1 = 1;
    }
  }
  if (!failed && t0 < t1) {
    const bool ok = wait_bar(bar2, ph2);
    if (__syncthreads_or(!ok)) {
      failed = true;
    } else {
      ph2 ^= 1;
      pending2 = 0;
      fence_after();
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        float re[16], im[16];
        tmem_ld16x2(tmem + lane_base + COL_D2 + 64 * half + 16 * p, tmem + lane_base + COL_D2 + 128 + 64 * half + 16 * p,
                    re, im);
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[16 * p + j] = fmaf(wprev, fmaf(re[j], re[j], im[j] * im[j]), acc[16 * p + j]);
      }
      const long long qp = (t1 - 1) / F;
      const long long slot = blockIdx.x - cta_of(qp * F, a.tasks, G);
      float* out = a.coarse + (slot * a.images + qp) * (long long)(MR * MC) + sc;
#pragma unroll
      for (int j = 0; j < 64; ++j) out[(64 * half + j) * MC] = acc[j];
    }
  }
  if (failed) {
    if (tid == 0) atomicExch(&g_device_status, 1);
    // let outstanding MMAs finish (bounded) before tensor memory is released
    if (pending2) wait_bar(bar2, ph2);
    if (pending1) wait_bar(bar1, ph1);
  }
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOLS) : "memory");
  }
}

}  // namespace tc

// Slots of partial sums per image for `tasks` = images * fields cut into `ctas` ranges.
static long long tc_parts(long long images, long long fields, long long ctas) {
  const long long tasks = images * fields;
  long long parts = 1;
  for (long long q = 0; q < images; ++q) {
    const long long n = tc::cta_of(q * fields + fields - 1, tasks, ctas) - tc::cta_of(q * fields, tasks, ctas) + 1;
    if (n > parts) parts = n;
  }
  return parts;
}

}  // namespace oi

extern "C" int oi_coherent_tc_layout(long long images, int fields, int* ctas, int* nparts) {
  using namespace oi;
  if (images <= 0 || fields <= 0 || !ctas || !nparts) return fail(OI_EINVAL, "oi_coherent_tc_layout: bad arguments");
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return fail(OI_ECUDA, "oi_coherent_tc_layout: no CUDA device");
  const long long tasks = images * (long long)fields;
  const long long g = tasks < sms ? tasks : sms;
  *ctas = (int)g;
  *nparts = (int)tc_parts(images, fields, g);
  return OI_OK;
}

extern "C" int oi_coherent_coarse_tc(const void* band, int batch, int nch, int m0r, int br, int m0c, int bc,
                                     const void* pupil, long long pupil_batch_stride, const float* weight, int nz,
                                     int nk, const void* wr, const void* wc, int ctas, int nparts, float* coarse,
                                     void* stream) {
  using namespace oi;
  if (!band || !pupil || !weight || !wr || !wc || !coarse || batch <= 0 || nch <= 0 || br <= 0 || bc <= 0 ||
      nz <= 0 || nk <= 0 || ctas <= 0 || nparts <= 0 || pupil_batch_stride < 0)
    return fail(OI_EINVAL, "oi_coherent_coarse_tc: bad arguments");
  if (br > tc::BMAX || bc > tc::BMAX || 2 * br - 1 > tc::MR || 2 * bc - 1 > tc::MC)
    return fail(OI_ERANGE, "oi_coherent_coarse_tc: band %dx%d exceeds 64x64", br, bc);
  const long long images = (long long)batch * nz, fields = (long long)nk * nch;
  if (ctas > images * fields || ctas > 65535)
    return fail(OI_ERANGE, "oi_coherent_coarse_tc: %d CTAs for %lld tasks", ctas, images * fields);
  const long long need = tc_parts(images, fields, ctas);
  if (need > nparts)
    return fail(OI_ERANGE, "oi_coherent_coarse_tc: %d partial slots given, %lld needed", nparts, need);
  tc::Args a{(const float2*)band, (long long)nch * br * bc, nch, br, bc, m0r, m0c, (const float2*)pupil,
             pupil_batch_stride, weight, nz, nk, images, images * fields, nparts, (const float2*)wr,
             (const float2*)wc, coarse};
  int rc = ensure_smem((const void*)tc::coherent_tc_kernel, tc::SMEM_BYTES, "oi_coherent_coarse_tc");
  if (rc) return rc;
  tc::coherent_tc_kernel<<<(unsigned)ctas, tc::T, tc::SMEM_BYTES, (cudaStream_t)stream>>>(a);
  oi::note_launch();
  return check_launch("oi_coherent_coarse_tc");
}

extern "C" int oi_device_status(int* status, int reset) {
  using namespace oi;
  if (!status) return fail(OI_EINVAL, "oi_device_status: null status");
  if (cudaMemcpyFromSymbol(status, g_device_status, sizeof(int)) != cudaSuccess)
    return fail(OI_ECUDA, "oi_device_status: %s", cudaGetErrorString(cudaGetLastError()));
  if (reset) {
    const int zero = 0;
    if (cudaMemcpyToSymbol(g_device_status, &zero, sizeof(int)) != cudaSuccess)
      return fail(OI_ECUDA, "oi_device_status: %s", cudaGetErrorString(cudaGetLastError()));
  }
  return OI_OK;
}
