// Split-BF16x3 form of the coherent sum on a 128 x 128 coarse grid, on the 5th-generation tensor cores
// (tcgen05.mma, accumulators in tensor memory).  Same result as coherent_fft.cu -- the |fft2(.)|^2
// accumulation of CalculateAbbeImage (CalculateAerialImage.py:76-92) and CalculateAerialImage_SOCS
// (CalculateAerialImage_SOCS.py:5-10) -- with the band-to-coarse transform written as two dense DFT
// contractions:
//   E^T[sc][sr] = sum_ir sum_ic Cr[sr][ir] A[ir][ic] Cc[sc][ic],   A = P[z][k] .* band[b][c]  (<= 64 x 64),
//   Cc[sc][ic] = exp(-2 pi i (m0c+ic) sc / 128),  Cr[sr][ir] = exp(-2 pi i (m0r+ir) sr / 128).
// Stage 1 (M = sc, N = (re|im, ir), K = ic):   H^T = Cc A^T    A operand Cc (shared memory, constant), B operand
//   the stacked field [-Ai; Ar; Ai] (shared memory, built per field): Ccr x [Ar; Ai] + Cci x [-Ai; Ar].
// Stage 2 (M = sc, N = (re|im, sr), K = (re|im, ir)):   E^T = H^T Cr^T   A operand [Hr | Hi] (tensor memory,
//   converted from the stage-1 accumulator), B operand the stacked constant [-Cri; Crr; Cri]:
//   Hr x [Crr; Cri] + Hi x [-Cri; Crr].
// Every real operand x is split x = hi + lo with hi = bf16(x), lo = bf16(x - hi), and a product is
// hi*hi + hi*lo + lo*hi with FP32 accumulation (the lo*lo term, ~2^-16 relative, is dropped): about 16
// significant bits, against 24 for the FP32 forms.  Per field: 24 MMAs of 128x128x16 and 24 of 128x256x16.
// When m0r == m0c the row and column DFT matrices are the same and Cc is read from the Crr / Cri blocks.
//
// Work: the images' fields form one list of tasks t = (b*nz + z)*F + f, F = nk*nch, cut into equal
// contiguous ranges, one per CTA (one CTA per SM: the CTA holds all 512 tensor-memory columns).  A CTA
// accumulates w |E|^2 of its fields in registers and writes one partial coarse image per image it touches,
// to slot (CTA - first CTA of that image); the first CTA of an image zero-fills the slots no CTA owns, so
// the partial sums fold in a fixed order (deterministic).
//
// Pipeline (warp 0 lane 0 issues every MMA; all 8 warps read tensor memory, two per lane quarter):
//   barrier A | warp 0: issue stage 2 of t    | warps 1-7: build the stage-1 operand of t+1 from the staged
//             |                               |            pupil and band (copied ahead with cp.async)
//   barrier B | warp 0: issue stage 1 of t+1  | all: copy the pupil and band of t+2 into the stage
//   all: wait stage 2 of t, accumulate |E|^2 (overlaps stage 1 of t+1); wait stage 1 of t+1, convert its
//   accumulator to the stage-2 operand -> barrier A of the next task.
//
// Waits on the MMA-completion barriers are bounded (2 s of %globaltimer) and warp-uniform; on expiry the CTA
// records a status (oi_device_status), waits a bounded time for its outstanding MMAs, frees tensor memory and
// exits.
#include "tc_common.cuh"

namespace oi {

__device__ int g_device_status = 0;

namespace tc {

constexpr int T = 256;              // threads per CTA (8 warps: two per tensor-memory lane quarter)
constexpr int MC = 128, MR = 128;   // coarse grid
constexpr int BMAX = 64;            // band rows / columns (padded)
// Shared memory, from a 1024-byte aligned base.  Every operand is K-major with 64 bf16 (128 bytes) per row,
// 128-byte swizzled: element (row, k) at row*128 + (((k/8) ^ (row%8)) * 16) + (k%8)*2.
constexpr uint32_t ROWS = 128;                                // bytes per operand row
constexpr uint32_t CR3_BYTES = 384 * ROWS;                    // [-Cri; Crr; Cri], one precision
constexpr uint32_t CC_BYTES = 256 * ROWS;                     // [Ccr; Cci], one precision (m0r != m0c)
constexpr uint32_t B1_BYTES = 192 * ROWS;                     // [-Ai; Ar; Ai], one precision
constexpr uint32_t MISC_BYTES = 64;
// tensor memory columns (128 lanes x 512 columns of 32 bits)
constexpr uint32_t COL_D2 = 0;      // E^T: re [0,128), im [128,256)
constexpr uint32_t COL_D1 = 256;    // H^T: re [256,320), im [320,384)
constexpr uint32_t COL_A2H = 384;   // H^T as bf16 pairs, hi: [Hr | Hi] along K (64 columns)
constexpr uint32_t COL_A2L = 448;   // lo
constexpr uint32_t NCOLS = 512;

struct Layout {
  uint32_t cr3, cc, cc_lo, b1, stage, stage_arr, misc, bytes;  // cc: Ccr hi; Cci = cc + 128 rows; lo = cc + cc_lo
  uint32_t consts;                                             // bytes of the constant image (cr3 [+ cc])
  bool staged;
};

// Shared-memory layout for a band of `plane` elements.  The constant image (CR3 hi, lo, then Cc hi, lo when the
// column DFT differs) comes first, as oi_tc_constants writes it.  The stage holds the pupil and the band of a
// coming field (float2, `plane` + 2 elements each: element e at 8 (e + d), d in {0, 1} aligning the bulk copy)
// and is used when it fits.
__host__ __device__ inline Layout make_layout(bool sym, int plane) {
  Layout l;
  l.cr3 = 0;
  uint32_t off = 2 * CR3_BYTES;
  if (sym) {
    l.cc = l.cr3 + 128 * ROWS;
    l.cc_lo = CR3_BYTES;
  } else {
    l.cc = off;
    l.cc_lo = CC_BYTES;
    off += 2 * CC_BYTES;
  }
  l.consts = off;
  l.b1 = off;
  off += 2 * B1_BYTES;
  l.stage_arr = (uint32_t)(8 * (plane + 2) + 15) & ~15u;
  l.staged = off + 2 * l.stage_arr + MISC_BYTES + 1024 <= SMEM_LIMIT;
  l.stage = off;
  if (l.staged) off += 2 * l.stage_arr;
  l.misc = off;
  l.bytes = off + MISC_BYTES + 1024;
  return l;
}

// Writes rows of the DFT matrix C[s][i] = exp(-2 pi i (m0+i) s / 128), s < 128, i < 64, into an operand image
// (same bytes as the shared-memory operands): re at rows [re_row, +128), im at [im_row, +128) and, if
// neg_row >= 0, -im at [neg_row, +128); lo halves `lo` bytes after the hi halves.  One thread per 8 columns.
__device__ void dft_rows(unsigned char* img, uint32_t lo, int re_row, int im_row, int neg_row,
                         const float2* __restrict__ w, int m0, int chunk) {
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
  auto put = [&](int row, uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3, uint32_t off) {
    *(uint4*)(img + off + swz(row, g)) = make_uint4(x0, x1, x2, x3);
  };
  put(re_row + s, rh[0], rh[1], rh[2], rh[3], 0);
  put(re_row + s, rl[0], rl[1], rl[2], rl[3], lo);
  put(im_row + s, ih[0], ih[1], ih[2], ih[3], 0);
  put(im_row + s, il[0], il[1], il[2], il[3], lo);
  if (neg_row >= 0) {
    const uint32_t sg = 0x80008000u;
    put(neg_row + s, ih[0] ^ sg, ih[1] ^ sg, ih[2] ^ sg, ih[3] ^ sg, 0);
    put(neg_row + s, il[0] ^ sg, il[1] ^ sg, il[2] ^ sg, il[3] ^ sg, lo);
  }
}

// The constant image: CR3 = [-Cri; Crr; Cri] (from wr, m0r) and, when m0c != m0r, Cc = [Ccr; Cci].
__global__ void tc_constants_kernel(unsigned char* img, const float2* wr, int m0r, const float2* wc, int m0c) {
  const int chunk = blockIdx.x * blockDim.x + threadIdx.x;
  if (chunk >= 128 * 8) return;
  dft_rows(img, CR3_BYTES, 128, 256, 0, wr, m0r, chunk);
  if (m0c != m0r) dft_rows(img + 2 * CR3_BYTES, CC_BYTES, 0, 128, -1, wc, m0c, chunk);
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
  float* coarse;              // [nparts][images][128][128]
  const unsigned char* consts;  // constant operand image (oi_tc_constants)
};

// CTA owning task t when `tasks` are cut into gridDim.x ranges [floor(i T / G), floor((i+1) T / G)).
__host__ __device__ __forceinline__ long long cta_of(long long t, long long tasks, long long g) {
  return ((t + 1) * g - 1) / tasks;
}

struct FieldSrc {
  const float2* pupil;
  const float2* band;
  float w;
};

// Position of task t = (image q = b * nz + z, kernel k, channel c): divided out once per CTA, then advanced by
// counters (64-bit division is a long emulated sequence on the device).
struct TaskPos {
  long long q, b;
  int z, k, c;
  __device__ __forceinline__ void init(const Args& a, long long t) {
    const int F = a.nk * a.nch;
    q = t / F;
    const int f = (int)(t - q * F);
    k = f / a.nch;
    c = f - k * a.nch;
    b = q / a.nz;
    z = (int)(q - b * a.nz);
  }
  __device__ __forceinline__ void next(const Args& a) {
    if (++c == a.nch) {
      c = 0;
      if (++k == a.nk) {
        k = 0;
        ++q;
        if (++z == a.nz) {
          z = 0;
          ++b;
        }
      }
    }
  }
  __device__ __forceinline__ bool first() const { return k == 0 && c == 0; }   // first field of image q
};

__device__ __forceinline__ FieldSrc field_src(const Args& a, const TaskPos& p) {
  const long long plane = (long long)a.br * a.bc;
  FieldSrc s;
  s.pupil = a.pupil + p.b * a.pupil_batch_stride + ((long long)p.z * a.nk + p.k) * plane;
  s.band = a.band + p.b * a.band_img_stride + (long long)p.c * plane;
  s.w = __ldg(a.weight + (long long)p.z * a.nk + p.k);
  return s;
}

// Alignment shift of a float2 array in the stage: element e sits at 8 (e + d).
__device__ __forceinline__ int stage_shift(const float2* p) { return (int)(((uintptr_t)p >> 3) & 1); }

// Copy of n float2 from p into the stage array at s (16-byte aligned): the 16-byte aligned body by one bulk
// copy completing on `bar`, the (at most two) unaligned end elements by plain loads.  Returns the bulk bytes.
__device__ __forceinline__ uint32_t stage_array(uint32_t s, const float2* p, int n, uint32_t bar) {
  const int d = stage_shift(p);
  const int nb = (n - d) & ~1;
  if (nb > 0) bulk_g2s(s + 8 * (2 * d), p + d, 8u * nb, bar);
  if (d && n > 0) {
    const float2 v = __ldg(p);
    asm volatile("st.shared.v2.f32 [%0], {%1, %2};" ::"r"(s + 8), "f"(v.x), "f"(v.y) : "memory");
  }
  if (d + nb < n) {
    const float2 v = __ldg(p + n - 1);
    asm volatile("st.shared.v2.f32 [%0], {%1, %2};" ::"r"(s + 8 * (n - 1 + d)), "f"(v.x), "f"(v.y) : "memory");
  }
  return nb > 0 ? 8u * nb : 0u;
}

// Stage copy of task t's pupil and band (issued by one thread; completes on `bar`).
// The band is copied only when it differs from the one the stage holds (consecutive fields of one image and
// channel share it: the SOCS kernels of a clip).
__device__ __forceinline__ void stage_copy(const Args& a, const FieldSrc& f, uint32_t stage, uint32_t arr, uint32_t bar,
                                           bool with_band) {
  const int plane = a.br * a.bc;
  const uint32_t bytes = 8u * ((plane - stage_shift(f.pupil)) & ~1) +
                         (with_band ? 8u * ((plane - stage_shift(f.band)) & ~1) : 0u);
  expect_tx(bar, bytes);
  stage_array(stage, f.pupil, plane, bar);
  if (with_band) stage_array(stage + arr, f.band, plane, bar);
}

// The stage-1 B operand of a field, A = P .* band zero-padded to 64 x 64: rows [0,64) = -Ai, [64,128) = Ar,
// [128,192) = Ai (K = ic), hi at b1, lo at b1 + B1_BYTES.  pk / hc are generic pointers (stage or global).
// Threads bt = 0 .. nthreads-1 share the 512 chunks of 8 columns.
__device__ __forceinline__ void build_field(const float2* pk, const float2* hc, int br, int bc, uint32_t b1, int bt,
                                            int nthreads) {
  for (int chunk = bt; chunk < 64 * 8; chunk += nthreads) {
    const int ir = chunk >> 3, g = chunk & 7;
    float2 v[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int ic = 8 * g + e;
      v[e] = make_float2(0.f, 0.f);
      if (ir < br && ic < bc) {
        const int o = ir * bc + ic;
        v[e] = cmul(pk[o], hc[o]);
      }
    }
    uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      split2(v[2 * e].x, v[2 * e + 1].x, rh[e], rl[e]);
      split2(v[2 * e].y, v[2 * e + 1].y, ih[e], il[e]);
    }
    const uint32_t sg = 0x80008000u;
    const uint32_t o_ng = b1 + swz(ir, g), o_re = b1 + swz(64 + ir, g), o_im = b1 + swz(128 + ir, g);
    st_shared_v4(o_ng, ih[0] ^ sg, ih[1] ^ sg, ih[2] ^ sg, ih[3] ^ sg);
    st_shared_v4(o_ng + B1_BYTES, il[0] ^ sg, il[1] ^ sg, il[2] ^ sg, il[3] ^ sg);
    st_shared_v4(o_re, rh[0], rh[1], rh[2], rh[3]);
    st_shared_v4(o_re + B1_BYTES, rl[0], rl[1], rl[2], rl[3]);
    st_shared_v4(o_im, ih[0], ih[1], ih[2], ih[3]);
    st_shared_v4(o_im + B1_BYTES, il[0], il[1], il[2], il[3]);
  }
}

// Stage 1: D1[sc][n] = sum_ic Cc[sc][ic] B1[n][ic], n < 64 re / n >= 64 im of H^T:  Ccr x [Ar; Ai] (B1 rows
// 64..191) + Cci x [-Ai; Ar] (rows 0..127).  24 MMAs of 128 x 128 x 16.
__device__ __forceinline__ void issue_stage1(uint32_t tmem, uint32_t cc, uint32_t cc_lo, uint32_t b1) {
  constexpr uint32_t ID = idesc(128, false);
  const uint32_t d = tmem + COL_D1;
#pragma unroll
  for (int term = 0; term < 2; ++term) {
    const uint32_t x = cc + term * 128 * ROWS;
    const uint32_t y = b1 + (term ? 0u : 64 * ROWS);
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      const uint32_t ko = 32 * ks;
      mma_ss(d, sdesc(x + ko), sdesc(y + ko), ID, (term | ks) ? 1u : 0u);   // hi hi
      mma_ss(d, sdesc(x + ko), sdesc(y + B1_BYTES + ko), ID, 1);            // hi lo
      mma_ss(d, sdesc(x + cc_lo + ko), sdesc(y + ko), ID, 1);               // lo hi
    }
  }
}

// Stage 2: D2[sc][n] = sum_k A2[sc][k] CR3[row(n)][k], n < 128 re / n >= 128 im of E^T:  Hr x [Crr; Cri]
// (CR3 rows 128..383) + Hi x [-Cri; Crr] (rows 0..255).  24 MMAs of 128 x 256 x 16.
__device__ __forceinline__ void issue_stage2(uint32_t tmem, uint32_t cr3) {
  constexpr uint32_t ID = idesc(256, false);
  const uint32_t d = tmem + COL_D2;
#pragma unroll
  for (int ks = 0; ks < 8; ++ks) {
    const uint32_t bm = cr3 + ((ks >> 2) ? 0u : 128 * ROWS) + 32 * (ks & 3);
    const uint32_t ah = tmem + COL_A2H + 8 * ks, al = tmem + COL_A2L + 8 * ks;
    mma_ts(d, ah, sdesc(bm), ID, ks ? 1u : 0u);                              // hi hi
    mma_ts(d, ah, sdesc(bm + CR3_BYTES), ID, 1);                              // hi lo
    mma_ts(d, al, sdesc(bm), ID, 1);                                          // lo hi
  }
}

// w |E|^2 of the finished stage 2 into acc (this warp's lane quarter and column half).
__device__ __forceinline__ void accumulate(float (&acc)[64], uint32_t taddr, int half, float w) {
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    float re[32], im[32];
    tmem_ld32x2(taddr + COL_D2 + 64 * half + 32 * p, taddr + COL_D2 + 128 + 64 * half + 32 * p, re, im);
#pragma unroll
    for (int j = 0; j < 32; ++j) acc[32 * p + j] = fmaf(w, fmaf(re[j], re[j], im[j] * im[j]), acc[32 * p + j]);
  }
}

// The stage-1 accumulator (H^T, FP32) -> the stage-2 A operand (bf16 hi / lo pairs); half 0 converts Hr, 1 Hi.
__device__ __forceinline__ void convert(uint32_t taddr, int half) {
  float h[32], h2[32];
  tmem_ld32x2(taddr + COL_D1 + 64 * half, taddr + COL_D1 + 64 * half + 32, h, h2);
  uint32_t hi[32], lo[32];
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    split2(h[2 * j], h[2 * j + 1], hi[j], lo[j]);
    split2(h2[2 * j], h2[2 * j + 1], hi[16 + j], lo[16 + j]);
  }
  tmem_st32(taddr + COL_A2H + 32 * half, hi);
  tmem_st32(taddr + COL_A2L + 32 * half, lo);
  wait_st();
}

__global__ void __launch_bounds__(T, 1) coherent_tc_kernel(Args a) {
  extern __shared__ unsigned char smem_raw[];
  const bool sym = a.m0r == a.m0c;
  const int plane = a.br * a.bc;
  const Layout L = make_layout(sym, plane);
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char* gbase = smem_raw + (base - raw);
  const uint32_t bar1 = base + L.misc, bar2 = bar1 + 8, bar3 = bar1 + 16, bar4 = bar1 + 24;
  volatile uint32_t* tmem_slot = (volatile uint32_t*)(gbase + L.misc + 32);
  const float2* st_p = (const float2*)(gbase + L.stage);
  const float2* st_h = (const float2*)(gbase + L.stage + L.stage_arr);
  const uint32_t cr3 = base + L.cr3, cc = base + L.cc, b1 = base + L.b1, stage = base + L.stage;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long G = gridDim.x;
  const long long t0 = (long long)blockIdx.x * a.tasks / G, t1 = ((long long)blockIdx.x + 1) * a.tasks / G;
  const int F = a.nk * a.nch;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(base + L.misc + 32),
                 "r"(NCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  TaskPos pt;                                   // position of task t (t0 before the loop)
  pt.init(a, t0);
  FieldSrc cur = field_src(a, pt);
  if (tid == 0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar1 + 8 * i) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    // constant operands: one bulk copy per 16 KB
    expect_tx(bar4, L.consts);
    for (uint32_t o = 0; o < L.consts; o += 16384)
      bulk_g2s(base + o, a.consts + o, L.consts - o < 16384 ? L.consts - o : 16384, bar4);
    pdl_wait();   // the band comes from the spectrum pass
    if (L.staged) stage_copy(a, cur, stage, L.stage_arr, bar3, true);
  }
  __syncthreads();  // barrier inits and the stage's unaligned end elements
  pdl_trigger();
  pdl_wait();
  uint32_t ph3 = 0;
  bool bad = false;
  if (L.staged) {
    bad = !warp_wait(bar3, ph3);
    ph3 ^= 1;
  }
  if (!bad) {
    const float2* pk = L.staged ? st_p + stage_shift(cur.pupil) : cur.pupil;
    const float2* hc = L.staged ? st_h + stage_shift(cur.band) : cur.band;
    build_field(pk, hc, a.br, a.bc, b1, tid, T);
  }
  if (tid == 0) bad |= !wait_bar(bar4, 0);  // the constants have landed
  fence_async_smem();
  fence_before();
  bool failed = __syncthreads_or(bad);
  fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t taddr = tmem + ((uint32_t)(32 * (warp & 3)) << 16);  // this warp's lane quarter
  const int half = warp >> 2;                                          // column half this warp reads
  const int sc = 32 * (warp & 3) + lane;                               // coarse column = accumulator row
  uint32_t ph1 = 0, ph2 = 0;
  int pending1 = 0, pending2 = 0, pending3 = 0;
  if (!failed) {
    if (tid == 0) {
      issue_stage1(tmem, cc, L.cc_lo, b1);
      commit(bar1);
    }
    pending1 = 1;
    FieldSrc nxt = cur;
    TaskPos p1 = pt;
    p1.next(a);
    if (t0 + 1 < t1) nxt = field_src(a, p1);
    if (L.staged && t0 + 1 < t1) {
      if (tid == 32) stage_copy(a, nxt, stage, L.stage_arr, bar3, nxt.band != cur.band);
      pending3 = 1;
    }
  }

  float acc[64];
#pragma unroll
  for (int j = 0; j < 64; ++j) acc[j] = 0.f;
  float wprev = 0.f;

  for (long long t = t0; t < t1 && !failed; ++t) {
    bad = false;
    TaskPos p1 = pt, p2;
    p1.next(a);
    p2 = p1;
    p2.next(a);
    // (1) |E|^2 of task t-1 (overlaps stage 1 of t on the tensor pipe)
    if (t > t0) {
      if (warp_wait(bar2, ph2)) {
        fence_after();
        accumulate(acc, taddr, half, wprev);
      } else {
        bad = true;
      }
      ph2 ^= 1;
      pending2 = 0;
      if (pt.first()) {  // task t-1 was the last of its image in this range
        const long long qp = pt.q - 1;
        const long long slot = blockIdx.x - cta_of(qp * F, a.tasks, G);
        float* out = a.coarse + (slot * a.images + qp) * (long long)(MR * MC) + sc;
#pragma unroll
        for (int j = 0; j < 64; ++j) {
          out[(64 * half + j) * MC] = acc[j];
          acc[j] = 0.f;
        }
      }
    }
    // (2) stage-1 accumulator of t -> stage-2 A operand
    if (warp_wait(bar1, ph1)) {
      fence_after();
      convert(taddr, half);
    } else {
      bad = true;
    }
    ph1 ^= 1;
    pending1 = 0;
    wprev = cur.w;
    if (t + 1 < t1) cur = field_src(a, p1);
    // zero-fill the partial slots of this image that no CTA owns (done by the image's first CTA)
    if (pt.first()) {
      const long long q = pt.q;
      const long long first = cta_of(q * F, a.tasks, G), last = cta_of(q * F + F - 1, a.tasks, G);
      for (long long slot = last - first + 1; slot < a.nparts; ++slot) {
        float* out = a.coarse + (slot * a.images + q) * (long long)(MR * MC);
        for (int e = tid; e < MR * MC / 4; e += T) ((float4*)out)[e] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
    if (pending3) {  // the stage holds task t+1
      bad |= !warp_wait(bar3, ph3);
      ph3 ^= 1;
      pending3 = 0;
    }
    fence_before();
    if (__syncthreads_or(bad)) {  // barrier A
      failed = true;
      break;
    }
    if (warp == 0) {
      if (lane == 0) {
        fence_after();
        issue_stage2(tmem, cr3);
        commit(bar2);
      }
      __syncwarp();
    } else if (t + 1 < t1) {
      const float2* pk = L.staged ? st_p + stage_shift(cur.pupil) : cur.pupil;
      const float2* hc = L.staged ? st_h + stage_shift(cur.band) : cur.band;
      build_field(pk, hc, a.br, a.bc, b1, tid - 32, T - 32);
    }
    pending2 = 1;
    fence_async_smem();
    __syncthreads();  // barrier B: the stage-1 operand of t+1 is built and the stage is free
    if (t + 1 < t1) {
      if (tid == 0) {
        fence_after();
        issue_stage1(tmem, cc, L.cc_lo, b1);
        commit(bar1);
      }
      pending1 = 1;
      if (L.staged && t + 2 < t1) {
        if (tid == 32) {
          const FieldSrc f2 = field_src(a, p2);
          stage_copy(a, f2, stage, L.stage_arr, bar3, f2.band != cur.band);   // cur: field t+1, in the stage
        }
        pending3 = 1;
      }
    }
    pt = p1;
  }
  if (!failed) {
    if (warp_wait(bar2, ph2)) {
      fence_after();
      accumulate(acc, taddr, half, wprev);
      pending2 = 0;
      const long long qp = (t1 - 1) / F;
      const long long slot = blockIdx.x - cta_of(qp * F, a.tasks, G);
      float* out = a.coarse + (slot * a.images + qp) * (long long)(MR * MC) + sc;
#pragma unroll
      for (int j = 0; j < 64; ++j) out[(64 * half + j) * MC] = acc[j];
    } else {
      failed = true;
    }
  }
  if (failed) {
    if (lane == 0) atomicExch(&g_device_status, 1);
    // let outstanding MMAs and copies finish (bounded) before tensor memory and shared memory are released
    if (pending2) wait_bar(bar2, ph2);
    if (pending1) wait_bar(bar1, ph1);
    if (pending3) wait_bar(bar3, ph3);
    if (tid == 0) wait_bar(bar4, 0);
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

extern "C" int oi_tc_constants(int m0r, int m0c, const void* wr, const void* wc, void* image, long long bytes,
                               void* stream) {
  using namespace oi;
  if (!wr || !wc || !image) return fail(OI_EINVAL, "oi_tc_constants: bad arguments");
  const long long need = 2LL * tc::CR3_BYTES + (m0r != m0c ? 2LL * tc::CC_BYTES : 0);
  if (bytes < need) return fail(OI_ERANGE, "oi_tc_constants: %lld bytes given, %lld needed", bytes, need);
  if ((uintptr_t)image % 16) return fail(OI_EINVAL, "oi_tc_constants: image not 16-byte aligned");
  tc::tc_constants_kernel<<<4, 256, 0, (cudaStream_t)stream>>>((unsigned char*)image, (const float2*)wr, m0r,
                                                                (const float2*)wc, m0c);
  oi::note_launch();
  return check_launch("oi_tc_constants");
}

extern "C" int oi_coherent_coarse_tc(const void* band, int batch, int nch, int m0r, int br, int m0c, int bc,
                                     const void* pupil, long long pupil_batch_stride, const float* weight, int nz,
                                     int nk, const void* consts, int ctas, int nparts, float* coarse, void* stream) {
  using namespace oi;
  if (!band || !pupil || !weight || !consts || !coarse || batch <= 0 || nch <= 0 || br <= 0 || bc <= 0 ||
      nz <= 0 || nk <= 0 || ctas <= 0 || nparts <= 0 || pupil_batch_stride < 0)
    return fail(OI_EINVAL, "oi_coherent_coarse_tc: bad arguments");
  if ((uintptr_t)consts % 16) return fail(OI_EINVAL, "oi_coherent_coarse_tc: constant image not 16-byte aligned");
  if (br > tc::BMAX || bc > tc::BMAX || 2 * br - 1 > tc::MR || 2 * bc - 1 > tc::MC)
    return fail(OI_ERANGE, "oi_coherent_coarse_tc: band %dx%d exceeds 64x64", br, bc);
  const long long images = (long long)batch * nz, fields = (long long)nk * nch;
  if (ctas > images * fields || ctas > 65535)
    return fail(OI_ERANGE, "oi_coherent_coarse_tc: %d CTAs for %lld tasks", ctas, images * fields);
  const long long need = tc_parts(images, fields, ctas);
  if (need > nparts)
    return fail(OI_ERANGE, "oi_coherent_coarse_tc: %d partial slots given, %lld needed", nparts, need);
  tc::Args a{(const float2*)band, (long long)nch * br * bc, nch, br, bc, m0r, m0c, (const float2*)pupil,
             pupil_batch_stride, weight, nz, nk, images, images * fields, nparts, coarse,
             (const unsigned char*)consts};
  const tc::Layout L = tc::make_layout(m0r == m0c, br * bc);
  int rc = ensure_smem((const void*)tc::coherent_tc_kernel, L.bytes, "oi_coherent_coarse_tc");
  if (rc) return rc;
  (void)launch_pdl(tc::coherent_tc_kernel, dim3((unsigned)ctas), dim3(tc::T), (size_t)L.bytes, (cudaStream_t)stream, a);
  oi::note_launch();
  return check_launch("oi_coherent_coarse_tc");
}

namespace oi {
namespace tc {

// The failure path every tensor-core kernel takes when a wait runs out, on its own: a CTA allocates tensor
// memory, waits with the bounded wait of the kernels (limit `limit_ns`) on a barrier phase that nothing
// completes, records the expiry in the device status, releases tensor memory and returns.  Nothing is in
// flight while it waits.
__global__ void wait_probe_kernel(unsigned long long limit_ns, unsigned cols) {
  __shared__ __align__(16) uint64_t bar;
  __shared__ uint32_t slot;
  const int warp = threadIdx.x >> 5;
  if (warp == 0) tmem_alloc(smem_u32(&slot), cols);
  if (threadIdx.x == 0) {
    mbar_init(smem_u32(&bar), 1);
    mbar_init_fence();
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = slot;
  const bool ok = warp_wait_for(smem_u32(&bar), 0, limit_ns);   // no thread arrives: the phase never completes
  if (!ok && threadIdx.x == 0) atomicExch(&g_device_status, 1);
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    tmem_dealloc(tmem, cols);
  }
}

}  // namespace tc
}  // namespace oi

extern "C" int oi_wait_probe(long long limit_ns, int tmem_cols, void* stream) {
  using namespace oi;
  if (limit_ns <= 0 || limit_ns > 100000000LL)
    return fail(OI_ERANGE, "oi_wait_probe: limit %lld ns outside (0, 100 ms]", limit_ns);
  if (tmem_cols < 32 || tmem_cols > 512 || (tmem_cols & (tmem_cols - 1)))
    return fail(OI_EINVAL, "oi_wait_probe: tensor-memory columns must be a power of two in [32, 512]");
  tc::wait_probe_kernel<<<1, 64, 0, (cudaStream_t)stream>>>((unsigned long long)limit_ns, (unsigned)tmem_cols);
  oi::note_launch();
  return check_launch("oi_wait_probe");
}

extern "C" int oi_device_status(int* status, int reset) {
  using namespace oi;
  if (!status) return fail(OI_EINVAL, "oi_device_status: null status");
  int rows = 0, synth = 0;
  if (cudaMemcpyFromSymbol(status, g_device_status, sizeof(int)) != cudaSuccess || rows_tc_status(&rows, reset) ||
      synth_tc_status(&synth, reset))
    return fail(OI_ECUDA, "oi_device_status: %s", cudaGetErrorString(cudaGetLastError()));
  *status |= rows | synth;
  if (reset) {
    const int zero = 0;
    if (cudaMemcpyToSymbol(g_device_status, &zero, sizeof(int)) != cudaSuccess)
      return fail(OI_ECUDA, "oi_device_status: %s", cudaGetErrorString(cudaGetLastError()));
  }
  return OI_OK;
}
