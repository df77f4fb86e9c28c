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
// Pipeline (12 warps, each role waiting on mbarriers only):
//   warps 0-7   tensor-memory warps, two per lane quarter: convert the stage-1 accumulator of field i, in place,
//               into its stage-2 A operand (bf16 hi / lo), build 224 of the 512 chunks of a coming field's
//               stage-1 B operand, and accumulate w |E|^2 of field i-1 from the stage-2 accumulator into registers;
//   warps 8-10  build the other 288 chunks of the stage-1 B operand of the coming fields (P .* band, read from
//               global memory where both stay L2-resident) into a ring of B1 slots: 2 for a symmetric band, 1 when
//               Cc needs its own 64 KB; every warp but the MMA warp builds the first slots' fields at the start;
//   warp 11     lane 0 issues the MMAs in the order S1(i), S2(i-1), S1(i+1), S2(i), ...
// Tensor memory holds E^T (256 columns) and two regions of 128 columns, each the stage-1 accumulator H^T of a
// field and, after its conversion, that field's stage-2 operand.  So the tensor pipe runs S1(i+1) while field
// i-1's |E|^2 is read out and S2(i) while field i+1 is converted and later fields are built: the conversions and
// builds leave its critical path.  S1(i+1) reuses the region S2(i-1) read and is issued once S2(i-1) completes.
//
// Every wait is bounded (2 s of %globaltimer); on expiry a role records a status (oi_device_status) and stops,
// the roles waiting on it then expire in turn, and the MMA thread waits (bounded) for the MMAs it issued before
// the CTA frees tensor memory and exits.
#include "tc_common.cuh"

namespace oi {

__device__ int g_device_status = 0;

namespace tc {

constexpr int T = 384;              // threads per CTA: 8 tensor-memory warps, 3 build warps, the MMA warp
constexpr int NBUILD = 3;           // build warps (8 .. 10)
constexpr int MMA_WARP = 11;
constexpr int MC = 128, MR = 128;   // coarse grid
constexpr int BMAX = 64;            // band rows / columns (padded)
// Shared memory, from a 1024-byte aligned base.  Every operand is K-major with 64 bf16 (128 bytes) per row,
// 128-byte swizzled: element (row, k) at row*128 + (((k/8) ^ (row%8)) * 16) + (k%8)*2.
constexpr uint32_t ROWS = 128;                                // bytes per operand row
constexpr uint32_t CR3_BYTES = 384 * ROWS;                    // [-Cri; Crr; Cri], one precision
constexpr uint32_t CC_BYTES = 256 * ROWS;                     // [Ccr; Cci], one precision (m0r != m0c)
constexpr uint32_t B1_BYTES = 192 * ROWS;                     // [-Ai; Ar; Ai], one precision
constexpr uint32_t MISC_BYTES = 128;
// tensor memory columns (128 lanes x 512 columns of 32 bits)
constexpr uint32_t COL_D2 = 0;      // E^T: re [0,128), im [128,256)
constexpr uint32_t COL_R = 256;     // regions 256 + 128 r, r = field index mod 2: H^T re [0,64), im [64,128);
                                    // converted: [Hr hi | Hr lo | Hi hi | Hi lo], 32 columns of bf16 pairs each
constexpr uint32_t NCOLS = 512;

struct Layout {
  uint32_t cr3, cc, cc_lo, b1, nb1, misc, bytes;  // cc: Ccr hi; Cci = cc + 128 rows; lo = cc + cc_lo
  uint32_t consts;                                // bytes of the constant image (cr3 [+ cc])
};

// Shared-memory layout.  The constant image (CR3 hi, lo, then Cc hi, lo when the column DFT differs) comes first,
// as oi_tc_constants writes it, then the B1 slots (hi, lo each).
__host__ __device__ inline Layout make_layout(bool sym) {
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
  l.nb1 = sym ? 2 : 1;
  off += l.nb1 * 2 * B1_BYTES;
  l.misc = off;
  l.bytes = off + MISC_BYTES + 1024;
  return l;
}
static_assert(2 * CR3_BYTES + 2 * 2 * B1_BYTES + MISC_BYTES + 1024 <= SMEM_LIMIT, "coherent_tc: shared memory");
static_assert(2 * CR3_BYTES + 2 * CC_BYTES + 2 * B1_BYTES + MISC_BYTES + 1024 <= SMEM_LIMIT,
              "coherent_tc: shared memory");

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

// The stage-1 B operand of a field, A = P .* band zero-padded to 64 x 64: rows [0,64) = -Ai, [64,128) = Ar,
// [128,192) = Ai (K = ic), hi at b1, lo at b1 + B1_BYTES, in 512 chunks of 8 columns.  The calling thread builds
// chunks c0, c0 + step, ... (COUNT of them), two at a time (all 32 loads of a pair issued before any product).
template <int COUNT>
__device__ __forceinline__ void build_chunks(const float2* __restrict__ pk, const float2* __restrict__ hc, int br,
                                             int bc, uint32_t b1, int c0, int step) {
  constexpr int count = COUNT;
#pragma unroll
  for (int k = 0; k < count; k += 2) {
    float2 p[2][8], h[2][8];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int chunk = c0 + (k + u) * step, ir = chunk >> 3, g = chunk & 7;
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int ic = 8 * g + e;
        const bool in = k + u < count && ir < br && ic < bc;
        const int o = ir * bc + ic;
        p[u][e] = in ? __ldg(pk + o) : make_float2(0.f, 0.f);
        h[u][e] = in ? __ldg(hc + o) : make_float2(0.f, 0.f);
      }
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      if (k + u >= count) break;
      const int chunk = c0 + (k + u) * step, ir = chunk >> 3, g = chunk & 7;
      uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float2 v0 = cmul(p[u][2 * e], h[u][2 * e]), v1 = cmul(p[u][2 * e + 1], h[u][2 * e + 1]);
        split2(v0.x, v1.x, rh[e], rl[e]);
        split2(v0.y, v1.y, ih[e], il[e]);
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
}

// Chunks of a field's B1 per thread: the build warps take chunks [0, 288) (three each), tensor-memory threads
// 0 .. 223 one each of [288, 512).
constexpr int BUILD_CHUNKS = 3 * 32 * NBUILD;
static_assert(BUILD_CHUNKS + 224 == 512 && 224 <= 256, "coherent_tc: B1 chunks");
__device__ __forceinline__ void build_share(const FieldSrc& f, int br, int bc, uint32_t b1, int tid) {
  if (tid >= 256) build_chunks<3>(f.pupil, f.band, br, bc, b1, tid - 256, 32 * NBUILD);
  else if (tid < 224) build_chunks<1>(f.pupil, f.band, br, bc, b1, BUILD_CHUNKS + tid, 0);
}

// Stage 1: D1[sc][n] = sum_ic Cc[sc][ic] B1[n][ic], n < 64 re / n >= 64 im of H^T:  Ccr x [Ar; Ai] (B1 rows
// 64..191) + Cci x [-Ai; Ar] (rows 0..127).  24 MMAs of 128 x 128 x 16 into the region at column d.
__device__ __forceinline__ void issue_stage1(uint32_t d, uint32_t cc, uint32_t cc_lo, uint32_t b1) {
  constexpr uint32_t ID = idesc(128, false);
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
// (CR3 rows 128..383) + Hi x [-Cri; Crr] (rows 0..255), A2 the converted region at column r.  24 MMAs of
// 128 x 256 x 16.
__device__ __forceinline__ void issue_stage2(uint32_t tmem, uint32_t r, uint32_t cr3) {
  constexpr uint32_t ID = idesc(256, false);
  const uint32_t d = tmem + COL_D2;
#pragma unroll
  for (int ks = 0; ks < 8; ++ks) {
    const uint32_t bm = cr3 + ((ks >> 2) ? 0u : 128 * ROWS) + 32 * (ks & 3);
    const uint32_t ah = tmem + r + 64 * (ks >> 2) + 8 * (ks & 3), al = ah + 32;
    mma_ts(d, ah, sdesc(bm), ID, ks ? 1u : 0u);                              // hi hi
    mma_ts(d, ah, sdesc(bm + CR3_BYTES), ID, 1);                              // hi lo
    mma_ts(d, al, sdesc(bm), ID, 1);                                          // lo hi
  }
}

// w |E|^2 of the finished stage 2 into acc (this warp's lane quarter and column half).
__device__ __forceinline__ void accumulate(float (&acc)[64], uint32_t taddr, int half, float w) {
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    float re[16], im[16];
    tmem_ld16x2(taddr + COL_D2 + 64 * half + 16 * p, taddr + COL_D2 + 128 + 64 * half + 16 * p, re, im);
#pragma unroll
    for (int j = 0; j < 16; ++j) acc[16 * p + j] = fmaf(w, fmaf(re[j], re[j], im[j] * im[j]), acc[16 * p + j]);
  }
}

// The stage-1 accumulator in the region at column r (H^T, FP32) -> the stage-2 A operand in place: half 0
// converts Hr (columns [0,64) -> hi at [0,32), lo at [32,64)), half 1 Hi (columns [64,128)), 32 columns at a
// time; every column a warp writes is one it has already read.
__device__ __forceinline__ void convert(uint32_t taddr, uint32_t r, int half) {
  const uint32_t c = taddr + r + 64 * half;
  float x[32];
  uint32_t hi[16], lo[16], lo2[16];
  tmem_ld32(c, x);
#pragma unroll
  for (int j = 0; j < 16; ++j) split2(x[2 * j], x[2 * j + 1], hi[j], lo[j]);
  tmem_st16(c, hi);        // columns [0,16): read
  tmem_ld32(c + 32, x);
#pragma unroll
  for (int j = 0; j < 16; ++j) split2(x[2 * j], x[2 * j + 1], hi[j], lo2[j]);
  tmem_st16(c + 16, hi);
  tmem_st16(c + 32, lo);   // columns [32,64): read by the second load
  tmem_st16(c + 48, lo2);
  wait_st();
}

__global__ void __launch_bounds__(T, 1) coherent_tc_kernel(Args a) {
  extern __shared__ unsigned char smem_raw[];
  const Layout L = make_layout(a.m0r == a.m0c);
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char* gbase = smem_raw + (base - raw);
  const uint32_t misc = base + L.misc;
  // barriers: cbar (constants landed), bfull[2] (B1 slot built), bfree[2] (S1 reading the slot finished),
  // s1done[2] (S1 into region r finished), conv[2] (region r converted), s2done (S2 finished: E^T complete and
  // its region free), d2free (E^T read out), fin (every issued MMA finished, at the end)
  const uint32_t cbar = misc, bfull = misc + 8, bfree = misc + 24, s1done = misc + 40, conv = misc + 56,
                 s2done = misc + 72, d2free = misc + 80, fin = misc + 88;
  volatile uint32_t* tmem_slot = (volatile uint32_t*)(gbase + L.misc + 96);
  const uint32_t cr3 = base + L.cr3, cc = base + L.cc, b1 = base + L.b1;
  const int nb1 = (int)L.nb1;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long G = gridDim.x;
  const long long t0 = (long long)blockIdx.x * a.tasks / G, t1 = ((long long)blockIdx.x + 1) * a.tasks / G;
  const int n = (int)(t1 - t0);   // fields of this CTA, >= 1
  const int F = a.nk * a.nch;

  if (warp == 0) tmem_alloc(misc + 96, NCOLS);
  if (tid == 32 * MMA_WARP) {
    mbar_init(cbar, 1);
    for (int r = 0; r < 2; ++r) {
      mbar_init(bfull + 8 * r, 8 + NBUILD);
      mbar_init(bfree + 8 * r, 1);
      mbar_init(s1done + 8 * r, 1);
      mbar_init(conv + 8 * r, 8);
    }
    mbar_init(s2done, 1);
    mbar_init(d2free, 8);
    mbar_init(fin, 1);
    mbar_init_fence();
    // constant operands: one bulk copy per 16 KB
    expect_tx(cbar, L.consts);
    for (uint32_t o = 0; o < L.consts; o += 16384)
      bulk_g2s(base + o, a.consts + o, L.consts - o < 16384 ? L.consts - o : 16384, cbar);
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;
  pdl_trigger();
  pdl_wait();   // bands, pupils and weights are read, and partial sums written, from here on
  if (warp != MMA_WARP) {   // every warp but the MMA warp builds the first fields' B1 (one per slot)
    TaskPos p;
    p.init(a, t0);
    for (int f = 0; f < n && f < nb1; ++f) {
      build_share(field_src(a, p), a.br, a.bc, b1 + f * 2 * B1_BYTES, tid);
      fence_async_smem();
      __syncwarp();
      if (lane == 0) arrive(bfull + 8 * f);
      p.next(a);
    }
  }

  if (warp == MMA_WARP) {
    // ---- MMA issue: S1(i) into region i & 1 (its B1 slot built, S2(i-2) done with the region), then S2(i-1)
    // (region converted, E^T of field i-2 read out)
    if (lane == 0) {
      const bool cok = wait_bar(cbar, 0);
      bool ok = cok, issued = false;
      Ring bs{0, 0};
      for (int i = 0; i <= n && ok; ++i) {
        if (i < n) {
          ok = wait_bar(bfull + 8 * bs.slot, bs.phase);
          if (ok && i >= 2) ok = wait_bar(s2done, (uint32_t)((i - 2) & 1));
          if (!ok) break;
          fence_after();
          issue_stage1(tmem + COL_R + 128u * (i & 1), cc, L.cc_lo, b1 + bs.slot * 2 * B1_BYTES);
          commit(s1done + 8 * (i & 1));
          commit(bfree + 8 * bs.slot);
          issued = true;
          bs.next(nb1);
        }
        if (i >= 1) {
          const int j = i - 1;
          ok = wait_bar(conv + 8 * (j & 1), (uint32_t)((j >> 1) & 1));
          if (ok && j >= 1) ok = wait_bar(d2free, (uint32_t)((j - 1) & 1));
          if (!ok) break;
          fence_after();
          issue_stage2(tmem, COL_R + 128u * (j & 1), cr3);
          commit(s2done);
        }
      }
      if (!ok) atomicExch(&g_device_status, 1);
      if (!cok) wait_bar(cbar, 0);   // the constant copies land before shared memory is released
      if (issued) {                  // every MMA issued has finished before tensor and shared memory are released
        commit(fin);
        wait_bar(fin, 0);
      }
    }
  } else if (warp >= 8) {
    // ---- build warps: their share of B1 of field i >= nb1 into slot i mod nb1 once S1(i - nb1) has read it; the
    // first CTA of an image zero-fills the partial slots of that image that no CTA owns
    const int bt = tid - 256;
    TaskPos p;
    p.init(a, t0);
    Ring bs{0, 0};
    bool ok = true;
    for (int i = 0; i < n; ++i) {
      if (i >= nb1) {
        ok = warp_wait(bfree + 8 * bs.slot, bs.phase ^ 1u);
        if (!ok) break;
        build_share(field_src(a, p), a.br, a.bc, b1 + bs.slot * 2 * B1_BYTES, tid);
        fence_async_smem();
        __syncwarp();
        if (lane == 0) arrive(bfull + 8 * bs.slot);
      }
      if (p.first()) {
        const long long q = p.q;
        const long long first = cta_of(q * F, a.tasks, G), last = cta_of(q * F + F - 1, a.tasks, G);
        for (long long slot = last - first + 1; slot < a.nparts; ++slot) {
          float* out = a.coarse + (slot * a.images + q) * (long long)(MR * MC);
          for (int e = bt; e < MR * MC / 4; e += 32 * NBUILD) ((float4*)out)[e] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
      }
      bs.next(nb1);
      p.next(a);
    }
    if (!ok && lane == 0) atomicExch(&g_device_status, 1);
  } else {
    // ---- tensor-memory warps: convert(i), their share of B1 of field i + nb1 (its slot was read by S1(i)), then
    // w |E|^2 of field i-1; a finished image's partial sum is stored
    const uint32_t taddr = tmem + ((uint32_t)(32 * (warp & 3)) << 16);   // this warp's lane quarter
    const int half = warp >> 2;                                           // column half this warp handles
    const int sc = 32 * (warp & 3) + lane;                                // coarse column = accumulator row
    float acc[64];
#pragma unroll
    for (int j = 0; j < 64; ++j) acc[j] = 0.f;
    TaskPos pj, pb;   // field j = i - 1, field i + nb1
    pj.init(a, t0);
    pb = pj;
    for (int f = 0; f < nb1; ++f) pb.next(a);
    bool ok = true;
    for (int i = 0; i <= n; ++i) {
      if (i < n) {
        ok = warp_wait(s1done + 8 * (i & 1), (uint32_t)((i >> 1) & 1));
        if (!ok) break;
        fence_after();
        convert(taddr, COL_R + 128u * (i & 1), half);
        fence_before();
        __syncwarp();
        if (lane == 0) arrive(conv + 8 * (i & 1));
        if (i + nb1 < n) {
          const int slot = i % nb1;
          build_share(field_src(a, pb), a.br, a.bc, b1 + slot * 2 * B1_BYTES, tid);
          fence_async_smem();
          __syncwarp();
          if (lane == 0) arrive(bfull + 8 * slot);
          pb.next(a);
        }
      }
      if (i >= 1) {
        const int j = i - 1;
        ok = warp_wait(s2done, (uint32_t)(j & 1));
        if (!ok) break;
        fence_after();
        accumulate(acc, taddr, half, __ldg(a.weight + (long long)pj.z * a.nk + pj.k));
        fence_before();
        __syncwarp();
        if (lane == 0) arrive(d2free);
        const long long q = pj.q;
        pj.next(a);
        if (j == n - 1 || pj.first()) {   // field j was the last of image q in this range
          const long long slot = blockIdx.x - cta_of(q * F, a.tasks, G);
          float* out = a.coarse + (slot * a.images + q) * (long long)(MR * MC) + sc;
#pragma unroll
          for (int jj = 0; jj < 64; ++jj) {
            out[(64 * half + jj) * MC] = acc[jj];
            acc[jj] = 0.f;
          }
        }
      }
    }
    if (!ok && lane == 0) atomicExch(&g_device_status, 1);
  }
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    tmem_dealloc(tmem, NCOLS);
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
  const tc::Layout L = tc::make_layout(m0r == m0c);
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
