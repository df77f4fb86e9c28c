// FFT form of the coherent sum on the coarse grid (the |fft2(.)|^2 accumulation of CalculateAbbeImage,
// CalculateAerialImage.py:76-92, and of CalculateAerialImage_SOCS, CalculateAerialImage_SOCS.py:5-10), for
// coarse grids of 64 or 128 per axis and of 256 x 256.
//
// For one (image b, plane z, subset of fields), each field A = P[z][k] .* band[b][c] (Br x Bc, on the band)
// is taken to the Mr x Mc coarse grid by a 2-D inverse transform
//   E[sr][sc] = sum_{ir,ic} A[ir][ic] exp(-2 pi i ((m0r+ir) sr/Mr + (m0c+ic) sc/Mc))
// done as Br pruned row FFTs (Mc points, only Bc inputs non-zero) into shared memory, then Mc pruned column
// FFTs (Mr points, only Br inputs non-zero).  Each thread owns one column task (sc, n1) for the whole field
// loop and accumulates w |E|^2 of its 32 outputs in registers, so E never leaves the SM.  Every FFT is the
// four-step 32 x N1 form of fft.cu (32-point transform in registers).  A 256 x 256 coarse grid (bands of 65 to
// 128) has its own kernel, coherent_fft256_kernel, whose accumulator lives in tensor memory.
//
// Fields of one (b, z) are split over `nsplit` blocks; block s writes its partial sum to
// coarse[s][b][z][sr][sc] and the coarse-spectrum stage adds the partials (a fixed order: deterministic).
#include "fft_common.cuh"
#include "tc_common.cuh"

namespace oi {

using cg::brev5;
using cg::gather_ifft;
using cg::ifft32;

struct CoherentFftArgs {
  const float2* band;
  long long band_img_stride;
  int nch, br, bc, m0r, m0c;
  const float2* pupil;
  long long pupil_batch_stride;
  const float* weight;
  int nz, nk, nsplit;
  const float2* wr;  // exp(+2 pi i j / mr), j < mr
  const float2* wc;  // exp(+2 pi i j / mc), j < mc
  float* coarse;     // [nsplit][batch][nz][mr][mc]
  long long split_stride;
};

// grid (nsplit, nz, batch); block = mc * N1R threads (column tasks); mr = 32 N1R, mc = 32 N1C.
template <int N1R, int N1C>
__global__ void __launch_bounds__(32 * N1C * N1R) coherent_fft_kernel(CoherentFftArgs a) {
  constexpr int MR = 32 * N1R, MC = 32 * N1C, T = MC * N1R;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* wr = (float2*)smem_raw;   // [MR]
  float2* wc = wr + MR;             // [MC]
  float2* as = wc + MC;             // [br][bc]
  float2* e1 = as + a.br * a.bc;    // [br][MC + 1] (padded against bank conflicts)
  const int tid = threadIdx.x;
  const int split = blockIdx.x, z = blockIdx.y;
  const long long b = blockIdx.z;
  for (int j = tid; j < MR; j += T) wr[j] = a.wr[j];
  for (int j = tid; j < MC; j += T) wc[j] = a.wc[j];
  const int sc = tid % MC, n1r = tid / MC;  // column task of this thread
  float acc[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) acc[i] = 0.f;
  const int nfield = a.nk * a.nch;
  const long long plane = (long long)a.br * a.bc;
  const float2* pup = a.pupil + b * a.pupil_batch_stride + (long long)z * a.nk * plane;
  for (int f = split; f < nfield; f += a.nsplit) {
    const int k = f / a.nch, c = f % a.nch;
    const float w = __ldg(a.weight + (long long)z * a.nk + k);
    const float2* pk = pup + (long long)k * plane;
    const float2* hc = a.band + b * a.band_img_stride + (long long)c * plane;
    __syncthreads();  // previous field's readers are done with as / e1; tables are loaded
    for (long long e = tid; e < plane; e += T) as[e] = cmul(__ldg(pk + e), __ldg(hc + e));
    __syncthreads();
    // row pass: br rows x N1C tasks, Mc-point transforms of the bc band columns
    for (int task = tid; task < a.br * N1C; task += T) {
      const int ir = task / N1C, n1 = task % N1C;
      float2 zr[32];
      gather_ifft<N1C>(zr, as + ir * a.bc, 1, a.m0c, a.bc, wc, n1);
#pragma unroll
      for (int i = 0; i < 32; ++i) e1[ir * (MC + 1) + n1 + N1C * brev5(i)] = zr[i];
    }
    __syncthreads();
    // column pass: thread (sc, n1r), Mr-point transform of the br band rows of column sc
    float2 zc[32];
    gather_ifft<N1R>(zc, e1 + sc, MC + 1, a.m0r, a.br, wr, n1r);
#pragma unroll
    for (int i = 0; i < 32; ++i) acc[i] = fmaf(w, fmaf(zc[i].x, zc[i].x, zc[i].y * zc[i].y), acc[i]);
  }
  float* out = a.coarse + split * a.split_stride + ((b * a.nz + z) * (long long)MR) * MC;
#pragma unroll
  for (int i = 0; i < 32; ++i) out[(n1r + N1R * brev5(i)) * MC + sc] = acc[i];
}

// ---- 256 x 256 coarse grid (bands of 65..128 per axis): the |E|^2 accumulator in tensor memory.
//
// 65,536 accumulators do not fit in the registers of one CTA, but they are exactly the 128 lanes x 512 columns
// of 32 bits of tensor memory.  One CTA of 512 threads per (split, z, b) holds all 512 columns (one CTA per SM).
// The band offsets only turn the phase of E: E[sr][sc] = exp(-2 pi i (m0r sr + m0c sc) / 256) E0[sr][sc], E0 the
// 256 x 256 transform of A = P .* band placed at the origin, so |E|^2 = |E0|^2 and the kernel transforms E0.
// Per field, in two halves h of the columns (sc mod 8 in 4h .. 4h+3), with 256 = 32 x 8 four-step transforms:
//   row pass     task (ir, n1) for ir < br and the half's 4 values of n1: the transform of band row ir of A
//                (products formed as the row is read from global memory), keeping its outputs
//                sc = n1 + 8 brev5(i), i < 32, at e1[ir][lc], lc = (n1 - 4h) + 4 brev5(i);
//   column pass  task (lc, n1r), 128 x 8 tasks, two per thread: the transform of column lc of e1 (rows br..127
//                stay zero), giving E0[n1r + 8 brev5(i)][sc(lc)], i < 32, and w |E0|^2 accumulated into
//                tensor-memory lane lc, columns (8h + n1r) 32 + i.
// Warp w may only address the lanes 32 (w % 4) .. + 31 of tensor memory, so thread (w, lane) takes the tasks
// lc = 32 (w % 4) + lane, n1r = w / 4 + 4r (r = 0, 1): every (lane, column) has one owner, and the accumulator
// needs no synchronisation beyond the thread's own store -> load ordering (tcgen05.wait::st).
constexpr int F256_T = 512;
constexpr int F256_S = 132;          // e1 row stride in float2: 4 (mod 16) keeps the row pass's stores conflict-free
constexpr size_t F256_MIN_SMEM = 120832;   // above half an SM's shared memory: one CTA per SM

// Four-step gather of the 256-point transform of x[0..b) (b <= 128, zero beyond):
//   z[t] = W^{t n1} sum_{s < 4} x[t + 32 s] V^{s n1},  W = exp(-2 pi i / 256), V = exp(-2 pi i / 8),
// then the 32-point transform: on return z[i] = X[n1 + 8 brev5(i)], X[s] = sum_j x[j] exp(-2 pi i j s / 256).
// tw8[s][n1] = V^{s n1} (s < 4), tw256[t][n1] = W^{t n1}.  PROD: x[j] = src[j] * src2[j] (global memory), else
// x[j] = src[j * stride] (shared memory).  FULL: x is stored up to 128 (no bound checks).
template <bool PROD, bool FULL>
__device__ __forceinline__ void gather256(float2 (&z)[32], const float2* src, const float2* src2, int stride, int b,
                                          const float2* tw8, const float2* tw256, int n1) {
  const float2 v1 = tw8[8 + n1], v2 = tw8[16 + n1], v3 = tw8[24 + n1];
  auto x = [&](int j) { return PROD ? cmul(__ldg(src + j), __ldg(src2 + j)) : src[j * stride]; };
#pragma unroll
  for (int t = 0; t < 32; ++t) {
    float2 acc = (FULL || t < b) ? x(t) : make_float2(0.f, 0.f);
    if (FULL || t + 32 < b) cfma(acc, x(t + 32), v1);
    if (FULL || t + 64 < b) cfma(acc, x(t + 64), v2);
    if (FULL || t + 96 < b) cfma(acc, x(t + 96), v3);
    z[t] = t == 0 ? acc : cmul(acc, tw256[t * 8 + n1]);
  }
  ifft32(z);
}

__global__ void __launch_bounds__(F256_T, 1) coherent_fft256_kernel(CoherentFftArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* tw8 = (float2*)smem_raw;                 // [4][8]
  float2* tw256 = tw8 + 32;                        // [32][8]
  uint32_t* slot = (uint32_t*)(tw256 + 256);       // tensor-memory base address (16 bytes reserved)
  float2* e1 = tw256 + 258;                        // [128][F256_S]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int split = blockIdx.x, z = blockIdx.y;
  const long long b = blockIdx.z;
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(slot), 512);
  for (int j = tid; j < 32 + 256; j += F256_T) {   // tw8 then tw256, contiguous; a.wr[j] = exp(+2 pi i j / 256)
    const int n1 = j & 7, k = (j < 32 ? j : j - 32) >> 3;
    const float2 t = __ldg(a.wr + ((j < 32 ? 32 * k * n1 : k * n1) & 255));
    tw8[j] = make_float2(t.x, -t.y);
  }
  const int br = a.br, bc = a.bc;
  for (int j = br * F256_S + tid; j < 128 * F256_S; j += F256_T) e1[j] = make_float2(0.f, 0.f);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem_q = *slot + ((uint32_t)(32 * (warp & 3)) << 16);   // this warp's lane quarter
  const int ir = tid >> 2, n1l = tid & 3;          // row task
  const int lc = 32 * (warp & 3) + lane;           // column task
  const int nfield = a.nk * a.nch;
  const long long plane = (long long)br * bc;
  const float2* pup = a.pupil + b * a.pupil_batch_stride + (long long)z * a.nk * plane;
  bool first = true;
  for (int f = split; f < nfield; f += a.nsplit) {
    const int k = f / a.nch, c = f - k * a.nch;
    const float w = __ldg(a.weight + (long long)z * a.nk + k);
    const float2* pk = pup + (long long)k * plane;
    const float2* hc = a.band + b * a.band_img_stride + (long long)c * plane;
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
      if (ir < br) {
        float2 zr[32];
        gather256<true, false>(zr, pk + (long long)ir * bc, hc + (long long)ir * bc, 1, bc, tw8, tw256, 4 * h + n1l);
#pragma unroll
        for (int i = 0; i < 32; ++i) e1[ir * F256_S + n1l + 4 * brev5(i)] = zr[i];
      }
      __syncthreads();
#pragma unroll 1
      for (int r = 0; r < 2; ++r) {
        const int n1r = (warp >> 2) + 4 * r;
        float2 zc[32];
        gather256<false, true>(zc, e1 + lc, nullptr, F256_S, 128, tw8, tw256, n1r);
        const uint32_t ta = tmem_q + (uint32_t)((8 * h + n1r) * 32);
        uint32_t v[32];
        if (first) {
#pragma unroll
          for (int i = 0; i < 32; ++i) v[i] = __float_as_uint(w * fmaf(zc[i].x, zc[i].x, zc[i].y * zc[i].y));
        } else {
          float acc[32];
          tc::wait_st();
          tc::tmem_ld32(ta, acc);
#pragma unroll
          for (int i = 0; i < 32; ++i) v[i] = __float_as_uint(fmaf(w, fmaf(zc[i].x, zc[i].x, zc[i].y * zc[i].y), acc[i]));
        }
        tc::tmem_st32(ta, v);
      }
      __syncthreads();   // the next row pass overwrites e1
    }
    first = false;
  }
  tc::wait_st();
  float* out = a.coarse + split * a.split_stride + (b * a.nz + z) * 65536LL;
#pragma unroll 1
  for (int h = 0; h < 2; ++h) {
    const int sc = 4 * h + (lc & 3) + 8 * (lc >> 2);
#pragma unroll 1
    for (int r = 0; r < 2; ++r) {
      const int n1r = (warp >> 2) + 4 * r;
      float acc[32];
      tc::tmem_ld32(tmem_q + (uint32_t)((8 * h + n1r) * 32), acc);
#pragma unroll
      for (int i = 0; i < 32; ++i) out[(n1r + 8 * brev5(i)) * 256 + sc] = acc[i];
    }
  }
  tc::fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after();
    tc::tmem_dealloc(*slot, 512);
  }
}

static int launch_cfft256(const CoherentFftArgs& a, int batch, cudaStream_t s) {
  size_t smem = sizeof(float2) * (32 + 256 + 2 + 128 * F256_S);
  if (smem < F256_MIN_SMEM) smem = F256_MIN_SMEM;
  {
    int rc_smem = ensure_smem((const void*)coherent_fft256_kernel, smem, "oi_coherent_coarse_fft");
    if (rc_smem) return rc_smem;
  }
  dim3 grid((unsigned)a.nsplit, (unsigned)a.nz, (unsigned)batch);
  coherent_fft256_kernel<<<grid, F256_T, smem, s>>>(a);
  oi::note_launch();
  return check_launch("oi_coherent_coarse_fft");
}

template <int N1R, int N1C>
static int launch_cfft(const CoherentFftArgs& a, int batch, cudaStream_t s) {
  constexpr int MR = 32 * N1R, MC = 32 * N1C, T = MC * N1R;
  size_t smem = sizeof(float2) * ((size_t)MR + MC + (size_t)a.br * a.bc + (size_t)a.br * (MC + 1));
  auto kern = coherent_fft_kernel<N1R, N1C>;
  {
    int rc_smem = ensure_smem((const void*)kern, smem, "oi_coherent_coarse_fft");
    if (rc_smem) return rc_smem;
  }
  dim3 grid((unsigned)a.nsplit, (unsigned)a.nz, (unsigned)batch);
  kern<<<grid, T, smem, s>>>(a);
  oi::note_launch();
  return check_launch("oi_coherent_coarse_fft");
}

}  // namespace oi

extern "C" int oi_coherent_coarse_fft(const void* band, int batch, int nch, int m0r, int br, int m0c, int bc,
                                      const void* pupil, long long pupil_batch_stride, const float* weight, int nz,
                                      int nk, int mr, int mc, const void* wr, const void* wc, int nsplit,
                                      float* coarse, void* stream) {
  using namespace oi;
  if (!band || !pupil || !weight || !wr || !wc || !coarse || batch <= 0 || nch <= 0 || br <= 0 || bc <= 0 ||
      nz <= 0 || nk <= 0 || nsplit <= 0 || pupil_batch_stride < 0)
    return fail(OI_EINVAL, "oi_coherent_coarse_fft: bad arguments");
  const bool big = mr == 256 && mc == 256;
  if ((!big && ((mr != 64 && mr != 128) || (mc != 64 && mc != 128))) || 2 * br - 1 > mr || 2 * bc - 1 > mc ||
      nz > 65535 || batch > 65535 || nsplit > nk * nch)
    return fail(OI_ERANGE, "oi_coherent_coarse_fft: coarse %dx%d / band %dx%d / split %d unsupported", mr, mc, br, bc,
                nsplit);
  CoherentFftArgs a{(const float2*)band, (long long)nch * br * bc, nch, br, bc, m0r, m0c, (const float2*)pupil,
                    pupil_batch_stride, weight, nz, nk, nsplit, (const float2*)wr, (const float2*)wc, coarse,
                    (long long)batch * nz * mr * mc};
  cudaStream_t s = (cudaStream_t)stream;
  if (big) return launch_cfft256(a, batch, s);
  if (mr == 128 && mc == 128) return launch_cfft<4, 4>(a, batch, s);
  if (mr == 64 && mc == 64) return launch_cfft<2, 2>(a, batch, s);
  if (mr == 128) return launch_cfft<4, 2>(a, batch, s);
  return launch_cfft<2, 4>(a, batch, s);
}
