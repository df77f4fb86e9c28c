// FP64 TCC assembly: TCC = sum_e h_e h_e^H with h[e][p][j] the weighted shifted pupils (GetTCCMatrix,
// CalculateTCCMatrix.py:58-75, with the diagonal source-weight matrix folded into h as sqrt(w)).
// The TCC is Hermitian: only lower-triangle 64x64 tiles are computed; each off-diagonal tile is written
// twice, once as is and once conjugate-transposed.
#include "oi_common.cuh"

namespace oi {

constexpr int TC_T = 64, TC_K = 16;

__global__ void __launch_bounds__(256) tcc_assemble_kernel(const double2* __restrict__ h, int ne, int fg, int nsrc,
                                                           double2* __restrict__ tcc) {
  __shared__ double2 as[TC_K][TC_T + 1];
  __shared__ double2 bs[TC_K][TC_T + 1];
  // lower-triangle tile index -> (tp, tq), tp >= tq
  long long t = blockIdx.x;
  int tp = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) / 2.0);
  while ((long long)tp * (tp + 1) / 2 > t) --tp;
  while ((long long)(tp + 1) * (tp + 2) / 2 <= t) ++tp;
  int tq = (int)(t - (long long)tp * (tp + 1) / 2);
  const int p0 = tp * TC_T, q0 = tq * TC_T;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0.0, 0.0);
  const long long plane = (long long)fg * nsrc;
  for (int e = 0; e < ne; ++e) {
    const double2* he = h + e * plane;
    for (int j0 = 0; j0 < nsrc; j0 += TC_K) {
#pragma unroll
      for (int i = 0; i < (TC_K * TC_T) / 256; ++i) {
        int idx = tid + 256 * i, r = idx / TC_K, kk = idx % TC_K;
        int j = j0 + kk, p = p0 + r, q = q0 + r;
        as[kk][r] = (j < nsrc && p < fg) ? he[(long long)p * nsrc + j] : make_double2(0.0, 0.0);
        bs[kk][r] = (j < nsrc && q < fg) ? he[(long long)q * nsrc + j] : make_double2(0.0, 0.0);
      }
      __syncthreads();
#pragma unroll 4
      for (int kk = 0; kk < TC_K; ++kk) {
        double2 a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = as[kk][ty * 4 + i];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = bs[kk][tx * 4 + j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) cfma_conj(acc[i][j], a[i], b[j]);
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int p = p0 + ty * 4 + i;
    if (p >= fg) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int q = q0 + tx * 4 + j;
      if (q >= fg) continue;
      tcc[(long long)p * fg + q] = acc[i][j];
      if (tp != tq) tcc[(long long)q * fg + p] = make_double2(acc[i][j].x, -acc[i][j].y);
    }
  }
}

}  // namespace oi

extern "C" int oi_tcc_assemble64(const void* h, int ne, int fg, int nsrc, void* tcc, void* stream) {
  using namespace oi;
  if (!h || !tcc || (ne != 1 && ne != 3) || fg <= 0 || nsrc <= 0)
    return fail(OI_EINVAL, "oi_tcc_assemble64: bad arguments (ne=%d fg=%d nsrc=%d)", ne, fg, nsrc);
  long long nt = ceil_div(fg, TC_T);
  long long tiles = nt * (nt + 1) / 2;
  if (tiles > 0x7fffffffLL) return fail(OI_ERANGE, "oi_tcc_assemble64: fg=%d too large", fg);
  tcc_assemble_kernel<<<(unsigned)tiles, 256, 0, (cudaStream_t)stream>>>((const double2*)h, ne, fg, nsrc,
                                                                          (double2*)tcc);
  oi::note_launch();
  return check_launch("oi_tcc_assemble64");
}
