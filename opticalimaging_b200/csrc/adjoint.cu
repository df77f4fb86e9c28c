// Adjoint of the coherent sum, for inverse lithography (gradients of a loss L through the aerial image).
//
// Forward (coherent_fft.cu):  I(r) = sum_f w_f |E_f(r)|^2,  E_f(r) = sum_{m in band} A_f(m) exp(-2 pi i m.r/N),
// A_f = P_k .* c, c(m) = 1/(Ny Nx) sum_y t(y) exp(+2 pi i m.y/N).  Given g = dL/dI (real, Ny x Nx):
//   dL/dt(y) = 2/(Ny Nx) Re sum_{m in band} W(m) exp(-2 pi i m.y/N),   W(m) = sum_f w_f conj(P_f(m)) F_f(m),
//   F_f(m)   = sum_r g(r) E_f(r) exp(+2 pi i m.r/N).
// F_f is evaluated exactly on the coarse grid: with g^c(s) = 1/(Mr Mc) sum_{|q|<B} ghat(q) exp(-2 pi i q.s/M)
// (the band-limited coarse copy of g, ghat(q) = sum_r g(r) exp(+2 pi i q.r/N)),
//   F_f(m) = sum_s g^c(s) E_f^c(s) exp(+2 pi i m.s/M)      for M >= 2B - 1 (no alias of m - m' reaches the band).
// The same coarse quantities give <g, |E_f|^2> = sum_s g^c(s) |E_f^c(s)|^2, the per-field dot products from
// which the source-weight gradient of the Abbe image follows (dI/dw_j = (n I_j - I) / sum w).
//
// One block per (field split, plane, image): for each of its fields it recomputes E^c (row and column inverse
// FFTs, as the forward kernel), multiplies by g^c, and takes the product back to the band with two direct DFTs
// (column then row; the band is small), accumulating W in registers.  Nothing per field reaches global memory.
#include "fft_common.cuh"

namespace oi {

using cg::brev5;
using cg::gather_ifft;

constexpr int ADJ_T = 512;
constexpr int ADJ_RB = 16;  // band-rows x columns tasks per thread in the column DFT: br * MC <= 16 * 512

struct AdjointArgs {
  const float2* band;       // [batch][nch][br][bc]
  long long band_img_stride;
  int nch, br, bc, m0r, m0c;
  const float2* pupil;      // [nz][nk][br][bc]
  const float* weight;      // [nz][nk]
  const float* gcoarse;     // [batch][nz][mr][mc]
  int nz, nk, nsplit;
  const float2* wr;         // exp(+2 pi i j / mr)
  const float2* wc;         // exp(+2 pi i j / mc)
  float2* wout;             // [nsplit][batch][nz][nch][br][bc]
  float* field_dot;         // [batch][nz][nk*nch] or null
};

template <int N1R, int N1C>
__global__ void __launch_bounds__(ADJ_T) coherent_adjoint_kernel(AdjointArgs a) {
  constexpr int MR = 32 * N1R, MC = 32 * N1C, T = ADJ_T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* wr = (float2*)smem_raw;            // [MR]
  float2* wc = wr + MR;                      // [MC]
  float2* as = wc + MC;                      // [br][bc]
  float2* x = as + a.br * a.bc;              // [MR][MC + 1]
  float* red = (float*)(x + MR * (MC + 1));  // [T / 32] block reduction scratch
  const int tid = threadIdx.x;
  const int split = blockIdx.x, z = blockIdx.y;
  const long long b = blockIdx.z;
  for (int j = tid; j < MR; j += T) wr[j] = a.wr[j];
  for (int j = tid; j < MC; j += T) wc[j] = a.wc[j];
  const int br = a.br, bc = a.bc, plane = br * bc;
  const float* gc = a.gcoarse + ((b * a.nz + z) * (long long)MR) * MC;
  const int nfield = a.nk * a.nch;
  const float2* pup = a.pupil + (long long)z * a.nk * plane;
  // band accumulators W[ir][ic] for the fixed task set e = tid + T j, one per channel in turn
  constexpr int NW = 8;   // plane <= NW * T (checked on the host)
  const int sc = tid % MC, n1r = tid / MC;  // column task of the inverse column pass (T = MC * N1R)
  for (int c = 0; c < a.nch; ++c) {
    float2 wacc[NW];
#pragma unroll
    for (int j = 0; j < NW; ++j) wacc[j] = make_float2(0.f, 0.f);
    for (int f = split; f < nfield; f += a.nsplit) {
      if (f % a.nch != c) continue;
      const int k = f / a.nch;
      const float w = __ldg(a.weight + (long long)z * a.nk + k);
      const float2* pk = pup + (long long)k * plane;
      const float2* hc = a.band + b * a.band_img_stride + (long long)c * plane;
      __syncthreads();
      for (int e = tid; e < plane; e += T) as[e] = cmul(__ldg(pk + e), __ldg(hc + e));
      __syncthreads();
      // E^c: row inverse FFTs of the band rows into x[0..br), then column inverse FFTs
      for (int task = tid; task < br * N1C; task += T) {
        const int ir = task / N1C, n1 = task % N1C;
        float2 zr[32];
        gather_ifft<N1C>(zr, as + ir * bc, 1, a.m0c, bc, wc, n1);
#pragma unroll
        for (int i = 0; i < 32; ++i) x[ir * (MC + 1) + n1 + N1C * brev5(i)] = zr[i];
      }
      __syncthreads();
      float2 zc[32];
      gather_ifft<N1R>(zc, x + sc, MC + 1, a.m0r, br, wr, n1r);
      __syncthreads();  // every column task has read its band rows: x may now hold Y = g^c E^c
      float dot = 0.f;
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const int sr = n1r + N1R * brev5(i);
        const float g = __ldg(gc + sr * MC + sc);
        dot = fmaf(g, fmaf(zc[i].x, zc[i].x, zc[i].y * zc[i].y), dot);
        x[sr * (MC + 1) + sc] = make_float2(g * zc[i].x, g * zc[i].y);
      }
      if (a.field_dot) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
        if ((tid & 31) == 0) red[tid >> 5] = dot;
      }
      __syncthreads();
      if (a.field_dot && tid < 32) {
        float v = tid < T / 32 ? red[tid] : 0.f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (tid == 0) a.field_dot[(b * a.nz + z) * (long long)nfield + f] = v;
      }
      // column DFT back to the band rows: F1[ir][sc] = sum_sr Y[sr][sc] exp(+2 pi i (m0r+ir) sr / MR)
      float2 f1[ADJ_RB];
#pragma unroll
      for (int j = 0; j < ADJ_RB; ++j) {
        const int e = tid + T * j;
        float2 acc = make_float2(0.f, 0.f);
        if (e < br * MC) {
          const int ir = e / MC, col = e % MC, m = a.m0r + ir;
          for (int sr = 0; sr < MR; ++sr) cfma(acc, x[sr * (MC + 1) + col], wr[(m * sr) & (MR - 1)]);
        }
        f1[j] = acc;
      }
      __syncthreads();
#pragma unroll
      for (int j = 0; j < ADJ_RB; ++j) {
        const int e = tid + T * j;
        if (e < br * MC) x[(e / MC) * (MC + 1) + e % MC] = f1[j];
      }
      __syncthreads();
      // row DFT back to the band columns and accumulation W += w conj(P) F
#pragma unroll
      for (int j = 0; j < NW; ++j) {
        const int e = tid + T * j;
        if (e < plane) {
          const int ir = e / bc, ic = e % bc, m = a.m0c + ic;
          float2 acc = make_float2(0.f, 0.f);
          const float2* row = x + ir * (MC + 1);
          for (int s = 0; s < MC; ++s) cfma(acc, row[s], wc[(m * s) & (MC - 1)]);
          const float2 p = __ldg(pk + e);
          const float2 cp = make_float2(w * p.x, -w * p.y);
          cfma(wacc[j], cp, acc);
        }
      }
    }
    float2* out = a.wout + ((((long long)split * gridDim.z + b) * a.nz + z) * a.nch + c) * plane;
#pragma unroll
    for (int j = 0; j < NW; ++j) {
      const int e = tid + T * j;
      if (e < plane) out[e] = wacc[j];
    }
  }
}

template <int N1R, int N1C>
static int launch_adjoint(const AdjointArgs& a, int batch, cudaStream_t s) {
  constexpr int MR = 32 * N1R, MC = 32 * N1C;
  static_assert(MC * N1R == ADJ_T, "one inverse column task per thread");
  size_t smem = sizeof(float2) * ((size_t)MR + MC + (size_t)a.br * a.bc + (size_t)MR * (MC + 1)) +
                sizeof(float) * (ADJ_T / 32);
  auto kern = coherent_adjoint_kernel<N1R, N1C>;
  int rc = ensure_smem((const void*)kern, smem, "oi_coherent_adjoint");
  if (rc) return rc;
  dim3 grid((unsigned)a.nsplit, (unsigned)a.nz, (unsigned)batch);
  kern<<<grid, ADJ_T, smem, s>>>(a);
  oi::note_launch();
  return check_launch("oi_coherent_adjoint");
}

}  // namespace oi

extern "C" int oi_coherent_adjoint(const void* band, int batch, int nch, int m0r, int br, int m0c, int bc,
                                   const void* pupil, const float* weight, int nz, int nk, const float* gcoarse,
                                   int mr, int mc, const void* wr, const void* wc, int nsplit, void* wout,
                                   float* field_dot, void* stream) {
  using namespace oi;
  if (!band || !pupil || !weight || !gcoarse || !wr || !wc || !wout || batch <= 0 || nch <= 0 || br <= 0 ||
      bc <= 0 || nz <= 0 || nk <= 0 || nsplit <= 0)
    return fail(OI_EINVAL, "oi_coherent_adjoint: bad arguments");
  if (!(mr == 128 && mc == 128) || 2 * br - 1 > mr || 2 * bc - 1 > mc || br * bc > 8 * ADJ_T ||
      br * mc > ADJ_RB * ADJ_T || nsplit > nk * nch || batch > 65535 || nz > 65535)
    return fail(OI_ERANGE, "oi_coherent_adjoint: coarse %dx%d / band %dx%d / split %d unsupported (coarse grid "
                "must be 128x128, band at most 64x64)", mr, mc, br, bc, nsplit);
  AdjointArgs a{(const float2*)band, (long long)nch * br * bc, nch, br, bc, m0r, m0c, (const float2*)pupil, weight,
                gcoarse, nz, nk, nsplit, (const float2*)wr, (const float2*)wc, (float2*)wout, field_dot};
  return launch_adjoint<4, 4>(a, batch, (cudaStream_t)stream);
}
