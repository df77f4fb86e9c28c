// FFT form of the coherent sum on the coarse grid (the |fft2(.)|^2 accumulation of CalculateAbbeImage,
// CalculateAerialImage.py:76-92, and of CalculateAerialImage_SOCS, CalculateAerialImage_SOCS.py:5-10), for
// coarse grids of 64 or 128 per axis.
//
// For one (image b, plane z, subset of fields), each field A = P[z][k] .* band[b][c] (Br x Bc, on the band)
// is taken to the Mr x Mc coarse grid by a 2-D inverse transform
//   E[sr][sc] = sum_{ir,ic} A[ir][ic] exp(-2 pi i ((m0r+ir) sr/Mr + (m0c+ic) sc/Mc))
// done as Br pruned row FFTs (Mc points, only Bc inputs non-zero) into shared memory, then Mc pruned column
// FFTs (Mr points, only Br inputs non-zero).  Each thread owns one column task (sc, n1) for the whole field
// loop and accumulates w |E|^2 of its 32 outputs in registers, so E never leaves the SM.  Every FFT is the
// four-step 32 x N1 form of fft.cu (32-point transform in registers).
//
// Fields of one (b, z) are split over `nsplit` blocks; block s writes its partial sum to
// coarse[s][b][z][sr][sc] and the coarse-spectrum stage adds the partials (a fixed order: deterministic).
#include "fft_common.cuh"

namespace oi {

using cg::brev5;
using cg::gather_ifft;

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
  if ((mr != 64 && mr != 128) || (mc != 64 && mc != 128) || 2 * br - 1 > mr || 2 * bc - 1 > mc ||
      nz > 65535 || batch > 65535 || nsplit > nk * nch)
    return fail(OI_ERANGE, "oi_coherent_coarse_fft: coarse %dx%d / band %dx%d / split %d unsupported", mr, mc, br, bc,
                nsplit);
  CoherentFftArgs a{(const float2*)band, (long long)nch * br * bc, nch, br, bc, m0r, m0c, (const float2*)pupil,
                    pupil_batch_stride, weight, nz, nk, nsplit, (const float2*)wr, (const float2*)wc, coarse,
                    (long long)batch * nz * mr * mc};
  cudaStream_t s = (cudaStream_t)stream;
  if (mr == 128 && mc == 128) return launch_cfft<4, 4>(a, batch, s);
  if (mr == 64 && mc == 64) return launch_cfft<2, 2>(a, batch, s);
  if (mr == 128) return launch_cfft<4, 2>(a, batch, s);
  return launch_cfft<2, 4>(a, batch, s);
}
