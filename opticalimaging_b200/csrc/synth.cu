// Exact band-limited resampling of the coarse intensity to the output grid: the last step of both imaging
// paths (the fftshift + normalisation of CalculateAerialImage.py:89-92 and CalculateAerialImage_SOCS.py:10).
//
// The intensity of fields band-limited to Br x Bc has a spectrum supported on |qr| < Br, |qc| < Bc.  Its
// samples on the coarse Mr x Mc grid (Mr >= 2Br-1, Mc >= 2Bc-1) determine that spectrum exactly:
//   Ihat(q) = 1/(Mr Mc) sum_s coarse[s] exp(+2 pi i (qr sr/Mr + qc sc/Mc))             (spec kernel)
// (the coarse intensity may arrive as `nparts` partial sums laid out one after another; they are added here)
// and the output is its trigonometric polynomial evaluated on the Ny x Nx grid.  The intensity is real, so
// only qc >= 0 is kept (qc > 0 doubled) and the x synthesis is a real dot product:
//   V[y][qc]   = sum_qr Ihat(qr, qc) exp(-2 pi i qr y/Ny)
//   out[y][x]  = sum_qc Re(V[y][qc] exp(-2 pi i qc x/Nx))                                 (synth kernel)
#include "oi_common.cuh"

namespace oi {

constexpr int SP_QT = 16;  // qc per spec block

// grid (ceil(bc/16), count).  ihat[i][jr][qc], jr = qr + br - 1.
__global__ void __launch_bounds__(256) coarse_spec_kernel(const float* __restrict__ coarse, int nparts,
                                                          long long part_stride, int mr, int mc, int br,
                                                          int bc, const float2* __restrict__ gc,
                                                          const float2* __restrict__ gr, float2* __restrict__ ihat) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* us = (float2*)smem_raw;  // [mr][SP_QT]
  const int tid = threadIdx.x, ql = tid % SP_QT, rg = tid / SP_QT;  // rg 0..15
  const int qc0 = blockIdx.x * SP_QT;
  const long long img = blockIdx.y;
  const float* cimg = coarse + img * (long long)mr * mc;
  const int qc = qc0 + ql;
  const int nq = 2 * br - 1;
  // U[sr][qc] = sum_sc coarse[sr][sc] gc[sc][qc]
  for (int sr = rg; sr < mr; sr += 16) {
    float2 u = make_float2(0.f, 0.f);
    if (qc < bc) {
      const float* row = cimg + (long long)sr * mc;
      for (int sc = 0; sc < mc; ++sc) {
        float v = __ldg(row + sc);
        for (int p = 1; p < nparts; ++p) v += __ldg(row + p * part_stride + sc);
        float2 t = __ldg(gc + (long long)sc * bc + qc);
        u.x = fmaf(v, t.x, u.x);
        u.y = fmaf(v, t.y, u.y);
      }
    }
    us[sr * SP_QT + ql] = u;
  }
  __syncthreads();
  const float norm = (qc == 0 ? 1.0f : 2.0f) / ((float)mr * (float)mc);
  for (int jr = rg; jr < nq; jr += 16) {
    if (qc >= bc) continue;
    float2 acc = make_float2(0.f, 0.f);
    for (int sr = 0; sr < mr; ++sr) cfma(acc, __ldg(gr + (long long)sr * nq + jr), us[sr * SP_QT + ql]);
    ihat[(img * nq + jr) * (long long)bc + qc] = make_float2(acc.x * norm, acc.y * norm);
  }
}

constexpr int SY_TY = 8;  // output rows per synth block

// grid (ceil(ny/8), count).
template <int NV>
__global__ void __launch_bounds__(256) synth_kernel(const float2* __restrict__ ihat, int br, int bc,
                                                    const float2* __restrict__ sy, const float2* __restrict__ sx,
                                                    int ny, int nx, float* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* vs = (float2*)smem_raw;  // [SY_TY][bc]
  const int tid = threadIdx.x;
  const int y0 = blockIdx.x * SY_TY;
  const long long img = blockIdx.y;
  const int nq = 2 * br - 1;
  const float2* ih = ihat + img * (long long)nq * bc;
  // V[r][qc] = sum_jr sy[y0+r][jr] ihat[jr][qc]
  for (int e = tid; e < SY_TY * bc; e += 256) {
    int r = e / bc, qc = e - r * bc, y = y0 + r;
    float2 acc = make_float2(0.f, 0.f);
    if (y < ny) {
      const float2* srow = sy + (long long)y * nq;
      for (int jr = 0; jr < nq; ++jr) cfma(acc, __ldg(srow + jr), __ldg(ih + (long long)jr * bc + qc));
    }
    vs[e] = acc;
  }
  __syncthreads();
  // out[y][x] = sum_qc (V.re * sx.re - V.im * sx.im)
  float acc[SY_TY][NV];
#pragma unroll
  for (int r = 0; r < SY_TY; ++r)
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[r][v] = 0.f;
  for (int qc = 0; qc < bc; ++qc) {
    float2 t[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      int x = tid + 256 * v;
      t[v] = x < nx ? __ldg(sx + (long long)qc * nx + x) : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int r = 0; r < SY_TY; ++r) {
      float2 vv = vs[r * bc + qc];
#pragma unroll
      for (int v = 0; v < NV; ++v) acc[r][v] = fmaf(vv.x, t[v].x, fmaf(-vv.y, t[v].y, acc[r][v]));
    }
  }
  float* o = out + img * (long long)ny * nx;
#pragma unroll
  for (int r = 0; r < SY_TY; ++r) {
    int y = y0 + r;
    if (y >= ny) continue;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      int x = tid + 256 * v;
      if (x < nx) o[(long long)y * nx + x] = acc[r][v];
    }
  }
}

// part[0][i] += part[1][i] + ... + part[nparts-1][i], in place (float4 lanes; n is a multiple of 4).
__global__ void sum_parts_kernel(float* __restrict__ coarse, int nparts, long long n) {
  long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 4;
  if (i >= n) return;
  float4 acc = *(const float4*)(coarse + i);
  for (int p = 1; p < nparts; ++p) {
    const float4 v = __ldg((const float4*)(coarse + p * n + i));
    acc.x += v.x;
    acc.y += v.y;
    acc.z += v.z;
    acc.w += v.w;
  }
  *(float4*)(coarse + i) = acc;
}

int fold_parts(float* coarse, int nparts, long long n, cudaStream_t s) {
  if (nparts <= 1) return OI_OK;
  if (n % 4 != 0) return fail(OI_EINVAL, "partial sums of %lld floats are not float4 aligned", n);
  sum_parts_kernel<<<(unsigned)ceil_div(n / 4, 256), 256, 0, s>>>(coarse, nparts, n);
  oi::note_launch();
  return check_launch("coarse spectrum/sum parts");
}

int coarse_spectrum(float* coarse, int count, int mr, int mc, int br, int bc, const void* gc, const void* gr,
                    void* ihat, cudaStream_t s, int nparts) {
  if (mr < 2 * br - 1 || mc < 2 * bc - 1)
    return fail(OI_EINVAL, "coarse grid %dx%d too small for band %dx%d", mr, mc, br, bc);
  if (mr > 1024 || count > 65535) return fail(OI_ERANGE, "coarse grid mr=%d or count=%d out of range", mr, count);
  int rc = fold_parts(coarse, nparts, (long long)count * mr * mc, s);
  if (rc) return rc;
  nparts = 1;
  size_t smem = sizeof(float2) * (size_t)mr * SP_QT;
  {
    int rc_smem = ensure_smem((const void*)coarse_spec_kernel, smem, "coarse spectrum");
    if (rc_smem) return rc_smem;
  }
  dim3 g1((unsigned)ceil_div(bc, SP_QT), (unsigned)count);
  coarse_spec_kernel<<<g1, 256, smem, s>>>(coarse, nparts, (long long)count * mr * mc, mr, mc, br, bc,
                                           (const float2*)gc, (const float2*)gr, (float2*)ihat);
  oi::note_launch();
  return check_launch("coarse spectrum");
}

template <int NV>
static void launch_synth(const float2* ihat, int count, int br, int bc, const float2* sy, const float2* sx, int ny,
                         int nx, float* out, cudaStream_t s) {
  dim3 grid((unsigned)ceil_div(ny, SY_TY), (unsigned)count);
  synth_kernel<NV><<<grid, 256, sizeof(float2) * SY_TY * bc, s>>>(ihat, br, bc, sy, sx, ny, nx, out);
  oi::note_launch();
}

}  // namespace oi

extern "C" int oi_coarse_to_image(float* coarse, int nparts, int count, int mr, int mc, int br, int bc,
                                  const void* gc, const void* gr, const void* sy, const void* sx, int ny, int nx,
                                  void* scratch, float* out, void* stream) {
  using namespace oi;
  if (!coarse || !gc || !gr || !sy || !sx || !scratch || !out || nparts <= 0 || count <= 0 || mr <= 0 || mc <= 0 ||
      br <= 0 || bc <= 0 || ny <= 0 || nx <= 0)
    return fail(OI_EINVAL, "oi_coarse_to_image: bad arguments");
  if (mr < 2 * br - 1 || mc < 2 * bc - 1)
    return fail(OI_EINVAL, "oi_coarse_to_image: coarse grid %dx%d too small for band %dx%d", mr, mc, br, bc);
  if (mr > 1024 || bc > 512 || nx > 2048 || count > 65535)
    return fail(OI_ERANGE, "oi_coarse_to_image: sizes out of range (mr=%d bc=%d nx=%d)", mr, bc, nx);
  cudaStream_t s = (cudaStream_t)stream;
  int rc = coarse_spectrum(coarse, count, mr, mc, br, bc, gc, gr, scratch, s, nparts);
  if (rc) return rc;
  const float2* ih = (const float2*)scratch;
  switch ((nx + 255) / 256) {
    case 1: launch_synth<1>(ih, count, br, bc, (const float2*)sy, (const float2*)sx, ny, nx, out, s); break;
    case 2: launch_synth<2>(ih, count, br, bc, (const float2*)sy, (const float2*)sx, ny, nx, out, s); break;
    case 3: case 4:
      launch_synth<4>(ih, count, br, bc, (const float2*)sy, (const float2*)sx, ny, nx, out, s); break;
    case 5: case 6: case 7: case 8:
      launch_synth<8>(ih, count, br, bc, (const float2*)sy, (const float2*)sx, ny, nx, out, s); break;
    default:
      return fail(OI_ERANGE, "oi_coarse_to_image: nx=%d above 2048 not supported", nx);
  }
  return check_launch("oi_coarse_to_image/synth");
}

extern "C" int oi_spectrum_to_image(const void* ihat, int count, int br, int bc, const void* sy, const void* sx,
                                    int ny, int nx, float* out, void* stream) {
  using namespace oi;
  if (!ihat || !sy || !sx || !out || count <= 0 || br <= 0 || bc <= 0 || ny <= 0 || nx <= 0)
    return fail(OI_EINVAL, "oi_spectrum_to_image: bad arguments");
  if (bc > 512 || nx > 2048 || count > 65535)
    return fail(OI_ERANGE, "oi_spectrum_to_image: sizes out of range (bc=%d nx=%d)", bc, nx);
  cudaStream_t s = (cudaStream_t)stream;
  const float2* ih = (const float2*)ihat;
  switch ((nx + 255) / 256) {
    case 1: launch_synth<1>(ih, count, br, bc, (const float2*)sy, (const float2*)sx, ny, nx, out, s); break;
    case 2: launch_synth<2>(ih, count, br, bc, (const float2*)sy, (const float2*)sx, ny, nx, out, s); break;
    case 3: case 4:
      launch_synth<4>(ih, count, br, bc, (const float2*)sy, (const float2*)sx, ny, nx, out, s); break;
    default:
      launch_synth<8>(ih, count, br, bc, (const float2*)sy, (const float2*)sx, ny, nx, out, s); break;
  }
  return check_launch("oi_spectrum_to_image");
}
