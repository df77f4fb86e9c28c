// Coherent sum of partially coherent imaging on the coarse grid: the |fft2(.)|^2 accumulation of
// CalculateAbbeImage (CalculateAerialImage.py:76-92, over source points x field components x channels) and of
// CalculateAerialImage_SOCS (CalculateAerialImage_SOCS.py:5-10, over SOCS kernels x channels).
//
// For one image b and plane z, every field (k, c) is band-limited to the Br x Bc band, so its intensity is
// band-limited to (2Br-1) x (2Bc-1) and is fully determined by its samples on any Mr x Mc grid with
// Mr >= 2Br-1, Mc >= 2Bc-1.  This kernel evaluates
//   coarse[b][z][sr][sc] = sum_{k,c} w[z][k] |sum_{ir,ic} frow[sr][ir] (P[z][k] .* band[b][c])[ir][ic] fcol[ic][sc]|^2
// as two small complex contractions per field, accumulating |E|^2 in registers: no per-field array ever
// reaches global memory.  One block owns 16 coarse rows of one (image, plane).
#include "oi_common.cuh"

namespace oi {

constexpr int CO_TR = 16;   // coarse rows per block
constexpr int CO_RC = 16;   // band rows per stage-1 chunk
constexpr int CO_CC = 16;   // band columns per stage-2 chunk
constexpr int CO_BMAX = 256;

struct CoherentArgs {
  const float2* band;
  long long band_img_stride;   // elements between images' band sets (nch * br * bc)
  int nch, br, bc;
  const float2* pupil;
  long long pupil_batch_stride;
  const float* weight;
  int nz, nk, mr, mc;
  const float2* frow;  // [mr][br]
  const float2* fcol;  // [bc][mc]
  float* coarse;       // [nsplit][batch][nz][mr][mc]
  int nsplit;          // fields f = split, split + nsplit, ... go to partial sum `split`
  long long split_stride;
};

// NU = ceil(bc / 64) column groups of stage 1, NJ = mc / 64 column groups of stage 2.
template <int NU, int NJ>
__global__ void __launch_bounds__(256) coherent_coarse_kernel(CoherentArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int bcp = NU * 64;  // padded band width
  float2* a_chunk = (float2*)smem_raw;          // [CO_RC][bcp]
  float2* f_chunk = a_chunk + CO_RC * bcp;      // [CO_TR][CO_RC]
  float2* gs = f_chunk + CO_TR * CO_RC;         // [CO_TR][bcp]
  float2* c_chunk = gs + CO_TR * bcp;           // [CO_CC][mc]

  const int tid = threadIdx.x, lane64 = tid & 63, grp = tid >> 6;  // grp 0..3 -> 4 coarse rows each
  const int rblocks = (a.mr + CO_TR - 1) / CO_TR;
  const int split = blockIdx.x / rblocks, sr0 = (blockIdx.x % rblocks) * CO_TR, z = blockIdx.y;
  const long long b = blockIdx.z;
  const int br = a.br, bc = a.bc, mr = a.mr, mc = a.mc;

  float acc[4][NJ];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j) acc[i][j] = 0.f;

  const float2* pup_base = a.pupil + b * a.pupil_batch_stride + (long long)z * a.nk * br * bc;
  for (int f = split; f < a.nk * a.nch; f += a.nsplit) {
    const int k = f / a.nch, c = f % a.nch;
    const float2* pk = pup_base + (long long)k * br * bc;
    const float w = __ldg(a.weight + (long long)z * a.nk + k);
    {
      const float2* hc = a.band + b * a.band_img_stride + (long long)c * br * bc;
      // ---- stage 1: G[r][ic] = sum_ir frow[sr0+r][ir] * P[ir][ic] * band[ir][ic]
      float2 g[4][NU];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int u = 0; u < NU; ++u) g[i][u] = make_float2(0.f, 0.f);
      for (int ir0 = 0; ir0 < br; ir0 += CO_RC) {
        for (int e = tid; e < CO_RC * bcp; e += 256) {
          int rr = e / bcp, cc = e - rr * bcp, ir = ir0 + rr;
          float2 v = make_float2(0.f, 0.f);
          if (ir < br && cc < bc) {
            long long off = (long long)ir * bc + cc;
            v = cmul(__ldg(pk + off), __ldg(hc + off));
          }
          a_chunk[e] = v;
        }
        {
          int r = tid / CO_RC, cc = tid % CO_RC;  // 256 = CO_TR * CO_RC
          int sr = sr0 + r, ir = ir0 + cc;
          f_chunk[tid] = (sr < mr && ir < br) ? __ldg(a.frow + (long long)sr * br + ir) : make_float2(0.f, 0.f);
        }
        __syncthreads();
#pragma unroll 4
        for (int rr = 0; rr < CO_RC; ++rr) {
          float2 f[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) f[i] = f_chunk[(grp * 4 + i) * CO_RC + rr];
#pragma unroll
          for (int u = 0; u < NU; ++u) {
            float2 av = a_chunk[rr * bcp + u * 64 + lane64];
#pragma unroll
            for (int i = 0; i < 4; ++i) cfma(g[i][u], f[i], av);
          }
        }
        __syncthreads();
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int u = 0; u < NU; ++u) gs[(grp * 4 + i) * bcp + u * 64 + lane64] = g[i][u];
      __syncthreads();
      // ---- stage 2: E[r][sc] = sum_ic G[r][ic] * fcol[ic][sc];  acc += w |E|^2
      float2 e2[4][NJ];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) e2[i][j] = make_float2(0.f, 0.f);
      for (int ic0 = 0; ic0 < bc; ic0 += CO_CC) {
        for (int e = tid; e < CO_CC * mc; e += 256) {
          int rr = e / mc, sc = e - rr * mc, ic = ic0 + rr;
          c_chunk[e] = (ic < bc) ? __ldg(a.fcol + (long long)ic * mc + sc) : make_float2(0.f, 0.f);
        }
        __syncthreads();
        const int lim = min(CO_CC, bc - ic0);
        for (int rr = 0; rr < lim; ++rr) {
          float2 gv[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) gv[i] = gs[(grp * 4 + i) * bcp + ic0 + rr];
#pragma unroll
          for (int j = 0; j < NJ; ++j) {
            float2 fv = c_chunk[rr * mc + j * 64 + lane64];
#pragma unroll
            for (int i = 0; i < 4; ++i) cfma(e2[i][j], gv[i], fv);
          }
        }
        __syncthreads();
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) acc[i][j] = fmaf(w, fmaf(e2[i][j].x, e2[i][j].x, e2[i][j].y * e2[i][j].y), acc[i][j]);
    }
  }
  float* out = a.coarse + split * a.split_stride + ((b * a.nz + z) * (long long)mr) * mc;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int sr = sr0 + grp * 4 + i;
    if (sr >= mr) continue;
#pragma unroll
    for (int j = 0; j < NJ; ++j) out[(long long)sr * mc + j * 64 + lane64] = acc[i][j];
  }
}

template <int NU, int NJ>
static int launch_coherent(const CoherentArgs& a, int batch, cudaStream_t s) {
  size_t smem = sizeof(float2) * ((size_t)CO_RC * NU * 64 + CO_TR * CO_RC + (size_t)CO_TR * NU * 64 +
                                  (size_t)CO_CC * a.mc);
  auto kern = coherent_coarse_kernel<NU, NJ>;
  {
    int rc_smem = ensure_smem((const void*)kern, smem, "oi_coherent_coarse");
    if (rc_smem) return rc_smem;
  }
  dim3 grid((unsigned)(ceil_div(a.mr, CO_TR) * a.nsplit), (unsigned)a.nz, (unsigned)batch);
  kern<<<grid, 256, smem, s>>>(a);
  oi::note_launch();
  return check_launch("oi_coherent_coarse");
}

template <int NU>
static int dispatch_nj(const CoherentArgs& a, int batch, cudaStream_t s) {
  switch (a.mc / 64) {
    case 1: return launch_coherent<NU, 1>(a, batch, s);
    case 2: return launch_coherent<NU, 2>(a, batch, s);
    case 3: return launch_coherent<NU, 3>(a, batch, s);
    case 4: return launch_coherent<NU, 4>(a, batch, s);
  }
  return fail(OI_ERANGE, "oi_coherent_coarse: mc=%d unsupported", a.mc);
}

}  // namespace oi

extern "C" int oi_coherent_coarse(const void* band, int batch, int nch, int br, int bc, const void* pupil,
                                  long long pupil_batch_stride, const float* weight, int nz, int nk, int mr, int mc,
                                  const void* frow, const void* fcol, int nsplit, float* coarse, void* stream) {
  using namespace oi;
  if (!band || !pupil || !weight || !frow || !fcol || !coarse || batch <= 0 || nch <= 0 || br <= 0 || bc <= 0 ||
      nz <= 0 || nk <= 0 || mr <= 0 || mc <= 0 || pupil_batch_stride < 0 || nsplit <= 0)
    return fail(OI_EINVAL, "oi_coherent_coarse: bad arguments");
  if (mc % 64 != 0 || mc > 256 || br > CO_BMAX || bc > CO_BMAX || nz > 65535 || batch > 65535 ||
      nsplit > nk * nch || (long long)ceil_div(mr, CO_TR) * nsplit > 2147483647LL)
    return fail(OI_ERANGE, "oi_coherent_coarse: sizes out of range (br=%d bc=%d mc=%d nsplit=%d)", br, bc, mc, nsplit);
  CoherentArgs a{(const float2*)band, (long long)nch * br * bc, nch, br, bc, (const float2*)pupil,
                 pupil_batch_stride, weight, nz, nk, mr, mc, (const float2*)frow, (const float2*)fcol, coarse,
                 nsplit, (long long)batch * nz * mr * mc};
  cudaStream_t s = (cudaStream_t)stream;
  switch ((bc + 63) / 64) {
    case 1: return dispatch_nj<1>(a, batch, s);
    case 2: return dispatch_nj<2>(a, batch, s);
    case 3: return dispatch_nj<3>(a, batch, s);
    case 4: return dispatch_nj<4>(a, batch, s);
  }
  return fail(OI_ERANGE, "oi_coherent_coarse: bc=%d unsupported", bc);
}
