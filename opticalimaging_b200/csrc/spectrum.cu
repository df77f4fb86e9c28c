// Band-limited forward spectrum of the mask near field (the numerical core of Scatter.CalculateSpectrum,
// Scatter.py:10-35, restricted to the frequencies the pupil can pass).
//
// Two separable passes, FP32 on the CUDA cores:
//   pass x: t[b][c][y][ic]    = sum_x h[b][y][x][c] * wx[x][ic]              (rows x Nx  by  Nx x Bc)
//   pass y: band[b][c][ir][ic] = scale * sum_y wy[y][ir] * t[b][c][y][ic]    (Br x Ny  by  Ny x Bc)
// The x pass streams the whole mask once; it is the HBM-facing part.  The y pass reads the small t.
#include "oi_common.cuh"
#include <cstdint>
#include <mutex>

namespace oi {

template <int KIND> struct FieldT;
template <> struct FieldT<OI_FIELD_REAL_F32> { using T = float; };
template <> struct FieldT<OI_FIELD_U8> { using T = float; };
template <> struct FieldT<OI_FIELD_COMPLEX_C64> { using T = float2; };

template <int KIND>
__device__ __forceinline__ typename FieldT<KIND>::T load_field(const void* f, long long idx);
template <>
__device__ __forceinline__ float load_field<OI_FIELD_REAL_F32>(const void* f, long long idx) {
  return __ldg((const float*)f + idx);
}
template <>
__device__ __forceinline__ float load_field<OI_FIELD_U8>(const void* f, long long idx) {
  return (float)__ldg((const uint8_t*)f + idx);
}
template <>
__device__ __forceinline__ float2 load_field<OI_FIELD_COMPLEX_C64>(const void* f, long long idx) {
  return __ldg((const float2*)f + idx);
}

__device__ __forceinline__ void mac(float2& acc, float a, float2 b) {
  acc.x = fmaf(a, b.x, acc.x);
  acc.y = fmaf(a, b.y, acc.y);
}
__device__ __forceinline__ void mac(float2& acc, float2 a, float2 b) { cfma(acc, a, b); }

__device__ __forceinline__ float zero_of(float) { return 0.f; }
__device__ __forceinline__ float2 zero_of(float2) { return make_float2(0.f, 0.f); }

constexpr int XB_M = 64, XB_N = 64, XB_K = 32;

// pass x.  Row R of t is (b, c, y) with R = (b*nch + c)*ny + y.
template <int KIND>
__global__ void __launch_bounds__(256) band_x_kernel(const void* __restrict__ field, int ny, int nx, int nch,
                                                     long long nrows, int bc, const float2* __restrict__ wx,
                                                     float2* __restrict__ t) {
  using T = typename FieldT<KIND>::T;
  __shared__ T as[XB_M][XB_K + 1];
  __shared__ __align__(16) float2 bs[XB_K][XB_N];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const long long row0 = (long long)blockIdx.x * XB_M;
  const int col0 = blockIdx.y * XB_N;
  float2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_float2(0.f, 0.f);

  for (int x0 = 0; x0 < nx; x0 += XB_K) {
#pragma unroll
    for (int i = 0; i < (XB_M * XB_K) / 256; ++i) {
      int e = tid + 256 * i, r = e / XB_K, kk = e % XB_K;
      long long R = row0 + r;
      int x = x0 + kk;
      T v = zero_of(T());
      if (R < nrows && x < nx) {
        long long bcidx = R / ny;
        int y = (int)(R - bcidx * ny);
        int c = (int)(bcidx % nch);
        long long b = bcidx / nch;
        v = load_field<KIND>(field, ((b * ny + y) * (long long)nx + x) * nch + c);
      }
      as[r][kk] = v;
    }
#pragma unroll
    for (int i = 0; i < (XB_K * XB_N) / 256; ++i) {
      int e = tid + 256 * i, kk = e / XB_N, cc = e % XB_N;
      int x = x0 + kk, col = col0 + cc;
      bs[kk][cc] = (x < nx && col < bc) ? __ldg(wx + (long long)x * bc + col) : make_float2(0.f, 0.f);
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < XB_K; ++kk) {
      T a[4];
      float2 b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = as[ty * 4 + i][kk];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mac(acc[i][j], a[i], b[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    long long R = row0 + ty * 4 + i;
    if (R >= nrows) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int col = col0 + tx * 4 + j;
      if (col < bc) t[R * bc + col] = acc[i][j];
    }
  }
}

constexpr int YB_M = 32, YB_N = 64, YB_K = 32;

// pass y: per image-channel matrix, band = scale * wy^T t.
__global__ void __launch_bounds__(256) band_y_kernel(const float2* __restrict__ t, int ny, int br, int bc,
                                                     const float2* __restrict__ wy, float scale,
                                                     float2* __restrict__ band) {
  __shared__ float2 ws[YB_K][YB_M + 1];
  __shared__ __align__(16) float2 ts[YB_K][YB_N];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int col0 = blockIdx.x * YB_N, r0 = blockIdx.y * YB_M;
  const long long mat = blockIdx.z;
  const float2* tm = t + mat * (long long)ny * bc;
  float2 acc[2][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_float2(0.f, 0.f);
  for (int y0 = 0; y0 < ny; y0 += YB_K) {
#pragma unroll
    for (int i = 0; i < (YB_K * YB_M) / 256; ++i) {
      int e = tid + 256 * i, kk = e / YB_M, r = e % YB_M;
      int y = y0 + kk, row = r0 + r;
      ws[kk][r] = (y < ny && row < br) ? __ldg(wy + (long long)y * br + row) : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int i = 0; i < (YB_K * YB_N) / 256; ++i) {
      int e = tid + 256 * i, kk = e / YB_N, cc = e % YB_N;
      int y = y0 + kk, col = col0 + cc;
      ts[kk][cc] = (y < ny && col < bc) ? tm[(long long)y * bc + col] : make_float2(0.f, 0.f);
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < YB_K; ++kk) {
      float2 a0 = ws[kk][ty * 2], a1 = ws[kk][ty * 2 + 1];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        float2 b = ts[kk][tx * 4 + j];
        cfma(acc[0][j], a0, b);
        cfma(acc[1][j], a1, b);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    int row = r0 + ty * 2 + i;
    if (row >= br) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int col = col0 + tx * 4 + j;
      if (col < bc)
        band[(mat * br + row) * (long long)bc + col] = make_float2(acc[i][j].x * scale, acc[i][j].y * scale);
    }
  }
}

}  // namespace oi

extern "C" int oi_band_spectrum(const void* field, int kind, int batch, int ny, int nx, int nch, int br, int bc,
                                const void* wx, const void* wy, float scale, void* scratch, void* band,
                                void* stream) {
  using namespace oi;
  if (!field || !wx || !wy || !scratch || !band || batch <= 0 || ny <= 0 || nx <= 0 || nch <= 0 || br <= 0 ||
      bc <= 0)
    return fail(OI_EINVAL, "oi_band_spectrum: bad arguments (batch=%d ny=%d nx=%d nch=%d br=%d bc=%d)", batch, ny,
                nx, nch, br, bc);
  if (kind != OI_FIELD_COMPLEX_C64 && nch != 1)
    return fail(OI_EINVAL, "oi_band_spectrum: real and u8 fields have one channel (nch=%d)", nch);
  if (br > 65535 * YB_M || bc > 65535 * XB_N || (long long)batch * nch > 65535)
    return fail(OI_ERANGE, "oi_band_spectrum: band or batch too large");
  cudaStream_t s = (cudaStream_t)stream;
  long long nrows = (long long)batch * nch * ny;
  dim3 gx((unsigned)ceil_div(nrows, XB_M), (unsigned)ceil_div(bc, XB_N));
  switch (kind) {
    case OI_FIELD_REAL_F32:
      band_x_kernel<OI_FIELD_REAL_F32><<<gx, 256, 0, s>>>(field, ny, nx, nch, nrows, bc, (const float2*)wx,
                                                           (float2*)scratch);
      oi::note_launch();
      break;
    case OI_FIELD_U8:
      band_x_kernel<OI_FIELD_U8><<<gx, 256, 0, s>>>(field, ny, nx, nch, nrows, bc, (const float2*)wx,
                                                     (float2*)scratch);
      oi::note_launch();
      break;
    case OI_FIELD_COMPLEX_C64:
      band_x_kernel<OI_FIELD_COMPLEX_C64><<<gx, 256, 0, s>>>(field, ny, nx, nch, nrows, bc, (const float2*)wx,
                                                              (float2*)scratch);
      oi::note_launch();
      break;
    default:
      return fail(OI_EINVAL, "oi_band_spectrum: unknown field kind %d", kind);
  }
  int rc = check_launch("oi_band_spectrum/x");
  if (rc) return rc;
  dim3 gy((unsigned)ceil_div(bc, YB_N), (unsigned)ceil_div(br, YB_M), (unsigned)(batch * nch));
  band_y_kernel<<<gy, 256, 0, s>>>((const float2*)scratch, ny, br, bc, (const float2*)wy, scale, (float2*)band);
  oi::note_launch();
  return check_launch("oi_band_spectrum/y");
}

// ---------------------------------------------------------------------------------------------------
// Band spectrum for callers that cannot allocate device memory.
//
// oi_band_spectrum needs a caller-provided scratch buffer for the intermediate row transform.  Some callers
// cannot provide one: code that only ever receives device pointers from a host application that owns every
// allocation (and forbids its plug-ins from calling cudaMalloc), or code running where an allocation would
// stall or fail (inside a fixed memory budget that is already fully handed out).  This entry point serves
// them: its scratch is a fixed-size array compiled into the library, one copy on each GPU that loads it,
// kept until the process exits.  Only the inputs and the output come from the caller.
namespace oi {

constexpr long long kStaticScratchF2 = OI_NOALLOC_SCRATCH_COMPLEX;  // complex values: 16 MiB per device
static __device__ __align__(256) float2 g_static_scratch[kStaticScratchF2];

// Device address of g_static_scratch on each device.  In host code the symbol itself is only a host-side handle,
// so the address comes from cudaGetSymbolAddress.  It is looked up again on every call whose stream is not
// capturing (a context torn down and created again -- cudaDeviceReset -- loads the module anew, possibly
// elsewhere, so an address kept from before would be stale); a call on a capturing stream makes no lookup and
// uses the address the last call on that device found.
static float2* g_static_scratch_ptr[64] = {nullptr};
static std::mutex g_static_scratch_mu;

static int static_scratch(cudaStream_t stream, float2** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(OI_ECUDA, "oi_band_spectrum_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) return fail(OI_ERANGE, "oi_band_spectrum_noalloc: device %d out of range", dev);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(stream, &cap);
  if (e != cudaSuccess)
    return fail(OI_ECUDA, "oi_band_spectrum_noalloc: cudaStreamIsCapturing: %s", cudaGetErrorString(e));
  std::lock_guard<std::mutex> lock(g_static_scratch_mu);
  if (cap == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p)
      return fail(OI_ECUDA, "oi_band_spectrum_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    g_static_scratch_ptr[dev] = (float2*)p;
  } else if (!g_static_scratch_ptr[dev]) {
    return fail(OI_EINVAL, "oi_band_spectrum_noalloc: the first call on device %d is being captured into a "
                           "graph; make one call on that device before any stream capture", dev);
  }
  *out = g_static_scratch_ptr[dev];
  return OI_OK;
}

}  // namespace oi

extern "C" int oi_band_spectrum_noalloc(const void* field, int kind, int batch, int ny, int nx, int nch, int br,
                                        int bc, const void* wx, const void* wy, float scale, void* band,
                                        void* stream) {
  using namespace oi;
  if (!field || !wx || !wy || !band || batch <= 0 || ny <= 0 || nx <= 0 || nch <= 0 || br <= 0 || bc <= 0)
    return fail(OI_EINVAL, "oi_band_spectrum_noalloc: bad arguments (batch=%d ny=%d nx=%d nch=%d br=%d bc=%d)",
                batch, ny, nx, nch, br, bc);
  const long long need = (long long)batch * nch * ny * bc;
  if (need > kStaticScratchF2)
    return fail(OI_ERANGE,
                "oi_band_spectrum_noalloc: needs %lld complex scratch values (batch*nch*ny*bc) but the built-in "
                "scratch holds %lld; use oi_band_spectrum with a caller buffer or split the batch",
                need, kStaticScratchF2);
  float2* scratch = nullptr;
  int rc = static_scratch((cudaStream_t)stream, &scratch);
  if (rc) return rc;
  // every scratch entry the y pass reads is written by the x pass first: nothing needs clearing
  return oi_band_spectrum(field, kind, batch, ny, nx, nch, br, bc, wx, wy, scale, scratch, band, stream);
}
