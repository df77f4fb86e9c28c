// Phase tables, status reporting and version of liboi_b200.
#include <atomic>
#include "oi_common.cuh"
#include <cstring>
#include <mutex>
#include <set>
#include <utility>

namespace oi {

static thread_local char g_err[512] = "";

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int ensure_smem(const void* kern, size_t bytes, const char* what) {
  if (bytes <= 48 * 1024) return OI_OK;
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(OI_ECUDA, "%s: cudaGetDevice: %s", what, cudaGetErrorString(e));
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;  // (kernel, device) pairs raised to the opt-in maximum
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({kern, dev})) return OI_OK;
  int optin = 0;
  e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return fail(OI_ECUDA, "%s: shared memory limit: %s", what, cudaGetErrorString(e));
  cudaFuncAttributes fa;   // the kernel's static shared memory counts against the same per-block limit
  e = cudaFuncGetAttributes(&fa, kern);
  if (e != cudaSuccess) return fail(OI_ECUDA, "%s: kernel attributes: %s", what, cudaGetErrorString(e));
  const int room = optin - (int)fa.sharedSizeBytes;
  if (bytes > (size_t)room)
    return fail(OI_ERANGE, "%s: needs %zu + %zu bytes of shared memory, the device allows %d", what, bytes,
                fa.sharedSizeBytes, optin);
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, room);
  if (e != cudaSuccess) return fail(OI_ECUDA, "%s: smem attribute: %s", what, cudaGetErrorString(e));
  done.insert({kern, dev});
  return OI_OK;
}

static std::atomic<long long> g_launches{0};

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(OI_ECUDA, "%s: %s", what, cudaGetErrorString(e));
  return OI_OK;
}

// out[a][b] = scale * exp(sign * 2 pi i * ((a + a0)(b + b0) mod n) / n).  The phase index is reduced in
// exact 64-bit integer arithmetic so the angle handed to sincospi is in [0, 2).
__global__ void twiddle_kernel(float2* out, int rows, int cols, long long a0, long long b0, long long n,
                               int sign, double scale) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)rows * cols) return;
  long long a = idx / cols + a0, b = idx % cols + b0;
  long long am = ((a % n) + n) % n, bm = ((b % n) + n) % n;
  // (am * bm) mod n without overflow for n < 2^31
  long long r = (long long)(((unsigned long long)am * (unsigned long long)bm) % (unsigned long long)n);
  double s, c;
  sincospi(2.0 * (double)r / (double)n, &s, &c);
  out[idx] = make_float2((float)(scale * c), (float)(scale * sign * s));
}

}  // namespace oi

extern "C" const char* oi_last_error(void) { return oi::g_err; }

extern "C" int oi_version(void) { return 1; }

extern "C" int oi_twiddle(void* out, int rows, int cols, long long a0, long long b0, long long n, int sign,
                          double scale, void* stream) {
  if (!out || rows <= 0 || cols <= 0 || n <= 0 || n >= (1LL << 31) || (sign != 1 && sign != -1))
    return oi::fail(OI_EINVAL, "oi_twiddle: bad arguments (rows=%d cols=%d n=%lld sign=%d)", rows, cols, n, sign);
  long long total = (long long)rows * cols;
  int threads = 256;
  long long blocks = (total + threads - 1) / threads;
  oi::twiddle_kernel<<<(unsigned)blocks, threads, 0, (cudaStream_t)stream>>>((float2*)out, rows, cols, a0, b0, n,
                                                                             sign, scale);
  oi::note_launch();
  return oi::check_launch("oi_twiddle");
}

extern "C" int oi_launch_count(long long* count) {
  if (!count) return oi::fail(OI_EINVAL, "oi_launch_count: null count");
  *count = oi::g_launches.load(std::memory_order_relaxed);
  return OI_OK;
}
