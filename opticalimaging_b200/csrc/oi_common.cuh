// Shared helpers of the engine's CUDA sources: status reporting and small complex arithmetic.
#pragma once
#include <cuda_runtime.h>
#include <cstdio>
#include <cstdarg>
#include "../../include/oi_b200.h"

namespace oi {

// Records a formatted message as the calling thread's last error and returns `code`.
int fail(int code, const char* fmt, ...);

// Counts one kernel launch (oi_launch_count reports the total, for launch accounting in benchmarks).
void note_launch();

// Checks the launch just enqueued; returns OI_OK or OI_ECUDA with the CUDA error text recorded.
int check_launch(const char* what);

// Lets `kern` use `bytes` of dynamic shared memory.  Above the 48 KB default the kernel's limit is raised to
// the device's opt-in maximum, once per (kernel, device) -- so later launches, including ones inside CUDA-graph
// capture, make no attribute call.
int ensure_smem(const void* kern, size_t bytes, const char* what);

// Programmatic dependent launch.  The kernels of the split-form step are launched with programmatic stream
// serialisation (launch_pdl): a kernel's CTAs may start -- allocate tensor memory, initialise barriers, load
// constant operands -- while the previous kernel's last CTAs finish.  Before reading anything an earlier kernel
// wrote, and before writing global memory, a thread calls pdl_wait(), which returns once the preceding grids
// have completed and their writes are visible; pdl_trigger() lets the next such kernel launch once every CTA of
// this one has started.  A kernel launched this way after any other work is correct too (the wait covers it).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, args...);
}

__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// acc += a * b
__device__ __forceinline__ void cfma(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(-a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(a.y, b.x, acc.y);
}
__device__ __forceinline__ void cfma(double2& acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
// acc += a * conj(b)
__device__ __forceinline__ void cfma_conj(double2& acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.y, b.x, acc.y);
  acc.y = fma(-a.x, b.y, acc.y);
}

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// The coarse-intensity spectrum stage shared by oi_coarse_to_image and oi_coarse_to_image_fft (synth.cu):
// ihat[i][jr][qc] = (qc ? 2 : 1) / (mr mc) * sum_s coarse[i][s] exp(+2 pi i (qr sr/mr + qc sc/mc)).
// Adds partial sums 1..nparts-1 (each n floats, one after another) into the first, in place.
int fold_parts(float* coarse, int nparts, long long n, cudaStream_t s);

// The coarse intensity may be split in `nparts` partial sums, each count*mr*mc floats, added in order.
int coarse_spectrum(float* coarse, int count, int mr, int mc, int br, int bc, const void* gc, const void* gr,
                    void* ihat, cudaStream_t s, int nparts);

}  // namespace oi
