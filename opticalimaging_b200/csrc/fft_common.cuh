// Device helpers shared by the coarse-grid kernels (coherent_fft.cu, coherent_tc.cu, adjoint.cu): the 32-point
// transform in registers and the inverse four-step gather of a band-limited input.
#pragma once
#include "oi_common.cuh"

namespace oi {
namespace cg {

// cos(2 pi t / 32), t = 0..15 (exact decimal expansions of the standard values); sin via the quarter shift
__host__ __device__ constexpr float c32(int t) {
  return t == 0 ? 1.0f : t == 1 ? 0.980785280403230449f : t == 2 ? 0.923879532511286756f
       : t == 3 ? 0.831469612302545237f : t == 4 ? 0.707106781186547524f : t == 5 ? 0.555570233019602225f
       : t == 6 ? 0.382683432365089772f : t == 7 ? 0.195090322016128268f : t == 8 ? 0.0f
       : t == 9 ? -0.195090322016128268f : t == 10 ? -0.382683432365089772f : t == 11 ? -0.555570233019602225f
       : t == 12 ? -0.707106781186547524f : t == 13 ? -0.831469612302545237f : t == 14 ? -0.923879532511286756f
       : -0.980785280403230449f;
}
__host__ __device__ constexpr float s32(int t) { return t <= 8 ? c32(8 - t) : c32(t - 8); }
__host__ __device__ constexpr int brev5(int i) {
  return ((i & 1) << 4) | ((i & 2) << 2) | (i & 4) | ((i & 8) >> 2) | ((i & 16) >> 4);
}

// 32-point DFT with exp(-2 pi i k n / 32) in registers, decimation in frequency: v[i] = X[brev5(i)].
__device__ __forceinline__ void ifft32(float2 (&v)[32]) {
#pragma unroll
  for (int len = 32; len >= 2; len >>= 1) {
    const int half = len >> 1, step = 32 / len;
#pragma unroll
    for (int blk = 0; blk < 32; blk += len) {
#pragma unroll
      for (int j = 0; j < half; ++j) {
        float2 u = v[blk + j], w = v[blk + j + half];
        v[blk + j] = make_float2(u.x + w.x, u.y + w.y);
        float2 d = make_float2(u.x - w.x, u.y - w.y);
        const int t = j * step;
        if (t == 0) {
          v[blk + j + half] = d;
        } else if (t == 8) {
          v[blk + j + half] = make_float2(d.y, -d.x);  // * (-i)
        } else {
          const float c = c32(t), s = -s32(t);
          v[blk + j + half] = make_float2(d.x * c - d.y * s, d.x * s + d.y * c);
        }
      }
    }
  }
}

// Inverse four-step for an M = 32 N1 point transform of a band-limited input: thread n1 forms
//   z[k2] = W_M^{-k2 n1} sum_k1 x[k2 + 32 k1] W_N1^{-k1 n1},  x[k] = src[((k - m0) mod M) * stride] if < b else 0,
// then the 32-point transform; on return z[i] = X[n1 + N1 brev5(i)], X[s] = sum_m x_m exp(-2 pi i m s / M).
// w: exp(+2 pi i j / M), j < M.
template <int N1>
__device__ __forceinline__ void gather_ifft(float2 (&z)[32], const float2* src, int stride, int m0, int b,
                                            const float2* w, int n1) {
  constexpr int M = 32 * N1;
#pragma unroll
  for (int k2 = 0; k2 < 32; ++k2) {
    float2 acc = make_float2(0.f, 0.f);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
      const int idx = (k2 + 32 * k1 - m0) & (M - 1);
      if (idx < b) {
        const float2 tw = w[(32 * k1 * n1) & (M - 1)];
        cfma(acc, src[idx * stride], make_float2(tw.x, -tw.y));
      }
    }
    const float2 tw = w[(k2 * n1) & (M - 1)];
    z[k2] = cmul(acc, make_float2(tw.x, -tw.y));
  }
  ifft32(z);
}

}  // namespace cg
}  // namespace oi
