// FFT form of the two N-point transforms of the imaging path, FP32 on the CUDA cores:
//   forward  mask -> band spectrum      (Scatter.CalculateSpectrum, Scatter.py:10-35, on the band only)
//   inverse  intensity spectrum -> image (the final synthesis of CalculateAerialImage_SOCS.py:7-10)
//
// Four-step decomposition N = 32 * N1 (N1 = 8, 16, 32, 64 for N = 256 .. 2048), x = n1 + N1 n2, k = k2 + 32 k1:
//   X[k2 + 32 k1] = sum_n1 W_N1^{k1 n1} W_N^{k2 n1} [ sum_n2 x[n1 + N1 n2] W_32^{k2 n2} ]
// Each of the N1 threads of a group owns one n1 and runs the 32-point transform in registers; the groups
// exchange through shared memory.  Only the band is wanted, so:
//   forward: the outer N1-term sum is evaluated for the band bins only (59 of 1024 at configuration 3);
//   inverse: the input is zero outside the band, so the first N1-term stage sums the few non-zero k1 only.
// Real rows travel in pairs as one complex row (x = a + i b); the forward pass separates the two spectra,
// the inverse pass builds one Hermitian spectrum per row so that the real and imaginary parts of one complex
// transform are the two output rows.
//
// Memory: the forward row pass reads each mask row once (coalesced: thread n1 reads x[n1 + N1 n2]) and writes
// the band columns transposed, [b][ic][y], so the column pass reads contiguous columns; the inverse passes
// write [b][qc][y] then rows [b][y][x], again coalesced.
#include "tc_common.cuh"
#include <cstdint>

namespace oi {

// cos / sin of 2 pi t / 32 for t = 0..15 (exact decimal expansions of the standard values)
__host__ __device__ constexpr float c32(int t) {
  return t == 0 ? 1.0f : t == 1 ? 0.980785280403230449f : t == 2 ? 0.923879532511286756f
       : t == 3 ? 0.831469612302545237f : t == 4 ? 0.707106781186547524f : t == 5 ? 0.555570233019602225f
       : t == 6 ? 0.382683432365089772f : t == 7 ? 0.195090322016128268f : t == 8 ? 0.0f
       : t == 9 ? -0.195090322016128268f : t == 10 ? -0.382683432365089772f : t == 11 ? -0.555570233019602225f
       : t == 12 ? -0.707106781186547524f : t == 13 ? -0.831469612302545237f : t == 14 ? -0.923879532511286756f
       : -0.980785280403230449f;
}
__host__ __device__ constexpr float s32(int t) { return t <= 8 ? c32(8 - t) : c32(t - 8); }
__host__ __device__ constexpr int bitrev5(int i) {
  return ((i & 1) << 4) | ((i & 2) << 2) | (i & 4) | ((i & 8) >> 2) | ((i & 16) >> 4);
}

// d * exp(SIGN 2 pi i t / 32), t a compile-time constant after unrolling
template <int SIGN>
__device__ __forceinline__ float2 rot32(float2 d, int t) {
  if (t == 0) return d;
  if (t == 8) return SIGN > 0 ? make_float2(-d.y, d.x) : make_float2(d.y, -d.x);
  const float c = c32(t), s = SIGN * s32(t);
  return make_float2(d.x * c - d.y * s, d.x * s + d.y * c);
}

// In-register 32-point DFT, X[k] = sum_n v[n] exp(SIGN 2 pi i k n / 32), decimation in frequency.
// Natural-order input; on return v[i] = X[bitrev5(i)].
template <int SIGN>
__device__ __forceinline__ void fft32(float2 (&v)[32]) {
#pragma unroll
  for (int len = 32; len >= 2; len >>= 1) {
    const int half = len >> 1, step = 32 / len;
#pragma unroll
    for (int blk = 0; blk < 32; blk += len) {
#pragma unroll
      for (int j = 0; j < half; ++j) {
        float2 u = v[blk + j], w = v[blk + j + half];
        v[blk + j] = make_float2(u.x + w.x, u.y + w.y);
        v[blk + j + half] = rot32<SIGN>(make_float2(u.x - w.x, u.y - w.y), j * step);
      }
    }
  }
}

template <typename K>
static int set_smem(K kern, size_t bytes, const char* what) {
  return ensure_smem((const void*)kern, bytes, what);
}

template <int KIND> __device__ __forceinline__ float load_real(const void* f, long long i);
template <> __device__ __forceinline__ float load_real<OI_FIELD_REAL_F32>(const void* f, long long i) {
  return __ldg((const float*)f + i);
}
template <> __device__ __forceinline__ float load_real<OI_FIELD_U8>(const void* f, long long i) {
  return (float)__ldg((const uint8_t*)f + i);
}

// Twiddle tables, laid out so that a warp reading one k for all n1 touches consecutive entries:
//   t2[k2][n1] = W_N^{k2 n1}  (32 x N1)      t1[k1][n1] = W_N1^{k1 n1} = W_N^{32 k1 n1}  (N1 x N1)
// with W_N = exp(+2 pi i / N).  The four N-point kernels read them from global memory (one table per N, built
// by oi_twiddle: warp-coalesced, L1-resident); the coarse-spectrum kernel builds them in shared memory from the
// 1-D table W_M^j.  (Reading a 1-D table at index k n1 mod N across a warp is a stride-k access, up to 32-way
// bank conflicts.)
template <int N1>
__device__ __forceinline__ void build_tables(const float2* __restrict__ wn_g, float2* t2, float2* t1, int tid,
                                             int nthreads) {
  constexpr int N = 32 * N1;
  for (int e = tid; e < 32 * N1; e += nthreads) {
    const int k2 = e / N1, n1 = e % N1;
    t2[e] = __ldg(wn_g + ((k2 * n1) & (N - 1)));
  }
  for (int e = tid; e < N1 * N1; e += nthreads) {
    const int k1 = e / N1, n1 = e % N1;
    t1[e] = __ldg(wn_g + ((32 * k1 * n1) & (N - 1)));
  }
}
template <int N1>
constexpr int table_f2() { return 32 * N1 + N1 * N1; }

template <int SIGN>
__device__ __forceinline__ float2 sgn(float2 w) { return SIGN > 0 ? w : make_float2(w.x, -w.y); }

// Stage 2 + transpose: z holds the bit-reversed 32-point result of thread n1; multiply by W_N^{n1 k2} and
// store to ys[k2][n1] (row stride N1 + 1).
template <int SIGN, int N1>
__device__ __forceinline__ void twiddle_store(const float2 (&z)[32], const float2* t2, int n1, float2* ys) {
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    const int k2 = bitrev5(i);
    ys[k2 * (N1 + 1) + n1] = cmul(z[i], sgn<SIGN>(t2[k2 * N1 + n1]));
  }
}

// Z[k] = sum_n1 W_N1^{k1 n1} ys[k2][n1]  (forward outer stage for one bin k = k2 + 32 k1)
template <int SIGN, int N1>
__device__ __forceinline__ float2 outer_bin(const float2* ys, const float2* t1, int k) {
  const int k2 = k & 31, k1 = k >> 5;
  const float2* row = ys + k2 * (N1 + 1);
  const float2* tw = t1 + k1 * N1;
  float2 acc = make_float2(0.f, 0.f);
#pragma unroll 8
  for (int n1 = 0; n1 < N1; ++n1) cfma(acc, row[n1], sgn<SIGN>(tw[n1]));
  return acc;
}
// Two bins at once (ka, kb), each summed in two interleaved halves: four independent chains.
template <int SIGN, int N1>
__device__ __forceinline__ void outer_bin2(const float2* ys, const float2* t1, int ka, int kb, float2& va, float2& vb) {
  const float2* ra = ys + (ka & 31) * (N1 + 1);
  const float2* rb = ys + (kb & 31) * (N1 + 1);
  const float2* ta = t1 + (ka >> 5) * N1;
  const float2* tb = t1 + (kb >> 5) * N1;
  float2 a0 = make_float2(0.f, 0.f), a1 = a0, b0 = a0, b1 = a0;
#pragma unroll 4
  for (int n1 = 0; n1 < N1; n1 += 2) {
    cfma(a0, ra[n1], sgn<SIGN>(ta[n1]));
    cfma(a1, ra[n1 + 1], sgn<SIGN>(ta[n1 + 1]));
    cfma(b0, rb[n1], sgn<SIGN>(tb[n1]));
    cfma(b1, rb[n1 + 1], sgn<SIGN>(tb[n1 + 1]));
  }
  va = make_float2(a0.x + a1.x, a0.y + a1.y);
  vb = make_float2(b0.x + b1.x, b0.y + b1.y);
}

// --------------------------------------------------------------------------------- forward, rows
// field rows [nrows = batch*ny][N] (real or u8) -> t[b][ic][y], ic over the band m0c .. m0c+bc-1.
// Z is evaluated on the contiguous frequency range u0 .. u0+nu-1 that holds the band and its mirror.
template <int N1, int KIND>
__global__ void __launch_bounds__(256, 3) fft_rows_fwd_kernel(const void* __restrict__ field, long long nrows, int ny,
                                                           const float2* __restrict__ wn_g, int m0c, int bc, int u0,
                                                           int nu, float2* __restrict__ t, int nparts,
                                                           long long pstride) {
  // nparts > 1 (float32 only): the field is the sum of nparts arrays pstride elements apart
  constexpr int N = 32 * N1, G = 256 / N1;  // G row pairs per block
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const float2* t2 = wn_g;                    // global [32][N1], read through L1 (warp-coalesced)
  const float2* t1 = wn_g + 32 * N1;          // global [N1][N1]
  float2* ys = (float2*)smem_raw;             // [G][32][N1+1]
  float2* zs = ys + G * 32 * (N1 + 1);        // [G][nu]
  const int tid = threadIdx.x, g = tid / N1, n1 = tid % N1;
  const long long r0 = (long long)blockIdx.x * (2 * G) + 2 * g;
  float2 z[32];
  if (r0 + 1 < nrows) {
    const long long o0 = r0 * N, o1 = o0 + N;
#pragma unroll
    for (int n2 = 0; n2 < 32; ++n2)
      z[n2] = make_float2(load_real<KIND>(field, o0 + n1 + N1 * n2), load_real<KIND>(field, o1 + n1 + N1 * n2));
    for (int p = 1; p < nparts; ++p) {
      const long long op = p * pstride;
#pragma unroll
      for (int n2 = 0; n2 < 32; ++n2) {
        z[n2].x += load_real<KIND>(field, op + o0 + n1 + N1 * n2);
        z[n2].y += load_real<KIND>(field, op + o1 + n1 + N1 * n2);
      }
    }
  } else {
#pragma unroll
    for (int n2 = 0; n2 < 32; ++n2) z[n2] = make_float2(0.f, 0.f);
  }
  fft32<+1>(z);
  __syncthreads();  // tables ready
  float2* yg = ys + g * 32 * (N1 + 1);
  twiddle_store<+1, N1>(z, t2, n1, yg);
  __syncthreads();
  float2* zg = zs + g * nu;
  for (int q = n1; q < nu; q += N1) zg[q] = outer_bin<+1, N1>(yg, t1, (u0 + q) & (N - 1));
  __syncthreads();
  // separate the two real rows and write t[b][ic][y] with y fastest (2G consecutive rows of one image)
  const long long rblk = (long long)blockIdx.x * (2 * G);
  for (int e = tid; e < bc * 2 * G; e += 256) {
    const int ic = e / (2 * G), rr = e % (2 * G), gg = rr >> 1;
    const long long r = rblk + rr;
    if (r >= nrows) continue;
    const int m = m0c + ic;
    const float2 zp = zs[gg * nu + (m - u0)], zm = zs[gg * nu + (-m - u0)];
    float2 v;
    if ((rr & 1) == 0) v = make_float2(0.5f * (zp.x + zm.x), 0.5f * (zp.y - zm.y));   // (Z(m) + conj Z(-m)) / 2
    else v = make_float2(0.5f * (zp.y + zm.y), -0.5f * (zp.x - zm.x));               // (Z(m) - conj Z(-m)) / 2i
    const long long b = r / ny;
    const int y = (int)(r - b * ny);
    t[(b * bc + ic) * (long long)ny + y] = v;
  }
}

// ------------------------------------------------------------------------------ forward, columns
// t[b][ic][y] (N = ny) -> band[b][ir][ic] = scale * sum_y t exp(+2 pi i (m0r+ir) y / ny).
// SYM: t holds the non-negative columns kx = 0 .. bc-1 of a real mask's row transform and the band is the
// symmetric bco x br band (m0c = -(bco-1)/2, m0r = -(br-1)/2): column kx lands at ic = kx + (bco-1)/2 and, for
// kx > 0, its mirror band[-ky][-kx] = conj(band[ky][kx]) at row br-1-ir, column (bco-1)/2 - kx.
// Blocks of COLS_T threads (G = COLS_T / N1 columns each, 32 KB of t): the block's columns are contiguous in t
// and are staged into shared memory by 16-byte asynchronous copies (cp.async, completed per thread: no waits on
// another thread's progress), from where each thread reads its 32 strided values; the twiddled rows then reuse
// the same shared memory.  At the symmetric band's 30 columns per image a batch of 64 has 1920 columns: 480
// blocks, all resident at once.
constexpr int COLS_T = 128;

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

template <int N1, bool SYM>
__global__ void __launch_bounds__(COLS_T, 6) fft_cols_fwd_kernel(const float2* __restrict__ t, long long ncols, int bc,
                                                              const float2* __restrict__ wn_g, int m0r, int br,
                                                              float scale, float2* __restrict__ band, int bco,
                                                              int dbl_from) {
  constexpr int N = 32 * N1, G = COLS_T / N1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const float2* t2 = wn_g;
  const float2* t1 = wn_g + 32 * N1;
  float2* ys = (float2*)smem_raw;
  const int tid = threadIdx.x, g = tid / N1, n1 = tid % N1;
  const long long col0 = (long long)blockIdx.x * G, col = col0 + g;
  pdl_trigger();
  pdl_wait();   // t comes from the row pass
  {
    const long long cols = ncols - col0 < G ? ncols - col0 : G;
    const int chunks = (int)(cols * N / 2);   // 16-byte pieces of the block's contiguous columns
    const float4* src = (const float4*)(t + col0 * N);
    float4* dst = (float4*)smem_raw;
    for (int c = tid; c < chunks; c += COLS_T) cp_async16(dst + c, src + c);
    cp_async_wait_all();
    __syncthreads();
  }
  float2 z[32];
  if (col < ncols) {
    const float2* stg = ys + g * N;
#pragma unroll
    for (int n2 = 0; n2 < 32; ++n2) z[n2] = stg[n1 + N1 * n2];
  } else {
#pragma unroll
    for (int n2 = 0; n2 < 32; ++n2) z[n2] = make_float2(0.f, 0.f);
  }
  __syncthreads();   // the stage is overwritten by the twiddled rows below
  fft32<+1>(z);
  float2* yg = ys + g * 32 * (N1 + 1);
  twiddle_store<+1, N1>(z, t2, n1, yg);
  __syncthreads();
  if (col >= ncols) return;
  const long long b = col / bc;
  const int ic = (int)(col - b * bc);
  if (!SYM) {   // columns ic >= dbl_from are doubled (a Hermitian half-spectrum standing for both halves)
    const float sc = ic >= dbl_from ? 2.f * scale : scale;
    for (int ir = n1; ir < br; ir += N1) {
      float2 v = outer_bin<+1, N1>(yg, t1, (m0r + ir) & (N - 1));
      band[(b * br + ir) * (long long)bc + ic] = make_float2(v.x * sc, v.y * sc);
    }
  } else {   // bins ir and ir + N1 together
    const int h = (bco - 1) / 2;
    for (int ir = n1; ir < br; ir += 2 * N1) {
      float2 v[2];
      outer_bin2<+1, N1>(yg, t1, (m0r + ir) & (N - 1), (m0r + ir + N1) & (N - 1), v[0], v[1]);
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int r = ir + u * N1;
        if (r >= br) break;
        band[(b * br + r) * (long long)bco + h + ic] = make_float2(v[u].x * scale, v[u].y * scale);
        if (ic > 0) band[(b * br + br - 1 - r) * (long long)bco + h - ic] = make_float2(v[u].x * scale, -v[u].y * scale);
      }
    }
  }
}

// --------------------------------------------------------------------------- inverse, shared part
// Thread n1 of a group: z[k2] = W_N^{-k2 n1} sum_{k1} coef(k2 + 32 k1) W_N1^{-k1 n1} over the non-zero
// coefficients, which sit at frequencies q in [-qmax, qmax] (index q mod N); coef(q) = cq[q + qmax].
template <int N1>
__device__ __forceinline__ void inverse_gather(float2 (&z)[32], const float2* cq, int qmax, const float2* t2,
                                               const float2* t1, int n1) {
  constexpr int N = 32 * N1;
  if (qmax < 64) {
    // |q| <= 63: the only non-zero inputs of k2 are q = k2, k2 + 32 (k1 = 0, 1) and q = k2 - 32, k2 - 64
    // (k1 = N1 - 1, N1 - 2).  Four predicated terms with their twiddles in registers: no runtime loops, so
    // the 32 independent k2 chains interleave.
    const float2 w1 = sgn<-1>(t1[1 * N1 + n1]);            // W_N1^{-n1}
    const float2 wm1 = sgn<-1>(t1[(N1 - 1) * N1 + n1]);    // W_N1^{-(N1-1) n1}
    const float2 wm2 = sgn<-1>(t1[(N1 - 2) * N1 + n1]);    // W_N1^{-(N1-2) n1}
    const float2* c0 = cq + qmax;                          // c0[q] = coefficient of frequency q
#pragma unroll
    for (int k2 = 0; k2 < 32; ++k2) {
      float2 acc = k2 <= qmax ? c0[k2] : make_float2(0.f, 0.f);
      if (k2 + 32 <= qmax) cfma(acc, c0[k2 + 32], w1);
      if (k2 - 32 >= -qmax) cfma(acc, c0[k2 - 32], wm1);
      if (k2 - 64 >= -qmax) cfma(acc, c0[k2 - 64], wm2);
      z[k2] = cmul(acc, sgn<-1>(t2[k2 * N1 + n1]));
    }
    fft32<-1>(z);
    return;
  }
#pragma unroll
  for (int k2 = 0; k2 < 32; ++k2) {
    float2 acc = make_float2(0.f, 0.f);
    for (int k1 = 0; k2 + 32 * k1 <= qmax; ++k1)  // q = k2 + 32 k1 >= 0
      cfma(acc, cq[k2 + 32 * k1 + qmax], sgn<-1>(t1[k1 * N1 + n1]));
    for (int k1 = N1 - 1; k1 > 0 && k2 + 32 * k1 >= N - qmax; --k1)  // q = k2 + 32 k1 - N < 0
      cfma(acc, cq[k2 + 32 * k1 - N + qmax], sgn<-1>(t1[k1 * N1 + n1]));
    z[k2] = cmul(acc, sgn<-1>(t2[k2 * N1 + n1]));
  }
  fft32<-1>(z);
}

// ------------------------------------------------------------------------------ inverse, columns
// ihat[i][jr][qc] (qr = jr - (br-1)) -> v[i][qc][y] = sum_qr ihat exp(-2 pi i qr y / ny)
template <int N1>
__global__ void __launch_bounds__(256, 3) fft_cols_inv_kernel(const float2* __restrict__ ihat, long long ncols, int br,
                                                           int bc, const float2* __restrict__ wn_g,
                                                           float2* __restrict__ v) {
  constexpr int N = 32 * N1, G = 256 / N1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const float2* t2 = wn_g;
  const float2* t1 = wn_g + 32 * N1;
  const int nq = 2 * br - 1;
  float2* cs = (float2*)smem_raw;  // [G][nq]
  const int tid = threadIdx.x, g = tid / N1, n1 = tid % N1;
  const long long col0 = (long long)blockIdx.x * G;
  for (int e = tid; e < G * nq; e += 256) {
    const int jr = e / G, gg = e % G;
    const long long col = col0 + gg;
    float2 c = make_float2(0.f, 0.f);
    if (col < ncols) {
      const long long i = col / bc;
      const int qc = (int)(col - i * bc);
      c = ihat[(i * nq + jr) * (long long)bc + qc];
    }
    cs[gg * nq + jr] = c;
  }
  __syncthreads();
  const long long col = col0 + g;
  float2 z[32];
  inverse_gather<N1>(z, cs + g * nq, br - 1, t2, t1, n1);
  if (col >= ncols) return;
  float2* dst = v + col * N;
#pragma unroll
  for (int i = 0; i < 32; ++i) dst[n1 + N1 * bitrev5(i)] = z[i];
}

// ---------------------------------------------------------------- inverse, columns into V operand tiles
// The column pass of the tensor-core synthesis: for image i and band columns qc0 .. qc0+G-1 (G = max(8, 256/N1),
// zero beyond bc) the inverse column FFTs as fft_cols_inv_kernel, kept in shared memory, then written directly as
// the bf16 hi / lo V operand tiles of the row pass (rows y of 128-row blocks, K = re | im of 64 band columns,
// 128-byte swizzled: [hi: re | im][lo: re | im] x [128][64]) -- v itself never reaches global memory.
template <int N1, int G>
__global__ void __launch_bounds__(G * N1) cols_inv_tiles_kernel(const float2* __restrict__ ihat, int br, int bc,
                                                              int ny, const float2* __restrict__ wn_g,
                                                              unsigned char* __restrict__ tiles) {
  constexpr int N = 32 * N1, T = G * N1;
  constexpr uint32_t OPER = 128 * 128, TILE = 4 * OPER;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const float2* t2 = wn_g;
  const float2* t1 = wn_g + 32 * N1;
  const int nq = 2 * br - 1;
  float2* cs = (float2*)smem_raw;                        // [G][nq]
  float2* vs = cs + ((G * nq + 1) & ~1);                 // [G][N / 2]: one half of the rows, column-major so that
                                                         // consecutive lanes (rows) hit consecutive banks
  const int tid = threadIdx.x, g = tid / N1, n1 = tid % N1;
  const long long i = blockIdx.y;
  const int qc0 = blockIdx.x * G;
  pdl_trigger();
  pdl_wait();   // ihat comes from the coarse spectrum
  for (int e = tid; e < G * nq; e += T) {
    const int jr = e / G, gg = e % G, qc = qc0 + gg;
    cs[gg * nq + jr] = qc < bc ? ihat[(i * nq + jr) * (long long)bc + qc] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2 z[32];
  inverse_gather<N1>(z, cs + g * nq, br - 1, t2, t1, n1);
  // z[k] is row n1 + N1 bitrev5(k): even k give the first half of the rows, odd k the second.  The rows are
  // transposed through shared memory one half at a time (half the buffer: more blocks per SM, one wave).
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    if (h) __syncthreads();   // the first half has been stored
#pragma unroll
    for (int k = h; k < 32; k += 2) vs[g * (N / 2) + n1 + N1 * (bitrev5(k) - 16 * h)] = z[k];
    __syncthreads();
    // QPT band columns per store: 8 (one 16-byte chunk of the bf16 row) or, for G = 4, 4 (half a chunk)
    constexpr int QPT = G < 8 ? G : 8;
    for (int it = tid; it < (N / 2) * (G / QPT); it += T) {
      const int yh = it % (N / 2), gq = it / (N / 2), y = yh + h * (N / 2);
      const int qf = qc0 + QPT * gq, q = qf >> 3;
      const float2* src = vs + (QPT * gq) * (N / 2) + yh;
      float re[QPT], im[QPT];
#pragma unroll
      for (int e = 0; e < QPT; ++e) {
        const float2 x = src[e * (N / 2)];
        re[e] = x.x, im[e] = x.y;
      }
      uint32_t rh[QPT / 2], rl[QPT / 2], ih[QPT / 2], il[QPT / 2];
#pragma unroll
      for (int e = 0; e < QPT / 2; ++e) {
        tc::split2(re[2 * e], re[2 * e + 1], rh[e], rl[e]);
        tc::split2(im[2 * e], im[2 * e + 1], ih[e], il[e]);
      }
      const long long row = i * ny + y;
      unsigned char* o = tiles + (row >> 7) * TILE + tc::swz((int)(row & 127), q);
      if constexpr (QPT == 8) {
        *(uint4*)o = make_uint4(rh[0], rh[1], rh[2], rh[3]);
        *(uint4*)(o + OPER) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
        *(uint4*)(o + 2 * OPER) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
        *(uint4*)(o + 3 * OPER) = make_uint4(il[0], il[1], il[2], il[3]);
      } else {
        o += 2 * (qf & 7);   // the half of the chunk holding band columns qf .. qf + 3
        *(uint2*)o = make_uint2(rh[0], rh[1]);
        *(uint2*)(o + OPER) = make_uint2(ih[0], ih[1]);
        *(uint2*)(o + 2 * OPER) = make_uint2(rl[0], rl[1]);
        *(uint2*)(o + 3 * OPER) = make_uint2(il[0], il[1]);
      }
    }
  }
}

template <int N1, int G>
static int cols_inv_tiles(const float2* ihat, int count, int br, int bc, int ny, const float2* wn_y,
                          unsigned char* tiles, cudaStream_t s) {
  const size_t smem = sizeof(float2) * (((size_t)G * (2 * br - 1) + 1) & ~(size_t)1) + sizeof(float2) * 16 * N1 * G;
  int rc = set_smem(cols_inv_tiles_kernel<N1, G>, smem, "oi_coarse_to_image_tc/cols");
  if (rc) return rc;
  dim3 grid(64 / G, (unsigned)count);
  (void)launch_pdl(cols_inv_tiles_kernel<N1, G>, grid, dim3(G * N1), smem, s, ihat, br, bc, ny, wn_y, tiles);
  oi::note_launch();
  return check_launch("oi_coarse_to_image_tc/cols");
}

// --------------------------------------------------------------------------------- inverse, rows
// v[i][qc][y] (qc = 0..bc-1, qc > 0 doubled) -> out[i][y][x] = sum_qc Re(v exp(-2 pi i qc x / nx))
template <int N1>
__global__ void __launch_bounds__(256, 3) fft_rows_inv_kernel(const float2* __restrict__ v, long long nrows, int ny,
                                                           int bc, const float2* __restrict__ wn_g,
                                                           float* __restrict__ out) {
  constexpr int N = 32 * N1, G = 256 / N1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const float2* t2 = wn_g;
  const float2* t1 = wn_g + 32 * N1;
  const int nq = 2 * bc - 1;
  float2* vs = (float2*)smem_raw;      // [bc][2G + 1] (padded against bank conflicts)
  float2* cs = vs + bc * (2 * G + 1);  // [G][nq]
  const int tid = threadIdx.x, g = tid / N1, n1 = tid % N1;
  const long long rblk = (long long)blockIdx.x * (2 * G);
  for (int e = tid; e < bc * 2 * G; e += 256) {
    const int qc = e / (2 * G), rr = e % (2 * G);
    const long long r = rblk + rr;
    float2 c = make_float2(0.f, 0.f);
    if (r < nrows) {
      const long long i = r / ny;
      const int y = (int)(r - i * ny);
      c = v[(i * bc + qc) * (long long)ny + y];
    }
    vs[qc * (2 * G + 1) + rr] = c;
  }
  __syncthreads();
  // Hermitian spectra of the row pair packed as F_a + i F_b, q in [-(bc-1), bc-1]
  for (int e = tid; e < G * nq; e += 256) {
    const int gg = e / nq, j = e % nq, q = j - (bc - 1), aq = q < 0 ? -q : q;
    float2 a = vs[aq * (2 * G + 1) + 2 * gg], b = vs[aq * (2 * G + 1) + 2 * gg + 1];
    const float h = aq == 0 ? 1.0f : 0.5f;
    if (q < 0) {
      a.y = -a.y;
      b.y = -b.y;
    }
    cs[e] = make_float2(h * (a.x - b.y), h * (a.y + b.x));  // h (a + i b)
  }
  __syncthreads();
  const long long r0 = rblk + 2 * g;
  float2 z[32];
  inverse_gather<N1>(z, cs + g * nq, bc - 1, t2, t1, n1);
  if (r0 >= nrows) return;
  float* o0 = out + r0 * N;
  float* o1 = o0 + N;
  const bool second = r0 + 1 < nrows;
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    const int x = n1 + N1 * bitrev5(i);
    o0[x] = z[i].x;
    if (second) o1[x] = z[i].y;
  }
}

// --------------------------------------------------------------- coarse intensity -> its spectrum
// COARSE_PARTS blocks per coarse image, each for a range of the band columns qc (mr = 32 N1R, mc = 32 N1C, each
// 64 or 128; U holds the block's columns only, so that two blocks fit an SM):
//   ihat[i][jr][qc] = (qc ? 2 : 1) / (mr mc) * sum_{sr,sc} coarse[i][sr][sc] exp(+2 pi i (qr sr/mr + qc sc/mc))
// for qr = jr - (br-1) in [-(br-1), br-1] and qc in [0, bc).  Row FFTs of the real image in pairs (two rows per
// complex transform), the band bins of each separated into U[sr][qc]; then column FFTs of U at the qr bins.
constexpr int COARSE_PARTS = 2;
template <int N1R, int N1C>
__global__ void __launch_bounds__(512) coarse_spec_fft_kernel(const float* __restrict__ coarse, int nparts,
                                                              long long part_stride, int br, int bc,
                                                              const float2* __restrict__ wr_g,
                                                              const float2* __restrict__ wc_g, int area_f2,
                                                              float2* __restrict__ ihat) {
  constexpr int MR = 32 * N1R, MC = 32 * N1C, T = 512;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* r2 = (float2*)smem_raw;      // row-axis (MR) tables: [32][N1R], [N1R][N1R]
  float2* r1 = r2 + 32 * N1R;
  float2* c2 = r1 + N1R * N1R;         // column-axis (MC) tables: [32][N1C], [N1C][N1C]
  float2* c1t = c2 + 32 * N1C;
  float2* area = c1t + N1C * N1C;      // [area_f2] union: coarse image / row transposes / column transposes
  float2* u = area + area_f2;          // [MR][cw]: this block's band columns
  const int tid = threadIdx.x;
  const long long img = blockIdx.x;
  // this block's band columns: blockIdx.y-th of gridDim.y equal ranges of [0, bc)
  const int cw = (bc + gridDim.y - 1) / gridDim.y, c0 = blockIdx.y * cw, c1 = min(bc, c0 + cw);
  build_tables<N1R>(wr_g, r2, r1, tid, T);
  build_tables<N1C>(wc_g, c2, c1t, tid, T);
  pdl_trigger();
  pdl_wait();   // the partial coarse images come from the coherent sum
  float* cimg = (float*)area;
  const float4* src = (const float4*)(coarse + img * (long long)MR * MC);
  constexpr int PER = MR * MC / 4 / T;   // float4 per thread
  float4 acc[PER];
#pragma unroll
  for (int k = 0; k < PER; ++k) acc[k] = __ldg(src + tid + T * k);
  for (int p = 1; p < nparts; ++p) {   // the partial sums, added in order; all loads of a part in flight together
    float4 x[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) x[k] = __ldg(src + p * (part_stride / 4) + tid + T * k);
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      acc[k].x += x[k].x;
      acc[k].y += x[k].y;
      acc[k].z += x[k].z;
      acc[k].w += x[k].w;
    }
  }
#pragma unroll
  for (int k = 0; k < PER; ++k) ((float4*)cimg)[tid + T * k] = acc[k];
  __syncthreads();
  // row pass: pair p = rows (2p, 2p+1), thread n1
  const int p = tid / N1C, n1 = tid % N1C;
  const bool row_task = p < MR / 2;
  float2 z[32];
  if (row_task) {
#pragma unroll
    for (int n2 = 0; n2 < 32; ++n2)
      z[n2] = make_float2(cimg[(2 * p) * MC + n1 + N1C * n2], cimg[(2 * p + 1) * MC + n1 + N1C * n2]);
    fft32<+1>(z);
  }
  __syncthreads();  // the image is consumed; the area now holds row transposes
  if (row_task) twiddle_store<+1, N1C>(z, c2, n1, area + p * 32 * (N1C + 1));
  __syncthreads();
  for (int e = tid; e < (MR / 2) * (c1 - c0); e += T) {
    const int pp = e / (c1 - c0), qc = c0 + e % (c1 - c0);
    const float2* ys = area + pp * 32 * (N1C + 1);
    const float2 zp = outer_bin<+1, N1C>(ys, c1t, qc & (MC - 1));
    const float2 zm = outer_bin<+1, N1C>(ys, c1t, (-qc) & (MC - 1));
    u[(2 * pp) * cw + qc - c0] = make_float2(0.5f * (zp.x + zm.x), 0.5f * (zp.y - zm.y));
    u[(2 * pp + 1) * cw + qc - c0] = make_float2(0.5f * (zp.y + zm.y), -0.5f * (zp.x - zm.x));
  }
  __syncthreads();
  // column pass: column qc of U, thread n1r
  const int qc = c0 + tid / N1R, n1r = tid % N1R;
  const bool col_task = qc < c1;
  if (col_task) {
#pragma unroll
    for (int n2 = 0; n2 < 32; ++n2) z[n2] = u[(n1r + N1R * n2) * cw + qc - c0];
    fft32<+1>(z);
  }
  __syncthreads();  // row transposes are consumed; the area now holds column transposes
  if (col_task) twiddle_store<+1, N1R>(z, r2, n1r, area + (qc - c0) * 32 * (N1R + 1));
  __syncthreads();
  const int nq = 2 * br - 1;
  const float norm = 1.0f / ((float)MR * (float)MC);
  for (int e = tid; e < nq * (c1 - c0); e += T) {
    const int jr = e / (c1 - c0), c = c0 + e % (c1 - c0);
    const float2 v = outer_bin<+1, N1R>(area + (c - c0) * 32 * (N1R + 1), r1, (jr - (br - 1)) & (MR - 1));
    const float s = (c == 0 ? 1.0f : 2.0f) * norm;
    ihat[(img * nq + jr) * (long long)bc + c] = make_float2(v.x * s, v.y * s);
  }
}

template <int N1R, int N1C>
static int launch_coarse_spec_fft(float* coarse, int nparts, int count, int br, int bc, const float2* wr,
                                  const float2* wc, float2* ihat, cudaStream_t s) {
  constexpr int MR = 32 * N1R, MC = 32 * N1C;
  const int cw = (bc + COARSE_PARTS - 1) / COARSE_PARTS;   // band columns per block (as in the kernel)
  const int rows_ys = (MR / 2) * 32 * (N1C + 1), c_f2 = MR * MC / 2, cols_ys = cw * 32 * (N1R + 1);
  const int area_f2 = max(rows_ys, max(c_f2, cols_ys));
  const size_t smem = sizeof(float2) * ((size_t)table_f2<N1R>() + table_f2<N1C>() + area_f2 + (size_t)MR * cw);
  auto kern = coarse_spec_fft_kernel<N1R, N1C>;
  int rc = set_smem(kern, smem, "coarse spectrum fft");
  if (rc) return rc;
  (void)launch_pdl(kern, dim3((unsigned)count, COARSE_PARTS), dim3(512), smem, s, (const float*)coarse, nparts,
                   (long long)count * MR * MC, br, bc, wr, wc, area_f2, ihat);
  oi::note_launch();
  return check_launch("coarse spectrum fft");
}

template <int N1>
static size_t smem_rows_fwd(int nu) { return sizeof(float2) * ((256 / N1) * 32 * (N1 + 1) + (256 / N1) * nu); }
template <int N1>
static size_t smem_cols_fwd() { return sizeof(float2) * ((COLS_T / N1) * 32 * (N1 + 1)); }


template <int N1>
static int band_fft(const void* field, int kind, int batch, int ny, int nx, int m0r, int br, int m0c, int bc,
                    const float2* wn_x, const float2* wn_y, float scale, float2* t, float2* band, cudaStream_t s,
                    int nparts = 1, long long pstride = 0) {
  // row transforms have length nx = 32 * N1; the column kernel picks its own N1 for ny
  const int u0 = min(m0c, -(m0c + bc - 1)), u1 = max(m0c + bc - 1, -m0c), nu = u1 - u0 + 1;
  constexpr int G = 256 / N1;
  const long long nrows = (long long)batch * ny;
  size_t smem = smem_rows_fwd<N1>(nu);
  int rc;
  if (kind == OI_FIELD_U8) {
    rc = set_smem(fft_rows_fwd_kernel<N1, OI_FIELD_U8>, smem, "oi_band_spectrum_fft/rows");
    if (rc) return rc;
    fft_rows_fwd_kernel<N1, OI_FIELD_U8><<<(unsigned)ceil_div(nrows, 2 * G), 256, smem, s>>>(
        field, nrows, ny, wn_x, m0c, bc, u0, nu, t, 1, 0LL);
    oi::note_launch();
  } else {
    rc = set_smem(fft_rows_fwd_kernel<N1, OI_FIELD_REAL_F32>, smem, "oi_band_spectrum_fft/rows");
    if (rc) return rc;
    fft_rows_fwd_kernel<N1, OI_FIELD_REAL_F32><<<(unsigned)ceil_div(nrows, 2 * G), 256, smem, s>>>(
        field, nrows, ny, wn_x, m0c, bc, u0, nu, t, nparts, pstride);
    oi::note_launch();
  }
  return check_launch("oi_band_spectrum_fft/rows");
}

// bco: the output band width (SYM: bc = (bco + 1) / 2 input columns; else bco = bc)
template <int N1, bool SYM = false>
static int cols_fwd(const float2* t, int batch, int bc, const float2* wn_y, int m0r, int br, float scale,
                    float2* band, cudaStream_t s, int bco = 0, int dbl_from = 0x7fffffff) {
  constexpr int G = COLS_T / N1;
  if ((uintptr_t)t % 16) return fail(OI_EINVAL, "oi_band_spectrum_fft/cols: scratch must be 16-byte aligned");
  size_t smem = smem_cols_fwd<N1>();
  int rc = set_smem(fft_cols_fwd_kernel<N1, SYM>, smem, "oi_band_spectrum_fft/cols");
  if (rc) return rc;
  const long long ncols = (long long)batch * bc;
  (void)launch_pdl(fft_cols_fwd_kernel<N1, SYM>, dim3((unsigned)ceil_div(ncols, G)), dim3(COLS_T), smem, s,
                   (const float2*)t, ncols, bc, wn_y, m0r, br, scale, band, SYM ? bco : bc, dbl_from);
  oi::note_launch();
  return check_launch("oi_band_spectrum_fft/cols");
}

template <int N1>
static int cols_inv(const float2* ihat, int count, int br, int bc, const float2* wn_y, float2* v, cudaStream_t s) {
  constexpr int G = 256 / N1;
  size_t smem = sizeof(float2) * (G * (2 * br - 1));
  int rc = set_smem(fft_cols_inv_kernel<N1>, smem, "oi_coarse_to_image_fft/cols");
  if (rc) return rc;
  const long long ncols = (long long)count * bc;
  fft_cols_inv_kernel<N1><<<(unsigned)ceil_div(ncols, G), 256, smem, s>>>(ihat, ncols, br, bc, wn_y, v);
  oi::note_launch();
  return check_launch("oi_coarse_to_image_fft/cols");
}

template <int N1>
static int rows_inv(const float2* v, int count, int ny, int bc, const float2* wn_x, float* out, cudaStream_t s) {
  constexpr int G = 256 / N1;
  size_t smem = sizeof(float2) * (bc * (2 * G + 1) + G * (2 * bc - 1));
  int rc = set_smem(fft_rows_inv_kernel<N1>, smem, "oi_coarse_to_image_fft/rows");
  if (rc) return rc;
  const long long nrows = (long long)count * ny;
  fft_rows_inv_kernel<N1><<<(unsigned)ceil_div(nrows, 2 * G), 256, smem, s>>>(v, nrows, ny, bc, wn_x, out);
  oi::note_launch();
  return check_launch("oi_coarse_to_image_fft/rows");
}

static int n1_of(int n) {
  switch (n) {
    case 256: return 8;
    case 512: return 16;
    case 1024: return 32;
    case 2048: return 64;
  }
  return 0;
}

}  // namespace oi

extern "C" int oi_fft_supported(int ny, int nx) {
  return oi::n1_of(ny) != 0 && oi::n1_of(nx) != 0 ? 1 : 0;
}

extern "C" int oi_band_spectrum_fft(const void* field, int kind, int batch, int ny, int nx, int m0r, int br, int m0c,
                                    int bc, const void* wn_x, const void* wn_y, float scale, void* scratch,
                                    void* band, void* stream) {
  using namespace oi;
  if (!field || !wn_x || !wn_y || !scratch || !band || batch <= 0 || br <= 0 || bc <= 0)
    return fail(OI_EINVAL, "oi_band_spectrum_fft: bad arguments");
  if (kind != OI_FIELD_REAL_F32 && kind != OI_FIELD_U8)
    return fail(OI_EINVAL, "oi_band_spectrum_fft: real float32 or uint8 masks only (kind=%d)", kind);
  const int nx1 = n1_of(nx), ny1 = n1_of(ny);
  if (!nx1 || !ny1) return fail(OI_ERANGE, "oi_band_spectrum_fft: grid %dx%d is not 256..2048, power of 2", ny, nx);
  const int maxc = max(abs(m0c), abs(m0c + bc - 1));
  if (2 * maxc >= nx || br > ny)
    return fail(OI_ERANGE, "oi_band_spectrum_fft: band (%d+%d, %d+%d) too wide for %dx%d", m0r, br, m0c, bc, ny, nx);
  cudaStream_t s = (cudaStream_t)stream;
  float2* t = (float2*)scratch;
  int rc;
  switch (nx1) {
    case 8: rc = band_fft<8>(field, kind, batch, ny, nx, m0r, br, m0c, bc, (const float2*)wn_x, (const float2*)wn_y, scale, t, (float2*)band, s); break;
    case 16: rc = band_fft<16>(field, kind, batch, ny, nx, m0r, br, m0c, bc, (const float2*)wn_x, (const float2*)wn_y, scale, t, (float2*)band, s); break;
    case 32: rc = band_fft<32>(field, kind, batch, ny, nx, m0r, br, m0c, bc, (const float2*)wn_x, (const float2*)wn_y, scale, t, (float2*)band, s); break;
    default: rc = band_fft<64>(field, kind, batch, ny, nx, m0r, br, m0c, bc, (const float2*)wn_x, (const float2*)wn_y, scale, t, (float2*)band, s); break;
  }
  if (rc) return rc;
  switch (ny1) {
    case 8: return cols_fwd<8>(t, batch, bc, (const float2*)wn_y, m0r, br, scale, (float2*)band, s);
    case 16: return cols_fwd<16>(t, batch, bc, (const float2*)wn_y, m0r, br, scale, (float2*)band, s);
    case 32: return cols_fwd<32>(t, batch, bc, (const float2*)wn_y, m0r, br, scale, (float2*)band, s);
    default: return cols_fwd<64>(t, batch, bc, (const float2*)wn_y, m0r, br, scale, (float2*)band, s);
  }
}

// The Hermitian half-spectrum of a coarse intensity held as nparts partial sums (oi_coherent_coarse_fft's output,
// [nparts][count][mr][mc] float32): ihat[i][qr + br-1][qc] = w(qc) / (mr mc) sum_{y,x} (sum_p coarse[p][i][y][x])
// exp(+2 pi i (qr y / mr + qc x / mc)), |qr| < br, 0 <= qc < bc, w(0) = 1 and w(qc > 0) = 2 -- the input of
// oi_spectrum_to_image_fft.  The parts are summed in the row pass's loads; scratch: count * mr * bc complex.
extern "C" int oi_coarse_half_spectrum_fft(const float* coarse, int nparts, int count, int mr, int mc, int br, int bc,
                                           const void* wn_c, const void* wn_r, void* scratch, void* ihat,
                                           void* stream) {
  using namespace oi;
  if (!coarse || !wn_c || !wn_r || !scratch || !ihat || nparts <= 0 || count <= 0 || br <= 0 || bc <= 0)
    return fail(OI_EINVAL, "oi_coarse_half_spectrum_fft: bad arguments");
  const int nx1 = n1_of(mc), ny1 = n1_of(mr);
  if (!nx1 || !ny1)
    return fail(OI_ERANGE, "oi_coarse_half_spectrum_fft: coarse grid %dx%d is not 256..2048, power of 2", mr, mc);
  if (2 * (bc - 1) >= mc || 2 * br - 1 > mr)
    return fail(OI_ERANGE, "oi_coarse_half_spectrum_fft: band %dx%d too wide for %dx%d", br, bc, mr, mc);
  cudaStream_t s = (cudaStream_t)stream;
  float2* t = (float2*)scratch;
  float2* out = (float2*)ihat;
  const int nq = 2 * br - 1, m0r = -(br - 1);
  const float scale = 1.f / ((float)mr * (float)mc);
  const long long pstride = (long long)count * mr * mc;
  int rc;
  switch (nx1) {
    case 8: rc = band_fft<8>(coarse, OI_FIELD_REAL_F32, count, mr, mc, m0r, nq, 0, bc, (const float2*)wn_c, (const float2*)wn_r, scale, t, out, s, nparts, pstride); break;
    case 16: rc = band_fft<16>(coarse, OI_FIELD_REAL_F32, count, mr, mc, m0r, nq, 0, bc, (const float2*)wn_c, (const float2*)wn_r, scale, t, out, s, nparts, pstride); break;
    case 32: rc = band_fft<32>(coarse, OI_FIELD_REAL_F32, count, mr, mc, m0r, nq, 0, bc, (const float2*)wn_c, (const float2*)wn_r, scale, t, out, s, nparts, pstride); break;
    default: rc = band_fft<64>(coarse, OI_FIELD_REAL_F32, count, mr, mc, m0r, nq, 0, bc, (const float2*)wn_c, (const float2*)wn_r, scale, t, out, s, nparts, pstride); break;
  }
  if (rc) return rc;
  switch (ny1) {
    case 8: return cols_fwd<8>(t, count, bc, (const float2*)wn_r, m0r, nq, scale, out, s, 0, 1);
    case 16: return cols_fwd<16>(t, count, bc, (const float2*)wn_r, m0r, nq, scale, out, s, 0, 1);
    case 32: return cols_fwd<32>(t, count, bc, (const float2*)wn_r, m0r, nq, scale, out, s, 0, 1);
    default: return cols_fwd<64>(t, count, bc, (const float2*)wn_r, m0r, nq, scale, out, s, 0, 1);
  }
}

extern "C" int oi_coarse_to_image_fft(float* coarse, int nparts, int count, int mr, int mc, int br, int bc,
                                      const void* gc, const void* gr, const void* wm_r, const void* wm_c,
                                      const void* wn_y, const void* wn_x, int ny, int nx, void* scratch_ihat,
                                      void* scratch_v, float* out, void* stream) {
  using namespace oi;
  if (!coarse || !gc || !gr || !wn_y || !wn_x || !scratch_ihat || !scratch_v || !out || count <= 0 || nparts <= 0)
    return fail(OI_EINVAL, "oi_coarse_to_image_fft: bad arguments");
  const int nx1 = n1_of(nx), ny1 = n1_of(ny);
  if (!nx1 || !ny1) return fail(OI_ERANGE, "oi_coarse_to_image_fft: grid %dx%d is not 256..2048, power of 2", ny, nx);
  if (2 * br - 1 > ny || 2 * bc - 1 > nx) return fail(OI_ERANGE, "oi_coarse_to_image_fft: band too wide for grid");
  cudaStream_t s = (cudaStream_t)stream;
  int rc;
  if (wm_r && wm_c && (mr == 64 || mr == 128) && (mc == 64 || mc == 128) && bc <= 64) {
    float2* ih = (float2*)scratch_ihat;
    const float2 *tr = (const float2*)wm_r, *tc = (const float2*)wm_c;
    if (mr == 128 && mc == 128) rc = launch_coarse_spec_fft<4, 4>(coarse, nparts, count, br, bc, tr, tc, ih, s);
    else if (mr == 64 && mc == 64) rc = launch_coarse_spec_fft<2, 2>(coarse, nparts, count, br, bc, tr, tc, ih, s);
    else if (mr == 128) rc = launch_coarse_spec_fft<4, 2>(coarse, nparts, count, br, bc, tr, tc, ih, s);
    else rc = launch_coarse_spec_fft<2, 4>(coarse, nparts, count, br, bc, tr, tc, ih, s);
  } else {
    rc = coarse_spectrum(coarse, count, mr, mc, br, bc, gc, gr, scratch_ihat, s, nparts);
  }
  if (rc) return rc;
  const float2* ih = (const float2*)scratch_ihat;
  float2* v = (float2*)scratch_v;
  switch (ny1) {
    case 8: rc = cols_inv<8>(ih, count, br, bc, (const float2*)wn_y, v, s); break;
    case 16: rc = cols_inv<16>(ih, count, br, bc, (const float2*)wn_y, v, s); break;
    case 32: rc = cols_inv<32>(ih, count, br, bc, (const float2*)wn_y, v, s); break;
    default: rc = cols_inv<64>(ih, count, br, bc, (const float2*)wn_y, v, s); break;
  }
  if (rc) return rc;
  switch (nx1) {
    case 8: return rows_inv<8>(v, count, ny, bc, (const float2*)wn_x, out, s);
    case 16: return rows_inv<16>(v, count, ny, bc, (const float2*)wn_x, out, s);
    case 32: return rows_inv<32>(v, count, ny, bc, (const float2*)wn_x, out, s);
    default: return rows_inv<64>(v, count, ny, bc, (const float2*)wn_x, out, s);
  }
}

extern "C" int oi_spectrum_to_image_fft(const void* ihat, int count, int br, int bc, const void* wn_y,
                                        const void* wn_x, int ny, int nx, void* scratch_v, float* out,
                                        void* stream) {
  using namespace oi;
  if (!ihat || !wn_y || !wn_x || !scratch_v || !out || count <= 0 || br <= 0 || bc <= 0)
    return fail(OI_EINVAL, "oi_spectrum_to_image_fft: bad arguments");
  const int nx1 = n1_of(nx), ny1 = n1_of(ny);
  if (!nx1 || !ny1) return fail(OI_ERANGE, "oi_spectrum_to_image_fft: grid %dx%d is not 256..2048, power of 2", ny, nx);
  if (2 * br - 1 > ny || 2 * bc - 1 > nx) return fail(OI_ERANGE, "oi_spectrum_to_image_fft: band too wide for grid");
  cudaStream_t s = (cudaStream_t)stream;
  const float2* ih = (const float2*)ihat;
  float2* v = (float2*)scratch_v;
  int rc;
  switch (ny1) {
    case 8: rc = cols_inv<8>(ih, count, br, bc, (const float2*)wn_y, v, s); break;
    case 16: rc = cols_inv<16>(ih, count, br, bc, (const float2*)wn_y, v, s); break;
    case 32: rc = cols_inv<32>(ih, count, br, bc, (const float2*)wn_y, v, s); break;
    default: rc = cols_inv<64>(ih, count, br, bc, (const float2*)wn_y, v, s); break;
  }
  if (rc) return rc;
  switch (nx1) {
    case 8: return rows_inv<8>(v, count, ny, bc, (const float2*)wn_x, out, s);
    case 16: return rows_inv<16>(v, count, ny, bc, (const float2*)wn_x, out, s);
    case 32: return rows_inv<32>(v, count, ny, bc, (const float2*)wn_x, out, s);
    default: return rows_inv<64>(v, count, ny, bc, (const float2*)wn_x, out, s);
  }
}

// Split-BF16x3 tensor-core form of oi_band_spectrum_fft: the row pass is oi_rows_fwd_tc (a DFT contraction
// on the tensor cores against the constant image `wconsts` of oi_rows_tc_constants(0, ...)), the column pass
// the FFT above.
extern "C" int oi_band_spectrum_tc(const void* field, int kind, int batch, int ny, int nx, int m0r, int br, int m0c,
                                   int bc, const void* wconsts, const void* wn_y, float scale, void* scratch,
                                   void* band, void* stream) {
  using namespace oi;
  if (!field || !wconsts || !wn_y || !scratch || !band || batch <= 0 || br <= 0 || bc <= 0)
    return fail(OI_EINVAL, "oi_band_spectrum_tc: bad arguments");
  const int ny1 = n1_of(ny);
  if (!ny1 || nx % 128 != 0 || nx > 4096)
    return fail(OI_ERANGE, "oi_band_spectrum_tc: grid %dx%d unsupported", ny, nx);
  if (bc > 64 || br > ny) return fail(OI_ERANGE, "oi_band_spectrum_tc: band %dx%d unsupported", br, bc);
  int rc = oi_rows_fwd_tc(field, kind, batch, ny, nx, m0c, bc, wconsts, scratch, stream);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const float2* t = (const float2*)scratch;
  switch (ny1) {
    case 8: return cols_fwd<8>(t, batch, bc, (const float2*)wn_y, m0r, br, scale, (float2*)band, s);
    case 16: return cols_fwd<16>(t, batch, bc, (const float2*)wn_y, m0r, br, scale, (float2*)band, s);
    case 32: return cols_fwd<32>(t, batch, bc, (const float2*)wn_y, m0r, br, scale, (float2*)band, s);
    default: return cols_fwd<64>(t, batch, bc, (const float2*)wn_y, m0r, br, scale, (float2*)band, s);
  }
}

// oi_band_spectrum_tc for a symmetric band (m0r = -(br-1)/2, m0c = -(bc-1)/2, br and bc odd, bc <= 63): the row
// pass computes only the band's non-negative columns (oi_rows_fwd_tc_half against `hconsts` of
// oi_rows_tc_constants(2, nx, m0c, bc, ...)) and the column pass fills the negative ones from
// band[-ky][-kx] = conj(band[ky][kx]) (a real mask).  scratch: batch * ny * (bc+1)/2 complex.
extern "C" int oi_band_spectrum_tc_sym(const void* field, int kind, int batch, int ny, int nx, int br, int bc,
                                       const void* hconsts, const void* wn_y, float scale, void* scratch, void* band,
                                       void* stream) {
  using namespace oi;
  if (!field || !hconsts || !wn_y || !scratch || !band || batch <= 0 || br <= 0 || bc <= 0)
    return fail(OI_EINVAL, "oi_band_spectrum_tc_sym: bad arguments");
  const int ny1 = n1_of(ny);
  if (!ny1 || nx % 128 != 0 || nx > 4096)
    return fail(OI_ERANGE, "oi_band_spectrum_tc_sym: grid %dx%d unsupported", ny, nx);
  if (bc % 2 == 0 || br % 2 == 0 || bc > 63 || br > ny)
    return fail(OI_ERANGE, "oi_band_spectrum_tc_sym: band %dx%d is not an odd symmetric band of width <= 63", br, bc);
  const int bch = (bc + 1) / 2, m0r = -(br - 1) / 2;
  int rc = oi_rows_fwd_tc_half(field, kind, batch, ny, nx, bch, hconsts, scratch, stream);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const float2* t = (const float2*)scratch;
  switch (ny1) {
    case 8: return cols_fwd<8, true>(t, batch, bch, (const float2*)wn_y, m0r, br, scale, (float2*)band, s, bc);
    case 16: return cols_fwd<16, true>(t, batch, bch, (const float2*)wn_y, m0r, br, scale, (float2*)band, s, bc);
    case 32: return cols_fwd<32, true>(t, batch, bch, (const float2*)wn_y, m0r, br, scale, (float2*)band, s, bc);
    default: return cols_fwd<64, true>(t, batch, bch, (const float2*)wn_y, m0r, br, scale, (float2*)band, s, bc);
  }
}

// Split-BF16x3 tensor-core form of oi_coarse_to_image_fft on the 128 x 128 coarse grid: fold, coarse spectrum
// and column pass as there; the row pass is oi_rows_inv_tc against `cconsts` of oi_rows_tc_constants(1, ...).
extern "C" int oi_coarse_to_image_tc(float* coarse, int nparts, int count, int br, int bc, const void* wm_r,
                                     const void* wm_c, const void* wn_y, const void* cconsts, int ny, int nx,
                                     void* scratch_ihat, void* scratch_v, void* scratch_tiles, float* out,
                                     void* stream) {
  using namespace oi;
  (void)scratch_v;
  if (!coarse || !wm_r || !wm_c || !wn_y || !cconsts || !scratch_ihat || !scratch_tiles || !out || count <= 0 ||
      nparts <= 0 || br <= 0 || bc <= 0)
    return fail(OI_EINVAL, "oi_coarse_to_image_tc: bad arguments");
  const int ny1 = n1_of(ny);
  if (!ny1 || nx % 128 != 0 || nx > 4096 || bc > 64 || 2 * br - 1 > 128 || 2 * br - 1 > ny)
    return fail(OI_ERANGE, "oi_coarse_to_image_tc: grid %dx%d / band %dx%d unsupported", ny, nx, br, bc);
  cudaStream_t s = (cudaStream_t)stream;
  float2* ih = (float2*)scratch_ihat;
  int rc = launch_coarse_spec_fft<4, 4>(coarse, nparts, count, br, bc, (const float2*)wm_r, (const float2*)wm_c, ih, s);
  if (rc) return rc;
  unsigned char* tiles = (unsigned char*)scratch_tiles;
  const float2* wy = (const float2*)wn_y;
  switch (ny1) {
    case 8: rc = cols_inv_tiles<8, 32>(ih, count, br, bc, ny, wy, tiles, s); break;
    case 16: rc = cols_inv_tiles<16, 16>(ih, count, br, bc, ny, wy, tiles, s); break;
    case 32: rc = cols_inv_tiles<32, 8>(ih, count, br, bc, ny, wy, tiles, s); break;
    default: rc = cols_inv_tiles<64, 8>(ih, count, br, bc, ny, wy, tiles, s); break;
  }
  if (rc) return rc;
  return rows_inv_from_tiles(tiles, count, ny, nx, cconsts, out, s);
}
