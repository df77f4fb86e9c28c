// FP64 top-K eigenpairs of a Hermitian positive semi-definite operator, for the SOCS decomposition
// (DecomposeTCC_SOCS.py:7-9, where the reference takes a full torch.svd of its complex64 TCC and keeps the
// leading K singular pairs).  Block subspace iteration with Rayleigh-Ritz, on the GPU, in double precision:
//
//   X = orthonormal(random n x p)
//   repeat:   Y = T X,   X = CholQR2(Y)                      (Cholesky QR twice: X^H X = I to rounding)
//   every `check` iterations: Z = T X, H = X^H Z (p x p), H = Q diag(w) Q^H (cyclic Jacobi), residuals
//             ||Z q_i - w_i X q_i|| of the leading k; stop when their maximum is below tol * w_0.
//   result:   the Ritz pairs (w_i, X q_i), i < k, eigenvalues descending and clamped at zero.
//
// The subspace converges like (lambda_{p+1} / lambda_k)^iterations; the TCC's spectrum decays, so a block of
// p = 64 vectors resolves the leading 24 of the 2048 nm configuration (lambda_65 / lambda_24 = 0.21) to a
// rank-24 projector error of 1e-12 in about 16 iterations.  T is a dense n x n matrix or the factored form
// T = sum_e h_e h_e^H (h [ne][n][s], the scaled pupil matrix of CalculateTCCMatrix.py:33-51), applied without
// forming T.  Kernels: a tiled complex FP64 GEMM (row-major, optional conjugate transpose of A, split over K
// with partial sums added in a fixed order), and one-CTA kernels for the p x p steps (Cholesky and triangular
// inverse, Jacobi eigendecomposition, residual norms).
#include "oi_common.cuh"
#include <cstdint>
#include <vector>
#include <cmath>

namespace oi {
namespace eg {

constexpr int BM = 32, BN = 32, BK = 16;   // GEMM tile
constexpr int PMAX = 64;                   // block size limit of the one-CTA steps

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 conjd(double2 a) { return make_double2(a.x, -a.y); }

// C[z][m][n] = sum_{kk in chunk z} op(A)[i][kk] B[kk][j]; op(A) = A (A [m][lda]) or A^H (A [k][lda]).
// With one chunk and acc = 1 the result is added to C.
template <bool AH>
__global__ void __launch_bounds__(256) zgemm_kernel(int m, int n, int k, const double2* __restrict__ A, long long lda,
                                                    const double2* __restrict__ B, long long ldb, double2* C,
                                                    long long ldc, int kchunk, int acc) {
  __shared__ double2 As[BK][BM + 1];
  __shared__ double2 Bs[BK][BN + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN, z = blockIdx.z;
  const int k0 = z * kchunk, k1 = min(k, k0 + kchunk);
  double2 c00 = make_double2(0, 0), c01 = c00, c10 = c00, c11 = c00;
  for (int kt = k0; kt < k1; kt += BK) {
    for (int e = threadIdx.x; e < BM * BK; e += 256) {
      int i, kk;
      if (AH) {   // coalesced along i: A[kt + kk][m0 + i]
        i = e % BM;
        kk = e / BM;
      } else {    // coalesced along kk: A[m0 + i][kt + kk]
        kk = e % BK;
        i = e / BK;
      }
      const int gi = m0 + i, gk = kt + kk;
      double2 v = make_double2(0, 0);
      if (gi < m && gk < k1) v = AH ? conjd(A[(long long)gk * lda + gi]) : A[(long long)gi * lda + gk];
      As[kk][i] = v;
    }
    for (int e = threadIdx.x; e < BK * BN; e += 256) {
      const int j = e % BN, kk = e / BN, gj = n0 + j, gk = kt + kk;
      Bs[kk][j] = (gj < n && gk < k1) ? B[(long long)gk * ldb + gj] : make_double2(0, 0);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      const double2 a0 = As[kk][2 * ty], a1 = As[kk][2 * ty + 1], b0 = Bs[kk][2 * tx], b1 = Bs[kk][2 * tx + 1];
      cfma(c00, a0, b0);
      cfma(c01, a0, b1);
      cfma(c10, a1, b0);
      cfma(c11, a1, b1);
    }
    __syncthreads();
  }
  const int i0 = m0 + 2 * ty, j0 = n0 + 2 * tx;
  double2* Cz = C + (long long)z * m * ldc;
  auto put = [&](int i, int j, double2 v) {
    if (i < m && j < n) {
      double2* p = Cz + (long long)i * ldc + j;
      *p = acc ? cadd(*p, v) : v;
    }
  };
  put(i0, j0, c00);
  put(i0, j0 + 1, c01);
  put(i0 + 1, j0, c10);
  put(i0 + 1, j0 + 1, c11);
}

// out[e] (+)= sum_z parts[z][e], z = 0 .. nparts-1 in order.
__global__ void reduce_parts_kernel(const double2* __restrict__ parts, int nparts, long long count, double2* out,
                                    int acc) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count) return;
  double2 s = acc ? out[e] : make_double2(0, 0);
  for (int z = 0; z < nparts; ++z) s = cadd(s, parts[(long long)z * count + e]);
  out[e] = s;
}

// Deterministic start block: entries uniform in [-1, 1] + i [-1, 1] from a 64-bit mix of their index.
__global__ void start_block_kernel(double2* X, long long count, unsigned long long seed) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count) return;
  auto mix = [](unsigned long long x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
  };
  const unsigned long long a = mix(seed ^ (2ull * e)), b = mix(seed ^ (2ull * e + 1));
  X[e] = make_double2((double)(a >> 11) * 0x1.0p-52 - 1.0, (double)(b >> 11) * 0x1.0p-52 - 1.0);
}

// One CTA: G (p x p Hermitian, row-major) = R^H R with R upper triangular (Cholesky, after adding
// shift_rel * max_j G_jj to the diagonal against rank deficiency), then Rinv = R^-1.
constexpr size_t CHOL_SMEM = sizeof(double2) * PMAX * (PMAX + 1) + 16;
__global__ void __launch_bounds__(256) chol_inv_kernel(int p, const double2* __restrict__ Gin, double2* Rinv,
                                                       double shift_rel) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2 (*G)[PMAX + 1] = (double2 (*)[PMAX + 1])smem_raw;
  double& dmax = *(double*)(smem_raw + sizeof(double2) * PMAX * (PMAX + 1));
  const int t = threadIdx.x;
  for (int e = t; e < p * p; e += 256) G[e / p][e % p] = Gin[e];
  __syncthreads();
  if (t == 0) {
    double m = 0;
    for (int j = 0; j < p; ++j) m = fmax(m, G[j][j].x);
    dmax = m;
  }
  __syncthreads();
  if (t < p) G[t][t].x += shift_rel * dmax;
  __syncthreads();
  for (int j = 0; j < p; ++j) {   // row j of R overwrites row j of G (upper part)
    if (t == 0) {
      const double d = G[j][j].x;
      G[j][j] = make_double2(sqrt(d > 1e-300 ? d : 1e-300), 0.0);
    }
    __syncthreads();
    const double r = G[j][j].x;
    for (int c = j + 1 + t; c < p; c += 256) G[j][c] = make_double2(G[j][c].x / r, G[j][c].y / r);
    __syncthreads();
    const int w = p - j - 1;
    for (int e = t; e < w * w; e += 256) {   // trailing update G[a][b] -= conj(R[j][a]) R[j][b], a <= b
      const int a = j + 1 + e / w, b = j + 1 + e % w;
      if (a <= b) {
        const double2 ra = G[j][a], rb = G[j][b];
        G[a][b].x -= ra.x * rb.x + ra.y * rb.y;
        G[a][b].y -= ra.x * rb.y - ra.y * rb.x;
      }
    }
    __syncthreads();
  }
  // Rinv: column c by back substitution, R Rinv[:, c] = e_c (upper triangular)
  if (t < p) {
    const int c = t;
    double2 x[PMAX];
    for (int i = p - 1; i >= 0; --i) {
      double2 s = make_double2(i == c ? 1.0 : 0.0, 0.0);
      if (i <= c) {
        for (int l = i + 1; l <= c; ++l) {
          const double2 rl = G[i][l];
          s.x -= rl.x * x[l].x - rl.y * x[l].y;
          s.y -= rl.x * x[l].y + rl.y * x[l].x;
        }
        const double r = G[i][i].x;
        x[i] = make_double2(s.x / r, s.y / r);
      } else {
        x[i] = make_double2(0.0, 0.0);
      }
    }
    for (int i = 0; i < p; ++i) Rinv[(long long)i * p + c] = x[i];
  }
}

// One CTA: eigendecomposition of a Hermitian p x p matrix (p even, <= 64) by cyclic Jacobi sweeps in the
// round-robin order (p/2 disjoint rotations per step).  w: eigenvalues descending; Q: row-major, column i the
// eigenvector of w[i].
constexpr size_t JACOBI_SMEM = 2 * sizeof(double2) * PMAX * (PMAX + 1);
__global__ void __launch_bounds__(256) heev_jacobi_kernel(int p, const double2* __restrict__ Hin, double* w,
                                                          double2* Q, int max_sweeps) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2 (*A)[PMAX + 1] = (double2 (*)[PMAX + 1])smem_raw;
  double2 (*V)[PMAX + 1] = (double2 (*)[PMAX + 1])(smem_raw + sizeof(double2) * PMAX * (PMAX + 1));
  __shared__ double2 J[PMAX / 2][4];
  __shared__ int pi[PMAX / 2], pj[PMAX / 2], order[PMAX], perm[PMAX];
  __shared__ double off, tot;
  const int t = threadIdx.x, h = p / 2;
  for (int e = t; e < p * p; e += 256) {
    const int r = e / p, c = e % p;
    A[r][c] = Hin[e];
    V[r][c] = make_double2(r == c ? 1.0 : 0.0, 0.0);
  }
  if (t < p) order[t] = t;
  __syncthreads();
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    if (t == 0) {
      double o = 0, a = 0;
      for (int r = 0; r < p; ++r)
        for (int c = 0; c < p; ++c) {
          const double v = A[r][c].x * A[r][c].x + A[r][c].y * A[r][c].y;
          a += v;
          if (r != c) o += v;
        }
      off = o;
      tot = a;
    }
    __syncthreads();
    if (!(off > 1e-30 * tot)) break;
    for (int step = 0; step < p - 1; ++step) {
      if (t < h) {   // pair t of this step and its rotation (from the matrix before the step)
        int i = order[t], j = order[p - 1 - t];
        if (i > j) {
          const int s = i;
          i = j;
          j = s;
        }
        pi[t] = i;
        pj[t] = j;
        const double a = A[i][i].x, b = A[j][j].x;
        const double2 c = A[i][j];
        const double g = sqrt(c.x * c.x + c.y * c.y);
        double2 j00 = make_double2(1, 0), j01 = make_double2(0, 0), j10 = make_double2(0, 0), j11 = make_double2(1, 0);
        if (g > 0) {
          const double ex = c.x / g, ey = -c.y / g;   // conj(e^{i phi})
          const double th = 0.5 * atan2(2 * g, a - b), cs = cos(th), sn = sin(th);
          j00 = make_double2(cs, 0);
          j01 = make_double2(-sn, 0);
          j10 = make_double2(ex * sn, ey * sn);
          j11 = make_double2(ex * cs, ey * cs);
        }
        J[t][0] = j00;
        J[t][1] = j01;
        J[t][2] = j10;
        J[t][3] = j11;
      }
      __syncthreads();
      for (int e = t; e < p * h; e += 256) {   // columns: A <- A J, V <- V J
        const int r = e / h, k = e % h, i = pi[k], j = pj[k];
        const double2 j00 = J[k][0], j01 = J[k][1], j10 = J[k][2], j11 = J[k][3];
        const double2 ai = A[r][i], aj = A[r][j], vi = V[r][i], vj = V[r][j];
        A[r][i] = cadd(cmul(ai, j00), cmul(aj, j10));
        A[r][j] = cadd(cmul(ai, j01), cmul(aj, j11));
        V[r][i] = cadd(cmul(vi, j00), cmul(vj, j10));
        V[r][j] = cadd(cmul(vi, j01), cmul(vj, j11));
      }
      __syncthreads();
      for (int e = t; e < p * h; e += 256) {   // rows: A <- J^H A
        const int c = e / h, k = e % h, i = pi[k], j = pj[k];
        const double2 j00 = conjd(J[k][0]), j01 = conjd(J[k][1]), j10 = conjd(J[k][2]), j11 = conjd(J[k][3]);
        const double2 ai = A[i][c], aj = A[j][c];
        A[i][c] = cadd(cmul(j00, ai), cmul(j10, aj));
        A[j][c] = cadd(cmul(j01, ai), cmul(j11, aj));
      }
      __syncthreads();
      if (t == 0) {   // next round-robin order: keep order[0], rotate the rest
        const int last = order[p - 1];
        for (int s = p - 1; s > 1; --s) order[s] = order[s - 1];
        order[1] = last;
      }
      __syncthreads();
    }
  }
  if (t == 0) {   // eigenvalues descending
    for (int i = 0; i < p; ++i) perm[i] = i;
    for (int i = 0; i < p; ++i) {
      int best = i;
      for (int k = i + 1; k < p; ++k)
        if (A[perm[k]][perm[k]].x > A[perm[best]][perm[best]].x) best = k;
      const int s = perm[i];
      perm[i] = perm[best];
      perm[best] = s;
    }
  }
  __syncthreads();
  if (t < p) w[t] = A[perm[t]][perm[t]].x;
  for (int e = t; e < p * p; e += 256) Q[e] = V[e / p][perm[e % p]];
}

// res[j] = || Z[:, j] - w[j] X[:, j] ||, j < k (block per column).
__global__ void residual_kernel(int n, int p, const double2* __restrict__ Z, const double2* __restrict__ X,
                                const double* __restrict__ w, double* res) {
  __shared__ double part[256];
  const int j = blockIdx.x;
  double s = 0;
  for (int i = threadIdx.x; i < n; i += 256) {
    const double2 z = Z[(long long)i * p + j], x = X[(long long)i * p + j];
    const double dx = z.x - w[j] * x.x, dy = z.y - w[j] * x.y;
    s += dx * dx + dy * dy;
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) res[j] = sqrt(part[0]);
}

// Output: vecs [n][k] = columns 0..k-1 of XQ (row-major n x p), vals[i] = max(w[i], 0).
__global__ void output_kernel(int n, int p, int k, const double2* __restrict__ XQ, const double* __restrict__ w,
                              double2* vecs, double* vals) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < (long long)n * k) vecs[e] = XQ[(e / k) * p + e % k];
  if (e < k) vals[e] = w[e] > 0 ? w[e] : 0.0;
}

// ------------------------------------------------------------------------------------------- host side
struct Solver {
  cudaStream_t s;
  double2* parts;
  long long parts_count;
  int status = OI_OK;

  // C = op(A) B (+ C), split over K when the output has few tiles.
  void gemm(bool ah, int m, int n, int k, const double2* A, long long lda, const double2* B, long long ldb, double2* C,
            long long ldc, bool acc) {
    if (status) return;
    const int tiles = ((m + BM - 1) / BM) * ((n + BN - 1) / BN);
    int splits = 1;
    while (tiles * splits < 256 && k / (splits * 2) >= 4 * BK && (long long)(splits * 2) * m * n <= parts_count)
      splits *= 2;
    const int kchunk = ((k + splits - 1) / splits + BK - 1) / BK * BK;
    splits = (k + kchunk - 1) / kchunk;
    dim3 grid((unsigned)((n + BN - 1) / BN), (unsigned)((m + BM - 1) / BM), (unsigned)splits);
    double2* out = splits > 1 ? parts : C;
    const long long ldo = splits > 1 ? n : ldc;
    if (ah)
      zgemm_kernel<true><<<grid, 256, 0, s>>>(m, n, k, A, lda, B, ldb, out, ldo, kchunk, splits > 1 ? 0 : acc);
    else
      zgemm_kernel<false><<<grid, 256, 0, s>>>(m, n, k, A, lda, B, ldb, out, ldo, kchunk, splits > 1 ? 0 : acc);
    oi::note_launch();
    if ((status = check_launch("oi_eig_topk64/gemm"))) return;
    if (splits > 1) {
      if (ldc != n) {
        status = fail(OI_EINVAL, "oi_eig_topk64: split GEMM into a strided output");
        return;
      }
      const long long cnt = (long long)m * n;
      reduce_parts_kernel<<<(unsigned)ceil_div(cnt, 256), 256, 0, s>>>(parts, splits, cnt, C, acc ? 1 : 0);
      oi::note_launch();
      status = check_launch("oi_eig_topk64/reduce");
    }
  }
};

}  // namespace eg
}  // namespace oi

extern "C" int oi_eig_topk64_workspace(int n, int p, int ne, int s, long long* bytes) {
  using namespace oi;
  if (!bytes || n <= 0 || p <= 0) return fail(OI_EINVAL, "oi_eig_topk64_workspace: bad arguments");
  const long long np = (long long)n * p, pp = (long long)p * p, sp = ne > 0 ? (long long)s * p : 0;
  const long long parts = 256LL * pp > 8 * np ? 256LL * pp : 8 * np;
  *bytes = 16 * (3 * np + sp + 4 * pp + parts) + 8 * (2 * (long long)p) + 256;
  return OI_OK;
}

extern "C" int oi_eig_topk64(const void* tcc, const void* h, int ne, int n, int s, int k, int p, int max_iter,
                             double tol, void* vecs, double* vals, void* work, long long work_bytes, int* iters,
                             void* stream) {
  using namespace oi;
  using namespace oi::eg;
  const bool dense = tcc != nullptr;
  if ((!tcc && !h) || (tcc && h) || !vecs || !vals || !work || n <= 0 || k <= 0 || p <= 0 || max_iter <= 0 ||
      (!dense && (ne <= 0 || s <= 0)))
    return fail(OI_EINVAL, "oi_eig_topk64: bad arguments");
  if (p > PMAX || p % 2 || k > p || p > n)
    return fail(OI_ERANGE, "oi_eig_topk64: need k <= p <= min(n, %d), p even (k=%d p=%d n=%d)", PMAX, k, p, n);
  long long need = 0;
  oi_eig_topk64_workspace(n, p, dense ? 0 : ne, s, &need);
  if (work_bytes < need) return fail(OI_ERANGE, "oi_eig_topk64: %lld workspace bytes given, %lld needed", work_bytes, need);
  if (int rc = ensure_smem((const void*)chol_inv_kernel, CHOL_SMEM, "oi_eig_topk64")) return rc;
  if (int rc = ensure_smem((const void*)heev_jacobi_kernel, JACOBI_SMEM, "oi_eig_topk64")) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const long long np = (long long)n * p, pp = (long long)p * p;
  double2* X = (double2*)(((uintptr_t)work + 255) & ~(uintptr_t)255);
  double2* Y = X + np;
  double2* Z = Y + np;
  double2* Wf = Z + np;                                // factored form: h_e^H X, [s][p]
  double2* G = Wf + (dense ? 0 : (long long)s * p);
  double2* Rinv = G + pp;
  double2* Q = Rinv + pp;
  double2* Hm = Q + pp;
  double2* parts = Hm + pp;
  const long long parts_count = 256LL * pp > 8 * np ? 256LL * pp : 8 * np;
  double* w = (double*)(parts + parts_count);
  double* res = w + p;
  Solver sv{st, parts, parts_count};
  const double2* T = (const double2*)tcc;
  const double2* hh = (const double2*)h;

  auto apply = [&](const double2* in, double2* out) {   // out = T in
    if (dense) {
      sv.gemm(false, n, p, n, T, n, in, p, out, p, false);
    } else {
      for (int e = 0; e < ne; ++e) {
        const double2* he = hh + (long long)e * n * s;
        sv.gemm(true, s, p, n, he, s, in, p, Wf, p, false);   // h_e^H in
        sv.gemm(false, n, p, s, he, s, Wf, p, out, p, e > 0);  // out (+)= h_e (h_e^H in)
      }
    }
  };
  auto orth = [&](const double2* in, double2* out) {   // out = CholQR2(in), through Z (in and out distinct)
    for (int pass = 0; pass < 2 && !sv.status; ++pass) {
      const double2* src = pass == 0 ? in : Z;
      double2* dst = pass == 0 ? Z : out;
      sv.gemm(true, p, p, n, src, p, src, p, G, p, false);   // Gram matrix
      if (sv.status) return;
      chol_inv_kernel<<<1, 256, CHOL_SMEM, st>>>(p, G, Rinv, pass == 0 ? 1e-13 : 1e-15);
      oi::note_launch();
      if ((sv.status = check_launch("oi_eig_topk64/chol"))) return;
      sv.gemm(false, n, p, p, src, p, Rinv, p, dst, p, false);
    }
  };

  start_block_kernel<<<(unsigned)ceil_div(np, 256), 256, 0, st>>>(Y, np, 0x5eed0f71ull + (unsigned long long)n);
  oi::note_launch();
  if (int rc = check_launch("oi_eig_topk64/start")) return rc;
  orth(Y, X);
  int it = 0;
  bool converged = false;
  std::vector<double> hres(k), hw(p);
  const int check = 4;
  while (!sv.status && it < max_iter) {
    apply(X, Y);
    orth(Y, X);
    ++it;
    if (it % check == 0 || it == max_iter) {
      apply(X, Z);                                                    // Rayleigh-Ritz
      sv.gemm(true, p, p, n, X, p, Z, p, Hm, p, false);
      if (sv.status) break;
      heev_jacobi_kernel<<<1, 256, JACOBI_SMEM, st>>>(p, Hm, w, Q, 40);
      oi::note_launch();
      if ((sv.status = check_launch("oi_eig_topk64/jacobi"))) break;
      sv.gemm(false, n, p, p, X, p, Q, p, Y, p, false);               // Y = X Q (Ritz vectors)
      sv.gemm(false, n, p, p, Z, p, Q, p, X, p, false);               // X = Z Q = T X Q
      if (sv.status) break;
      residual_kernel<<<(unsigned)k, 256, 0, st>>>(n, p, X, Y, w, res);
      oi::note_launch();
      if ((sv.status = check_launch("oi_eig_topk64/residual"))) break;
      if (cudaMemcpyAsync(hres.data(), res, 8 * k, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaMemcpyAsync(hw.data(), w, 8 * p, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess) {
        sv.status = fail(OI_ECUDA, "oi_eig_topk64: %s", cudaGetErrorString(cudaGetLastError()));
        break;
      }
      double worst = 0;
      for (int i = 0; i < k; ++i) worst = std::fmax(worst, hres[i]);
      const double scale = std::fabs(hw[0]) > 0 ? std::fabs(hw[0]) : 1.0;
      cudaMemcpyAsync(X, Y, 16 * np, cudaMemcpyDeviceToDevice, st);   // continue from the Ritz vectors
      if (worst <= tol * scale) {
        converged = true;
        break;
      }
    }
  }
  if (sv.status) return sv.status;
  if (iters) *iters = converged ? it : -it;
  // X holds the Ritz vectors (columns by descending w)
  output_kernel<<<(unsigned)ceil_div((long long)n * k > p ? (long long)n * k : p, 256), 256, 0, st>>>(
      n, p, k, X, w, (double2*)vecs, vals);
  oi::note_launch();
  return check_launch("oi_eig_topk64/output");
}
