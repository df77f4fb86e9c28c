// The two N-point row passes of the split-BF16x3 form as dense DFT contractions on the tensor cores
// (tcgen05.mma, split BF16x3, FP32 accumulate in tensor memory):
//
//   forward   (oi_rows_fwd_tc)  t[b][ic][y] = sum_x mask[b][y][x] exp(+2 pi i (m0c+ic) x / nx)
//             -- the row half of the band spectrum (Scatter.CalculateSpectrum, Scatter.py:10-35, on the band);
//   inverse   (oi_rows_inv_tc)  out[i][y][x] = sum_qc Re(v[i][qc][y] exp(-2 pi i qc x / nx))
//             -- the last pass of the synthesis (qc > 0 terms already doubled by the caller).
//
// Forward: D[y][n] (M = 128 rows, N = 128: n < 64 re / n >= 64 im of band column ic = n mod 64, K = x in
// chunks of 64) = A x W^T, A = the mask rows (converted to bf16 hi / lo), W = [cos; sin] of the band columns
// (a constant operand image, streamed per chunk).  Inverse: D[x][y] (M = 128 columns x of one x tile,
// N = 128 rows, K = (re | im) x 64 band columns) = C x V^T, C = [cos | sin] of the x tile (constant image,
// resident per x tile), V = v converted to bf16 hi / lo.  The accumulator's lanes are the rows (forward) or
// the columns (inverse), so every warp store of the result is one coalesced segment.
//
// Roles (320 threads): warps 0-7 convert the staged inputs into the K-major, 128-byte swizzled bf16 operand
// and drain finished accumulators to global memory (two warps per tensor-memory lane quarter); warp 8 issues
// the loads into the staging buffers (one 2-D tensor-map box per tile and 1-D bulk copies of the constants; no
// multicast); warp 9 lane 0 issues the MMAs and
// commits them to mbarriers.  Staging and operands are double-buffered (forward) or single (inverse); the
// accumulator is double-buffered in tensor memory so that draining one block overlaps the MMAs of the next.
// Every mbarrier wait is bounded (2 s); on expiry the role records the status (oi_device_status) and stops,
// the others then expire in turn, and the CTA frees tensor memory and exits.
#include <cuda.h>
#include "tc_common.cuh"

namespace oi {

static __device__ int g_rows_status = 0;

int rows_tc_status(int* status, bool reset) {
  if (cudaMemcpyFromSymbol(status, g_rows_status, sizeof(int)) != cudaSuccess) return OI_ECUDA;
  if (reset) {
    const int zero = 0;
    if (cudaMemcpyToSymbol(g_rows_status, &zero, sizeof(int)) != cudaSuccess) return OI_ECUDA;
  }
  return OI_OK;
}

namespace rt {

using namespace tc;

constexpr int NT = 320;                    // threads: 8 converter warps, producer warp, MMA warp
constexpr int NCONV = 256;
constexpr uint32_t OPER = 128 * 128;       // one [128 rows][64 bf16] swizzled operand block (16 KB)
constexpr uint32_t ACC_COLS = 128;         // one accumulator: 128 lanes x 128 fp32 columns
constexpr uint32_t TMEM_COLS = 256;        // two accumulators

__device__ __forceinline__ void fail_status() { atomicExch(&g_rows_status, 1); }

__device__ __forceinline__ void arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// 8 floats -> 4 packed bf16 hi words and 4 lo words
__device__ __forceinline__ void split8(const float (&v)[8], uint32_t (&hi)[4], uint32_t (&lo)[4]) {
#pragma unroll
  for (int e = 0; e < 4; ++e) split2(v[2 * e], v[2 * e + 1], hi[e], lo[e]);
}

// 2-D tiled bulk-tensor load of the box at element coordinates (x, y) of `map` (no multicast), completing on bar.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

// ------------------------------------------------------------------------------------------ forward
// Shared memory: two stages of { staging (mask rows: 128 x 64 f32 or u8), W chunk (hi, lo), A operand (hi, lo) }.
constexpr uint32_t F_STG = 128 * 64 * 4;
constexpr uint32_t F_STAGE = F_STG + 2 * OPER + 2 * OPER;
constexpr uint32_t F_MISC = 2 * F_STAGE;
constexpr uint32_t F_SMEM = F_MISC + 128 + 1024;

struct FwdArgs {
  const void* field;        // [rows][nx] float32 or uint8
  long long rows;           // batch * ny (a multiple of 128)
  int ny, nx, bc, kind;
  const unsigned char* w;   // constant image: per 64-column chunk, [hi | lo] x [128 rows][64]
  float2* t;                // [batch][bc][ny]
};

template <int KIND>
__global__ void __launch_bounds__(NT, 1) rows_fwd_tc_kernel(FwdArgs a, const __grid_constant__ CUtensorMap mask_map) {
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char* gbase = smem_raw + (base - raw);
  const uint32_t misc = base + F_MISC;
  // barriers: full[2] (staging + W landed), conv[2] (A operand written), done[2] (MMAs of the stage finished),
  // accf[2] (accumulator complete), acce[2] (accumulator drained)
  const uint32_t full = misc, conv = misc + 16, done = misc + 32, accf = misc + 48, acce = misc + 64;
  volatile uint32_t* tmem_slot = (volatile uint32_t*)(gbase + F_MISC + 96);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int KC = a.nx / 64;
  const long long items = a.rows / 128;
  const long long G = gridDim.x;
  const long long i0 = (long long)blockIdx.x * items / G, i1 = ((long long)blockIdx.x + 1) * items / G;
  const long long nchunks = (i1 - i0) * KC;
  const uint32_t stg_bytes = KIND == OI_FIELD_U8 ? 128 * 64 : F_STG;

  if (warp == 0) tmem_alloc(misc + 96, TMEM_COLS);
  if (tid == 0) {
    for (int s = 0; s < 2; ++s) {
      mbar_init(full + 8 * s, 1);
      mbar_init(conv + 8 * s, 8);
      mbar_init(done + 8 * s, 1);
      mbar_init(accf + 8 * s, 1);
      mbar_init(acce + 8 * s, 8);
    }
    mbar_init_fence();
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 8) {
    // ---- producer: staging rows and the W chunk of chunk g into stage g & 1
    for (long long g = 0; g < nchunks; ++g) {
      const int s = (int)(g & 1);
      if (g >= 2 && !warp_wait(done + 8 * s, (uint32_t)(((g - 2) >> 1) & 1))) {
        if (lane == 0) fail_status();
        break;
      }
      const long long item = i0 + g / KC;
      const int c = (int)(g % KC);
      const uint32_t st = base + s * F_STAGE;
      if (lane == 0) {
        // the 128 x 64 mask box (one tensor-map load) and the W chunk (one bulk copy)
        expect_tx(full + 8 * s, stg_bytes + 2 * OPER);
        tma_load_2d(st, &mask_map, 64 * c, (int)(item * 128), full + 8 * s);
        bulk_g2s(st + F_STG, a.w + (long long)c * 2 * OPER, 2 * OPER, full + 8 * s);
      }
    }
  } else if (warp == 9) {
    // ---- MMA issue: D[buf] += A_s x W_s^T over the 64-column chunk (K steps of 16), split BF16x3
    if (lane == 0) {
      constexpr uint32_t ID = idesc(128, false);
      for (long long g = 0; g < nchunks; ++g) {
        const int s = (int)(g & 1);
        const long long n = g / KC;
        const int c = (int)(g % KC), buf = (int)(n & 1);
        bool ok = wait_bar(conv + 8 * s, (uint32_t)((g >> 1) & 1));
        if (ok && c == 0 && n >= 2) ok = wait_bar(acce + 8 * buf, (uint32_t)(((n - 2) >> 1) & 1));
        if (!ok) {
          fail_status();
          break;
        }
        fence_after();
        const uint32_t st = base + s * F_STAGE, wch = st + F_STG, aop = wch + 2 * OPER;
        const uint32_t d = tmem + buf * ACC_COLS;
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
          const uint32_t ko = 32 * ks;
          mma_ss(d, sdesc(aop + ko), sdesc(wch + ko), ID, (c | ks) ? 1u : 0u);        // hi hi
          mma_ss(d, sdesc(aop + ko), sdesc(wch + OPER + ko), ID, 1);                  // hi lo
          if (KIND != OI_FIELD_U8) mma_ss(d, sdesc(aop + OPER + ko), sdesc(wch + ko), ID, 1);  // lo hi
        }
        commit(done + 8 * s);
        if (c == KC - 1) commit(accf + 8 * buf);
      }
    }
  } else {
    // ---- converters (warps 0-7): staging -> A operand; drain finished accumulators
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
    const int half = warp >> 2;
    bool ok = true;
    auto drain = [&](long long n) {
      // accumulator of item n: lanes = rows, columns re [0,64) / im [64,128) of band column ic
      const int buf = (int)(n & 1);
      if (!warp_wait(accf + 8 * buf, (uint32_t)((n >> 1) & 1))) return false;
      fence_after();
      float re[32], im[32];
      tmem_ld32x2(tmem + lane_base + buf * ACC_COLS + 32 * half, tmem + lane_base + buf * ACC_COLS + 64 + 32 * half,
                  re, im);
      fence_before();
      __syncwarp();
      if (lane == 0) arrive(acce + 8 * buf);
      const long long row = (i0 + n) * 128 + 32 * (warp & 3) + lane;
      const long long b = row / a.ny;
      const int y = (int)(row - b * a.ny);
      float2* dst = a.t + (b * a.bc + 32 * half) * (long long)a.ny + y;
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if (32 * half + j < a.bc) dst[(long long)j * a.ny] = make_float2(re[j], im[j]);
      return true;
    };
    for (long long g = 0; g < nchunks && ok; ++g) {
      const int s = (int)(g & 1);
      ok = warp_wait(full + 8 * s, (uint32_t)((g >> 1) & 1));
      if (ok && g >= 2) ok = warp_wait(done + 8 * s, (uint32_t)(((g - 2) >> 1) & 1));
      if (!ok) break;
      const uint32_t st = base + s * F_STAGE, aop = st + F_STG + 2 * OPER;
      const unsigned char* gst = gbase + s * F_STAGE;
      if (KIND == OI_FIELD_U8) {
#pragma unroll
        for (int p = 0; p < 4; ++p) {
          const int id = tid + NCONV * p, r = id >> 3, q = id & 7;   // row r, columns 8q .. 8q+7 (exact in bf16)
          const uint2 u = *(const uint2*)(gst + r * 64 + 8 * q);
          float v[8];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            v[e] = (float)((u.x >> (8 * e)) & 0xFF);
            v[4 + e] = (float)((u.y >> (8 * e)) & 0xFF);
          }
          uint32_t hi[4], lo[4];
          split8(v, hi, lo);
          st_shared_v4(aop + swz(r, q), hi[0], hi[1], hi[2], hi[3]);
        }
      } else {
#pragma unroll
        for (int p = 0; p < 8; ++p) {
          const int id = tid + NCONV * p, r = id >> 4, k = id & 15;  // row r, columns 4k .. 4k+3
          const float4 x = *(const float4*)(gst + r * 256 + 16 * k);
          uint32_t h0, l0, h1, l1;
          split2(x.x, x.y, h0, l0);
          split2(x.z, x.w, h1, l1);
          const uint32_t o = aop + swz(r, k >> 1) + 8 * (k & 1);
          asm volatile("st.shared.v2.b32 [%0], {%1, %2};" ::"r"(o), "r"(h0), "r"(h1) : "memory");
          asm volatile("st.shared.v2.b32 [%0], {%1, %2};" ::"r"(o + OPER), "r"(l0), "r"(l1) : "memory");
        }
      }
      fence_async_smem();
      __syncwarp();
      if (lane == 0) arrive(conv + 8 * s);
      // the previous item's accumulator is complete once this item's first chunk is converted
      const long long n = g / KC;
      if (g % KC == 0 && n >= 1) ok = drain(n - 1);
    }
    if (ok && nchunks > 0) ok = drain(i1 - i0 - 1);
    if (!ok && lane == 0) fail_status();
  }
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    tmem_dealloc(tmem, TMEM_COLS);
  }
}

// ------------------------------------------------------------------------------------------ inverse
// Shared memory: C tile of the current x tile (hi, lo: [kc][128 rows][64]), V operand (hi, lo), staging of v
// ([bc][128] float2).
constexpr uint32_t I_CX = 0;
constexpr uint32_t I_VOP = 4 * OPER;
constexpr uint32_t I_STG = 8 * OPER;
constexpr uint32_t I_MISC = I_STG + 64 * 128 * 8;
constexpr uint32_t I_SMEM = I_MISC + 128 + 1024;

struct InvArgs {
  const float2* v;          // [count][bc][ny]
  long long rows;           // count * ny (a multiple of 128)
  int ny, nx, bc;
  const unsigned char* c;   // constant image: per 128-column x tile, [hi | lo] x [kc][128 rows][64]
  float* out;               // [count][ny][nx]
};

// Drain the accumulator of item `it` (tensor-memory buffer `buf`): lanes = x of this warp's quarter, columns =
// rows y0 .. y0+127 of the block (this warp's half), stored as coalesced 128-byte rows segments.
__device__ __forceinline__ void inv_drain(const InvArgs& a, uint32_t taddr, uint32_t acce, int half, int warp,
                                          int lane, long long it, int buf, long long R) {
  fence_after();
  const long long j = it / R, r = it % R;
  float* dst = a.out + (r * 128 + 64 * half) * (long long)a.nx + j * 128 + 32 * (warp & 3) + lane;
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    float o0[16], o1[16];
    tmem_ld16x2(taddr + buf * ACC_COLS + 64 * half + 32 * p, taddr + buf * ACC_COLS + 64 * half + 32 * p + 16, o0,
                o1);
#pragma unroll
    for (int k = 0; k < 16; ++k) __stcs(dst + (long long)(32 * p + k) * a.nx, o0[k]);
#pragma unroll
    for (int k = 0; k < 16; ++k) __stcs(dst + (long long)(32 * p + 16 + k) * a.nx, o1[k]);
  }
  fence_before();
  __syncwarp();
  if (lane == 0) arrive(acce + 8 * buf);
}

__global__ void __launch_bounds__(NT, 1) rows_inv_tc_kernel(InvArgs a, const __grid_constant__ CUtensorMap v_map) {
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char* gbase = smem_raw + (base - raw);
  const uint32_t misc = base + I_MISC;
  // barriers: full (staging landed), cx (C tile landed), conv (V written), done (MMAs finished),
  // acce[2] (accumulator drained)
  const uint32_t full = misc, cxb = misc + 8, conv = misc + 16, done = misc + 24, acce = misc + 32;
  volatile uint32_t* tmem_slot = (volatile uint32_t*)(gbase + I_MISC + 96);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long R = a.rows / 128;                // row blocks
  const long long items = (long long)(a.nx / 128) * R;
  const long long G = gridDim.x;
  const long long i0 = (long long)blockIdx.x * items / G, i1 = ((long long)blockIdx.x + 1) * items / G;
  const long long N = i1 - i0;

  if (warp == 0) tmem_alloc(misc + 96, TMEM_COLS);
  if (tid == 0) {
    mbar_init(full, 1);
    mbar_init(cxb, 1);
    mbar_init(conv, 8);
    mbar_init(done, 1);
    mbar_init(acce, 8);
    mbar_init(acce + 8, 8);
    mbar_init_fence();
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 8) {
    // ---- producer: the C tile when the x tile changes, then the staging of v for item n
    int reloads = 0;
    for (long long n = 0; n < N; ++n) {
      const long long it = i0 + n, j = it / R, r = it % R;
      bool ok = true;
      if (n >= 1) ok = warp_wait(conv, (uint32_t)((n - 1) & 1));            // staging consumed
      const bool reload = n == 0 || (it - 1) / R != j;
      if (ok && reload && n >= 1) ok = warp_wait(done, (uint32_t)((n - 1) & 1));   // old C tile no longer read
      if (!ok) {
        if (lane == 0) fail_status();
        break;
      }
      if (reload) {
        if (lane == 0) {
          expect_tx(cxb, 4 * OPER);
          for (int q = 0; q < 4; ++q) bulk_g2s(base + I_CX + q * OPER, a.c + j * 4 * OPER + q * OPER, OPER, cxb);
        }
        ++reloads;
      }
      // v of image i, band columns 0 .. bc-1, rows y0 .. y0+127: one [bc][256 float] tensor-map box
      const long long row0 = r * 128, i = row0 / a.ny;
      const int y0 = (int)(row0 - i * a.ny);
      if (lane == 0) {
        expect_tx(full, (uint32_t)a.bc * 1024);
        tma_load_2d(base + I_STG, &v_map, 2 * y0, (int)(i * a.bc), full);
      }
    }
    (void)reloads;
  } else if (warp == 9) {
    if (lane == 0) {
      constexpr uint32_t ID = idesc(128, false);
      int reloads = 0;
      for (long long n = 0; n < N; ++n) {
        const long long it = i0 + n, j = it / R;
        const int buf = (int)(n & 1);
        const bool reload = n == 0 || (it - 1) / R != j;
        bool ok = wait_bar(conv, (uint32_t)(n & 1));
        if (ok && reload) ok = wait_bar(cxb, (uint32_t)(reloads & 1));
        if (ok && n >= 2) ok = wait_bar(acce + 8 * buf, (uint32_t)(((n - 2) >> 1) & 1));
        if (!ok) {
          fail_status();
          break;
        }
        if (reload) ++reloads;
        fence_after();
        const uint32_t d = tmem + buf * ACC_COLS;
#pragma unroll
        for (int ks = 0; ks < 8; ++ks) {
          const uint32_t ko = (uint32_t)(ks >> 2) * OPER + 32 * (ks & 3);
          const uint32_t ah = base + I_CX + ko, al = ah + 2 * OPER;
          const uint32_t bh = base + I_VOP + ko, bl = bh + 2 * OPER;
          mma_ss(d, sdesc(ah), sdesc(bh), ID, ks ? 1u : 0u);   // hi hi
          mma_ss(d, sdesc(ah), sdesc(bl), ID, 1);              // hi lo
          mma_ss(d, sdesc(al), sdesc(bh), ID, 1);              // lo hi
        }
        commit(done);
      }
    }
  } else {
    // ---- converters: staging [qc][y] float2 -> V operand rows y, K = (re | im) x qc; drain accumulators
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
    const int half = warp >> 2;
    const float2* stg = (const float2*)(gbase + I_STG);
    bool ok = true;
    for (long long n = 0; n < N && ok; ++n) {
      ok = warp_wait(full, (uint32_t)(n & 1));
      if (ok && n >= 1) ok = warp_wait(done, (uint32_t)((n - 1) & 1));    // V free, accumulator n-1 complete
      if (!ok) break;
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        const int id = tid + NCONV * p, y = id & 127, q = id >> 7;    // row y, band columns 8q .. 8q+7
        float re[8], im[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int qc = 8 * q + e;
          const float2 x = qc < a.bc ? stg[qc * 128 + y] : make_float2(0.f, 0.f);
          re[e] = x.x;
          im[e] = x.y;
        }
        uint32_t hi[4], lo[4];
        split8(re, hi, lo);
        const uint32_t o = base + I_VOP + swz(y, q);
        st_shared_v4(o, hi[0], hi[1], hi[2], hi[3]);
        st_shared_v4(o + 2 * OPER, lo[0], lo[1], lo[2], lo[3]);
        split8(im, hi, lo);
        st_shared_v4(o + OPER, hi[0], hi[1], hi[2], hi[3]);
        st_shared_v4(o + 3 * OPER, lo[0], lo[1], lo[2], lo[3]);
      }
      fence_async_smem();
      __syncwarp();
      if (lane == 0) arrive(conv);
      if (n >= 1) inv_drain(a, tmem + lane_base, acce, half, warp, lane, i0 + n - 1, (int)((n - 1) & 1), R);
    }
    if (ok && N > 0) {
      ok = warp_wait(done, (uint32_t)((N - 1) & 1));
      if (ok) inv_drain(a, tmem + lane_base, acce, half, warp, lane, i0 + N - 1, (int)((N - 1) & 1), R);
    }
    if (!ok && lane == 0) fail_status();
  }
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    tmem_dealloc(tmem, TMEM_COLS);
  }
}

// --------------------------------------------------------------------------------- constant images
// Forward: for each 64-column chunk c, W rows n < 64: cos(2 pi (m0c+n) x / nx), rows 64+n: sin(...) (n < bc;
// zero rows above), K = x = 64c .. 64c+63; [hi | lo].  One thread per (chunk, row, 8 columns).
__global__ void rows_fwd_consts_kernel(int nx, int m0c, int bc, unsigned char* img) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int kc = nx / 64;
  if (id >= (long long)kc * 128 * 8) return;
  const int c = (int)(id / 1024), row = (int)((id / 8) % 128), q = (int)(id % 8);
  const int n = row & 63;
  float v[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const long long x = 64LL * c + 8 * q + e;
    double s = 0.0, co = 0.0;
    if (n < bc) {
      const long long m = m0c + n;
      long long p = (m * x) % nx;
      if (p < 0) p += nx;
      sincospi(2.0 * (double)p / (double)nx, &s, &co);
    }
    v[e] = (float)(row < 64 ? co : s);
  }
  uint32_t hi[4], lo[4];
  split8(v, hi, lo);
  unsigned char* o = img + (long long)c * 2 * OPER + swz(row, q);
  *(uint4*)o = make_uint4(hi[0], hi[1], hi[2], hi[3]);
  *(uint4*)(o + OPER) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
}

// Inverse: for each 128-column x tile j, rows x (128), K kc = 0: cos(2 pi qc x / nx), kc = 1: sin(...),
// qc = 0 .. 63 (zero for qc >= bc); [hi | lo] x [kc].
__global__ void rows_inv_consts_kernel(int nx, int bc, unsigned char* img) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int nt = nx / 128;
  if (id >= (long long)nt * 2 * 128 * 8) return;
  const int j = (int)(id / 2048), kc = (int)((id / 1024) % 2), row = (int)((id / 8) % 128), q = (int)(id % 8);
  const long long x = 128LL * j + row;
  float v[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const int qc = 8 * q + e;
    double s = 0.0, co = 0.0;
    if (qc < bc) {
      const long long p = ((long long)qc * x) % nx;
      sincospi(2.0 * (double)p / (double)nx, &s, &co);
    }
    v[e] = (float)(kc == 0 ? co : s);
  }
  uint32_t hi[4], lo[4];
  split8(v, hi, lo);
  unsigned char* o = img + (long long)j * 4 * OPER + kc * OPER + swz(row, q);
  *(uint4*)o = make_uint4(hi[0], hi[1], hi[2], hi[3]);
  *(uint4*)(o + 2 * OPER) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
}

typedef CUresult (*EncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// A 2-D tensor map (dim0 contiguous, rows `stride1` bytes apart) with a box0 x box1 box, no swizzle.
static int encode_2d(CUtensorMap* map, CUtensorMapDataType type, const void* base, unsigned long long dim0,
                     unsigned long long dim1, unsigned long long stride1, unsigned box0, unsigned box1) {
  static EncodeTiled encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn)
      return fail(OI_ECUDA, "cuTensorMapEncodeTiled is not available");
    encode = (EncodeTiled)fn;
  }
  const cuuint64_t dims[2] = {dim0, dim1}, strides[1] = {stride1};
  const cuuint32_t box[2] = {box0, box1}, estr[2] = {1, 1};
  const CUresult r = encode(map, type, 2, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(OI_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return OI_OK;
}

static int sm_count() {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 0;
  return sms;
}

}  // namespace rt
}  // namespace oi

extern "C" int oi_rows_tc_constants(int which, int nx, int m0c, int bc, void* image, long long bytes, void* stream) {
  using namespace oi;
  if (!image || nx <= 0 || bc <= 0 || bc > 64 || (which != 0 && which != 1))
    return fail(OI_EINVAL, "oi_rows_tc_constants: bad arguments");
  if (nx % 128 != 0 || nx > 4096) return fail(OI_ERANGE, "oi_rows_tc_constants: nx=%d is not a multiple of 128", nx);
  const long long need = which == 0 ? (long long)(nx / 64) * 2 * rt::OPER : (long long)(nx / 128) * 4 * rt::OPER;
  if (bytes < need) return fail(OI_ERANGE, "oi_rows_tc_constants: %lld bytes given, %lld needed", bytes, need);
  if ((uintptr_t)image % 16) return fail(OI_EINVAL, "oi_rows_tc_constants: image not 16-byte aligned");
  const long long threads = need / 16 / 2;
  cudaStream_t s = (cudaStream_t)stream;
  if (which == 0)
    rt::rows_fwd_consts_kernel<<<(unsigned)ceil_div(threads, 256), 256, 0, s>>>(nx, m0c, bc, (unsigned char*)image);
  else
    rt::rows_inv_consts_kernel<<<(unsigned)ceil_div(threads, 256), 256, 0, s>>>(nx, bc, (unsigned char*)image);
  oi::note_launch();
  return check_launch("oi_rows_tc_constants");
}

extern "C" int oi_rows_fwd_tc(const void* field, int kind, int batch, int ny, int nx, int m0c, int bc,
                              const void* consts, void* t, void* stream) {
  using namespace oi;
  if (!field || !consts || !t || batch <= 0 || bc <= 0) return fail(OI_EINVAL, "oi_rows_fwd_tc: bad arguments");
  if (kind != OI_FIELD_REAL_F32 && kind != OI_FIELD_U8)
    return fail(OI_EINVAL, "oi_rows_fwd_tc: real float32 or uint8 masks only (kind=%d)", kind);
  if (ny % 128 != 0 || nx % 128 != 0 || nx > 4096 || bc > 64)
    return fail(OI_ERANGE, "oi_rows_fwd_tc: grid %dx%d / band width %d unsupported", ny, nx, bc);
  if ((uintptr_t)field % 16 || (uintptr_t)consts % 16)
    return fail(OI_EINVAL, "oi_rows_fwd_tc: field and constants must be 16-byte aligned");
  const long long rows = (long long)batch * ny, items = rows / 128;
  const int sms = rt::sm_count();
  if (!sms) return fail(OI_ECUDA, "oi_rows_fwd_tc: no CUDA device");
  const long long ctas = items < sms ? items : sms;
  rt::FwdArgs a{field, rows, ny, nx, bc, kind, (const unsigned char*)consts, (float2*)t};
  cudaStream_t s = (cudaStream_t)stream;
  const bool u8 = kind == OI_FIELD_U8;
  CUtensorMap map;
  int rc = rt::encode_2d(&map, u8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, field,
                         (unsigned long long)nx, (unsigned long long)rows, (unsigned long long)nx * (u8 ? 1 : 4), 64,
                         128);
  if (rc) return rc;
  if (u8) {
    rc = ensure_smem((const void*)rt::rows_fwd_tc_kernel<OI_FIELD_U8>, rt::F_SMEM, "oi_rows_fwd_tc");
    if (rc) return rc;
    rt::rows_fwd_tc_kernel<OI_FIELD_U8><<<(unsigned)ctas, rt::NT, rt::F_SMEM, s>>>(a, map);
    oi::note_launch();
  } else {
    rc = ensure_smem((const void*)rt::rows_fwd_tc_kernel<OI_FIELD_REAL_F32>, rt::F_SMEM, "oi_rows_fwd_tc");
    if (rc) return rc;
    rt::rows_fwd_tc_kernel<OI_FIELD_REAL_F32><<<(unsigned)ctas, rt::NT, rt::F_SMEM, s>>>(a, map);
    oi::note_launch();
  }
  return check_launch("oi_rows_fwd_tc");
}

extern "C" int oi_rows_inv_tc(const void* v, int count, int ny, int nx, int bc, const void* consts, float* out,
                              void* stream) {
  using namespace oi;
  if (!v || !consts || !out || count <= 0 || bc <= 0) return fail(OI_EINVAL, "oi_rows_inv_tc: bad arguments");
  if (ny % 128 != 0 || nx % 128 != 0 || nx > 4096 || bc > 64)
    return fail(OI_ERANGE, "oi_rows_inv_tc: grid %dx%d / band width %d unsupported", ny, nx, bc);
  if ((uintptr_t)v % 16 || (uintptr_t)consts % 16)
    return fail(OI_EINVAL, "oi_rows_inv_tc: v and constants must be 16-byte aligned");
  const long long rows = (long long)count * ny, items = (long long)(nx / 128) * (rows / 128);
  const int sms = rt::sm_count();
  if (!sms) return fail(OI_ECUDA, "oi_rows_inv_tc: no CUDA device");
  const long long ctas = items < sms ? items : sms;
  rt::InvArgs a{(const float2*)v, rows, ny, nx, bc, (const unsigned char*)consts, out};
  CUtensorMap map;   // v as float [count * bc][2 ny]: boxes of bc band columns x 128 complex rows
  int rc = rt::encode_2d(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, v, 2ULL * ny, (unsigned long long)count * bc,
                         8ULL * ny, 256, (unsigned)bc);
  if (rc) return rc;
  rc = ensure_smem((const void*)rt::rows_inv_tc_kernel, rt::I_SMEM, "oi_rows_inv_tc");
  if (rc) return rc;
  rt::rows_inv_tc_kernel<<<(unsigned)ctas, rt::NT, rt::I_SMEM, (cudaStream_t)stream>>>(a, map);
  oi::note_launch();
  return check_launch("oi_rows_inv_tc");
}
