// Synthesis preparation on the tensor cores (split BF16x3, FP32 accumulate): from the coarse intensity's
// partial sums to the V operand tiles of the synthesis row pass (rows_tc.cu), as two real GEMMs per image:
//
//   U[sr][n] = sum_sc c[sr][sc] G[sc][n],   G = ((qc ? 2 : 1) / M) (cos | sin)(2 pi qc sc / M),  n = (re | im, qc)
//   v[y][n]  = sum_sr A[y][sr] U[sr][n],    A = (1 / M) sum_{|qr| < br} cos(2 pi qr (sr / M - y / ny))
//
// with c the coarse intensity (M = 128 per axis, the sum of its partial sums).  This is the coarse spectrum
// Ihat[qr][qc] = (qc ? 2 : 1) / M^2 sum_s c[s] exp(+2 pi i (qr sr + qc sc) / M) (|qr| < br, 0 <= qc < bc) followed
// by the column synthesis v[qc][y] = sum_qr Ihat[qr][qc] exp(-2 pi i qr y / ny) -- the fftshift-free form of the
// reference's final transform (CalculateAerialImage_SOCS.py:7-10) on the intensity's band -- with the qr sum
// taken first: over a symmetric qr range it is a real Dirichlet kernel in (sr / M - y / ny).
//
// Items are (image, group of TP consecutive 128-row y tiles), one contiguous range per CTA.  Per item the
// converter warps fold the partial sums into the B operand of stage 1 (bf16 hi / lo, shared memory), one lane
// issues the 24 MMAs of U^T = G^T c^T (M = 128 n, N = 128 sr, K = 128 sc), the converters turn each tensor-memory
// lane (a row n of U^T) into the B operand of stage 2 (K = sr) in place, and per y tile 24 MMAs give
// v = A U (M = 128 y, N = 128, K = 128 sr), drained from tensor memory as the V tile's bf16 hi / lo blocks.  The
// constant operands (G, then the A tile of each y tile) stream through a ring of 16 KB pieces, 1.5 tiles deep,
// each piece released as soon as the MMAs reading it finish.  Per y tile a CTA moves the A tile's 64 KB in and
// the V tile's 64 KB out over its path to L2 (about 24 bytes per cycle for both together, measured: ~2.7 us
// per tile with the stores, ~1.5 us without them), which bounds the pass.
//
// Roles (320 threads): warps 0-7 convert (fold, U transpose, V drain; two warps per tensor-memory lane
// quarter), warp 8 streams the constant pieces (2-D tensor-map boxes, no multicast), warp 9 lane 0 issues the
// MMAs.  A V tile is staged in shared memory in its final (swizzled operand) layout -- in the stage-1 B region,
// free while the item's tiles drain -- and leaves as bulk copies issued by warp 0 lane 0: written straight from
// registers, each lane's 16-byte pieces of one row would touch 32 lines per warp store.  Every mbarrier wait is bounded (2 s); on expiry the role records the device status and stops, the
// producer waits for its copies in flight and the MMA thread for its issued MMAs before memory is released.
#include "tc_common.cuh"

namespace oi {

static __device__ int g_synth_status = 0;

int synth_tc_status(int* status, bool reset) {
  if (cudaMemcpyFromSymbol(status, g_synth_status, sizeof(int)) != cudaSuccess) return OI_ECUDA;
  if (reset) {
    const int zero = 0;
    if (cudaMemcpyToSymbol(g_synth_status, &zero, sizeof(int)) != cudaSuccess) return OI_ECUDA;
  }
  return OI_OK;
}

namespace st {

using namespace tc;

constexpr int M = 128;                     // coarse grid per axis
constexpr uint32_t OPER = 128 * 128;       // one [128 rows][64 bf16] swizzled operand block (16 KB)
constexpr int NR = 6;                      // constant pieces in the ring (1.5 tiles: a tile's A loads overlap
                                           // the previous tile's MMAs)
constexpr int T = 320;                     // 8 converter warps, producer warp, MMA warp
constexpr uint32_t R_OFF = 0;                            // ring of constant pieces
constexpr uint32_t A1_OFF = NR * OPER;                   // the folded coarse image (stage-1 B), later the V staging
constexpr uint32_t B2_OFF = A1_OFF + 4 * OPER;           // stage-2 B (U^T)
constexpr uint32_t MISC = B2_OFF + 4 * OPER;
constexpr uint32_t SMEM = MISC + 512 + 1024;
static_assert(A1_OFF % 1024 == 0 && B2_OFF % 1024 == 0, "operand alignment");
static_assert(SMEM <= SMEM_LIMIT, "synthesis preparation: shared memory");

struct Args {
  const float* coarse;      // [nparts][count][128][128]
  long long part_stride;    // floats between partial sums
  int nparts, count, ny, tp;
  unsigned char* tiles;     // V tiles [count * ny / 128][64 KB]
};

__device__ __forceinline__ void fail_status() { atomicExch(&g_synth_status, 1); }

// The k-th y tile of a CTA's group [t0, t1).
__device__ __forceinline__ int tile_of(int t0, int, int k) { return t0 + k; }

// Converter warps' share of the fold: image `img`, 2048 tasks (row sr, 8-column chunk q16) over 256 threads,
// partial sums added in order, written as the bf16 hi / lo stage-1 B operand (blocks [hi k0 | hi k1 | lo k0 |
// lo k1], K = sc).
__device__ __forceinline__ void fold(const Args& a, long long img, int tid, unsigned char* a1) {
  const float* src = a.coarse + img * (long long)(M * M);
  float4 acc[16], x[16];
#pragma unroll
  for (int t = 0; t < 8; ++t) {   // the first two partial sums' loads in flight together
    const int task = tid + 256 * t, sr = task >> 4, q16 = task & 15;
    const float4* p = (const float4*)(src + sr * M + 8 * q16);
    acc[2 * t] = __ldg(p);
    acc[2 * t + 1] = __ldg(p + 1);
    if (a.nparts > 1) {
      x[2 * t] = __ldg(p + a.part_stride / 4);
      x[2 * t + 1] = __ldg(p + a.part_stride / 4 + 1);
    }
  }
  for (int part = 1; part < a.nparts; ++part) {
    if (part > 1) {
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        const int task = tid + 256 * t, sr = task >> 4, q16 = task & 15;
        const float4* p = (const float4*)(src + part * a.part_stride + sr * M + 8 * q16);
        x[2 * t] = __ldg(p);
        x[2 * t + 1] = __ldg(p + 1);
      }
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      acc[k].x += x[k].x;
      acc[k].y += x[k].y;
      acc[k].z += x[k].z;
      acc[k].w += x[k].w;
    }
  }
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    const int task = tid + 256 * t, sr = task >> 4, q16 = task & 15, kb = q16 >> 3, q = q16 & 7;
    uint32_t hi[4], lo[4];
    split2(acc[2 * t].x, acc[2 * t].y, hi[0], lo[0]);
    split2(acc[2 * t].z, acc[2 * t].w, hi[1], lo[1]);
    split2(acc[2 * t + 1].x, acc[2 * t + 1].y, hi[2], lo[2]);
    split2(acc[2 * t + 1].z, acc[2 * t + 1].w, hi[3], lo[3]);
    const uint32_t o = swz(sr, q);
    *(uint4*)(a1 + kb * OPER + o) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *(uint4*)(a1 + (2 + kb) * OPER + o) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
  }
}

__global__ void __launch_bounds__(T, 1) synth_prep_tc_kernel(Args a, const __grid_constant__ CUtensorMap k_map) {
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char* gbase = smem_raw + (base - raw);
  const uint32_t misc = base + MISC;
  // barriers: rfull[6] / rfree[6] (constant pieces), a1full (stage-1 B written), d1full (U^T complete in tensor
  // memory), b2full (stage-2 B written), b2free (the item's stage-2 MMAs finished), accf[2] / acce[2] (v tile
  // complete / drained), fin (every issued MMA finished, at the end)
  // vstaged (a V tile is staged by all eight converter warps), vsfree (its bulk copies have read the staging)
  const uint32_t rfull = misc, rfree = misc + 8 * NR, a1full = misc + 16 * NR, d1full = a1full + 8, b2full = a1full + 16,
                 b2free = a1full + 24, accf = a1full + 32, acce = a1full + 48, fin = a1full + 64, vstaged = a1full + 72,
                 vsfree = a1full + 80;
  static_assert(16 * NR + 88 <= 256, "synthesis preparation: barrier block");
  volatile uint32_t* tmem_slot = (volatile uint32_t*)(gbase + MISC + 256);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int TY = a.ny / 128;                           // y tiles per image
  const int H = (TY + a.tp - 1) / a.tp;                // y-tile groups per image
  const long long items = (long long)a.count * H;
  const long long G = gridDim.x;
  const long long i0 = (long long)blockIdx.x * items / G, i1 = ((long long)blockIdx.x + 1) * items / G;
  const int NI = (int)(i1 - i0);

  if (warp == 0) tmem_alloc(misc + 256, 512);
  if (tid == 0) {
    for (int s = 0; s < NR; ++s) {
      mbar_init(rfull + 8 * s, 1);
      mbar_init(rfree + 8 * s, 1);
    }
    mbar_init(a1full, 8);
    mbar_init(d1full, 1);
    mbar_init(b2full, 8);
    mbar_init(b2free, 1);
    for (int s = 0; s < 2; ++s) {
      mbar_init(accf + 8 * s, 1);
      mbar_init(acce + 8 * s, 8);
    }
    mbar_init(fin, 1);
    mbar_init(vstaged, 8);
    mbar_init(vsfree, 1);
    mbar_init_fence();
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;
  pdl_trigger();
  pdl_wait();   // the coarse sums come from the coherent sum (and the constant image may be fresh on the stream)

  if (warp == 8) {
    // ---- constant pieces: per item G (4 pieces), then the A tile of each y tile (4 pieces each)
    if (lane == 0) {
      Ring rs{0, 0};
      int g = 0;
      bool ok = true;
      for (long long it = i0; it < i1 && ok; ++it) {
        const int grp = (int)(it % H), t0 = grp * a.tp, t1 = min(TY, t0 + a.tp);
        for (int k = -1; k < t1 - t0 && ok; ++k) {   // k = -1 stands for G (blocks 0-3), then A_t (4 + 4t ..)
          const int t = k < 0 ? t0 - 1 : tile_of(t0, t1, k);
          for (int p = 0; p < 4; ++p, ++g) {
            if (g >= NR && !wait_bar(rfree + 8 * rs.slot, rs.phase ^ 1u)) {
              ok = false;
              break;
            }
            const int blk = t < t0 ? p : 4 * (1 + t) + p;
            expect_tx(rfull + 8 * rs.slot, OPER);
            tma_load_2d(base + R_OFF + rs.slot * OPER, &k_map, 0, blk * 128, rfull + 8 * rs.slot);
            rs.next(NR);
          }
        }
      }
      if (!ok) fail_status();
      drain_ring(rfull, rs, g, NR);   // the copies in flight land before shared memory is released
    }
  } else if (warp == 9) {
    if (lane == 0) {
      constexpr uint32_t ID = idesc(128, false);
      const uint32_t a1 = base + A1_OFF, b2 = base + B2_OFF;
      Ring rs{0, 0}, ab{0, 0};
      bool ok = true, issued = false;
      int m = 0;   // v tiles issued
      // wait for the next ring piece: false on expiry, else its shared address in `addr`
      auto piece = [&](int& slot, uint32_t& addr) -> bool {
        if (!wait_bar(rfull + 8 * rs.slot, rs.phase)) return false;
        fence_after();
        slot = rs.slot;
        addr = base + R_OFF + rs.slot * OPER;
        rs.next(NR);
        return true;
      };
      for (int n = 0; n < NI && ok; ++n) {
        const long long it = i0 + n;
        const int grp = (int)(it % H), t0 = grp * a.tp, t1 = min(TY, t0 + a.tp);
        ok = wait_bar(a1full, (uint32_t)(n & 1));
        if (!ok) break;
        fence_after();
        // stage 1: D1 = G^T c^T = U^T (lanes n, columns sr); pieces G hi k0, G hi k1, G lo k0, G lo k1 (A),
        // the folded image (B)
        int sl[4];
        for (int p = 0; p < 4 && ok; ++p) {
          uint32_t gp = 0;
          if (!piece(sl[p], gp)) {
            ok = false;
            break;
          }
          issued = true;
          const int kb = p & 1;
          const uint32_t chi = a1 + kb * OPER, clo = a1 + (2 + kb) * OPER;
#pragma unroll
          for (int ks = 0; ks < 4; ++ks) {
            if (p < 2) {   // G hi: hi x hi, hi x lo
              mma_ss(tmem, sdesc(gp + 32 * ks), sdesc(chi + 32 * ks), ID, (p | ks) ? 1u : 0u);
              mma_ss(tmem, sdesc(gp + 32 * ks), sdesc(clo + 32 * ks), ID, 1);
            } else {       // G lo: lo x hi
              mma_ss(tmem, sdesc(gp + 32 * ks), sdesc(chi + 32 * ks), ID, 1);
            }
          }
          commit(rfree + 8 * sl[p]);   // the slot is refilled once these MMAs finish
        }
        if (!ok) break;
        commit(d1full);
        ok = wait_bar(b2full, (uint32_t)(n & 1));
        if (!ok) break;
        fence_after();
        // stage 2, per y tile: D2[buf] = A_t U; pieces A hi k0, A hi k1, A lo k0, A lo k1; B = U^T (b2)
        for (int k = 0; k < t1 - t0 && ok; ++k, ++m) {
          const int t = tile_of(t0, t1, k);
          if (m >= 2) {
            ok = wait_bar(acce + 8 * ab.slot, ab.phase ^ 1u);
            if (!ok) break;
          }
          const uint32_t d2 = tmem + 128 * (1 + ab.slot);
          for (int p = 0; p < 4 && ok; ++p) {
            uint32_t ap = 0;
            if (!piece(sl[p], ap)) {
              ok = false;
              break;
            }
            const int kb = p & 1;
            const uint32_t bhi = b2 + kb * OPER, blo = b2 + (2 + kb) * OPER;
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
              if (p < 2) {   // A hi: hi x hi, hi x lo
                mma_ss(d2, sdesc(ap + 32 * ks), sdesc(bhi + 32 * ks), ID, (p | ks) ? 1u : 0u);
                mma_ss(d2, sdesc(ap + 32 * ks), sdesc(blo + 32 * ks), ID, 1);
              } else {       // A lo: lo x hi
                mma_ss(d2, sdesc(ap + 32 * ks), sdesc(bhi + 32 * ks), ID, 1);
              }
            }
            commit(rfree + 8 * sl[p]);   // the slot is refilled once these MMAs finish (the next tile's piece)
          }
          if (!ok) break;
          commit(accf + 8 * ab.slot);
          ab.next(2);
        }
        if (!ok) break;
        commit(b2free);   // the item's stage-2 MMAs (the readers of b2) are complete when this arrives
      }
      if (!ok) fail_status();
      if (issued) {   // every MMA issued has finished before tensor and shared memory are released
        commit(fin);
        wait_bar(fin, 0);
      }
    }
  } else {
    // ---- warps 0-7: fold, U^T conversion, V drain
    unsigned char* a1 = gbase + A1_OFF;
    unsigned char* b2 = gbase + B2_OFF;
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
    const int half = warp >> 2, row = 32 * (warp & 3) + lane;
    Ring ab{0, 0};
    bool ok = true;
    uint32_t vt = 0;   // V tiles staged
    for (int n = 0; n < NI && ok; ++n) {
      const long long it = i0 + n, img = it / H;
      const int grp = (int)(it % H), t0 = grp * a.tp, t1 = min(TY, t0 + a.tp);
      if (vt >= 1) {   // the previous item's last V tile has left the staging (the stage-1 operand region)
        ok = warp_wait(vsfree, (vt - 1) & 1u);
        if (!ok) break;
      }
      fold(a, img, tid, a1);
      fence_async_smem();
      fence_before();
      __syncwarp();
      if (lane == 0) arrive(a1full);
      ok = warp_wait(d1full, (uint32_t)(n & 1));
      if (!ok) break;
      fence_after();
      if (n >= 1) {                                  // the previous item's stage 2 no longer reads b2
        ok = warp_wait(b2free, (uint32_t)((n - 1) & 1));
        if (!ok) break;
      }
      // B2 = U^T as bf16 hi / lo straight from tensor memory: lane = row n, this warp's half = K block (sr)
      {
        float u0[32], u1[32];
        const uint32_t ta = tmem + lane_base + 64 * half;
        tmem_ld32x2(ta, ta + 32, u0, u1);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const float* src = q < 4 ? u0 + 8 * q : u1 + 8 * (q - 4);
          uint32_t hi[4], lo[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) split2(src[2 * e], src[2 * e + 1], hi[e], lo[e]);
          const uint32_t o = swz(row, q);
          *(uint4*)(b2 + half * OPER + o) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
          *(uint4*)(b2 + (2 + half) * OPER + o) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
        }
      }
      fence_async_smem();
      fence_before();
      __syncwarp();
      if (lane == 0) arrive(b2full);
      // V tiles: lane = y of the tile, this warp's half = re (blocks hi 0, lo 2) or im (hi 1, lo 3)
      for (int k = 0; k < t1 - t0 && ok; ++k, ++vt) {
        const int t = tile_of(t0, t1, k);
        ok = warp_wait(accf + 8 * ab.slot, ab.phase);
        if (!ok) break;
        fence_after();
        float v0[32], v1[32];
        const uint32_t ta = tmem + lane_base + 128 * (1 + ab.slot) + 64 * half;
        tmem_ld32x2(ta, ta + 32, v0, v1);
        fence_before();
        __syncwarp();
        if (lane == 0) arrive(acce + 8 * ab.slot);
        if (vt >= 1 && k > 0) {   // the previous tile's copies have read the staging
          ok = warp_wait(vsfree, (vt - 1) & 1u);
          if (!ok) break;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const float* src = q < 4 ? v0 + 8 * q : v1 + 8 * (q - 4);
          uint32_t hi[4], lo[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) split2(src[2 * e], src[2 * e + 1], hi[e], lo[e]);
          const uint32_t o = swz(row, q);
          *(uint4*)(a1 + half * OPER + o) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
          *(uint4*)(a1 + (2 + half) * OPER + o) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
        }
        fence_async_smem();   // visible to the bulk copies
        __syncwarp();
        if (lane == 0) arrive(vstaged);
        if (tid == 0) {
          ok = wait_bar(vstaged, vt & 1u);
          if (ok) {
            unsigned char* tile = a.tiles + (img * TY + t) * (long long)(4 * OPER);
#pragma unroll
            for (int b = 0; b < 4; ++b) bulk_s2g(tile + b * OPER, base + A1_OFF + b * OPER, OPER);
            bulk_commit();
            bulk_wait_read();
            arrive(vsfree);
          }
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        ab.next(2);
      }
    }
    if (tid == 0) bulk_wait_all();   // the V tiles are written before the CTA exits
    if (!ok && lane == 0) fail_status();
  }
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// Constant image: G^T as [hi k0 | hi k1 | lo k0 | lo k1] x [128 n][64 sc] (n < 64: cos of qc = n, n >= 64: sin of
// qc = n - 64, times (qc ? 2 : 1) / M, zero for qc >= bc), then per 128-row y tile t the A operand in the same
// block order, [128 y][64 sr].  Phases reduced exactly in 64-bit integers, values in double precision.
__global__ void synth_consts_kernel(int ny, int br, int bc, unsigned char* img) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;   // (tile u, row, K block, chunk q)
  const int tiles = 1 + ny / 128;
  if (id >= (long long)tiles * 2048) return;
  const int u = (int)(id / 2048), r = (int)((id / 16) % 128), kb = (int)((id / 8) % 2), q = (int)(id % 8);
  float v[8];
#pragma unroll 1
  for (int e = 0; e < 8; ++e) {
    const int k = 64 * kb + 8 * q + e;
    double val = 0.0;
    if (u == 0) {   // G^T[n = r][sc = k]
      const int qc = r & 63;
      if (qc < bc) {
        double s, c;
        sincospi(2.0 * (double)(((long long)qc * k) % M) / M, &s, &c);
        val = (qc ? 2.0 : 1.0) / M * (r < 64 ? c : s);
      }
    } else {        // A[y][sr = k], y = 128 (u - 1) + r: (1/M) sum_{|qr|<br} cos(2 pi qr (k ny - y M) / (M ny))
      const long long y = 128LL * (u - 1) + r, den = (long long)M * ny, d = (long long)k * ny - y * M;
      for (int qr = -(br - 1); qr <= br - 1; ++qr) {
        long long p = ((long long)qr * d) % den;
        if (p < 0) p += den;
        val += cospi(2.0 * (double)p / (double)den);
      }
      val /= M;
    }
    v[e] = (float)val;
  }
  uint32_t hi[4], lo[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) split2(v[2 * e], v[2 * e + 1], hi[e], lo[e]);
  unsigned char* o = img + (long long)u * 4 * OPER + swz(r, q);
  *(uint4*)(o + kb * OPER) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
  *(uint4*)(o + (2 + kb) * OPER) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
}

}  // namespace st

// The V tiles of count images from their coarse intensities (nparts partial sums); `sconsts` from
// oi_synth_tc_constants for (ny, br, bc).
int synth_tiles_tc(const float* coarse, int nparts, int count, int br, int bc, const void* sconsts, int ny,
                   void* tiles, cudaStream_t s) {
  (void)br;
  (void)bc;
  const int sms = tc::sm_count();
  if (!sms) return fail(OI_ECUDA, "oi_synth_tiles_tc: no CUDA device");
  const int TY = ny / 128;
  // y tiles per item: the split minimising waves x (tiles per item + the item's fixed stage-1 cost)
  int best_tp = TY;
  double best = 0.0;
  for (int tp = 1; tp <= TY; ++tp) {
    const long long items = (long long)count * ((TY + tp - 1) / tp);
    const double cost = (double)((items + sms - 1) / sms) * (tp + 1.5);
    if (tp == 1 || cost < best) {
      best = cost;
      best_tp = tp;
    }
  }
  const long long items = (long long)count * ((TY + best_tp - 1) / best_tp), ctas = items < sms ? items : sms;
  st::Args a{coarse, (long long)count * st::M * st::M, nparts, count, ny, best_tp, (unsigned char*)tiles};
  CUtensorMap k_map;   // rows of 128 bytes of the constant image, boxes of [128 rows][64 uint16]
  int rc = tc::encode_2d(&k_map, CU_TENSOR_MAP_DATA_TYPE_UINT16, sconsts, 64, (unsigned long long)(1 + TY) * 512, 128,
                         64, 128);
  if (!rc) rc = ensure_smem((const void*)st::synth_prep_tc_kernel, st::SMEM, "oi_synth_tiles_tc");
  if (rc) return rc;
  (void)launch_pdl(st::synth_prep_tc_kernel, dim3((unsigned)ctas), dim3(st::T), st::SMEM, s, a, k_map);
  oi::note_launch();
  return check_launch("oi_synth_tiles_tc");
}

}  // namespace oi

extern "C" int oi_synth_tc_constants(int ny, int br, int bc, void* image, long long bytes, void* stream) {
  using namespace oi;
  if (!image || ny <= 0 || br <= 0 || bc <= 0) return fail(OI_EINVAL, "oi_synth_tc_constants: bad arguments");
  if (ny % 128 != 0 || ny > 4096 || bc > 64 || 2 * br - 1 > st::M)
    return fail(OI_ERANGE, "oi_synth_tc_constants: ny=%d / band %dx%d unsupported", ny, br, bc);
  const long long need = (long long)(1 + ny / 128) * 4 * st::OPER;
  if (bytes < need) return fail(OI_ERANGE, "oi_synth_tc_constants: %lld bytes given, %lld needed", bytes, need);
  if ((uintptr_t)image % 16) return fail(OI_EINVAL, "oi_synth_tc_constants: image not 16-byte aligned");
  const long long threads = (long long)(1 + ny / 128) * 2048;
  st::synth_consts_kernel<<<(unsigned)ceil_div(threads, 256), 256, 0, (cudaStream_t)stream>>>(ny, br, bc,
                                                                                             (unsigned char*)image);
  oi::note_launch();
  return check_launch("oi_synth_tc_constants");
}

extern "C" int oi_synth_tiles_tc(const float* coarse, int nparts, int count, int br, int bc, const void* sconsts,
                                 int ny, void* tiles, void* stream) {
  using namespace oi;
  if (!coarse || !sconsts || !tiles || nparts <= 0 || count <= 0 || br <= 0 || bc <= 0)
    return fail(OI_EINVAL, "oi_synth_tiles_tc: bad arguments");
  if (ny % 128 != 0 || ny > 4096 || bc > 64 || 2 * br - 1 > st::M)
    return fail(OI_ERANGE, "oi_synth_tiles_tc: ny=%d / band %dx%d unsupported", ny, br, bc);
  if ((uintptr_t)coarse % 16 || (uintptr_t)sconsts % 16 || (uintptr_t)tiles % 16)
    return fail(OI_EINVAL, "oi_synth_tiles_tc: coarse, constants and tiles must be 16-byte aligned");
  return synth_tiles_tc(coarse, nparts, count, br, bc, sconsts, ny, tiles, (cudaStream_t)stream);
}

extern "C" int oi_coarse_to_image_tcs(const float* coarse, int nparts, int count, int br, int bc, const void* sconsts,
                                      const void* cconsts, int ny, int nx, void* scratch_tiles, float* out,
                                      void* stream) {
  using namespace oi;
  if (!coarse || !sconsts || !cconsts || !scratch_tiles || !out || nparts <= 0 || count <= 0 || br <= 0 || bc <= 0)
    return fail(OI_EINVAL, "oi_coarse_to_image_tcs: bad arguments");
  if (ny % 128 != 0 || ny > 4096 || nx % 128 != 0 || nx > 4096 || bc > 64 || 2 * br - 1 > st::M)
    return fail(OI_ERANGE, "oi_coarse_to_image_tcs: grid %dx%d / band %dx%d unsupported", ny, nx, br, bc);
  if ((uintptr_t)coarse % 16 || (uintptr_t)sconsts % 16 || (uintptr_t)cconsts % 16 || (uintptr_t)scratch_tiles % 16)
    return fail(OI_EINVAL, "oi_coarse_to_image_tcs: coarse, constants and tiles must be 16-byte aligned");
  cudaStream_t s = (cudaStream_t)stream;
  int rc = synth_tiles_tc(coarse, nparts, count, br, bc, sconsts, ny, scratch_tiles, s);
  if (rc) return rc;
  return rows_inv_from_tiles(scratch_tiles, count, ny, nx, cconsts, out, s);
}
