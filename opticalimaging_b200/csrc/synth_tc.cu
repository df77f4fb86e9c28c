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
// constant operands G and A_t are generated by the converter warps in shared memory from small tables (the row
// Dirichlet kernel depends on y and sr only through sr ny/128 - y, so a table of ny values holds every A tile;
// G is the coarse grid's cos / sin), the next tile's A as soon as the MMAs of the current one finish.  Loading
// them instead cost 64 KB per y tile over the SM's path to L2 next to the V tile's 64 KB of stores (~2.7 us per
// tile against ~1.5 us with either stream alone).
//
// Roles (320 threads): warps 0-7 convert (fold, G and A generation, U^T conversion, V drain; two warps per
// tensor-memory lane quarter), warp 9 lane 0 issues the MMAs (warp 8 only helps load the tables).  A V tile is
// staged in shared memory in its final (swizzled operand) layout -- in the stage-1 B region, free while the
// item's tiles drain -- and leaves as bulk copies issued by warp 0 lane 0: written straight from registers, each
// lane's 16-byte pieces of one row would touch 32 lines per warp store.  Every mbarrier wait is bounded (2 s); on
// expiry the role records the device status and stops, warp 0 lane 0 waits for its bulk copies and the MMA thread
// for its issued MMAs before memory is released.
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
constexpr int T = 320;                     // 8 converter warps, an idle warp, MMA warp
constexpr uint32_t GA_OFF = 0;                           // generated constant operand: G (stage 1), then A_t
constexpr uint32_t A1_OFF = GA_OFF + 4 * OPER;           // the folded coarse image (stage-1 B), later the V staging
constexpr uint32_t B2_OFF = A1_OFF + 4 * OPER;           // stage-2 B (U^T)
constexpr uint32_t TAB_OFF = B2_OFF + 4 * OPER;          // tables: g [ny], cos [M], sin [M] (float)
constexpr uint32_t TAB_BYTES = (4096 + 2 * M) * 4;
constexpr uint32_t MISC = TAB_OFF + TAB_BYTES;
constexpr uint32_t SMEM = MISC + 512 + 1024;
static_assert(A1_OFF % 1024 == 0 && B2_OFF % 1024 == 0 && MISC % 16 == 0, "operand alignment");
static_assert(SMEM <= SMEM_LIMIT, "synthesis preparation: shared memory");

struct Args {
  const float* coarse;      // [nparts][count][128][128]
  long long part_stride;    // floats between partial sums
  int nparts, count, ny, tp, bc;
  const float* tables;      // oi_synth_tc_constants: g [ny], cos [M], sin [M]
  unsigned char* tiles;     // V tiles [count * ny / 128][64 KB]
};

__device__ __forceinline__ void fail_status() { atomicExch(&g_synth_status, 1); }

// Converter warps' share of generating a constant operand block set [hi k0 | hi k1 | lo k0 | lo k1] x [128 rows]
// [64] into `dst` from the tables: 2048 tasks (row, 8-column chunk) over 256 threads, lanes on consecutive rows.
//   G (u < 0):  row n, column sc: (qc ? 2 : 1)/M (n < 64 ? cos : sin)(2 pi qc sc / M), qc = n mod 64, zero for
//               qc >= bc -- the cos / sin tables hold float(cos / sin) and the scale is a power of two, so the
//               value is the float of the double product;
//   A_u (u >= 0): row y = 128 u + r, column sr: g[(sr ny/M - y) mod ny], the Dirichlet kernel of the row band.
__device__ __forceinline__ void generate(const float* tab, int ny, int bc, int u, int tid, unsigned char* dst) {
  const float* g = tab;
  const float* cs = tab + ny;
  const int TYm = ny / M;
#pragma unroll 1
  for (int t = 0; t < 8; ++t) {
    const int task = tid + 256 * t, r = task & 127, ch = task >> 7, kb = ch >> 3, q = ch & 7;
    float v[8];
    if (u < 0) {
      const int qc = r & 63;
      const float sc = qc ? 2.0f / M : 1.0f / M;
      const float* tb = cs + (r < 64 ? 0 : M);
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int k = 64 * kb + 8 * q + e;
        v[e] = qc < bc ? sc * tb[(qc * k) & (M - 1)] : 0.0f;
      }
    } else {
      const int y = 128 * u + r;
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int k = 64 * kb + 8 * q + e;
        const int d = k * TYm - y + ny;   // in (0, 2 ny): k TYm < ny and y < ny
        v[e] = g[d >= ny ? d - ny : d];
      }
    }
    uint32_t hi[4], lo[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) split2(v[2 * e], v[2 * e + 1], hi[e], lo[e]);
    const uint32_t o = swz(r, q);
    *(uint4*)(dst + kb * OPER + o) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *(uint4*)(dst + (2 + kb) * OPER + o) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
  }
}

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

__global__ void __launch_bounds__(T, 1) synth_prep_tc_kernel(Args a) {
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char* gbase = smem_raw + (base - raw);
  const uint32_t misc = base + MISC;
  // barriers: a1full (the folded image and G generated by all eight converter warps), d1full (U^T complete in
  // tensor memory), b2full (stage-2 B written), b2free (the item's stage-2 MMAs finished), afull (an A tile
  // generated), accf[2] / acce[2] (v tile complete / drained), fin (every issued MMA finished, at the end),
  // vstaged (a V tile staged by the eight converter warps), vsfree (its bulk copies have read the staging)
  const uint32_t a1full = misc, d1full = misc + 8, b2full = misc + 16, b2free = misc + 24, afull = misc + 32,
                 accf = misc + 40, acce = misc + 56, fin = misc + 72, vstaged = misc + 80, vsfree = misc + 88;
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
    mbar_init(a1full, 8);
    mbar_init(d1full, 1);
    mbar_init(b2full, 8);
    mbar_init(b2free, 1);
    mbar_init(afull, 8);
    for (int s = 0; s < 2; ++s) {
      mbar_init(accf + 8 * s, 1);
      mbar_init(acce + 8 * s, 8);
    }
    mbar_init(fin, 1);
    mbar_init(vstaged, 8);
    mbar_init(vsfree, 1);
    mbar_init_fence();
  }
  pdl_trigger();
  pdl_wait();   // the coarse sums come from the coherent sum (and the tables may be fresh on the stream)
  float* tab = (float*)(gbase + TAB_OFF);
  for (int i = tid; i < a.ny + 2 * M; i += T) tab[i] = __ldg(a.tables + i);
  fence_before();
  __syncthreads();   // barrier inits and the tables
  fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 9) {
    if (lane == 0) {
      constexpr uint32_t ID = idesc(128, false);
      const uint32_t ga = base + GA_OFF, a1 = base + A1_OFF, b2 = base + B2_OFF;
      Ring ab{0, 0};
      bool ok = true, issued = false;
      int m = 0;   // v tiles issued (A tiles consumed)
      for (int n = 0; n < NI && ok; ++n) {
        const long long it = i0 + n;
        const int grp = (int)(it % H), t0 = grp * a.tp, t1 = min(TY, t0 + a.tp);
        ok = wait_bar(a1full, (uint32_t)(n & 1));
        if (!ok) break;
        fence_after();
        issued = true;
        // stage 1: D1 = G^T c^T = U^T (lanes n, columns sr); A = G, B = the folded image; hi hi, hi lo, lo hi
#pragma unroll
        for (int kb = 0; kb < 2; ++kb) {
          const uint32_t ghi = ga + kb * OPER, glo = ga + (2 + kb) * OPER, chi = a1 + kb * OPER,
                         clo = a1 + (2 + kb) * OPER;
#pragma unroll
          for (int ks = 0; ks < 4; ++ks) {
            const uint32_t ko = 32 * ks;
            mma_ss(tmem, sdesc(ghi + ko), sdesc(chi + ko), ID, (kb | ks) ? 1u : 0u);
            mma_ss(tmem, sdesc(ghi + ko), sdesc(clo + ko), ID, 1);
            mma_ss(tmem, sdesc(glo + ko), sdesc(chi + ko), ID, 1);
          }
        }
        commit(d1full);
        ok = wait_bar(b2full, (uint32_t)(n & 1));
        if (!ok) break;
        fence_after();
        // stage 2, per y tile: D2[buf] = A_t U; A_t generated into the same region (B = U^T)
        for (int k = 0; k < t1 - t0 && ok; ++k, ++m) {
          if (m >= 2) {
            ok = wait_bar(acce + 8 * ab.slot, ab.phase ^ 1u);
            if (!ok) break;
          }
          ok = wait_bar(afull, (uint32_t)(m & 1));
          if (!ok) break;
          fence_after();
          const uint32_t d2 = tmem + 128 * (1 + ab.slot);
#pragma unroll
          for (int kb = 0; kb < 2; ++kb) {
            const uint32_t ahi = ga + kb * OPER, alo = ga + (2 + kb) * OPER, bhi = b2 + kb * OPER,
                           blo = b2 + (2 + kb) * OPER;
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
              const uint32_t ko = 32 * ks;
              mma_ss(d2, sdesc(ahi + ko), sdesc(bhi + ko), ID, (kb | ks) ? 1u : 0u);
              mma_ss(d2, sdesc(ahi + ko), sdesc(blo + ko), ID, 1);
              mma_ss(d2, sdesc(alo + ko), sdesc(bhi + ko), ID, 1);
            }
          }
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
  } else if (warp < 8) {
    // ---- warps 0-7: fold and G, U^T conversion, A tiles, V drain
    unsigned char* ga = gbase + GA_OFF;
    unsigned char* a1 = gbase + A1_OFF;
    unsigned char* b2 = gbase + B2_OFF;
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
    const int half = warp >> 2, row = 32 * (warp & 3) + lane;
    Ring ab{0, 0};
    bool ok = true;
    uint32_t vt = 0;   // V tiles staged
    // signal that this warp's part of a generated operand is in place for the MMAs
    auto done = [&](uint32_t bar) {
      fence_async_smem();
      fence_before();
      __syncwarp();
      if (lane == 0) arrive(bar);
    };
    for (int n = 0; n < NI && ok; ++n) {
      const long long it = i0 + n, img = it / H;
      const int grp = (int)(it % H), t0 = grp * a.tp, t1 = min(TY, t0 + a.tp);
      if (vt >= 1) {   // the previous item's last V tile has left the staging (the stage-1 B region)
        ok = warp_wait(vsfree, (vt - 1) & 1u);
        if (!ok) break;
      }
      // (the region of G / A: its last readers, the previous item's last tile of MMAs, completed before that
      // tile's accumulator was drained)
      fold(a, img, tid, a1);
      generate(tab, a.ny, a.bc, -1, tid, ga);
      done(a1full);
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
      done(b2full);
      generate(tab, a.ny, a.bc, t0, tid, ga);        // the stage-1 MMAs (readers of G) are complete
      done(afull);
      // V tiles: lane = y of the tile, this warp's half = re (blocks hi 0, lo 2) or im (hi 1, lo 3)
      for (int k = 0; k < t1 - t0 && ok; ++k, ++vt) {
        const int t = t0 + k;
        ok = warp_wait(accf + 8 * ab.slot, ab.phase);
        if (!ok) break;
        fence_after();
        if (k + 1 < t1 - t0) {   // the tile's MMAs are complete: the next tile's A replaces this one's
          generate(tab, a.ny, a.bc, t + 1, tid, ga);
          done(afull);
        }
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

// Tables of the generated constant operands, in double precision from exactly reduced phases, stored as float:
//   g[e]   = (1/M) sum_{|qr|<br} cos(2 pi qr e / ny),  e < ny  (A[y][sr] = g[(sr ny/M - y) mod ny]),
//   cos[j] = cos(2 pi j / M), sin[j] = sin(2 pi j / M),  j < M  (G).
__global__ void synth_consts_kernel(int ny, int br, float* tab) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id < ny) {
    const long long den = (long long)M * ny, d = (long long)M * id;
    double val = 0.0;
    for (int qr = -(br - 1); qr <= br - 1; ++qr) {
      long long p = ((long long)qr * d) % den;
      if (p < 0) p += den;
      val += cospi(2.0 * (double)p / (double)den);
    }
    tab[id] = (float)(val / M);
  } else if (id < ny + 2 * M) {
    const int j = id - ny, c = j % M;
    double sn, co;
    sincospi(2.0 * (double)c / M, &sn, &co);
    tab[id] = (float)(j < M ? co : sn);
  }
}

}  // namespace st

// The V tiles of count images from their coarse intensities (nparts partial sums); `sconsts` from
// oi_synth_tc_constants for (ny, br, bc).
int synth_tiles_tc(const float* coarse, int nparts, int count, int br, int bc, const void* sconsts, int ny,
                   void* tiles, cudaStream_t s) {
  (void)br;
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
  st::Args a{coarse, (long long)count * st::M * st::M, nparts, count, ny, best_tp, bc, (const float*)sconsts,
             (unsigned char*)tiles};
  int rc = ensure_smem((const void*)st::synth_prep_tc_kernel, st::SMEM, "oi_synth_tiles_tc");
  if (rc) return rc;
  (void)launch_pdl(st::synth_prep_tc_kernel, dim3((unsigned)ctas), dim3(st::T), st::SMEM, s, a);
  oi::note_launch();
  return check_launch("oi_synth_tiles_tc");
}

}  // namespace oi

extern "C" int oi_synth_tc_constants(int ny, int br, int bc, void* image, long long bytes, void* stream) {
  using namespace oi;
  if (!image || ny <= 0 || br <= 0 || bc <= 0) return fail(OI_EINVAL, "oi_synth_tc_constants: bad arguments");
  if (ny % 128 != 0 || ny > 4096 || bc > 64 || 2 * br - 1 > st::M)
    return fail(OI_ERANGE, "oi_synth_tc_constants: ny=%d / band %dx%d unsupported", ny, br, bc);
  const long long need = (long long)(ny + 2 * st::M) * 4;
  if (bytes < need) return fail(OI_ERANGE, "oi_synth_tc_constants: %lld bytes given, %lld needed", bytes, need);
  if ((uintptr_t)image % 16) return fail(OI_EINVAL, "oi_synth_tc_constants: image not 16-byte aligned");
  st::synth_consts_kernel<<<(unsigned)ceil_div((long long)ny + 2 * st::M, 256), 256, 0, (cudaStream_t)stream>>>(
      ny, br, (float*)image);
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
