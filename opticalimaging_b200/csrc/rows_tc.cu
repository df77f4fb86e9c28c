// The two N-point row passes of the split-BF16x3 form as dense DFT contractions on the tensor cores
// (tcgen05.mma, split BF16x3, FP32 accumulate in tensor memory):
//
//   forward   (oi_rows_fwd_tc)  t[b][ic][y] = sum_x mask[b][y][x] exp(+2 pi i (m0c+ic) x / nx)
//             -- the row half of the band spectrum (Scatter.CalculateSpectrum, Scatter.py:10-35, on the band);
//             (oi_rows_fwd_tc_half) the same for ic = 0 .. bch-1 at m0c = 0 only: for a real mask
//             t[-ic] = conj(t[ic]), so a symmetric band needs only its non-negative columns;
//   inverse   (oi_rows_inv_tc)  out[i][y][x] = sum_qc Re(v[i][qc][y] exp(-2 pi i qc x / nx))
//             -- the last pass of the synthesis (qc > 0 terms already doubled by the caller).
//
// Forward: D[y][n] (M = 128 rows, N = 128: n < 64 re / n >= 64 im of band column ic = n mod 64, K = x in
// chunks of 64) = A x W^T, A = the mask rows (converted to bf16 hi / lo), W = [cos; sin] of the band columns
// (a constant operand image, streamed per chunk).  Inverse: D[x][y] (M = 128 columns x of one x tile,
// N = 256 rows, K = (re | im) x 64 band columns) = C x V^T, C = [cos | sin] of the x tile (constant image,
// streamed in 16 KB pieces), V = v as bf16 hi / lo operand tiles (resident while the row-block pair lasts).  The
// accumulator's lanes are the rows (forward) or the columns (inverse), so every warp store of the result is one
// coalesced segment.  The forward pass takes its A operand (converted on the fly) from tensor memory, so its
// converters write no shared memory; the inverse reads both operands from shared memory, where its V tiles land
// by TMA.  (Measured issue rates, M = 128, K = 16: 64 cycles at N = 128 and 128 at N = 256 with either operand
// source; at N = 64, 48 cycles from shared memory and 56 with A in tensor memory, against 32.)
//
// Roles (352 threads): warps 0-7 convert the staged mask chunks into the A operand in tensor memory (forward)
// and drain finished accumulators to global memory (two warps per tensor-memory lane quarter); warps 8 and 10
// issue the loads into shared-memory rings (forward: 2-D tensor-map boxes of the masks and 1-D bulk copies of
// W; inverse: 2-D tensor-map boxes of the C pieces and of the V tiles; no multicast); warp 9 lane 0 issues the
// MMAs and commits them to mbarriers.  Accumulators are double-buffered so that draining
// overlaps the MMAs of the next blocks.
// Every mbarrier wait is bounded (2 s); on expiry the role records the status (oi_device_status) and stops,
// the others then expire in turn.  Before the CTA frees tensor memory and exits, each producer waits (bounded)
// for the copies it issued to land and the MMA thread commits its issued MMAs to a barrier and waits for them,
// so nothing writes shared or tensor memory after it is released.
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
constexpr uint32_t OPER = 128 * 128;       // one [128 rows][64 bf16] swizzled operand block (16 KB)

__device__ __forceinline__ void fail_status() { atomicExch(&g_rows_status, 1); }

// 8 floats -> 4 packed bf16 hi words and 4 lo words
__device__ __forceinline__ void split8(const float (&v)[8], uint32_t (&hi)[4], uint32_t (&lo)[4]) {
#pragma unroll
  for (int e = 0; e < 4; ++e) split2(v[2 * e], v[2 * e + 1], hi[e], lo[e]);
}

// ------------------------------------------------------------------------------------------ forward
// Items are pairs of 128-row blocks (rows 256 P .. 256 P + 255): one W chunk feeds both blocks' MMAs, so each
// 64-column chunk of mask costs 32 KB of mask plus 16 KB of W over the SM-to-L2 path instead of 32 + 32 (that
// path, about 30 bytes per cycle per SM, bounds this pass).  Shared memory: a ring of staging slots (the chunk
// of both blocks: per block two 128-byte-swizzled [128][32] float boxes, or one 64-byte-swizzled [128][64]
// uint8 box) and a ring of W chunks (hi, lo); FwdCfg sizes both rings to fill the 224 KB, so that as many mask
// bytes as fit are in flight from DRAM while a slot is converted.  Tensor memory: the two blocks' accumulators
// (columns 0 and 128, 128 each) and two A slots at 256 + 128 s (block h: hi at 64 h, lo at 64 h + 32), the
// chunk as bf16 hi / lo written by the converters, read by the MMA.  A pair past the last row block (odd count)
// reads zeros and stores nothing for its second block.
// NB = band columns per real / imaginary part of W: 64 (a band of up to 64 columns, N = 128), or 32 for the
// Hermitian half of a real mask's symmetric band (columns 0 .. bch-1 only, N = 64, a 16 KB W chunk: half the
// W bytes per mask byte over the SM-to-L2 path and half the MMA width).
constexpr uint32_t F_STG = 128 * 64 * 4;             // one row block's chunk (float)
constexpr uint32_t F_ACC = 128;                      // accumulator columns per block
constexpr uint32_t F_COL_A = 2 * F_ACC;
constexpr uint32_t F_TMEM_COLS = 512;

template <int KIND, int NB>
struct FwdCfg {
  static constexpr bool U8 = KIND == OI_FIELD_U8;
  static constexpr uint32_t BLK = U8 ? 128 * 64 : F_STG;   // one block's chunk
  static constexpr uint32_t PSTG = 2 * BLK;                 // one staging slot: both blocks
  static constexpr uint32_t WOP = 2 * NB * 128;             // one precision of a W chunk: [2 NB rows][64 bf16]
  static constexpr uint32_t FW = 2 * WOP;                   // one W chunk (hi, lo) and its slot
  // float32 chunks: 2 slots of 64 KB beside 3 W slots of 32 KB (NB = 64), 3 beside 2 of 16 KB (NB = 32);
  // uint8 chunks: 8 slots of 16 KB
  static constexpr int NS = U8 ? 8 : (NB == 32 ? 3 : 2);
  static constexpr int NWS = (!U8 && NB == 32) ? 2 : 3;
  static constexpr uint32_t WOFF = NS * PSTG;
  static constexpr uint32_t MISC = WOFF + NWS * FW;
  static constexpr uint32_t SMEM = MISC + 384 + 1024;
  // mbarriers from MISC: sfull[NS], sfree[NS], wfull[NWS], wdone[NWS], conv[2], adone[2], accf, acce, fin;
  // the tensor-memory address at MISC + 248, the lo flags at MISC + 256 .. 319
  static constexpr uint32_t SFULL = 0, SFREE = 8 * NS, WFULL = 16 * NS, WDONE = WFULL + 8 * NWS,
                            CONV = WDONE + 8 * NWS, ADONE = CONV + 16, ACCF = ADONE + 16, ACCE = ACCF + 8,
                            FIN = ACCE + 8;
  static_assert(FIN + 8 <= 248, "forward row pass: barriers");
  static_assert(SMEM <= SMEM_LIMIT, "forward row pass: shared memory");
};

struct FwdArgs {
  long long rows;           // batch * ny (a multiple of 128)
  int ny, nx, bc;
  const unsigned char* w;   // constant image: per 64-column chunk, [hi | lo] x [2 NB rows][64]
  float2* t;                // [batch][bc][ny]
};

constexpr int F_NT = NT + 32;   // + a warp issuing the W loads

template <int KIND, int NB>
__global__ void __launch_bounds__(F_NT, 1) rows_fwd_tc_kernel(FwdArgs a, const __grid_constant__ CUtensorMap mask_map) {
  static_assert(NB == 64 || NB == 32, "forward row pass: NB");
  using Cfg = FwdCfg<KIND, NB>;
  constexpr int F_NS = Cfg::NS, F_NWS = Cfg::NWS;
  constexpr uint32_t WOP = Cfg::WOP, FW = Cfg::FW;
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char* gbase = smem_raw + (base - raw);
  const uint32_t misc = base + Cfg::MISC;
  // barriers: sfull (staging landed), sfree (staging read), wfull (W landed), wdone (MMAs reading the W slot
  // finished), conv[2] (A slot written), adone[2] (MMAs reading the A slot finished), accf (accumulators
  // complete), acce (accumulators drained), fin (every issued MMA finished, at the end)
  const uint32_t sfull = misc + Cfg::SFULL, sfree = misc + Cfg::SFREE, wfull = misc + Cfg::WFULL,
                 wdone = misc + Cfg::WDONE, conv = misc + Cfg::CONV, adone = misc + Cfg::ADONE,
                 accf = misc + Cfg::ACCF, acce = misc + Cfg::ACCE, fin = misc + Cfg::FIN;
  volatile uint32_t* tmem_slot = (volatile uint32_t*)(gbase + Cfg::MISC + 248);
  // per A slot and converter warp: 1 when the warp's part of the chunk has a non-zero bf16 lo half (a mask value
  // not exact in bf16); when no warp sets it the lo x hi products are exactly zero and are not issued
  volatile uint32_t* lo_flags = (volatile uint32_t*)(gbase + Cfg::MISC + 256);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int KC = a.nx / 64;
  const long long R = a.rows / 128;                  // row blocks
  const long long items = (R + 1) / 2;               // pairs
  const long long G = gridDim.x;
  const long long i0 = (long long)blockIdx.x * items / G, i1 = ((long long)blockIdx.x + 1) * items / G;
  const long long nchunks = (i1 - i0) * KC;
  constexpr bool U8 = KIND == OI_FIELD_U8;
  constexpr uint32_t BLK = Cfg::BLK;

  if (warp == 0) tmem_alloc(misc + 248, F_TMEM_COLS);
  if (tid == 0) {
    for (int s = 0; s < F_NS; ++s) {
      mbar_init(sfull + 8 * s, 1);
      mbar_init(sfree + 8 * s, 8);
    }
    for (int s = 0; s < F_NWS; ++s) {
      mbar_init(wfull + 8 * s, 1);
      mbar_init(wdone + 8 * s, 1);
    }
    for (int s = 0; s < 2; ++s) {
      mbar_init(conv + 8 * s, 8);
      mbar_init(adone + 8 * s, 1);
    }
    mbar_init(accf, 1);
    mbar_init(acce, 8);
    mbar_init(fin, 1);
    mbar_init_fence();
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;
  pdl_trigger();
  pdl_wait();   // the masks and t are ordered after the preceding kernels from here on

  // Loop state advances incrementally (ring slot / phase, chunk / item): no integer division per chunk.
  const int NC = (int)nchunks;
  if (warp == 8) {
    // ---- mask producer: chunk g of both blocks into staging slot g % 2 as soon as the slot has been read
    if (lane == 0) {
      Ring st{0, 0};
      int c = 0, y = (int)(i0 * 256), g = 0;
      for (; g < NC; ++g) {
        if (g >= F_NS && !wait_bar(sfree + 8 * st.slot, st.phase ^ 1u)) {
          fail_status();
          break;
        }
        const uint32_t dst = base + st.slot * Cfg::PSTG;
        expect_tx(sfull + 8 * st.slot, 2 * BLK);
#pragma unroll
        for (int h = 0; h < 2; ++h) {   // rows past the tensor's end read as zeros
          tma_load_2d(dst + h * BLK, &mask_map, 64 * c, y + 128 * h, sfull + 8 * st.slot);
          if (!U8) tma_load_2d(dst + h * BLK + BLK / 2, &mask_map, 64 * c + 32, y + 128 * h, sfull + 8 * st.slot);
        }
        st.next(F_NS);
        if (++c == KC) {
          c = 0;
          y += 256;
        }
      }
      drain_ring(sfull, st, g, F_NS);   // the copies in flight land before shared memory is released
    }
  } else if (warp == 10) {
    // ---- W producer: chunk g's W into slot g % 3 once the MMAs of chunk g-3 have finished
    if (lane == 0) {
      Ring ws{0, 0};
      int c = 0, g = 0;
      for (; g < NC; ++g) {
        if (g >= F_NWS && !wait_bar(wdone + 8 * ws.slot, ws.phase ^ 1u)) {
          fail_status();
          break;
        }
        expect_tx(wfull + 8 * ws.slot, FW);
        bulk_g2s(base + Cfg::WOFF + ws.slot * FW, a.w + (long long)c * FW, FW, wfull + 8 * ws.slot);
        ws.next(F_NWS);
        if (++c == KC) c = 0;
      }
      drain_ring(wfull, ws, g, F_NWS);
    }
  } else if (warp == 9) {
    // ---- MMA issue: D[h] += A[h](tmem slot) x W^T over the chunk (K steps of 16), split BF16x3, h = both blocks
    if (lane == 0) {
      constexpr uint32_t ID = idesc(2 * NB, false);
      Ring as{0, 0}, ws{0, 0};
      int c = 0, n = 0;
      bool issued = false;
      for (int g = 0; g < NC; ++g) {
        bool ok = wait_bar(conv + 8 * as.slot, as.phase);
        if (ok) ok = wait_bar(wfull + 8 * ws.slot, ws.phase);
        if (ok && c == 0 && n >= 1) ok = wait_bar(acce, (uint32_t)((n - 1) & 1));   // previous pair drained
        if (!ok) {
          fail_status();
          break;
        }
        issued = true;
        fence_after();
        const uint32_t wch = base + Cfg::WOFF + ws.slot * FW;
        uint32_t lo_any = 0;
        if (!U8) {   // the eight warps' flags of this A slot, as two 16-byte reads
          uint32_t f0, f1, f2, f3, f4, f5, f6, f7;
          const uint32_t fa = smem_u32((const void*)(lo_flags + 8 * as.slot));
          asm volatile("ld.volatile.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(f0), "=r"(f1), "=r"(f2), "=r"(f3) : "r"(fa));
          asm volatile("ld.volatile.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(f4), "=r"(f5), "=r"(f6), "=r"(f7)
                       : "r"(fa + 16u));
          lo_any = f0 | f1 | f2 | f3 | f4 | f5 | f6 | f7;
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const uint32_t d = tmem + h * F_ACC, at = tmem + F_COL_A + 128 * as.slot + 64 * h;
#pragma unroll
          for (int ks = 0; ks < 4; ++ks) {
            const uint32_t ko = 32 * ks;
            mma_ts(d, at + 8 * ks, sdesc(wch + ko), ID, (c | ks) ? 1u : 0u);            // hi hi
            mma_ts(d, at + 8 * ks, sdesc(wch + WOP + ko), ID, 1);                      // hi lo
            if (lo_any) mma_ts(d, at + 32 + 8 * ks, sdesc(wch + ko), ID, 1);           // lo hi
          }
        }
        commit(adone + 8 * as.slot);
        commit(wdone + 8 * ws.slot);
        if (c == KC - 1) commit(accf);
        as.next(2);
        ws.next(F_NWS);
        if (++c == KC) {
          c = 0;
          ++n;
        }
      }
      if (issued) {   // every MMA issued has finished before tensor and shared memory are released
        commit(fin);
        wait_bar(fin, 0);
      }
    }
  } else if (warp < 8) {
    // ---- converters (warps 0-7): staging -> A slot in tensor memory; drain finished accumulators.
    // Warp w converts rows 32 (w & 3) .. +31 of both blocks (its tensor-memory lane quarter), columns
    // 32 (w >> 2) .. +31.
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
    const int half = warp >> 2, r = 32 * (warp & 3) + lane;
    bool ok = true;
    auto drain = [&](int n) {
      // accumulators of pair n: lanes = rows, columns re [0,NB) / im [NB,2NB) of band column ic (this warp:
      // DC columns from DC half); block by block, released (acce) once the second block is in registers
      constexpr int DC = NB / 2;
      if (!warp_wait(accf, (uint32_t)(n & 1))) return false;
      fence_after();
#pragma unroll 1
      for (int h = 0; h < 2; ++h) {
        float re[DC], im[DC];
        const uint32_t ta = tmem + lane_base + h * F_ACC + DC * half;
        if constexpr (DC == 32) tmem_ld32x2(ta, ta + NB, re, im);
        else tmem_ld16x2(ta, ta + NB, re, im);
        if (h == 1) {
          fence_before();
          __syncwarp();
          if (lane == 0) arrive(acce);
        }
        const long long rb = 2 * (i0 + n) + h;
        if (rb < R) {
          const int row = (int)(rb * 128) + r;
          const int b = row / a.ny, y = row - b * a.ny;
          float2* dst = a.t + ((long long)b * a.bc + DC * half) * a.ny + y;
#pragma unroll
          for (int j = 0; j < DC; ++j)
            if (DC * half + j < a.bc) dst[(long long)j * a.ny] = make_float2(re[j], im[j]);
        }
      }
      return true;
    };
    Ring st{0, 0}, as{0, 0};
    int c = 0, n = 0;
    for (int g = 0; g < NC && ok; ++g) {
      ok = warp_wait(sfull + 8 * st.slot, st.phase);
      if (ok && g >= 2) ok = warp_wait(adone + 8 * as.slot, as.phase ^ 1u);   // A slot free (chunk g-2 done)
      if (!ok) break;
      bool lo_nz = false;
#pragma unroll 1
      for (int h = 0; h < 2; ++h) {
        float v[32];
        const unsigned char* blk = gbase + st.slot * Cfg::PSTG + h * BLK;
        if (U8) {
          const unsigned char* row = blk + r * 64;   // 64-byte swizzle: chunk j at j ^ ((r >> 1) & 3)
#pragma unroll
          for (int jj = 0; jj < 2; ++jj) {
            const uint4 u = *(const uint4*)(row + (((2 * half + jj) ^ ((r >> 1) & 3)) << 4));
            const uint32_t w4[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
            for (int e = 0; e < 16; ++e) v[16 * jj + e] = (float)((w4[e >> 2] >> (8 * (e & 3))) & 0xFF);
          }
        } else {
          const unsigned char* row = blk + half * (F_STG / 2) + r * 128;   // 128-byte swizzle
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const float4 x = *(const float4*)(row + ((j ^ (r & 7)) << 4));
            v[4 * j] = x.x, v[4 * j + 1] = x.y, v[4 * j + 2] = x.z, v[4 * j + 3] = x.w;
          }
        }
        uint32_t hi[16], lo[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) split2(v[2 * e], v[2 * e + 1], hi[e], lo[e]);
        const uint32_t at = tmem + lane_base + F_COL_A + 128 * as.slot + 64 * h + 16 * half;
        tmem_st16(at, hi);
        if (!U8) {
#pragma unroll
          for (int e = 0; e < 16; ++e) lo_nz |= lo[e] != 0u;
          tmem_st16(at + 32, lo);          // always written: another warp's flag may make the MMAs read it
        }
      }
      __syncwarp();
      if (lane == 0) arrive(sfree + 8 * st.slot);          // the staging slot may be refilled
      if (!U8) lo_nz = __any_sync(0xffffffffu, lo_nz);
      wait_st();
      fence_before();
      __syncwarp();
      if (lane == 0) {
        if (!U8) lo_flags[8 * as.slot + warp] = lo_nz ? 1u : 0u;   // read by the MMA thread after `conv`
        arrive(conv + 8 * as.slot);
      }
      // the previous pair's accumulators are complete once this pair's first chunk is converted
      if (c == 0 && n >= 1) ok = drain(n - 1);
      st.next(F_NS);
      as.next(2);
      if (++c == KC) {
        c = 0;
        ++n;
      }
    }
    if (ok && NC > 0) ok = drain((int)(i1 - i0) - 1);
    if (!ok && lane == 0) fail_status();
  }
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    tmem_dealloc(tmem, F_TMEM_COLS);
  }
}

// ------------------------------------------------------------------------------------------ inverse
// v -> V operand tiles: for each block of 128 rows (image i, rows y0 .. y0+127) the bf16 hi / lo operand
// [hi: kc 0 (re of band column qc < 64), kc 1 (im)][lo: kc 0, kc 1] x [128 rows y][64], in the swizzled shared-
// memory layout, so that the row kernel loads it with one bulk copy.  One block per tile; v is read coalesced
// (128 consecutive y of one band column) into shared memory and written as 16-byte chunks.
constexpr uint32_t VT_BYTES = 4 * OPER;   // one V tile (64 KB)

__global__ void __launch_bounds__(256) v_tiles_kernel(const float2* __restrict__ v, int ny, int bc,
                                                       unsigned char* __restrict__ tiles) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* st = (float2*)smem_raw;   // [bc][128]
  const int tid = threadIdx.x;
  const long long r = blockIdx.x, row0 = r * 128, i = row0 / ny;
  const int y0 = (int)(row0 - i * ny);
  // bc rows of 128 complex = 64 float4 each; all loads of a thread issued before any store (16 in flight)
  constexpr int PER = 16;   // 16 x 256 float4 >= 64 x 64
  float4 buf[PER];
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    const int e = tid + 256 * p, qc = e >> 6, y2 = e & 63;
    buf[p] = qc < bc ? __ldg((const float4*)(v + (i * bc + qc) * (long long)ny + y0) + y2) : make_float4(0.f, 0.f, 0.f, 0.f);
  }
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    const int e = tid + 256 * p, qc = e >> 6;
    if (qc < bc) ((float4*)st)[e] = buf[p];
  }
  __syncthreads();
  unsigned char* out = tiles + r * VT_BYTES;
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int id = tid + 256 * p, y = id & 127, q = id >> 7;   // row y, band columns 8q .. 8q+7
    float re[8], im[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int qc = 8 * q + e;
      const float2 x = qc < bc ? st[qc * 128 + y] : make_float2(0.f, 0.f);
      re[e] = x.x;
      im[e] = x.y;
    }
    uint32_t hi[4], lo[4];
    const uint32_t o = swz(y, q);
    split8(re, hi, lo);
    *(uint4*)(out + o) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *(uint4*)(out + 2 * OPER + o) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    split8(im, hi, lo);
    *(uint4*)(out + OPER + o) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *(uint4*)(out + 3 * OPER + o) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
  }
}

// Items (row-block pair P = rows 256 P .. 256 P + 255, x tile j) in pair-major order, cut into one contiguous
// range per CTA.  A CTA keeps the V tiles of its pair (128 KB) and streams the C tiles of the nx / 128 x tiles
// (64 KB each, L2-resident for the whole launch) through a ring of 6 pieces of 16 KB ([128 x][64] blocks: hi or
// lo of kc 0 or 1), released one by one as soon as the MMAs reading them have finished.  One C tile serves 256
// output rows (N = 256), so the operand stream is half the output stream, and every V tile is read once.  A pair
// past the last row block (odd row-block count) reads zeros for its second half and stores nothing there.
// Tensor memory: two accumulators of 256 columns.
constexpr int I_NC = 6;                               // C pieces in the ring
constexpr int I_NT = NT + 32;                         // + a warp loading the V tiles
constexpr uint32_t I_ACC = 256;                       // accumulator columns (N)
constexpr uint32_t I_C = 0;
constexpr uint32_t I_V = I_NC * OPER;                 // V of the pair: block q (hi kc 0, hi kc 1, lo kc 0, lo kc 1)
                                                      // at 2 q OPER, [256 rows][64]
constexpr uint32_t I_MISC = I_V + 8 * OPER;
constexpr uint32_t I_SMEM = I_MISC + 512 + 1024;
constexpr uint32_t I_TMEM_COLS = 2 * I_ACC;
static_assert(I_SMEM <= SMEM_LIMIT, "inverse row pass: shared memory");

struct InvArgs {
  const unsigned char* vt;  // V tiles, [rows / 128][64 KB]: [hi kc 0 | hi kc 1 | lo kc 0 | lo kc 1] x [128 y][64]
  long long rows;           // count * ny (a multiple of 128)
  int ny, nx;
  const unsigned char* c;   // constant image: per 128-column x tile, [hi kc 0 | hi kc 1 | lo kc 0 | lo kc 1] x [128 x][64]
  float* out;               // [count][ny][nx]
};

// Block index (in the image layout above) of C piece p of an x tile: p = 0 hi kc 0, 1 lo kc 0, 2 hi kc 1, 3 lo kc 1.
__host__ __device__ constexpr int piece_block(int p) { return (p & 1) * 2 + (p >> 1); }

// Drain accumulator `buf` (item: pair P, x tile j): lanes = x of this warp's quarter, columns 128 half ..
// 128 half + 127 = rows of row block 2 P + half, stored as coalesced 128-byte row segments.
__device__ __forceinline__ void inv_drain(const InvArgs& a, uint32_t taddr, uint32_t acce, int half, int warp,
                                          int lane, int j, long long rb, bool store, int buf) {
  fence_after();
  if (store) {
    float* dst = a.out + rb * 128 * (long long)a.nx + j * 128 + 32 * (warp & 3) + lane;
    const uint32_t col = taddr + buf * I_ACC + 128 * half;
#pragma unroll 1
    for (int p = 0; p < 4; ++p) {
      float o0[16], o1[16];
      tmem_ld16x2(col + 32 * p, col + 32 * p + 16, o0, o1);
#pragma unroll
      for (int k = 0; k < 16; ++k) __stcs(dst + (long long)(32 * p + k) * a.nx, o0[k]);
#pragma unroll
      for (int k = 0; k < 16; ++k) __stcs(dst + (long long)(32 * p + 16 + k) * a.nx, o1[k]);
    }
  }
  fence_before();
  __syncwarp();
  if (lane == 0) arrive(acce + 8 * buf);
}

// Producers: warp 8 the C pieces of every item, warp 10 the V tiles of every pair (after the MMAs of the previous
// pair have finished).  MMA (warp 9): D[acc] = C x V^T, per C piece the MMAs that read it (C hi: hi x V hi and
// hi x V lo; C lo: lo x V hi), 24 of 128 x 256 x 16 per item, both operands from shared memory.  Warps 0-7 drain.
// The C and V images are read through 2-D tensor maps over their 128-byte rows (uint16, no swizzle: the images
// are stored pre-swizzled, so a box lands in shared memory exactly as the operand layout wants it), one box of
// 128 rows per 16 KB block.
__global__ void __launch_bounds__(I_NT, 1) rows_inv_tc_kernel(InvArgs a, const __grid_constant__ CUtensorMap c_map,
                                                               const __grid_constant__ CUtensorMap v_map) {
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char* gbase = smem_raw + (base - raw);
  const uint32_t misc = base + I_MISC;
  // barriers: cfull[6] (piece landed), cfree[6] (MMAs reading the piece finished), vfull[4] (V block q of the
  // pair landed), vfree[4] (MMAs reading V block q finished), accf[2] (accumulator complete), acce[2]
  // (accumulator drained), fin (MMAs finished, failure path)
  const uint32_t cfull = misc, cfree = misc + 48, vfull = misc + 96, vfree = misc + 128, accf = misc + 160,
                 acce = misc + 176, fin = misc + 192;
  volatile uint32_t* tmem_slot = (volatile uint32_t*)(gbase + I_MISC + 256);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int JT = a.nx / 128;                       // x tiles
  const long long R = a.rows / 128, PR = (R + 1) / 2;
  const long long items = PR * JT;
  const long long G = gridDim.x;
  const long long i0 = (long long)blockIdx.x * items / G, i1 = ((long long)blockIdx.x + 1) * items / G;
  const long long N = i1 - i0;

  if (warp == 0) tmem_alloc(misc + 256, I_TMEM_COLS);
  if (tid == 0) {
    for (int s = 0; s < I_NC; ++s) {
      mbar_init(cfull + 8 * s, 1);
      mbar_init(cfree + 8 * s, 1);
    }
    for (int s = 0; s < 2; ++s) {
      mbar_init(accf + 8 * s, 1);
      mbar_init(acce + 8 * s, 8);
    }
    for (int q = 0; q < 4; ++q) {
      mbar_init(vfull + 8 * q, 1);
      mbar_init(vfree + 8 * q, 1);
    }
    mbar_init(fin, 1);
    mbar_init_fence();
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;

  pdl_trigger();
  if (warp != 8) pdl_wait();   // warp 8 streams only the constant C tiles; the rest read V or write the image

  // item i0 + n = (pair P, x tile j); counters advance per item (the pair changes exactly when j wraps)
  const long long P0 = i0 / JT;
  const int j0 = (int)(i0 - P0 * JT);
  if (warp == 8) {
    // ---- C pieces: piece g of the range into ring slot g % 6 once the MMAs of piece g-6 have finished
    if (lane == 0) {
      Ring cs{0, 0};
      int j = j0, g = 0;
      bool ok = true;
      for (long long n = 0; n < N && ok; ++n) {
        for (int p = 0; p < 4; ++p, ++g) {
          if (g >= I_NC && !wait_bar(cfree + 8 * cs.slot, cs.phase ^ 1u)) {
            ok = false;
            break;
          }
          expect_tx(cfull + 8 * cs.slot, OPER);
          tma_load_2d(base + I_C + cs.slot * OPER, &c_map, 0, (j * 4 + piece_block(p)) * 128, cfull + 8 * cs.slot);
          cs.next(I_NC);
        }
        if (++j == JT) j = 0;
      }
      if (!ok) fail_status();
      drain_ring(cfull, cs, g, I_NC);   // the copies in flight land before shared memory is released
    }
  } else if (warp == 10) {
    // ---- V tiles of pair k of the range: block q (hi kc 0, hi kc 1, lo kc 0, lo kc 1; both row blocks) once the
    // MMAs of pair k-1 that read it have finished, in the order the MMAs first need them (0, 2, 1, 3)
    if (lane == 0) {
      const long long npairs = N > 0 ? (i1 - 1) / JT - P0 + 1 : 0;
      int lq[4] = {0, 0, 0, 0};   // loads issued per block
      bool ok = true;
      for (int k = 0; k < npairs && ok; ++k) {
        const long long rb = 2 * (P0 + k);
        for (int i = 0; i < 4; ++i) {
          const int q = ((i & 1) << 1) | (i >> 1);
          if (k >= 1 && !wait_bar(vfree + 8 * q, (uint32_t)((k - 1) & 1))) {
            ok = false;
            break;
          }
          expect_tx(vfull + 8 * q, 2 * OPER);
          for (int h = 0; h < 2; ++h)   // rows past the tensor's end read as zeros
            tma_load_2d(base + I_V + (2 * q + h) * OPER, &v_map, 0, (int)(((rb + h) * 4 + q) * 128), vfull + 8 * q);
          ++lq[q];
        }
      }
      if (!ok) fail_status();
      for (int q = 0; q < 4; ++q)   // the last tiles have landed
        if (lq[q] > 0) wait_bar(vfull + 8 * q, (uint32_t)((lq[q] - 1) & 1));
    }
  } else if (warp == 9) {
    if (lane == 0) {
      constexpr uint32_t ID = idesc(I_ACC, false);
      Ring cs{0, 0}, ab{0, 0};
      uint32_t vph = 1;
      int j = j0;
      bool ok = true;
      int issued = 0;
      for (long long n = 0; n < N && ok; ++n) {
        const bool first = n == 0 || j == 0, last = j == JT - 1;   // first / last item of its pair
        if (first) vph ^= 1u;                                       // parity of this pair's V loads
        if (++j == JT) j = 0;
        if (ok && n >= 2) ok = wait_bar(acce + 8 * ab.slot, ab.phase ^ 1u);
        const uint32_t d = tmem + ab.slot * I_ACC;
        for (int p = 0; p < 4 && ok; ++p) {
          if (first && (p & 1) == 0) {   // V hi and lo of this kc for the new pair
            ok = wait_bar(vfull + 8 * (p >> 1), vph) && wait_bar(vfull + 8 * ((p >> 1) + 2), vph);
            if (!ok) break;
          }
          ok = wait_bar(cfull + 8 * cs.slot, cs.phase);
          if (!ok) break;
          fence_after();
          const uint32_t cp = base + I_C + cs.slot * OPER;
          const uint32_t vhi = base + I_V + (uint32_t)(p >> 1) * 2 * OPER, vlo = vhi + 4 * OPER;
          if ((p & 1) == 0) {
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
              mma_ss(d, sdesc(cp + 32 * ks), sdesc(vhi + 32 * ks), ID, (p | ks) ? 1u : 0u);   // hi hi
              mma_ss(d, sdesc(cp + 32 * ks), sdesc(vlo + 32 * ks), ID, 1);                    // hi lo
            }
          } else {
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) mma_ss(d, sdesc(cp + 32 * ks), sdesc(vhi + 32 * ks), ID, 1);   // lo hi
          }
          issued = 1;
          commit(cfree + 8 * cs.slot);
          cs.next(I_NC);
          if (last && (p & 1)) {   // the pair's last MMAs on V hi / lo of this kc have been issued
            commit(vfree + 8 * (p >> 1));
            commit(vfree + 8 * ((p >> 1) + 2));
          }
        }
        if (!ok) break;
        commit(accf + 8 * ab.slot);
        ab.next(2);
      }
      if (!ok) fail_status();
      if (issued) {   // every MMA issued has finished before tensor and shared memory are released
        commit(fin);
        wait_bar(fin, 0);
      }
    }
  } else if (warp < 8) {
    // ---- warps 0-7: drain each finished accumulator (warps 0-3 the pair's first row block, 4-7 its second)
    const uint32_t taddr = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
    const int half = warp >> 2;
    Ring ab{0, 0};
    long long P = P0;
    int j = j0;
    bool ok = true;
    for (long long n = 0; n < N && ok; ++n) {
      ok = warp_wait(accf + 8 * ab.slot, ab.phase);
      if (!ok) break;
      const long long rb = 2 * P + half;
      inv_drain(a, taddr, acce, half, warp, lane, j, rb, rb < R, ab.slot);
      ab.next(2);
      if (++j == JT) {
        j = 0;
        ++P;
      }
    }
    if (!ok && lane == 0) fail_status();
  }
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    tmem_dealloc(tmem, I_TMEM_COLS);
  }
}

// --------------------------------------------------------------------------------- constant images
// Forward: for each 64-column chunk c, W rows n < nb: cos(2 pi (m0c+n) x / nx), rows nb+n: sin(...) (n < bc;
// zero rows above), K = x = 64c .. 64c+63; [hi | lo], 2 (2 nb) 128 bytes per chunk.  nb = 64, or 32 for the
// Hermitian half (m0c = 0).  One thread per (chunk, row, 8 columns).
__global__ void rows_fwd_consts_kernel(int nx, int m0c, int bc, int nb, unsigned char* img) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int kc = nx / 64;
  const uint32_t wop = 2u * nb * 128u;
  if (id >= (long long)kc * 2 * nb * 8) return;
  const int c = (int)(id / (16 * nb)), row = (int)((id / 8) % (2 * nb)), q = (int)(id % 8);
  const int n = row & (nb - 1);
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
    v[e] = (float)(row < nb ? co : s);
  }
  uint32_t hi[4], lo[4];
  split8(v, hi, lo);
  unsigned char* o = img + (long long)c * 2 * wop + swz(row, q);
  *(uint4*)o = make_uint4(hi[0], hi[1], hi[2], hi[3]);
  *(uint4*)(o + wop) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
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

}  // namespace rt
}  // namespace oi

extern "C" int oi_rows_tc_constants(int which, int nx, int m0c, int bc, void* image, long long bytes, void* stream) {
  using namespace oi;
  if (!image || nx <= 0 || bc <= 0 || bc > 64 || which < 0 || which > 2)
    return fail(OI_EINVAL, "oi_rows_tc_constants: bad arguments");
  if (nx % 128 != 0 || nx > 4096) return fail(OI_ERANGE, "oi_rows_tc_constants: nx=%d is not a multiple of 128", nx);
  // which 2: the Hermitian half of the symmetric band of width bc (m0c = -(bc-1)/2): columns 0 .. (bc-1)/2
  if (which == 2 && (bc % 2 == 0 || m0c != -(bc - 1) / 2 || (bc + 1) / 2 > 32))
    return fail(OI_ERANGE, "oi_rows_tc_constants: band %d at %d is not symmetric of width <= 63", bc, m0c);
  const long long need = which == 0 ? (long long)(nx / 64) * 2 * rt::OPER
                         : which == 2 ? (long long)(nx / 64) * rt::OPER : (long long)(nx / 128) * 4 * rt::OPER;
  if (bytes < need) return fail(OI_ERANGE, "oi_rows_tc_constants: %lld bytes given, %lld needed", bytes, need);
  if ((uintptr_t)image % 16) return fail(OI_EINVAL, "oi_rows_tc_constants: image not 16-byte aligned");
  const long long threads = need / 16 / 2;
  cudaStream_t s = (cudaStream_t)stream;
  if (which == 0)
    rt::rows_fwd_consts_kernel<<<(unsigned)ceil_div(threads, 256), 256, 0, s>>>(nx, m0c, bc, 64, (unsigned char*)image);
  else if (which == 2)
    rt::rows_fwd_consts_kernel<<<(unsigned)ceil_div(threads, 256), 256, 0, s>>>(nx, 0, (bc + 1) / 2, 32,
                                                                               (unsigned char*)image);
  else
    rt::rows_inv_consts_kernel<<<(unsigned)ceil_div(threads, 256), 256, 0, s>>>(nx, bc, (unsigned char*)image);
  oi::note_launch();
  return check_launch("oi_rows_tc_constants");
}

namespace oi {

// The forward row pass at NB band columns per part (64: oi_rows_fwd_tc; 32: oi_rows_fwd_tc_half); `what` names
// the entry point in errors.
template <int NB>
static int rows_fwd_launch(const void* field, int kind, int batch, int ny, int nx, int bc, const void* consts, void* t,
                           void* stream, const char* what) {
  if (!field || !consts || !t || batch <= 0 || bc <= 0) return fail(OI_EINVAL, "%s: bad arguments", what);
  if (kind != OI_FIELD_REAL_F32 && kind != OI_FIELD_U8)
    return fail(OI_EINVAL, "%s: real float32 or uint8 masks only (kind=%d)", what, kind);
  if (ny % 128 != 0 || nx % 128 != 0 || nx > 4096 || bc > NB)
    return fail(OI_ERANGE, "%s: grid %dx%d / band width %d unsupported", what, ny, nx, bc);
  if ((uintptr_t)field % 16 || (uintptr_t)consts % 16)
    return fail(OI_EINVAL, "%s: field and constants must be 16-byte aligned", what);
  const long long rows = (long long)batch * ny, items = (rows / 128 + 1) / 2;   // pairs of row blocks
  const int sms = rt::sm_count();
  if (!sms) return fail(OI_ECUDA, "%s: no CUDA device", what);
  if (rows + 256 > 0x7fffffffLL) return fail(OI_ERANGE, "%s: %lld rows exceed the tensor-map range", what, rows);
  const long long ctas = items < sms ? items : sms;
  rt::FwdArgs a{rows, ny, nx, bc, (const unsigned char*)consts, (float2*)t};
  cudaStream_t s = (cudaStream_t)stream;
  const bool u8 = kind == OI_FIELD_U8;
  CUtensorMap map;   // mask boxes: [128 rows][32 float] with the 128-byte swizzle, or [128][64 uint8], 64-byte
  int rc = rt::encode_2d(&map, u8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, field,
                         (unsigned long long)nx, (unsigned long long)rows, (unsigned long long)nx * (u8 ? 1 : 4),
                         u8 ? 64 : 32, 128, u8 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B);
  if (rc) return rc;
  if (u8) {
    constexpr uint32_t smem = rt::FwdCfg<OI_FIELD_U8, NB>::SMEM;
    rc = ensure_smem((const void*)rt::rows_fwd_tc_kernel<OI_FIELD_U8, NB>, smem, what);
    if (rc) return rc;
    (void)launch_pdl(rt::rows_fwd_tc_kernel<OI_FIELD_U8, NB>, dim3((unsigned)ctas), dim3(rt::F_NT), smem, s, a, map);
    oi::note_launch();
  } else {
    constexpr uint32_t smem = rt::FwdCfg<OI_FIELD_REAL_F32, NB>::SMEM;
    rc = ensure_smem((const void*)rt::rows_fwd_tc_kernel<OI_FIELD_REAL_F32, NB>, smem, what);
    if (rc) return rc;
    (void)launch_pdl(rt::rows_fwd_tc_kernel<OI_FIELD_REAL_F32, NB>, dim3((unsigned)ctas), dim3(rt::F_NT), smem, s, a,
                     map);
    oi::note_launch();
  }
  return check_launch(what);
}

}  // namespace oi

extern "C" int oi_rows_fwd_tc(const void* field, int kind, int batch, int ny, int nx, int m0c, int bc,
                              const void* consts, void* t, void* stream) {
  (void)m0c;   // carried by the constant image
  return oi::rows_fwd_launch<64>(field, kind, batch, ny, nx, bc, consts, t, stream, "oi_rows_fwd_tc");
}

extern "C" int oi_rows_fwd_tc_half(const void* field, int kind, int batch, int ny, int nx, int bch, const void* consts,
                                   void* t, void* stream) {
  return oi::rows_fwd_launch<32>(field, kind, batch, ny, nx, bch, consts, t, stream, "oi_rows_fwd_tc_half");
}

namespace oi {

int rows_inv_from_tiles(const void* vtiles, int count, int ny, int nx, const void* consts, float* out, cudaStream_t s) {
  const long long rows = (long long)count * ny, R = rows / 128, items = (long long)(nx / 128) * ((R + 1) / 2);
  const int sms = rt::sm_count();
  if (!sms) return fail(OI_ECUDA, "oi_rows_inv_tc: no CUDA device");
  if ((R + 1) * 512 > 0x7fffffffLL) return fail(OI_ERANGE, "oi_rows_inv_tc: %lld rows exceed the tensor-map range", rows);
  const long long ctas = items < sms ? items : sms;
  rt::InvArgs a{(const unsigned char*)vtiles, rows, ny, nx, (const unsigned char*)consts, out};
  CUtensorMap c_map, v_map;   // [rows of 128 bytes] of the constant image and of the V tiles
  int rc = rt::encode_2d(&c_map, CU_TENSOR_MAP_DATA_TYPE_UINT16, consts, 64, (unsigned long long)(nx / 128) * 512, 128,
                         64, 128);
  if (!rc) rc = rt::encode_2d(&v_map, CU_TENSOR_MAP_DATA_TYPE_UINT16, vtiles, 64, (unsigned long long)R * 512, 128, 64, 128);
  if (!rc) rc = ensure_smem((const void*)rt::rows_inv_tc_kernel, rt::I_SMEM, "oi_rows_inv_tc");
  if (rc) return rc;
  (void)launch_pdl(rt::rows_inv_tc_kernel, dim3((unsigned)ctas), dim3(rt::I_NT), rt::I_SMEM, s, a, c_map, v_map);
  oi::note_launch();
  return check_launch("oi_rows_inv_tc");
}

}  // namespace oi

extern "C" int oi_rows_inv_tc_tiles(const void* vtiles, int count, int ny, int nx, const void* consts, float* out,
                                    void* stream) {
  using namespace oi;
  if (!vtiles || !consts || !out || count <= 0) return fail(OI_EINVAL, "oi_rows_inv_tc_tiles: bad arguments");
  if (ny % 128 != 0 || nx % 128 != 0 || nx > 4096)
    return fail(OI_ERANGE, "oi_rows_inv_tc_tiles: grid %dx%d unsupported", ny, nx);
  if ((uintptr_t)consts % 16 || (uintptr_t)vtiles % 16)
    return fail(OI_EINVAL, "oi_rows_inv_tc_tiles: constants and V tiles must be 16-byte aligned");
  return rows_inv_from_tiles(vtiles, count, ny, nx, consts, out, (cudaStream_t)stream);
}

extern "C" int oi_rows_inv_tc(const void* v, int count, int ny, int nx, int bc, const void* consts, void* vtiles,
                              float* out, void* stream) {
  using namespace oi;
  if (!v || !consts || !vtiles || !out || count <= 0 || bc <= 0) return fail(OI_EINVAL, "oi_rows_inv_tc: bad arguments");
  if (ny % 128 != 0 || nx % 128 != 0 || nx > 4096 || bc > 64)
    return fail(OI_ERANGE, "oi_rows_inv_tc: grid %dx%d / band width %d unsupported", ny, nx, bc);
  if ((uintptr_t)consts % 16 || (uintptr_t)vtiles % 16)
    return fail(OI_EINVAL, "oi_rows_inv_tc: constants and V tiles must be 16-byte aligned");
  const long long R = (long long)count * ny / 128;
  cudaStream_t s = (cudaStream_t)stream;
  int rc = ensure_smem((const void*)rt::v_tiles_kernel, (size_t)bc * 128 * 8, "oi_rows_inv_tc/tiles");
  if (rc) return rc;
  rt::v_tiles_kernel<<<(unsigned)R, 256, (size_t)bc * 128 * 8, s>>>((const float2*)v, ny, bc, (unsigned char*)vtiles);
  oi::note_launch();
  rc = check_launch("oi_rows_inv_tc/tiles");
  if (rc) return rc;
  return rows_inv_from_tiles(vtiles, count, ny, nx, consts, out, s);
}
