// tcgen05 building blocks shared by the tensor-core kernels (coherent_tc.cu, rows_tc.cu): shared-memory
// operand descriptors (K-major, 128-byte swizzle), instruction descriptors (kind::f16, bf16 x bf16 -> f32,
// M = 128), MMA issue and commit, bounded mbarrier waits, tensor-memory loads and stores, 1-D bulk copies and
// the bf16 hi/lo split.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cstdint>
#include "oi_common.cuh"

namespace oi {

// Each translation unit with tensor-core kernels keeps its own status word (a kernel whose bounded wait
// expired sets it) and a host reader; oi_device_status combines them.
int rows_tc_status(int* status, bool reset);

// The tensor-core synthesis row pass (rows_tc.cu) from V operand tiles already in memory: tiles [count*ny/128]
// [64 KB] (bf16 hi/lo, [hi: re | im][lo: re | im] x [128 rows][64], 128-byte swizzled), consts from
// oi_rows_tc_constants(1, ...).
int rows_inv_from_tiles(const void* vtiles, int count, int ny, int nx, const void* consts, float* out, cudaStream_t s);

// The synthesis preparation on the tensor cores (synth_tc.cu): V operand tiles from the coarse partial sums, and
// its status word.
int synth_tiles_tc(const float* coarse, int nparts, int count, int br, int bc, const void* sconsts, int ny,
                   void* tiles, cudaStream_t s);
int synth_tc_status(int* status, bool reset);

namespace tc {

constexpr uint32_t SMEM_LIMIT = 232448;                 // opt-in maximum of dynamic shared memory per CTA
constexpr unsigned long long WAIT_NS = 2000000000ull;   // bound of every wait on an mbarrier

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// K-major, 128-byte swizzle, 8-row groups 1024 bytes apart, descriptor version 1 (sm_100).  Element (row, k)
// of a [rows][64] bf16 operand sits at row*128 + (((k/8) ^ (row%8)) * 16) + (k%8)*2 from a 1024-byte aligned
// base; a K step of 16 advances the start address by 32 bytes.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr) {
  const uint32_t lo = ((addr >> 4) & 0x3FFFu) | (1u << 16);
  const uint32_t hi = (1024u >> 4) | (1u << 14) | (2u << 29);
  return ((uint64_t)hi << 32) | lo;
}
// kind::f16, bf16 x bf16 -> f32, both K-major, M = 128.
__host__ __device__ constexpr uint32_t idesc(int n, bool neg_b) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (neg_b ? (1u << 14) : 0u) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(128 >> 4) << 24);
}
__device__ __forceinline__ void mma_ss(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(id), "r"(acc));
}
__device__ __forceinline__ void mma_ts(uint32_t d, uint32_t a_tmem, uint64_t b, uint32_t id, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(d),
      "r"(a_tmem), "l"(b), "r"(id), "r"(acc));
}
__device__ __forceinline__ void commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}
__device__ __forceinline__ bool try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the barrier phase of the given parity; false once `limit_ns` has passed without it.
__device__ __forceinline__ bool wait_bar_for(uint32_t bar, uint32_t parity, unsigned long long limit_ns) {
  if (try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer();
  while (!try_wait(bar, parity))
    if (globaltimer() - t0 > limit_ns) return false;
  return true;
}
// The bound every kernel uses.
__device__ __forceinline__ bool wait_bar(uint32_t bar, uint32_t parity) { return wait_bar_for(bar, parity, WAIT_NS); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Two 32-lane x 16-column loads and their completion wait in one asm statement: the destination registers are
// written asynchronously, so no use of them may be scheduled before tcgen05.wait::ld.
__device__ __forceinline__ void tmem_ld16x2(uint32_t addr_a, uint32_t addr_b, float (&va)[16], float (&vb)[16]) {
  uint32_t a[16], b[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%32];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%33];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3]), "=r"(a[4]), "=r"(a[5]), "=r"(a[6]), "=r"(a[7]),
        "=r"(a[8]), "=r"(a[9]), "=r"(a[10]), "=r"(a[11]), "=r"(a[12]), "=r"(a[13]), "=r"(a[14]), "=r"(a[15]),
        "=r"(b[0]), "=r"(b[1]), "=r"(b[2]), "=r"(b[3]), "=r"(b[4]), "=r"(b[5]), "=r"(b[6]), "=r"(b[7]),
        "=r"(b[8]), "=r"(b[9]), "=r"(b[10]), "=r"(b[11]), "=r"(b[12]), "=r"(b[13]), "=r"(b[14]), "=r"(b[15])
      : "r"(addr_a), "r"(addr_b)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    va[i] = __uint_as_float(a[i]);
    vb[i] = __uint_as_float(b[i]);
  }
}
__device__ __forceinline__ void tmem_st16(uint32_t addr, const uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::
          "r"(addr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
      "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
      : "memory");
}
#define OI_R8(b) "=r"(b[0]), "=r"(b[1]), "=r"(b[2]), "=r"(b[3]), "=r"(b[4]), "=r"(b[5]), "=r"(b[6]), "=r"(b[7])
#define OI_W8(b) "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7])
// Two 32-lane x 32-column loads and their completion wait in one asm statement (see tmem_ld16x2).
__device__ __forceinline__ void tmem_ld32x2(uint32_t addr_a, uint32_t addr_b, float (&va)[32], float (&vb)[32]) {
  uint32_t a[32], b[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
      "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%64];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,%48,"
      "%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%65];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : OI_R8(a), OI_R8((a + 8)), OI_R8((a + 16)), OI_R8((a + 24)), OI_R8(b), OI_R8((b + 8)), OI_R8((b + 16)),
        OI_R8((b + 24))
      : "r"(addr_a), "r"(addr_b)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    va[i] = __uint_as_float(a[i]);
    vb[i] = __uint_as_float(b[i]);
  }
}
// One 32-lane x 32-column load and its completion wait in one asm statement (see tmem_ld16x2).
__device__ __forceinline__ void tmem_ld32(uint32_t addr, float (&v)[32]) {
  uint32_t a[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
      "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : OI_R8(a), OI_R8((a + 8)), OI_R8((a + 16)), OI_R8((a + 24))
      : "r"(addr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(a[i]);
}
__device__ __forceinline__ void tmem_st32(uint32_t addr, const uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
      "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(addr),
      OI_W8(r), OI_W8((r + 8)), OI_W8((r + 16)), OI_W8((r + 24))
      : "memory");
}
#undef OI_R8
#undef OI_W8
// 1-D bulk copy global -> shared completing on an mbarrier (16-byte aligned addresses, size a multiple of 16).
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ uint32_t bf16x2_bits(__nv_bfloat162 h) {
  return (uint32_t)__bfloat16_as_ushort(h.x) | ((uint32_t)__bfloat16_as_ushort(h.y) << 16);
}
// (a, b) -> packed bf16 pairs hi = bf16(a, b), lo = bf16((a, b) - hi)
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  const float2 hf = __bfloat1622float2(h);
  hi = bf16x2_bits(h);
  lo = bf16x2_bits(__floats2bfloat162_rn(a - hf.x, b - hf.y));
}
__device__ __forceinline__ uint32_t swz(int row, int chunk) {
  return (uint32_t)(row * 128 + ((chunk ^ (row & 7)) << 4));
}
__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d)
               : "memory");
}


// Warp-uniform bounded wait: true when every lane saw the phase complete.
__device__ __forceinline__ bool warp_wait(uint32_t bar, uint32_t parity) {
  return __all_sync(0xffffffffu, wait_bar(bar, parity));
}
__device__ __forceinline__ bool warp_wait_for(uint32_t bar, uint32_t parity, unsigned long long limit_ns) {
  return __all_sync(0xffffffffu, wait_bar_for(bar, parity, limit_ns));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void tmem_alloc(uint32_t slot_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot_smem), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t tmem, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

__device__ __forceinline__ void arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Cursor over a ring of mbarrier-guarded slots: slot index and the parity of its current round.
struct Ring {
  int slot;
  uint32_t phase;
  __device__ __forceinline__ void next(int n) {
    if (++slot == n) {
      slot = 0;
      phase ^= 1u;
    }
  }
};

// Wait (bounded) for the last copies of a ring of n slots whose cursor is `c` after `g` issued copies (copy g-k
// went to slot (g-k) mod n, in the cursor's round when that slot is below the cursor, else the round before).
// Returns immediately for copies already consumed: their slot's barrier is then one phase further.
__device__ __forceinline__ void drain_ring(uint32_t full, const Ring& c, int g, int n) {
  const int last = g < n ? g : n;
  for (int k = 1; k <= last; ++k) {
    const int s = (c.slot - k + n) % n;
    wait_bar(full + 8 * s, s < c.slot ? c.phase : c.phase ^ 1u);
  }
}

// 2-D tiled bulk-tensor load of the box at element coordinates (x, y) of `map` (no multicast), completing on bar.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

// ---- host side
typedef CUresult (*EncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// A 1-D bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from shared to global memory, in
// the issuing thread's bulk async-group.
__device__ __forceinline__ void bulk_s2g(void* dst, uint32_t src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// the issuing thread's bulk groups have finished reading shared memory / have completed
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// A 2-D tensor map (dim0 contiguous, rows `stride1` bytes apart) with a box0 x box1 box, no swizzle.
inline int encode_2d(CUtensorMap* map, CUtensorMapDataType type, const void* base, unsigned long long dim0,
                     unsigned long long dim1, unsigned long long stride1, unsigned box0, unsigned box1,
                     CUtensorMapSwizzle swizzle = CU_TENSOR_MAP_SWIZZLE_NONE) {
  static EncodeTiled encode = nullptr;   // one per process (inline function)
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
                            swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(OI_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return OI_OK;
}

inline int sm_count() {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 0;
  return sms;
}

}  // namespace tc
}  // namespace oi
