// Complex trailing-update tile on the 5th-generation tensor cores (tcgen05, sm_100a):
//
//     C[128 x 64] -= L[128 x 32] U[32 x 64]        (complex64, FP32-accurate)
//
// as one real GEMM D[128 x 128] -= A[128 x 64] B[64 x 128] with
//     A[m][2k + t] = (Re, Im)[t] of L[m][k]                   (the interleaved complex layout read as reals)
//     B[2k + t][2c + s]: (t,s) = (0,0) Re U, (1,0) -Im U, (0,1) Im U, (1,1) Re U     (U = U[k][c])
//     D[m][2c + s] = (Re, Im)[s] of C[m][c]
// so D's columns are C's interleaved complex columns.  FP32 accuracy from TF32 inputs by the three-term
// split x = x_hi + x_lo (x_hi = x rounded to TF32): A B ~ A_hi B_hi + A_hi B_lo + A_lo B_hi (the dropped
// A_lo B_lo term is 2^-22 relative).  D lives in tensor memory (128 lanes = rows, 128 fp32 columns); A and B
// are K-major in shared memory without swizzle: element (row, kk) of a 128 x 64 operand at float offset
// (row / 8) * 512 + (kk / 4) * 32 + (row % 8) * 4 + kk % 4, i.e. 8-row x 16-byte core matrices, adjacent along
// K 128 bytes apart (leading byte offset) and along rows 2048 bytes apart (stride byte offset).
//
// Every wait on the MMA's completion barrier is bounded; a wait that runs out reports false and the caller
// flags the item instead of using the tile.
#pragma once

#include <stdint.h>

namespace dga {

constexpr int TC_M = 128;         // tile rows (TMEM lanes)
constexpr int TC_NR = 128;        // real tile columns (64 complex)
constexpr int TC_KR = 64;         // real K (32 complex)
constexpr int TC_OPERAND_FLOATS = TC_M * TC_KR;  // 8192 floats = 32 KB per operand buffer
constexpr long long TC_WAIT_LIMIT = 1LL << 22;   // try_wait polls before a wait gives up

__device__ __forceinline__ int tc_off(int row, int kk) {
  return (row >> 3) * 512 + (kk >> 2) * 32 + (row & 7) * 4 + (kk & 3);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: K-major, no swizzle, leading byte offset 128, stride byte offset 2048.
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(2048 >> 4) << 32) |
         (1ull << 46);
}

// Instruction descriptor of kind::tf32: D fp32, A and B tf32, A negated (D -= A B), both K-major, N = 128, M = 128.
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | (1u << 13) | ((uint32_t)(TC_NR >> 3) << 17) |
                              ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ float tf32_hi(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// Split x into the TF32 pair (hi, lo) and store both at float offset o of the two operand buffers.
__device__ __forceinline__ void tc_store_split(float* hi, float* lo, int o, float x) {
  const float h = tf32_hi(x);
  hi[o] = h;
  lo[o] = x - h;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// TMEM allocation by one whole warp; the address lands in *slot (shared memory).
__device__ __forceinline__ void tc_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tc_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count = 1) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for the barrier phase with the given parity (at most `limit` polls); false if it did not complete.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit = TC_WAIT_LIMIT) {
  const uint32_t a = smem_u32(bar);
  for (long long it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\tselp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// As mbar_wait, but each poll may suspend the thread for up to hint_ns nanoseconds while the phase is incomplete
// (it resumes as soon as the phase completes), so waiting warps leave the issue slots to the others: at most
// limit x hint_ns in all.
__device__ __forceinline__ bool mbar_wait_sleep(uint64_t* bar, uint32_t parity, long long limit, uint32_t hint_ns) {
  const uint32_t a = smem_u32(bar);
  for (long long it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\tselp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity), "r"(hint_ns)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Bulk copies between global and shared memory (the TMA engine, untiled form): the barrier expects `bytes` of
// transactions, then each copy (16-byte aligned addresses, size a multiple of 16) completes on it.  Source and
// destination are this CTA's own memory on this GPU; no multicast.
// A plain arrival on the barrier (for a thread that takes part in a phase without issuing work).
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst_smem)),
               "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// L2 eviction priorities: a policy covering every access it is given (fraction 1.0).
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
// bulk_g2s with an L2 cache policy for the source lines.
__device__ __forceinline__ void bulk_g2s_hint(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar,
                                              uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          smem_u32(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
      : "memory");
}
// Global store / load of 8 or 16 bytes with an L2 cache policy.
__device__ __forceinline__ void st_f2_hint(float2* p, float2 v, uint64_t policy) {
  asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(p), "f"(v.x), "f"(v.y), "l"(policy)
               : "memory");
}
__device__ __forceinline__ double2 ld_d2_hint(const double2* p, uint64_t policy) {
  double2 v;
  asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
               : "=d"(v.x), "=d"(v.y)
               : "l"(p), "l"(policy));
  return v;
}

// Hint to the TMA engine to bring [src, src + bytes) of global memory into L2 (16-byte aligned address, size a
// multiple of 16); nothing waits on it.
__device__ __forceinline__ void bulk_prefetch_l2(const void* src_gmem, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src_gmem), "r"(bytes) : "memory");
}
// Orders this thread's earlier generic-proxy memory accesses before later async-proxy (bulk copy) accesses.
__device__ __forceinline__ void fence_proxy_async_all() { asm volatile("fence.proxy.async;" ::: "memory"); }

// 32 consecutive fp32 columns of this thread's TMEM lane (32x32b shape: warp w % 4 owns lanes 32 (w % 4) ..).
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const float* v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
      "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
      "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]), "f"(v[8]), "f"(v[9]),
      "f"(v[10]), "f"(v[11]), "f"(v[12]), "f"(v[13]), "f"(v[14]), "f"(v[15]), "f"(v[16]), "f"(v[17]), "f"(v[18]),
      "f"(v[19]), "f"(v[20]), "f"(v[21]), "f"(v[22]), "f"(v[23]), "f"(v[24]), "f"(v[25]), "f"(v[26]), "f"(v[27]),
      "f"(v[28]), "f"(v[29]), "f"(v[30]), "f"(v[31])
      : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,"
      "%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7]), "=f"(v[8]),
        "=f"(v[9]), "=f"(v[10]), "=f"(v[11]), "=f"(v[12]), "=f"(v[13]), "=f"(v[14]), "=f"(v[15]), "=f"(v[16]),
        "=f"(v[17]), "=f"(v[18]), "=f"(v[19]), "=f"(v[20]), "=f"(v[21]), "=f"(v[22]), "=f"(v[23]), "=f"(v[24]),
        "=f"(v[25]), "=f"(v[26]), "=f"(v[27]), "=f"(v[28]), "=f"(v[29]), "=f"(v[30]), "=f"(v[31])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 16 consecutive fp32 columns of this thread's TMEM lane (32x32b shape, as tmem_st32 / tmem_ld32).
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float* v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
          taddr),
      "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]), "f"(v[8]), "f"(v[9]),
      "f"(v[10]), "f"(v[11]), "f"(v[12]), "f"(v[13]), "f"(v[14]), "f"(v[15])
      : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7]), "=f"(v[8]),
        "=f"(v[9]), "=f"(v[10]), "=f"(v[11]), "=f"(v[12]), "=f"(v[13]), "=f"(v[14]), "=f"(v[15])
      : "r"(taddr)
      : "memory");
}

// Shared-memory matrix descriptor, K-major without swizzle: 8-row x 16-byte core matrices, adjacent along K
// 128 bytes apart (leading byte offset) and along rows sbo bytes apart (stride byte offset).
__device__ __forceinline__ uint64_t tc_desc_sbo(uint32_t saddr, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) |
         (1ull << 46);
}

// One MMA of kind::tf32 with an explicit instruction descriptor: D = (accum ? D : 0) + op(A) B, operands K-major
// at the given shared-memory addresses (stride byte offset sbo).
__device__ __forceinline__ void tc_mma_desc(uint32_t d_tmem, uint32_t a_addr, uint32_t b_addr, uint32_t sbo,
                                            uint32_t idesc, uint32_t accum) {
  const uint64_t ad = tc_desc_sbo(a_addr, sbo), bd = tc_desc_sbo(b_addr, sbo);
  const uint32_t zero = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(ad), "l"(bd), "r"(idesc), "r"(accum), "r"(zero), "r"(zero), "r"(zero), "r"(zero)
      : "memory");
}

// One MMA of kind::tf32 with A in tensor memory (lane = row, one fp32 column per K element, a_tmem the column of
// the K step) and B K-major in shared memory: D = (accum ? D : 0) + op(A) B.
__device__ __forceinline__ void tc_mma_tmem_a(uint32_t d_tmem, uint32_t a_tmem, uint32_t b_addr, uint32_t sbo,
                                              uint32_t idesc, uint32_t accum) {
  const uint64_t bd = tc_desc_sbo(b_addr, sbo);
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "r"(a_tmem), "l"(bd), "r"(idesc), "r"(accum)
      : "memory");
}

// Arrives on bar when every tcgen05 operation the calling thread issued before has completed.
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// One MMA D (+)= -A B over K = 8 (reals) at K step j, A and B descriptors at the operand buffers' bases.
__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint32_t a_base, uint32_t b_base, int j) {
  const uint64_t ad = tc_desc(a_base + 256u * j), bd = tc_desc(b_base + 256u * j);
  const uint32_t accum = 1, zero = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(ad), "l"(bd), "r"(TC_IDESC), "r"(accum), "r"(zero), "r"(zero), "r"(zero), "r"(zero)
      : "memory");
}

// Issued by one thread after the operands and D are in place (and the caller's barrier): the three-term
// product over the full K, then a commit that arrives on bar when every MMA has completed.
__device__ __forceinline__ void tc_issue_tile(uint32_t d_tmem, const float* a_hi, const float* a_lo,
                                              const float* b_hi, const float* b_lo, uint64_t* bar) {
  const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo), bh = smem_u32(b_hi), bl = smem_u32(b_lo);
#pragma unroll
  for (int j = 0; j < TC_KR / 8; ++j) {
    tc_mma(d_tmem, al, bh, j);
    tc_mma(d_tmem, ah, bl, j);
    tc_mma(d_tmem, ah, bh, j);
  }
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

}  // namespace dga
