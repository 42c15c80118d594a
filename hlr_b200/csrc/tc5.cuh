// Blackwell (sm_100a) tensor-core primitives: tcgen05.mma with operands in
// shared memory and the accumulator in tensor memory (TMEM), mbarriers with
// bounded waits, and the 128-byte-swizzled operand layouts.
//
// Operand layouts (16-bit elements).  tcgen05.mma reads A (M x K) and B
// (N x K) through shared-memory descriptors.  Both kernels here use the
// 128-byte swizzle: an "atom" is 8 rows of 128 bytes (1 KB, 1024-byte
// aligned), and the 16-byte unit u of row r is stored at unit u ^ r.
//   MN-major (the M or N index contiguous): a row of the atom holds 64
//     consecutive M (N) elements of one K index; the 8 rows are K = 0..7.
//     Atoms along K are SBO bytes apart, atoms along M (N) LBO bytes apart.
//   K-major (the K index contiguous): a row holds 64 consecutive K elements
//     of one M (N) index; the 8 rows are 8 consecutive M (N) indices.  Atoms
//     along M (N) are SBO bytes apart; an MMA's K = 16 elements (32 bytes)
//     lie inside one row, and the next K step starts 32 bytes further.
// The descriptor holds the start address, LBO and SBO (in 16-byte units), a
// fixed version field (1) and the swizzle mode (2 = 128-byte swizzle).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace hlrc {
namespace tc5 {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of 16-byte unit `u` (0..7) of row `r` (0..7) inside a swizzled atom
__device__ __forceinline__ uint32_t swz(uint32_t r, uint32_t u) { return r * 128u + ((u ^ r) << 4); }

// shared-memory matrix descriptor, 128-byte swizzle
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= uint64_t((saddr >> 4) & 0x3fffu);
    d |= uint64_t((lbo >> 4) & 0x3fffu) << 16;
    d |= uint64_t((sbo >> 4) & 0x3fffu) << 32;
    d |= uint64_t(1) << 46;   // version
    d |= uint64_t(2) << 61;   // 128-byte swizzle
    return d;
}

// instruction descriptor of kind::f16: FP32 accumulator, A and B both FP16
// (bf16 = false) or both BF16, with their major-ness (1 = MN-major)
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N, bool bf16, bool a_mn, bool b_mn) {
    return (1u << 4)                                  // D: FP32
           | ((bf16 ? 1u : 0u) << 7)                  // A format
           | ((bf16 ? 1u : 0u) << 10)                 // B format
           | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16)
           | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

// ------------------------------------------------------------- mbarriers
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}
// Waits for phase `parity` of `bar` to complete, for at most `limit_ns` of
// wall-clock time; returns false (and leaves the wait) when the time ran out.
constexpr uint64_t WAIT_LIMIT_NS = 2000000000ull;   // 2 s: far above any legitimate wait here
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns = WAIT_LIMIT_NS) {
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = globaltimer();
    while (!mbar_try(bar, parity))
        if (globaltimer() - t0 > limit_ns) return false;
    return true;
}

// ------------------------------------------------------------ async proxy
// generic-proxy writes to shared memory (st.shared, cp.async) become
// visible to the tensor cores' async proxy
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// 16-byte copy global -> shared (L2 only); src_bytes 0 zero-fills
__device__ __forceinline__ void cp16(uint32_t dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// --------------------------------------------------------------------- TMA
// 2-D tile load (cp.async.bulk.tensor, no multicast) of this GPU's memory
// into shared memory, completing on `bar`; tmap points to a CUtensorMap
// kernel parameter (__grid_constant__).  c0 is the inner coordinate (in
// elements, a multiple of 16 bytes), c1 the row.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const void* tmap, int c0, int c1, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
            dst),
        "l"(tmap), "r"(c0), "r"(c1), "r"(smem_u32(bar))
        : "memory");
}
// one arrival on `bar` that also announces `bytes` of asynchronous copies
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(smem_u32(bar)),
        "r"(bytes)
        : "memory");
}

// ----------------------------------------------------------------- TMEM
// allocation by one whole warp; the address lands in *slot (shared memory)
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// D[tmem] (+)= A[adesc] * B[bdesc]^T, issued by one thread
__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// arrives once on `bar` when all MMAs issued so far by this thread are done
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 32 consecutive FP32 columns of the warp's 32 lanes: lane l of warp w
// (w % 4 = q) reads TMEM lane 32q + l; taddr must carry lane 32q.  The load
// and its wait are one asm statement, so no use of the registers can be
// placed between them.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc5
}  // namespace hlrc
