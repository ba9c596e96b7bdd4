// Fifth-generation tensor-core primitives for sm_100a (tcgen05 + TMEM), used
// by the traveltime surrogate's kernels.
//
// Operand tiles live in shared memory in the no-swizzle canonical layout of
// 8x8 core matrices: element (row, k) of a tile with R rows is at byte
//     (k / 8) * (R * 16) + (row / 8) * 128 + (row % 8) * 16 + (k % 8) * 2
// i.e. a core matrix is 8 rows x 16 bytes, core matrices of one 8-column
// group follow each other down the rows, and column groups are R*16 bytes
// apart.  The same bytes serve two descriptor views:
//   * K-major   (MN = rows, K = columns):  SBO = 128,    LBO = R * 16
//   * MN-major  (MN = columns, K = rows):  SBO = R * 16, LBO = 128
// (SBO: byte stride between 8-groups along MN; LBO: along K), so a tile of
// activations [points][features] is the A operand of a forward GEMM (K =
// features) and, unchanged, the transposed operand of a weight-gradient GEMM
// (K = points); a weight tile [out][in] is B of the forward GEMM and the
// MN-major B of the backward-data GEMM.
//
// Every wait on an mbarrier is bounded; a wait that gives up raises a flag
// the host reads (the kernel then finishes without further MMAs).
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

namespace kcig {
namespace tc {

constexpr uint32_t kWaitLimit = 1u << 24;  // polls of an mbarrier before giving up

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of element (row, k) in a canonical tile of R rows
__device__ __forceinline__ uint32_t canon_off(int row, int k, int R)
{
    return (uint32_t)((k >> 3) * (R * 16) + (row >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor, no swizzle, version 1 (sm_100)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100
    return d;                // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor of kind::f16: BF16 x BF16 -> FP32, M x N
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn_major, int b_mn_major)
{
    return (1u << 4)                      // D format F32
           | (1u << 7)                    // A format BF16
           | (1u << 10)                   // B format BF16
           | ((uint32_t)a_mn_major << 15) // A major
           | ((uint32_t)b_mn_major << 16) // B major
           | ((uint32_t)(N >> 3) << 17)   // N / 8
           | ((uint32_t)(M >> 4) << 24);  // M / 16
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// instruction descriptor of kind::tf32: TF32 x TF32 -> FP32, M x N, both
// operands K-major.  In the canonical layout a TF32 core matrix is 8 rows x
// 4 elements (16 bytes), so one MMA (K = 8) spans two core matrices along K,
// as a kind::f16 MMA (K = 16) does.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N)
{
    return (1u << 4)                      // D format F32
           | (2u << 7)                    // A format TF32
           | (2u << 10)                   // B format TF32
           | ((uint32_t)(N >> 3) << 17)   // N / 8
           | ((uint32_t)(M >> 4) << 24);  // M / 16
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// round to the nearest TF32 value (10 mantissa bits; the low 13 bits become 0)
__device__ __forceinline__ float to_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// all tcgen05 operations issued so far by this thread arrive on `bar` when done
__device__ __forceinline__ void commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor core
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// waits for the phase with parity `parity` to complete; false if it gave up
// (each try suspends the thread for up to a hardware time limit, so the
// bound is generous in time but finite)
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    const uint32_t a = smem_u32(bar);
    for (uint32_t i = 0; i < kWaitLimit; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity), "r"(0x989680u)
            : "memory");
        if (done) return true;
    }
    return false;
}

// non-blocking probe: has the phase with parity `parity` completed?
__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Adds `bytes` to the transaction count the current phase of `bar` waits for
// (no arrival): each thread that issues a bulk copy announces its bytes
// before issuing it, then one thread arrives once all have announced.
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
                 : "memory");
}

// Bulk asynchronous copy (the TMA engine, untiled form) of `bytes` from
// global memory to this CTA's shared memory, completing on `bar`'s
// transaction count.  Both addresses 16-byte aligned, bytes a multiple of
// 16.  No cluster multicast: the source is this GPU's own memory.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// one lane of a converged warp (elect.sync): the issuer of MMAs and commits
__device__ __forceinline__ bool elect_one()
{
    uint32_t pred = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t.reg .b32 r;\n\t"
        "elect.sync r|p, 0xffffffff;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(pred)
        :
        : "memory");
    return pred != 0;
}

// TMEM allocation by one whole warp; the base address is written to *slot
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes
// 32*(w%4) .. +31; `taddr` already carries the lane base)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    __syncwarp();  // the load is warp-collective (.sync.aligned)
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// Ordering contract used by the kernels: the MMAs of one step and the commit
// that tracks them are issued by one elected lane of a converged warp 0, in
// one block (every tcgen05 asm carries a memory clobber, so the commit cannot
// move above the MMAs it must track); all threads then wait on the mbarrier,
// fence::after_thread_sync, and only then read TMEM, warp by warp.

// one GEMM D[M=128][N] (+)= sum over K of A x B^T, K a multiple of 16, issued
// by the calling (single) thread; a/b are the tiles' shared addresses at K=0
// and the step between K=16 slices is 2 groups along K (2 * LBO)
__device__ __forceinline__ void gemm(uint32_t tmem_d, uint32_t a0, uint32_t a_lbo, uint32_t a_sbo, uint32_t b0,
                                     uint32_t b_lbo, uint32_t b_sbo, int K, uint32_t idesc, bool accumulate)
{
    for (int s = 0; s < K / 16; s++) {
        const uint64_t ad = sdesc(a0 + 2 * s * a_lbo, a_lbo, a_sbo);
        const uint64_t bd = sdesc(b0 + 2 * s * b_lbo, b_lbo, b_sbo);
        mma_bf16(tmem_d, ad, bd, idesc, (accumulate || s > 0) ? 1u : 0u);
    }
}

}  // namespace tc
}  // namespace kcig
