// ba_tc.cuh -- tcgen05 helpers of the dense Schur update (sm_100a): D = U U^T accumulated in tensor memory.
//
// The operand tile is 128 rows (the reduced system's 6P <= 120 rows, zero-padded) by TC_KT = 32 float columns, held
// twice: the columns rounded to TF32 (hi) and the remainders (lo), so that hi hi^T + hi lo^T + lo hi^T carries the
// product to FP32 accuracy through kind::tf32 MMAs (M = N = 128, K = 8 per instruction, A = B = the same K-major
// tile).  The tile uses the canonical no-swizzle K-major layout of the shared-memory descriptors: core matrices of
// 8 rows x 16 bytes (4 floats), the core matrices of one 8-row group consecutive along K (LBO = 128 B), the 8-row
// groups TC_KT / 4 core matrices apart (SBO = TC_KT * 32 B).  The accumulator is one 128-lane x 128-column FP32 block
// of tensor memory; one thread issues the MMAs and commits them to an mbarrier per tile stage, and at the end to a
// third one that drains them all; every wait is bounded.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define TC_M 128
#define TC_KT 32
#define TC_TILE_FLOATS (TC_M * TC_KT)          // one operand tile (hi or lo): 16 KB
#define TC_WAIT_LIMIT (1 << 24)                // polls of an mbarrier before giving up

// float index of element (r, k) of a tile (r < 128, k < TC_KT)
__device__ __forceinline__ int tc_off(int r, int k)
{
    return (((r >> 3) * (TC_KT / 4) + (k >> 2)) << 5) + ((r & 7) << 2) + (k & 3);
}

__device__ __forceinline__ uint32_t tc_smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// the value rounded to TF32 (round to nearest, ties away: cvt.rna) and the remainder
__device__ __forceinline__ void tc_split(float x, float& hi, float& lo)
{
    uint32_t h;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
    hi = __uint_as_float(h);
    lo = x - hi;
}

// shared-memory matrix descriptor: start address, LBO, SBO (bytes), version 1, no swizzle
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: kind::tf32, D F32, A and B TF32, both K-major, N = 128, M = 128
__host__ __device__ constexpr uint32_t tc_idesc()
{
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(128 >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void tc_mbar_init(uint64_t* bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem_addr(bar)));
}

// wait for phase `parity` of the mbarrier to complete; false when it did not within TC_WAIT_LIMIT polls
__device__ __forceinline__ bool tc_mbar_wait(uint64_t* bar, uint32_t parity)
{
    const uint32_t a = tc_smem_addr(bar);
    for (int i = 0; i < TC_WAIT_LIMIT; ++i) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (done) return true;
    }
    return false;
}

// the whole warp: allocate `ncols` tensor-memory columns, base address into *dst (shared memory)
__device__ __forceinline__ void tc_alloc(uint32_t* dst, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_addr(dst)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}

// the whole warp that allocated
__device__ __forceinline__ void tc_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
// generic-proxy writes of this thread to shared memory become visible to the tensor core's reads
__device__ __forceinline__ void tc_fence_proxy() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// one thread: arrive on bar once every tcgen05 operation the thread issued before has completed
__device__ __forceinline__ void tc_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(tc_smem_addr(bar))
                 : "memory");
}

// one thread: D (+)= hi hi^T + hi lo^T + lo hi^T over the TC_KT columns of the tile pair, then commit to bar
__device__ __forceinline__ void tc_issue(uint32_t tmem, const float* hi, const float* lo, bool accumulate,
                                         uint64_t* bar)
{
    const uint32_t idesc = tc_idesc();
    const uint32_t ah = tc_smem_addr(hi), al = tc_smem_addr(lo);
    const uint32_t sbo = TC_KT * 32, lbo = 128;
#pragma unroll
    for (int s = 0; s < TC_KT / 8; ++s) {
        const uint64_t dh = tc_desc(ah + 256 * s, lbo, sbo), dl = tc_desc(al + 256 * s, lbo, sbo);
        const uint64_t da[3] = {dh, dh, dl}, db[3] = {dh, dl, dh};
#pragma unroll
        for (int t = 0; t < 3; ++t) {
            const uint32_t acc = (accumulate || s > 0 || t > 0) ? 1u : 0u;
            asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                         "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
                         ::"r"(tmem), "l"(da[t]), "l"(db[t]), "r"(idesc), "r"(acc)
                         : "memory");
        }
    }
    tc_commit(bar);
}

// one thread, after the stage waits (or after one of them ran out): commit to a barrier of its own (`fin`, initialised,
// used once) and wait, bounded, until every tcgen05 operation the thread issued has completed (tcgen05.commit tracks
// all of the thread's earlier ones), so that tensor memory is freed with nothing in flight; false when it ran out
__device__ __forceinline__ bool tc_drain(uint64_t* fin)
{
    tc_commit(fin);
    return tc_mbar_wait(fin, 0);
}

// warp w (0..3) reads accumulator rows 32 w .. 32 w + 31 (its lane's row), columns c0 .. c0 + 15
__device__ __forceinline__ void tc_ld16(uint32_t tmem, int warp, int c0, float v[16])
{
    const uint32_t a = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0;
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                 "%14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15])
                 : "r"(a));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
