// ib_tma.cuh -- Tensor Memory Accelerator (cp.async.bulk.tensor) and mbarrier helpers for sm_100a,
// written as inline PTX, plus the host-side tensor-map encoder.
//
// Rules kept by every caller in this library:
//   * loads and stores are tiled, non-multicast, to and from this CTA's own shared memory;
//   * the innermost (x) box coordinate times 8 bytes is a multiple of 16 bytes (x even);
//   * stores start at non-negative in-range coordinates;
//   * every mbarrier wait is bounded (IB_TMA_SPIN_LIMIT polls; the tile waits take the limit from
//     their launch, which ib_setTileWaitLimit can lower); a wait that runs out sets the caller's
//     error word and the kernel drains what it issued, with the full limit, before returning.
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#ifndef IB_TMA_SPIN_LIMIT
#define IB_TMA_SPIN_LIMIT (1u << 26)
#endif

namespace ib {

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes the mbarrier initialisation visible to the async proxy (TMA).
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's generic-proxy shared-memory accesses before later async-proxy (TMA)
// accesses of the same memory.
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Polls the mbarrier phase with the given parity; false when the poll limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit = IB_TMA_SPIN_LIMIT)
{
    const uint32_t a = smem_u32(bar);
    for (uint32_t i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// CTA-wide wait with one poller: thread 0 polls (at most `limit` times), the CTA meets at a
// barrier that also agrees on the outcome, and every thread then takes its own acquire of the
// completed phase (a test that succeeds at once), so the other threads sleep in the barrier
// instead of polling.
__device__ __forceinline__ bool mbar_wait_cta(uint64_t *bar, uint32_t parity, uint32_t limit = IB_TMA_SPIN_LIMIT)
{
    bool ok = true;
    if (threadIdx.x == 0) ok = mbar_wait(bar, parity, limit);
    ok = __syncthreads_and(ok);
    if (ok) ok = mbar_wait(bar, parity);
    return ok;
}

// Tiled TMA loads into this CTA's shared memory, completing on `bar` (rank 3 and 4).
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_5d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3, int c4,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_u32(dst)),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
        : "memory");
}

// Untiled bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned) from global
// memory into this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"((uint64_t)src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Tiled TMA stores from this CTA's shared memory (bulk-group completion).
__device__ __forceinline__ void tma_store_3d(const CUtensorMap *map, const void *src, int c0, int c1, int c2)
{
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
                     (uint64_t)map),
                 "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(src))
                 : "memory");
}

__device__ __forceinline__ void tma_store_4d(const CUtensorMap *map, const void *src, int c0, int c1, int c2, int c3)
{
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(
                     (uint64_t)map),
                 "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(src))
                 : "memory");
}

__device__ __forceinline__ void tma_store_5d(const CUtensorMap *map, const void *src, int c0, int c1, int c2, int c3,
                                             int c4)
{
    asm volatile("cp.async.bulk.tensor.5d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4, %5}], [%6];" ::"l"(
                     (uint64_t)map),
                 "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(src))
                 : "memory");
}

__device__ __forceinline__ void bulk_commit()
{
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// Waits until every committed bulk store has finished reading its shared-memory source.
__device__ __forceinline__ void bulk_wait_read_all()
{
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// Waits until every committed bulk store has completed.
__device__ __forceinline__ void bulk_wait_all()
{
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap *map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)map) : "memory");
}

// Host: encodes a tiled FP64 tensor map (rank <= 5; dims innermost first, strides in bytes for
// dims 1..rank-1, box extents <= 256).  Returns 0 on success, else a status.
int encode_tmap_f64(CUtensorMap *map, void *base, int rank, const uint64_t *dims, const uint64_t *strides_bytes,
                    const uint32_t *box);

}  // namespace ib
