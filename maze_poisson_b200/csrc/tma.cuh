// TMA (cp.async.bulk.tensor) and mbarrier helpers for sm_100a, written as inline PTX.
// Every wait is bounded by a %globaltimer limit: a wait that expires reports failure to
// the caller instead of spinning forever.
#pragma once

#include <cuda.h>

#include "mzb_common.cuh"

namespace mzb {

constexpr unsigned long long kTmaWaitNs = 2000000000ull;  // 2 s per wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Make generic-proxy global writes that this thread has acquired visible to the async
// proxy (TMA reads issued afterwards by this thread).
__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Returns true once the barrier's phase with the given parity has completed, false if
// the wall-clock limit expired first.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    const unsigned long long t0 = global_ns();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (global_ns() - t0 > kTmaWaitNs) return false;
    }
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void prefetch_tensormap(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// Barrier among `count` threads (a multiple of 32) on hardware barrier `id` (1..15).
__device__ __forceinline__ void named_bar_sync(int id, int count) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// 3-D tiled bulk tensor load global -> shared, completing on `bar`.
// Coordinates are (x = k, y = j, z = i); x must be a multiple of 2 for 8-byte elements.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// ------------------------------------------------------------------------------------
// Grid barrier with a monotonic arrival counter: block b's e-th barrier completes when
// the counter reaches (e+1) * gridDim.x. One release-add per block, relaxed polls closed
// by an acquire fence, a bounded wait; `epoch` counts the barriers this block has passed
// in this launch.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned int ld_relaxed_u32(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ bool grid_sync_mono(GridBarrier* bar, unsigned int& epoch) {
    __shared__ int ok_sh;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(&bar->count) : "memory");
        const unsigned int target = (epoch + 1u) * gridDim.x;
        const unsigned long long t0 = global_ns();
        unsigned int polls = 0;
        while (ld_acquire_u32(&bar->count) < target) {
            if ((++polls & 255u) == 0u) {
                if (ld_relaxed_u32(&bar->err) != 0u) { ok = 0; break; }
                if (global_ns() - t0 > kBarrierTimeoutNs) {
                    atomicOr(&bar->err, 1u);
                    ok = 0;
                    break;
                }
            }
        }
        if (ok && ld_relaxed_u32(&bar->err) != 0u) ok = 0;
        ok_sh = ok;
    }
    epoch++;
    __syncthreads();
    return ok_sh != 0;
}

// Host: encode a 3-D tiled tensor map over an n^3 FP64 grid (x = k fastest) with box
// (bx, by, 1), no swizzle, no interleave, out-of-bounds fill zero.
bool encode_grid_map(CUtensorMap* map, const double* base, int n, int bx, int by);

}  // namespace mzb
