// Common device/host helpers for the B200 MD hot path (sm_100a).
//
// All FP64 kernels are compiled with --fmad=false so that every a*b+c is rounded twice,
// exactly like the reference's C (built without FMA); explicit fma() is used only where
// a kernel wants it (the mixed-precision inner solvers and the FFT butterflies).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>

namespace mzb {

constexpr double kPi = 3.14159265358979323846;
constexpr double kBoltzmannHartree = 3.1668e-6;  // Hartree / K

[[noreturn]] void fatal_cuda(cudaError_t e, const char* what, const char* file, int line);
[[noreturn]] void fatal(const char* msg);

// Number of kernels this library has launched (instrumentation for benchmarks).
extern unsigned long long g_kernel_launches;
inline void count_launch(unsigned long long k = 1) { g_kernel_launches += k; }

// Device blocks for the systems' arrays, reused across systems (devmem.cu): dev_free
// keeps a block for a later dev_alloc of the same size class once the device has
// synchronised; dev_trim releases every kept block.
void* dev_alloc(size_t bytes);
void dev_free(void* p);
void dev_trim();
size_t dev_cached_bytes();

}  // namespace mzb

#define MZB_CHECK(x)                                                       \
    do {                                                                   \
        cudaError_t mzb_e_ = (x);                                          \
        if (mzb_e_ != cudaSuccess) mzb::fatal_cuda(mzb_e_, #x, __FILE__, __LINE__); \
    } while (0)

namespace mzb {

// ------------------------------------------------------------------------------------
// Periodic index helpers on an n^3 grid, idx = (i*n + j)*n + k.
// ------------------------------------------------------------------------------------
__host__ __device__ __forceinline__ int wrap_inc(int a, int n) { return a + 1 == n ? 0 : a + 1; }
__host__ __device__ __forceinline__ int wrap_dec(int a, int n) { return a == 0 ? n - 1 : a - 1; }

// Correctly rounded x^3: x^2 = p + e exactly, p x = hi + lo exactly, one final rounding
// of hi + (lo + e x) (Dekker's exact product via FMA). glibc's pow(x, 3), which the
// reference calls for cubes (cubic spline weights, the PB transition switch), returns
// this value except in ~0.08 % of inputs where it is one ulp off.
__device__ __forceinline__ double cube_rn(double x) {
    const double p = x * x, e = fma(x, x, -p);
    const double hi = p * x, lo = fma(p, x, -hi);
    return hi + (lo + e * x);
}

// ------------------------------------------------------------------------------------
// Warp / block reductions (fixed trees: deterministic for a given launch shape; the xor
// butterfly leaves the identical value in every lane because IEEE addition commutes).
// ------------------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of up to 4 values; every thread gets the totals. `sh` holds
// 4*32 doubles. Requires blockDim.x to be a multiple of 32.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* sh) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; q++) v[q] = warp_sum(v[q]);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) sh[q * 32 + w] = v[q];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; q++) {
        double s = lane < nw ? sh[q * 32 + lane] : 0.0;
        v[q] = warp_sum(s);
    }
    __syncthreads();
}

// ------------------------------------------------------------------------------------
// Grid barrier for persistent cooperative kernels. Thread 0 of each block arrives on a
// counter; the last arriver resets it and bumps the generation. Every spin is bounded by
// a wall-clock limit read from %globaltimer: on expiry the waiter sets `err` and returns
// false, so a lost block can never hang the GPU.
// ------------------------------------------------------------------------------------
struct GridBarrier {
    unsigned int count;
    unsigned int gen;
    unsigned int err;
    unsigned int pad;
};

constexpr unsigned long long kBarrierTimeoutNs = 4000000000ull;  // 4 s per wait

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ bool grid_sync(GridBarrier* bar) {
    __shared__ int ok_sh;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned int g = ld_acquire_u32(&bar->gen);
        __threadfence();
        const unsigned int prev = atomicAdd(&bar->count, 1u);
        if (prev == gridDim.x - 1) {
            atomicExch(&bar->count, 0u);
            __threadfence();
            atomicAdd(&bar->gen, 1u);
        } else {
            // the acquire load that sees the new generation orders this CTA after the last
            // arriver's fence and, through the counter's RMW chain, after every arrival
            const unsigned long long t0 = global_ns();
            unsigned int polls = 0;
            while (ld_acquire_u32(&bar->gen) == g) {
                if ((++polls & 255u) == 0u && global_ns() - t0 > kBarrierTimeoutNs) {
                    atomicOr(&bar->err, 1u);
                    ok = 0;
                    break;
                }
            }
        }
        if (ld_acquire_u32(&bar->err) != 0u) ok = 0;
        ok_sh = ok;
    }
    __syncthreads();
    return ok_sh != 0;
}

}  // namespace mzb
