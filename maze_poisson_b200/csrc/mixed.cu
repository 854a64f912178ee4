// Mixed-precision field solve: FP64 iterative refinement around an FP32 geometric
// multigrid V-cycle (one cooperative launch per solve).
//
// Solves the same systems as the FP64 path -- L phi = -4 pi q / (h eps) for the LCG and
// MULTIGRID methods, L y = sigma for the MaZe methods (library/src/grid_lcg.c:126-149,
// verlet.c:31-71, grid_multigrid.c:110-212, verlet.c:86-149) -- to the same absolute
// inf-norm tolerance on the FP64 residual, but with a different inner solver:
//
//   repeat: r = b - L x            (FP64, residual checked against tol in FP64)
//           e = V-cycle(r)         (FP32: red-black GS V(nu1,nu2), 27-point full
//                                   weighting scaled by 4 = (2h/h)^2 for the unscaled
//                                   Laplacian, trilinear prolongation, down to a coarse
//                                   level solved exactly)
//           x += e - mean(e)       (FP64; the periodic Laplacian's null space is the
//                                   constants, and dropping e's mean keeps x's mean
//                                   where it started, as CG does)
//
// Work placement. Levels are swept by every CTA with a grid barrier between passes. When
// n/2 is 32, 64 or 128 the hierarchy has two levels and the coarse one is solved exactly by
// FFT (team_fft: three passes, each CTA transforming whole planes in its shared memory),
// which replaces the barrier-bound passes of the levels below. Otherwise levels go down to
// the first one of at most 16 points per side, which every CTA solves by its Green's
// function (team_direct). A plan kept for hierarchies that end at neither (mixed_small_level)
// loads the levels with n <= 16 (at most 3 x 4 x (16^3 + 8^3 + 4^3) B = 55 KB) into CTA 0's
// shared memory and works them there while the other CTAs wait at the next grid barrier;
// a coarsest level of at most 6^3 points is solved exactly by a convolution with its
// Green's function instead of by sweeps. Every V-cycle starts a level from
// x = 0, so the first red half-sweep (x_red = -b/6, no neighbour reads) is folded into the
// pass that writes the level's right-hand side (the FP64 residual pass, the
// restrictions), and the sum of the finest correction, whose mean is removed, is taken in
// the last two half-sweeps instead of by another pass.
#include <cuda_fp16.h>

#include <type_traits>
#include <vector>

#include "engine.cuh"
#include "mixed.cuh"
#include "tma.cuh"

namespace mzb {
namespace {

#ifndef MZB_MIXED_THREADS
#define MZB_MIXED_THREADS 1024
#endif
#ifndef MZB_MIXED_SWEEP_BATCH
#define MZB_MIXED_SWEEP_BATCH 2
#endif
#ifndef MZB_MIXED_BATCH
#define MZB_MIXED_BATCH 2
#endif
constexpr int kThreads = MZB_MIXED_THREADS;

__device__ __forceinline__ void stamp(const MixedArgs& a, int slot) {
    if (a.stamps != nullptr && blockIdx.x == 0 && threadIdx.x == 0 && slot < kMixedStampSlots)
        a.stamps[slot] = global_ns();
}
__device__ __forceinline__ void stamp_outer(const MixedArgs& a, int outer, int k) {
    if (outer < 8) stamp(a, 2 + 8 * outer + k);
}

// The CTAs that work one system: every CTA of a single-system launch, or one system's
// contiguous range of CTAs in a batched launch (mixed_batch_kernel).
struct Team {
    int nblk, b;        // CTAs in the team, this CTA's index in it
    GridBarrier* bar;   // the team's barrier (zeroed before the launch)
    double* partials;   // >= 4 nblk doubles
};

// Barrier over the team's CTAs (the monotonic barrier of tma.cuh with the team's count):
// each CTA's writes are ordered before its release-add by the entry __syncthreads; the
// acquire load that sees the final count synchronises with every release of the
// counter's release sequence, and the exit __syncthreads extends that to the whole CTA.
__device__ __forceinline__ bool team_sync(const Team& t, unsigned int& epoch) {
    __shared__ int ok_sh;
    if (t.nblk == 1) {  // a team of one CTA: the block barrier orders its global writes too
        __syncthreads();
        epoch++;
        return true;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(&t.bar->count) : "memory");
        const unsigned int target = (epoch + 1u) * (unsigned)t.nblk;
        const unsigned long long t0 = global_ns();
        unsigned int polls = 0;
        while (ld_acquire_u32(&t.bar->count) < target) {
            if ((++polls & 255u) == 0u) {
                if (ld_relaxed_u32(&t.bar->err) != 0u) {
                    ok = 0;
                    break;
                }
                if (global_ns() - t0 > kBarrierTimeoutNs) {
                    atomicOr(&t.bar->err, 1u);
                    ok = 0;
                    break;
                }
            }
        }
        if (ok && ld_relaxed_u32(&t.bar->err) != 0u) ok = 0;
        ok_sh = ok;
    }
    epoch++;
    __syncthreads();
    return ok_sh != 0;
}

// ---- loops ----

// whole-team loops: a warp per row of k
template <class F>
__device__ __forceinline__ void grid_pts(const Team& tm, int n, F&& f) {
    const int lane = threadIdx.x & 31;
    const long gw = (long)tm.b * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const long nw = (long)tm.nblk * (blockDim.x >> 5);
    const long rows = (long)n * n;
    for (long row = gw; row < rows; row += nw) {
        const int i = (int)(row / n), j = (int)(row - (long)i * n);
        for (int k = lane; k < n; k += 32) f(i, j, k);
    }
}
// CTA-0 loops (shared-memory levels): a thread per point
template <class F>
__device__ __forceinline__ void cta_pts(int n, F&& f) {
    const int n2 = n * n, tot = n2 * n;
    for (int p = threadIdx.x; p < tot; p += blockDim.x) {
        const int i = p / n2, rem = p - i * n2, j = rem / n;
        f(i, j, rem - j * n);
    }
}
template <class F>
__device__ __forceinline__ void cta_col(int n, int colour, F&& f) {
    const int h = n >> 1, hn = h * n, tot = hn * n;
    for (int p = threadIdx.x; p < tot; p += blockDim.x) {
        const int i = p / hn, rem = p - i * hn, j = rem / h, kk = rem - j * h;
        f(i, j, 2 * kk + ((i + j + colour) & 1));
    }
}

struct Nb {
    long c, ip, im, jp, jm, kp, km;
};
__device__ __forceinline__ Nb nb_of(int n, int i, int j, int k) {
    const long n2 = (long)n * n;
    Nb o;
    o.c = ((long)i * n + j) * n + k;
    o.ip = o.c + (i + 1 == n ? -(long)(n - 1) * n2 : n2);
    o.im = o.c + (i == 0 ? (long)(n - 1) * n2 : -n2);
    o.jp = o.c + (j + 1 == n ? -(long)(n - 1) * n : (long)n);
    o.jm = o.c + (j == 0 ? (long)(n - 1) * n : -(long)n);
    o.kp = o.c + (k + 1 == n ? -(long)(n - 1) : 1L);
    o.km = o.c + (k == 0 ? (long)(n - 1) : -1L);
    return o;
}

// Grid reduction of one sum and one max (deterministic fixed-order gather).
__device__ bool reduce_sum_max(double& s, double& mx, const Team& tm, unsigned& epoch, int& seq) {
    __shared__ double sh[2][32];
    __shared__ double res[2];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const long G = tm.nblk;
    s = warp_sum(s);
    mx = warp_max(mx);
    if (lane == 0) {
        sh[0][w] = s;
        sh[1][w] = mx;
    }
    __syncthreads();
    double* part = tm.partials + (long)(seq & 1) * 2 * G;
    if (w == 0) {
        double v0 = lane < nwarp ? sh[0][lane] : 0.0, v1 = lane < nwarp ? sh[1][lane] : 0.0;
        v0 = warp_sum(v0);
        v1 = warp_max(v1);
        if (lane == 0) {
            part[tm.b] = v0;
            part[G + tm.b] = v1;
        }
    }
    const bool ok = team_sync(tm, epoch);
    if (w == 0) {
        double v0 = 0.0, v1 = 0.0;
        for (long b = lane; b < G; b += 32) {
            v0 += __ldcg(part + b);
            v1 = fmax(v1, __ldcg(part + G + b));
        }
        v0 = warp_sum(v0);
        v1 = warp_max(v1);
        if (lane == 0) {
            res[0] = v0;
            res[1] = v1;
        }
    }
    __syncthreads();
    s = res[0];
    mx = res[1];
    __syncthreads();
    seq++;
    return ok;
}

// ---- multigrid point operations (pointers may be global or shared) ----
//
// The V-cycle is written once for the level scalar S: float for the mixed-precision form
// (FP32 levels inside FP64 refinement), double for the FP64 multigrid form (the same
// V-cycle and refinement loop with every value in FP64).

template <class S> __device__ __forceinline__ S neg_sixth();
template <> __device__ __forceinline__ float neg_sixth<float>() { return -1.0f / 6.0f; }
template <> __device__ __forceinline__ double neg_sixth<double>() { return -1.0 / 6.0; }
__device__ __forceinline__ float fma_s(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fma_s(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float warp_sum_s(float v) { return warp_sumf(v); }
__device__ __forceinline__ double warp_sum_s(double v) { return warp_sum(v); }
// level arrays of the hierarchy, stored as S
template <class S> __device__ __forceinline__ S* lev_x(const MixedArgs& a, int l) { return static_cast<S*>(a.lev_x[l]); }
template <class S> __device__ __forceinline__ S* lev_b(const MixedArgs& a, int l) { return static_cast<S*>(a.lev_b[l]); }
template <class S> __device__ __forceinline__ S* lev_r(const MixedArgs& a, int l) { return static_cast<S*>(a.lev_r[l]); }

// red-black Gauss-Seidel update of one point; returns the new value
template <class S>
__device__ __forceinline__ S gs_point(int n, const S* b, S* x, int i, int j, int k) {
    const Nb o = nb_of(n, i, j, k);
    S s = x[o.im] + x[o.ip];
    s += x[o.jm];
    s += x[o.jp];
    s += x[o.km];
    s += x[o.kp];
    const S v = (b[o.c] - s) * neg_sixth<S>();
    x[o.c] = v;
    return v;
}

template <class S>
__device__ __forceinline__ void resid_point(int n, const S* b, const S* x, S* r, int i, int j, int k) {
    const Nb o = nb_of(n, i, j, k);
    S s = x[o.ip] + x[o.im];
    s += x[o.jp];
    s += x[o.jm];
    s += x[o.kp];
    s += x[o.km];
    r[o.c] = b[o.c] - (s - S(6) * x[o.c]);
}

// Coarse point (I,J,K) of bc = 4 * R27(r) with its first red half-sweep from x = 0:
// xc = -bc/6 on red (I+J+K even) points, 0 on black ones.
template <class S>
__device__ __forceinline__ void restrict_point(int n, const S* r, S* bc, S* xc, int I, int J, int K) {
    const int nc = n / 2;
    const long n2 = (long)n * n;
    const int i = 2 * I, j = 2 * J, k = 2 * K;
    const long i0 = (long)i * n2, i1 = (long)(i + 1 == n ? 0 : i + 1) * n2, i2 = (long)(i == 0 ? n - 1 : i - 1) * n2;
    const long j0 = (long)j * n, j1 = (long)(j + 1 == n ? 0 : j + 1) * n, j2 = (long)(j == 0 ? n - 1 : j - 1) * n;
    const long k0 = k, k1 = (k + 1 == n ? 0 : k + 1), k2 = (k == 0 ? n - 1 : k - 1);
    const S f = r[i2 + j0 + k0] + r[i1 + j0 + k0] + r[i0 + j2 + k0] + r[i0 + j1 + k0] + r[i0 + j0 + k2] +
                    r[i0 + j0 + k1];
    const S e = r[i1 + j0 + k2] + r[i1 + j0 + k1] + r[i2 + j0 + k2] + r[i2 + j0 + k1] + r[i1 + j2 + k0] +
                    r[i1 + j1 + k0] + r[i2 + j2 + k0] + r[i2 + j1 + k0] + r[i0 + j2 + k2] + r[i0 + j2 + k1] +
                    r[i0 + j1 + k2] + r[i0 + j1 + k1];
    const S c = r[i1 + j1 + k2] + r[i1 + j1 + k1] + r[i1 + j2 + k2] + r[i1 + j2 + k1] + r[i2 + j1 + k2] +
                    r[i2 + j1 + k1] + r[i2 + j2 + k2] + r[i2 + j2 + k1];
    const long cc = ((long)I * nc + J) * nc + K;
    const S bv = (S(8) * r[i0 + j0 + k0] + S(4) * f + S(2) * e + c) * (S(0.0625));
    bc[cc] = bv;
    xc[cc] = ((I + J + K) & 1) == 0 ? bv * neg_sixth<S>() : S(0);
}

// fine x += P(coarse x) at (i,j,k), trilinear
template <class S>
__device__ __forceinline__ void prolong_point(int n, const S* xc, S* x, int i, int j, int k) {
    const int nc = n / 2;
    const long n2c = (long)nc * nc;
    const int ci = i >> 1, cj = j >> 1, ck = k >> 1;
    const long i0 = (long)ci * n2c, i1 = (long)(ci + 1 == nc ? 0 : ci + 1) * n2c;
    const long j0 = (long)cj * nc, j1 = (long)(cj + 1 == nc ? 0 : cj + 1) * nc;
    const long k0 = ck, k1 = (ck + 1 == nc ? 0 : ck + 1);
    const S wi = (i & 1) ? S(0.5) : S(0), wj = (j & 1) ? S(0.5) : S(0), wk = (k & 1) ? S(0.5) : S(0);
    const S a00 = xc[i0 + j0 + k0] * (S(1) - wk) + xc[i0 + j0 + k1] * wk;
    const S a01 = xc[i0 + j1 + k0] * (S(1) - wk) + xc[i0 + j1 + k1] * wk;
    const S a10 = xc[i1 + j0 + k0] * (S(1) - wk) + xc[i1 + j0 + k1] * wk;
    const S a11 = xc[i1 + j1 + k0] * (S(1) - wk) + xc[i1 + j1 + k1] * wk;
    const S b0 = a00 * (S(1) - wj) + a01 * wj, b1 = a10 * (S(1) - wj) + a11 * wj;
    x[((long)i * n + j) * n + k] += b0 * (S(1) - wi) + b1 * wi;
}

// ---- grid levels: red-black split layout ----
//
// On the levels worked by the whole grid, point (i,j,k) of colour c = (i+j+k) & 1 is
// stored at c n^3/2 + (i n + j) n/2 + (k >> 1): each colour is a contiguous half, and a
// row (i,j) of one colour is n/2 consecutive values. A half-sweep of colour c then reads
// the other colour and writes its own with unit-stride, fully coalesced accesses; in row
// (i,j) the points of colour c sit at k = 2 kk + s, s = (i+j+c) & 1, and their k-1 / k+1
// neighbours are the other colour's kk-1+s / kk+s, while their i+-1 / j+-1 neighbours are
// the other colour's kk in those rows.
//
// After a pre-smoothing that ends with a black half-sweep, the residual of every black
// point is zero (each black point satisfies its own equation exactly), so only the red
// residual is formed, the 27-point restriction keeps its 13 red taps (centre weight 8,
// the 12 edge points weight 2), and a prolongation that is followed by a red half-sweep
// only updates the black points (the red half-sweep overwrites the red ones without
// reading them).

constexpr int kBatch = MZB_MIXED_BATCH;  // points per lane whose loads are issued before any store
constexpr int kBatchSweep = MZB_MIXED_SWEEP_BATCH;  // the same for the red-black half-sweeps and red residuals

// Offsets within a level are 32-bit: the mixed solver takes n <= kMixedMaxN (n^3 < 2^31).
__device__ __forceinline__ int split_idx(int n, int i, int j, int k) {
    const int h = n >> 1;
    return ((i + j + k) & 1) * h * n * n + (i * n + j) * h + (k >> 1);
}

struct Rows {
    int c, im, ip, jm, jp;  // offsets of rows (i,j), (i-1,j), (i+1,j), (i,j-1), (i,j+1) in one colour
};
__device__ __forceinline__ Rows rows_of(int n, int i, int j) {
    const int h = n >> 1;
    const int ip = i + 1 == n ? 0 : i + 1, im = i == 0 ? n - 1 : i - 1;
    const int jp = j + 1 == n ? 0 : j + 1, jm = j == 0 ? n - 1 : j - 1;
    return Rows{(i * n + j) * h, (im * n + j) * h, (ip * n + j) * h, (i * n + jm) * h, (i * n + jp) * h};
}

// warp per row (i,j) of an n x n set of rows, over the team's CTAs
template <class F>
__device__ __forceinline__ void grid_rows(const Team& tm, int n, F&& f) {
    const int gw = tm.b * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int nw = tm.nblk * (blockDim.x >> 5);
    const int rows = n * n;
    for (int row = gw; row < rows; row += nw) {
        const int i = row / n;
        f(i, row - i * n);
    }
}

// Sums of the six other-colour neighbours of the T chunks kk = k0 + lane + 32 t of the
// colour in row o whose points sit at k = 2 kk + s. The four off-row neighbours and the
// in-row value at kk are loaded for all chunks first; the in-row neighbour on the other
// side (kk - 1 for s = 0, kk + 1 for s = 1) comes from the adjacent lane by a shuffle,
// and only at a chunk or row boundary from memory.
template <int T, class S>
__device__ __forceinline__ void split_nb_sums(const S* xo, const Rows& o, int h, int s, int k0, S (&sum)[T]) {
    const int lane = threadIdx.x & 31;
    S cen[T];
#pragma unroll
    for (int t = 0; t < T; t++) {
        const int kk = k0 + lane + 32 * t;
        sum[t] = S(0);
        cen[t] = S(0);
        if (kk < h) {
            const S a0 = xo[o.im + kk], a1 = xo[o.ip + kk], a2 = xo[o.jm + kk], a3 = xo[o.jp + kk];
            cen[t] = xo[o.c + kk];
            sum[t] = ((a0 + a1) + a2) + a3;
        }
    }
#pragma unroll
    for (int t = 0; t < T; t++) {
        const int kk = k0 + lane + 32 * t;
        const S up = __shfl_up_sync(0xffffffffu, cen[t], 1);
        const S dn = __shfl_down_sync(0xffffffffu, cen[t], 1);
        const S last_prev = __shfl_sync(0xffffffffu, cen[t > 0 ? t - 1 : 0], 31);
        const S first_next = __shfl_sync(0xffffffffu, cen[t + 1 < T ? t + 1 : t], 0);
        if (kk < h) {
            S side;
            if (s == 0) {
                if (lane > 0)
                    side = up;
                else if (t > 0)
                    side = last_prev;
                else
                    side = xo[o.c + (kk == 0 ? h - 1 : kk - 1)];
            } else {
                if (kk + 1 == h)
                    side = xo[o.c];
                else if (lane < 31)
                    side = dn;
                else if (t + 1 < T)
                    side = first_next;
                else
                    side = xo[o.c + kk + 1];
            }
            sum[t] = (sum[t] + cen[t]) + side;
        }
    }
}

// half-sweep of colour c; when acc is not null the new values are summed into it
template <class S>
__device__ void split_gs_scalar(const Team& tm, int n, int c, const S* b, S* x, double* acc) {
    const int lane = threadIdx.x & 31, h = n >> 1;
    const int hp = h * n * n;
    const S* xo = x + (1 - c) * hp;
    S* xc = x + c * hp;
    const S* bc = b + c * hp;
    double s_acc = 0.0;
    grid_rows(tm, n, [&](int i, int j) {
        const Rows o = rows_of(n, i, j);
        const int s = (i + j + c) & 1;
        for (int k0 = 0; k0 < h; k0 += 32 * kBatchSweep) {
            S bv[kBatchSweep], sum[kBatchSweep];
#pragma unroll
            for (int t = 0; t < kBatchSweep; t++) {
                const int kk = k0 + lane + 32 * t;
                bv[t] = kk < h ? bc[o.c + kk] : S(0);
            }
            split_nb_sums<kBatchSweep>(xo, o, h, s, k0, sum);
#pragma unroll
            for (int t = 0; t < kBatchSweep; t++) {
                const int kk = k0 + lane + 32 * t;
                if (kk < h) {
                    const S v = (bv[t] - sum[t]) * neg_sixth<S>();
                    xc[o.c + kk] = v;
                    s_acc += (double)v;
                }
            }
        }
    });
    if (acc != nullptr) *acc += s_acc;
}

// red residual r_red = b_red - L x at the red points (black residuals are zero)
template <class S>
__device__ void split_resid_red_scalar(const Team& tm, int n, const S* b, const S* x, S* r) {
    const int lane = threadIdx.x & 31, h = n >> 1;
    const int hp = h * n * n;
    const S* x1 = x + hp;
    grid_rows(tm, n, [&](int i, int j) {
        const Rows o = rows_of(n, i, j);
        const int s = (i + j) & 1;
        for (int k0 = 0; k0 < h; k0 += 32 * kBatchSweep) {
            S bv[kBatchSweep], xv[kBatchSweep], sum[kBatchSweep];
#pragma unroll
            for (int t = 0; t < kBatchSweep; t++) {
                const int kk = k0 + lane + 32 * t;
                bv[t] = kk < h ? b[o.c + kk] : S(0);
                xv[t] = kk < h ? x[o.c + kk] : S(0);
            }
            split_nb_sums<kBatchSweep>(x1, o, h, s, k0, sum);
#pragma unroll
            for (int t = 0; t < kBatchSweep; t++) {
                const int kk = k0 + lane + 32 * t;
                if (kk < h) r[o.c + kk] = bv[t] - (sum[t] - S(6) * xv[t]);
            }
        }
    });
}

// 4 x R27(r) at coarse point (I,J,K) from the red residual half of a split level n
// (the 13 red taps of the 27-point full weighting)
template <class S>
__device__ __forceinline__ S split_restrict_value(int n, const S* r, int I, int J, int K) {
    const int h = n >> 1;
    const int i = 2 * I, j = 2 * J;
    const int ip = i + 1, im = i == 0 ? n - 1 : i - 1, jp = j + 1, jm = j == 0 ? n - 1 : j - 1;
    auto R = [&](int fi, int fj) { return (fi * n + fj) * h; };
    const int Km = K == 0 ? h - 1 : K - 1;
    S e = r[R(ip, jp) + K] + r[R(ip, jm) + K];
    e += r[R(im, jp) + K];
    e += r[R(im, jm) + K];
    e += r[R(ip, j) + K];
    e += r[R(ip, j) + Km];
    e += r[R(im, j) + K];
    e += r[R(im, j) + Km];
    e += r[R(i, jp) + K];
    e += r[R(i, jp) + Km];
    e += r[R(i, jm) + K];
    e += r[R(i, jm) + Km];
    return (S(8) * r[R(i, j) + K] + S(2) * e) * (S(0.0625));
}

// coarse b = 4 R27(r), coarse x = its first red half-sweep from 0 (both split layout)
template <class S>
__device__ void split_restrict_scalar(const Team& tm, int n, const S* r, S* bc, S* xc) {
    const int lane = threadIdx.x & 31, nc = n / 2, hc = nc >> 1;
    const int hpc = hc * nc * nc;
    grid_rows(tm, nc, [&](int I, int J) {
        for (int k0 = 0; k0 < nc; k0 += 32 * kBatch) {
            S v[kBatch];
#pragma unroll
            for (int t = 0; t < kBatch; t++) {
                const int K = k0 + lane + 32 * t;
                if (K < nc) v[t] = split_restrict_value(n, r, I, J, K);
            }
#pragma unroll
            for (int t = 0; t < kBatch; t++) {
                const int K = k0 + lane + 32 * t;
                if (K < nc) {
                    const int C = (I + J + K) & 1;
                    const int idx = C * hpc + (I * nc + J) * hc + (K >> 1);
                    bc[idx] = v[t];
                    xc[idx] = C == 0 ? v[t] * neg_sixth<S>() : S(0);
                }
            }
        }
    });
}

// fine black x += P(coarse x), trilinear (both split layout)
template <class S>
__device__ void split_prolong_black_scalar(const Team& tm, int n, const S* xc, S* x) {
    const int lane = threadIdx.x & 31, h = n >> 1, nc = n / 2, hc = nc >> 1;
    const int hp = h * n * n, hpc = hc * nc * nc;
    S* x1 = x + hp;
    grid_rows(tm, n, [&](int i, int j) {
        const int s1 = (i + j + 1) & 1;  // black points of row (i,j) sit at k = 2 kk + s1
        const int ci = i >> 1, cj = j >> 1;
        const int ci1 = ci + 1 == nc ? 0 : ci + 1, cj1 = cj + 1 == nc ? 0 : cj + 1;
        const bool oi = i & 1, oj = j & 1, ok = s1;
        auto C = [&](int CI, int CJ, int CK) {
            return ((CI + CJ + CK) & 1) * hpc + (CI * nc + CJ) * hc + (CK >> 1);
        };
        auto line = [&](int CI, int CJ, int ck, int ck1) {
            const S a = xc[C(CI, CJ, ck)];
            return ok ? S(0.5) * (a + xc[C(CI, CJ, ck1)]) : a;
        };
        const int rowx = (i * n + j) * h;
        for (int k0 = 0; k0 < h; k0 += 32 * kBatch) {
            S v[kBatch], old[kBatch];
#pragma unroll
            for (int t = 0; t < kBatch; t++) {
                const int kk = k0 + lane + 32 * t;
                if (kk < h) {
                    const int ck = kk, ck1 = kk + 1 == nc ? 0 : kk + 1;
                    S p = line(ci, cj, ck, ck1);
                    if (oj) p = S(0.5) * (p + line(ci, cj1, ck, ck1));
                    if (oi) {
                        S q = line(ci1, cj, ck, ck1);
                        if (oj) q = S(0.5) * (q + line(ci1, cj1, ck, ck1));
                        p = S(0.5) * (p + q);
                    }
                    v[t] = p;
                    old[t] = x1[rowx + kk];
                }
            }
#pragma unroll
            for (int t = 0; t < kBatch; t++) {
                const int kk = k0 + lane + 32 * t;
                if (kk < h) x1[rowx + kk] = old[t] + v[t];
            }
        }
    });
}

// ---- vectorised split-layout passes (rows of h = 32 V floats, V = 2 or 4) ----
//
// A warp reads a whole row of one colour with one V-wide access per lane (lane l holds
// kk = V l .. V l + V - 1), so each lane keeps several independent 8- or 16-byte loads in
// flight; the scalar versions, one 4-byte value per access, reach only about a third of
// the HBM bandwidth. The in-row neighbour at either end of a lane's V values comes from
// the adjacent lane by a shuffle, wrapping from lane 0 to lane 31 as the periodic row
// does. Every sum keeps the scalar versions' order, so results are identical.

template <int V, class S>
__device__ __forceinline__ void ldv(const S* p, S (&v)[V]) {
    if constexpr (sizeof(S) == 4 && V == 4) {
        const float4 t = *reinterpret_cast<const float4*>(p);
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else if constexpr (sizeof(S) == 4) {
        const float2 t = *reinterpret_cast<const float2*>(p);
        v[0] = t.x; v[1] = t.y;
    } else {  // double: one 16-byte load per pair
#pragma unroll
        for (int e = 0; e < V; e += 2) {
            const double2 t = *reinterpret_cast<const double2*>(p + e);
            v[e] = t.x; v[e + 1] = t.y;
        }
    }
}
template <int V, class S>
__device__ __forceinline__ void stv(S* p, const S (&v)[V]) {
    if constexpr (sizeof(S) == 4 && V == 4)
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    else if constexpr (sizeof(S) == 4)
        *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
    else
#pragma unroll
        for (int e = 0; e < V; e += 2) *reinterpret_cast<double2*>(p + e) = make_double2(v[e], v[e + 1]);
}
// FP16 storage with FP32 arithmetic (level 0 of the mixed form): V = 8 values per 16-byte
// access, 4 per 8-byte, 2 per 4-byte access; stores round to nearest.
template <int V>
__device__ __forceinline__ void ldv(const __half* p, float (&v)[V]) {
    static_assert(V == 2 || V == 4 || V == 8, "FP16 rows take 2, 4 or 8 values per lane");
    if constexpr (V == 8) {
        const uint4 t = *reinterpret_cast<const uint4*>(p);
        const unsigned w[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w[q]));
            v[2 * q] = f.x;
            v[2 * q + 1] = f.y;
        }
    } else if constexpr (V == 4) {
        const uint2 t = *reinterpret_cast<const uint2*>(p);
        const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&t.x));
        const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&t.y));
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    } else {
        const float2 a = __half22float2(*reinterpret_cast<const __half2*>(p));
        v[0] = a.x; v[1] = a.y;
    }
}
template <int V>
__device__ __forceinline__ void stv(__half* p, const float (&v)[V]) {
    static_assert(V == 2 || V == 4 || V == 8, "FP16 rows take 2, 4 or 8 values per lane");
    if constexpr (V == 8) {
        unsigned w[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const __half2 h2 = __floats2half2_rn(v[2 * q], v[2 * q + 1]);
            w[q] = *reinterpret_cast<const unsigned*>(&h2);
        }
        *reinterpret_cast<uint4*>(p) = make_uint4(w[0], w[1], w[2], w[3]);
    } else if constexpr (V == 4) {
        const __half2 a = __floats2half2_rn(v[0], v[1]), b = __floats2half2_rn(v[2], v[3]);
        uint2 t;
        t.x = *reinterpret_cast<const unsigned*>(&a);
        t.y = *reinterpret_cast<const unsigned*>(&b);
        *reinterpret_cast<uint2*>(p) = t;
    } else {
        *reinterpret_cast<__half2*>(p) = __floats2half2_rn(v[0], v[1]);
    }
}
// arithmetic type of a storage type, and scalar conversions
template <class T> struct Calc { using type = T; };
template <> struct Calc<__half> { using type = float; };
__device__ __forceinline__ float to_calc(__half v) { return __half2float(v); }
__device__ __forceinline__ float to_calc(float v) { return v; }
__device__ __forceinline__ double to_calc(double v) { return v; }
template <class T> __device__ __forceinline__ T from_calc(typename Calc<T>::type v) {
    if constexpr (std::is_same<T, __half>::value) return __float2half_rn(v);
    else return v;
}
// V consecutive values of a row as one lane loads them: in the arithmetic type, or for FP16
// packed two to a register (converted where read), so that five rows of 8 FP16 values per
// lane fit the 64 registers of a 1024-thread CTA.
template <class T, int V>
struct RowVals {
    typename Calc<T>::type v[V];
    __device__ __forceinline__ void load(const T* p) { ldv<V>(p, v); }
    __device__ __forceinline__ typename Calc<T>::type operator[](int e) const { return v[e]; }
};
template <int V>
struct RowVals<__half, V> {
    static_assert(V == 8, "packed FP16 rows hold 8 values");
    uint4 w;
    __device__ __forceinline__ void load(const __half* p) { w = *reinterpret_cast<const uint4*>(p); }
    __device__ __forceinline__ float operator[](int e) const {
        const unsigned u = e < 2 ? w.x : e < 4 ? w.y : e < 6 ? w.z : w.w;
        const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&u));
        return (e & 1) ? f.y : f.x;
    }
};

// sum of the six other-colour neighbours of the lane's V points in row o (s as in
// split_nb_sums), from full-row vector loads
template <int V, class T, class S>
__device__ __forceinline__ void vec_nb_sums(const T* xo, const Rows& o, int s, S (&sum)[V]) {
    const int lane = threadIdx.x & 31;
    S a0[V], a1[V], a2[V], a3[V], cen[V];
    ldv<V>(xo + o.im + V * lane, a0);
    ldv<V>(xo + o.ip + V * lane, a1);
    ldv<V>(xo + o.jm + V * lane, a2);
    ldv<V>(xo + o.jp + V * lane, a3);
    ldv<V>(xo + o.c + V * lane, cen);
    const S prev = __shfl_sync(0xffffffffu, cen[V - 1], (lane + 31) & 31);
    const S next = __shfl_sync(0xffffffffu, cen[0], (lane + 1) & 31);
#pragma unroll
    for (int e = 0; e < V; e++) {
        const S side = s == 0 ? (e == 0 ? prev : cen[e - 1]) : (e == V - 1 ? next : cen[e + 1]);
        S t = ((a0[e] + a1[e]) + a2[e]) + a3[e];
        sum[e] = (t + cen[e]) + side;
    }
}

template <int V, class T>
__device__ void split_gs_vec(const Team& tm, int n, int c, const T* b, T* x, double* acc) {
    using S = typename Calc<T>::type;
    const int lane = threadIdx.x & 31, h = n >> 1;
    const int hp = h * n * n;
    const T* xo = x + (1 - c) * hp;
    T* xc = x + c * hp;
    const T* bc = b + c * hp;
    double s_acc = 0.0;
    grid_rows(tm, n, [&](int i, int j) {
        const Rows o = rows_of(n, i, j);
        S bv[V], sum[V], v[V];
        ldv<V>(bc + o.c + V * lane, bv);
        vec_nb_sums<V>(xo, o, (i + j + c) & 1, sum);
#pragma unroll
        for (int e = 0; e < V; e++) {
            v[e] = to_calc(from_calc<T>((bv[e] - sum[e]) * neg_sixth<S>()));  // the value stored
            s_acc += (double)v[e];
        }
        stv<V>(xc + o.c + V * lane, v);
    });
    if (acc != nullptr) *acc += s_acc;
}

template <int V, class T>
__device__ void split_resid_red_vec(const Team& tm, int n, const T* b, const T* x, T* r) {
    using S = typename Calc<T>::type;
    const int lane = threadIdx.x & 31, h = n >> 1;
    const int hp = h * n * n;
    const T* x1 = x + hp;
    grid_rows(tm, n, [&](int i, int j) {
        const Rows o = rows_of(n, i, j);
        S bv[V], xv[V], sum[V], v[V];
        ldv<V>(b + o.c + V * lane, bv);
        ldv<V>(x + o.c + V * lane, xv);
        vec_nb_sums<V>(x1, o, (i + j) & 1, sum);
#pragma unroll
        for (int e = 0; e < V; e++) v[e] = bv[e] - (sum[e] - S(6) * xv[e]);
        stv<V>(r + o.c + V * lane, v);
    });
}

// restriction with coarse rows of nc = h = 32 V points: lane l computes K = V l .. V l + V - 1
template <int V, class T, class S>
__device__ void split_restrict_vec(const Team& tm, int n, const T* r, S* bc, S* xc) {
    const int lane = threadIdx.x & 31, nc = n / 2, hc = nc >> 1, h = n >> 1;
    const int hpc = hc * nc * nc;
    grid_rows(tm, nc, [&](int I, int J) {
        const int i = 2 * I, j = 2 * J;
        const int ip = i + 1, im = i == 0 ? n - 1 : i - 1, jp = j + 1, jm = j == 0 ? n - 1 : j - 1;
        auto R = [&](int fi, int fj) { return r + (fi * n + fj) * h + V * lane; };
        S dpp[V], dpm[V], dmp[V], dmm[V], p0[V], m0[V], q0p[V], q0m[V], cc[V];
        ldv<V>(R(ip, jp), dpp);
        ldv<V>(R(ip, jm), dpm);
        ldv<V>(R(im, jp), dmp);
        ldv<V>(R(im, jm), dmm);
        ldv<V>(R(ip, j), p0);
        ldv<V>(R(im, j), m0);
        ldv<V>(R(i, jp), q0p);
        ldv<V>(R(i, jm), q0m);
        ldv<V>(R(i, j), cc);
        // values at K - 1: the previous element, or the previous lane's last one
        const S p0m = __shfl_sync(0xffffffffu, p0[V - 1], (lane + 31) & 31);
        const S m0m = __shfl_sync(0xffffffffu, m0[V - 1], (lane + 31) & 31);
        const S q0pm = __shfl_sync(0xffffffffu, q0p[V - 1], (lane + 31) & 31);
        const S q0mm = __shfl_sync(0xffffffffu, q0m[V - 1], (lane + 31) & 31);
        S bv[V];
#pragma unroll
        for (int e = 0; e < V; e++) {
            S ee = dpp[e] + dpm[e];
            ee += dmp[e];
            ee += dmm[e];
            ee += p0[e];
            ee += e == 0 ? p0m : p0[e - 1];
            ee += m0[e];
            ee += e == 0 ? m0m : m0[e - 1];
            ee += q0p[e];
            ee += e == 0 ? q0pm : q0p[e - 1];
            ee += q0m[e];
            ee += e == 0 ? q0mm : q0m[e - 1];
            bv[e] = (S(8) * cc[e] + S(2) * ee) * (S(0.0625));
        }
        // K = V lane + e has colour (I + J + e) & 1 and sits at K >> 1 of its half
        const int rowc = (I * nc + J) * hc;
        const int c0 = (I + J) & 1;
#pragma unroll
        for (int e = 0; e < V; e++) {
            const int C = (c0 + e) & 1;
            const int idx = C * hpc + rowc + ((V * lane + e) >> 1);
            bc[idx] = bv[e];
            xc[idx] = C == 0 ? bv[e] * neg_sixth<S>() : S(0);
        }
    });
}

// Coarse row (CI, CJ) of a level with nc = 32 V points per side as lane l reads it for the
// black points kk = V l .. V l + V - 1 of a fine row: the even ck = V l + 2 t from one
// colour half and the odd ck = V l + 2 t + 1 from the other, one vector load each.
template <int V, class S>
struct CoarseRun {
    S ev[V / 2], od[V / 2];
    __device__ __forceinline__ void load(const S* xc, int nc, int CI, int CJ) {
        const int lane = threadIdx.x & 31, hc = nc >> 1, hpc = hc * nc * nc;
        const int rowc = (CI * nc + CJ) * hc;
        const int c0 = (CI + CJ) & 1;  // colour of the even ck
        constexpr int H = V / 2;
        if constexpr (H == 1) {
            ev[0] = xc[c0 * hpc + rowc + lane];
            od[0] = xc[(c0 ^ 1) * hpc + rowc + lane];
        } else {
            ldv<H>(xc + c0 * hpc + rowc + H * lane, ev);
            ldv<H>(xc + (c0 ^ 1) * hpc + rowc + H * lane, od);
        }
    }
    // the values along k at the lane's V black points: coarse ck, or with ok the mean of
    // ck and ck + 1 (ck = V l + V, from the next lane, wraps to 0 at the row's end)
    __device__ __forceinline__ void line(bool ok, S (&L)[V]) const {
        const int lane = threadIdx.x & 31;
        const S last = __shfl_sync(0xffffffffu, ev[0], (lane + 1) & 31);
#pragma unroll
        for (int e = 0; e < V; e++) {
            const S c = (e & 1) ? od[e >> 1] : ev[e >> 1];
            const S c1 = e + 1 == V ? last : ((e & 1) ? ev[(e + 1) >> 1] : od[e >> 1]);
            L[e] = ok ? S(0.5) * (c + c1) : c;
        }
    }
};

// prolongation into the black points of rows of h = nc = 32 V values per colour: lane l adds
// the trilinear interpolation at black points kk = V l .. V l + V - 1 (same sums, in the same
// order, as split_prolong_black_scalar); the four coarse rows are loaded before any is used
template <int V, class S, class T>
__device__ void split_prolong_black_vec(const Team& tm, int n, const S* xc, T* x) {
    const int lane = threadIdx.x & 31, h = n >> 1, nc = n / 2;
    const int hp = h * n * n;
    T* x1 = x + hp;
    grid_rows(tm, n, [&](int i, int j) {
        const int s1 = (i + j + 1) & 1;
        const int ci = i >> 1, cj = j >> 1;
        const int ci1 = ci + 1 == nc ? 0 : ci + 1, cj1 = cj + 1 == nc ? 0 : cj + 1;
        const bool oi = i & 1, oj = j & 1, ok = s1;
        const int rowx = (i * n + j) * h + V * lane;
        S old[V], p[V], t[V], q[V];
        ldv<V>(x1 + rowx, old);
        CoarseRun<V, S> r00, r01, r10, r11;
        r00.load(xc, nc, ci, cj);
        r01.load(xc, nc, ci, cj1);
        r10.load(xc, nc, ci1, cj);
        r11.load(xc, nc, ci1, cj1);
        r00.line(ok, p);
        if (oj) {
            r01.line(ok, t);
#pragma unroll
            for (int e = 0; e < V; e++) p[e] = S(0.5) * (p[e] + t[e]);
        }
        if (oi) {
            r10.line(ok, q);
            if (oj) {
                r11.line(ok, t);
#pragma unroll
                for (int e = 0; e < V; e++) q[e] = S(0.5) * (q[e] + t[e]);
            }
#pragma unroll
            for (int e = 0; e < V; e++) p[e] = S(0.5) * (p[e] + q[e]);
        }
#pragma unroll
        for (int e = 0; e < V; e++) p[e] = old[e] + p[e];
        stv<V>(x1 + rowx, p);
    });
}

// Rows shorter than a warp's 32 V values (h = n/2 per colour, h % V == 0, h / V <= 32): a
// warp takes R = 32 / (h / V) consecutive rows at once, h / V lanes per row (the other
// lanes idle), each lane V values of its row. The in-row neighbours across a lane's ends
// come from the adjacent lanes of the same row, wrapping inside the row as the periodic
// row does. Same sums, in the same order, as the scalar and one-row versions.
struct RowLanes {
    int L, R, sub, q;  // lanes per row, rows per warp, this lane's row slot and chunk in it
    int lp, ln;        // lanes holding the previous and the next chunk of this lane's row
};
template <int V>
__device__ __forceinline__ RowLanes row_lanes(int h) {
    RowLanes t;
    const int lane = threadIdx.x & 31;
    t.L = h / V;
    t.R = 32 / t.L;
    t.sub = lane / t.L;
    t.q = lane - t.sub * t.L;
    t.lp = t.q == 0 ? lane + t.L - 1 : lane - 1;
    t.ln = t.q == t.L - 1 ? lane - (t.L - 1) : lane + 1;
    return t;
}
// warp per R rows of an n x n set of rows: f(i, j, active) for the lane's row (a clamped
// row of the warp's first when the lane idles, so that every lane takes the shuffles)
template <class F>
__device__ __forceinline__ void grid_row_groups(const Team& tm, int n, const RowLanes& t, F&& f) {
    const int gw = tm.b * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int nw = tm.nblk * (blockDim.x >> 5);
    const int rows = n * n;
    for (int r0 = gw * t.R; r0 < rows; r0 += nw * t.R) {
        const int row = r0 + t.sub;
        const bool act = t.sub < t.R && row < rows;
        const int rr = act ? row : r0;
        const int i = rr / n;
        f(i, rr - i * n, act);
    }
}
template <int V, class T, class S>
__device__ __forceinline__ void rows_nb_sums(const T* xo, const Rows& o, int s, int kk0, const RowLanes& t,
                                             S (&sum)[V]) {
    RowVals<T, V> a0, a1, a2, a3, cen;
    a0.load(xo + o.im + kk0);
    a1.load(xo + o.ip + kk0);
    a2.load(xo + o.jm + kk0);
    a3.load(xo + o.jp + kk0);
    cen.load(xo + o.c + kk0);
    const S prev = __shfl_sync(0xffffffffu, cen[V - 1], t.lp);
    const S next = __shfl_sync(0xffffffffu, cen[0], t.ln);
#pragma unroll
    for (int e = 0; e < V; e++) {
        const S side = s == 0 ? (e == 0 ? prev : cen[e - 1]) : (e == V - 1 ? next : cen[e + 1]);
        S u = ((a0[e] + a1[e]) + a2[e]) + a3[e];
        sum[e] = (u + cen[e]) + side;
    }
}
template <int V, class T>
__device__ void split_gs_rows(const Team& tm, int n, int c, const T* b, T* x, double* acc) {
    using S = typename Calc<T>::type;
    const int h = n >> 1, hp = h * n * n;
    const RowLanes t = row_lanes<V>(h);
    const T* xo = x + (1 - c) * hp;
    T* xc = x + c * hp;
    const T* bc = b + c * hp;
    const int kk0 = t.q * V;
    double s_acc = 0.0;
    grid_row_groups(tm, n, t, [&](int i, int j, bool act) {
        const Rows o = rows_of(n, i, j);
        RowVals<T, V> bv;
        S sum[V], v[V];
        bv.load(bc + o.c + kk0);
        rows_nb_sums<V>(xo, o, (i + j + c) & 1, kk0, t, sum);
#pragma unroll
        for (int e = 0; e < V; e++) v[e] = to_calc(from_calc<T>((bv[e] - sum[e]) * neg_sixth<S>()));  // as stored
        if (act) {
            stv<V>(xc + o.c + kk0, v);
#pragma unroll
            for (int e = 0; e < V; e++) s_acc += (double)v[e];
        }
    });
    if (acc != nullptr) *acc += s_acc;
}
template <int V, class T>
__device__ void split_resid_red_rows(const Team& tm, int n, const T* b, const T* x, T* r) {
    using S = typename Calc<T>::type;
    const int h = n >> 1, hp = h * n * n;
    const RowLanes t = row_lanes<V>(h);
    const T* x1 = x + hp;
    const int kk0 = t.q * V;
    grid_row_groups(tm, n, t, [&](int i, int j, bool act) {
        const Rows o = rows_of(n, i, j);
        RowVals<T, V> bv, xv;
        S sum[V], v[V];
        bv.load(b + o.c + kk0);
        xv.load(x + o.c + kk0);
        rows_nb_sums<V>(x1, o, (i + j) & 1, kk0, t, sum);
#pragma unroll
        for (int e = 0; e < V; e++) v[e] = bv[e] - (sum[e] - S(6) * xv[e]);
        if (act) stv<V>(r + o.c + kk0, v);
    });
}

// dispatch: rows of 128 floats (n = 256) as float4 and of 64 (n = 128) as float2, one row
// per warp; shorter rows several per warp (n % 8 == 0 as float4, n % 4 == 0 as float2)
// FP16 storage (level 0 of the mixed form, n = 256): half-sweeps and red residuals with 8
// values (16 bytes) per lane, several rows per warp; restriction and prolongation with 4.
template <class S>
__device__ __forceinline__ void split_gs(const Team& tm, int n, int c, const S* b, S* x, double* acc) {
    if constexpr (std::is_same<S, __half>::value) {  // 8 values (16 bytes) per lane, several rows per warp
        split_gs_rows<8>(tm, n, c, b, x, acc);
    } else {
        if (n == 256) split_gs_vec<4>(tm, n, c, b, x, acc);
        else if (n == 128) split_gs_vec<2>(tm, n, c, b, x, acc);
        else if (n < 256 && n % 8 == 0) split_gs_rows<4>(tm, n, c, b, x, acc);
        else if (n < 128 && n % 4 == 0) split_gs_rows<2>(tm, n, c, b, x, acc);
        else split_gs_scalar(tm, n, c, b, x, acc);
    }
}
template <class S>
__device__ __forceinline__ void split_resid_red(const Team& tm, int n, const S* b, const S* x, S* r) {
    if constexpr (std::is_same<S, __half>::value) {
        split_resid_red_rows<8>(tm, n, b, x, r);
    } else {
        if (n == 256) split_resid_red_vec<4>(tm, n, b, x, r);
        else if (n == 128) split_resid_red_vec<2>(tm, n, b, x, r);
        else if (n < 256 && n % 8 == 0) split_resid_red_rows<4>(tm, n, b, x, r);
        else if (n < 128 && n % 4 == 0) split_resid_red_rows<2>(tm, n, b, x, r);
        else split_resid_red_scalar(tm, n, b, x, r);
    }
}
template <class T, class S>
__device__ __forceinline__ void split_restrict(const Team& tm, int n, const T* r, S* bc, S* xc) {
    if constexpr (std::is_same<T, __half>::value) {
        if (n == 256) split_restrict_vec<4>(tm, n, r, bc, xc);
        else split_restrict_vec<2>(tm, n, r, bc, xc);
    } else {
        if (n == 256) split_restrict_vec<4>(tm, n, r, bc, xc);
        else if (n == 128) split_restrict_vec<2>(tm, n, r, bc, xc);
        else split_restrict_scalar(tm, n, r, bc, xc);
    }
}
template <class S, class T>
__device__ __forceinline__ void split_prolong_black(const Team& tm, int n, const S* xc, T* x) {
    if constexpr (std::is_same<T, __half>::value) {
        if (n == 256) split_prolong_black_vec<4>(tm, n, xc, x);
        else split_prolong_black_vec<2>(tm, n, xc, x);
    } else {
        if (n == 256) split_prolong_black_vec<4>(tm, n, xc, x);
        else if (n == 128) split_prolong_black_vec<2>(tm, n, xc, x);
        else split_prolong_black_scalar(tm, n, xc, x);
    }
}

// ---- the shared-memory part of the V-cycle (CTA 0) ----
//
// Shared memory holds x, b, r of levels lsmall..nlev-1 back to back, then (when the
// coarsest level is solved directly) the coarsest level's Green's function.
template <class S>
__device__ __forceinline__ S* small_arr(const MixedArgs& a, S* sm, int m, int which) {
    int off = 0;
    for (int l = a.lsmall; l < m; l++) off += 3 * a.lev_n[l] * a.lev_n[l] * a.lev_n[l];
    return sm + off + which * a.lev_n[m] * a.lev_n[m] * a.lev_n[m];
}

// Coarsest level solved exactly: x = G * b (circular convolution with the pseudo-inverse
// of the unscaled periodic 7-point Laplacian, precomputed on the host), i.e. the
// zero-mean solution of L x = b - mean(b). Several lanes share one output point.
template <class S>
__device__ void coarse_direct(int n, const S* g, const S* b, S* x) {
    const int N = n * n * n;
    int lanes = 1;  // lanes that share one output point
    while (lanes < 32 && 2 * lanes * N <= (int)blockDim.x) lanes *= 2;
    const int p = threadIdx.x / lanes, sub = threadIdx.x % lanes;
    S acc = S(0);
    if (p < N) {
        const int pi = p / (n * n), pj = (p / n) % n, pk = p % n;
        for (int q = sub; q < N; q += lanes) {
            const int qi = q / (n * n), qj = (q / n) % n, qk = q % n;
            const int d = (((pi - qi + n) % n) * n + ((pj - qj + n) % n)) * n + ((pk - qk + n) % n);
            acc += g[d] * b[q];
        }
    }
    for (int o = lanes >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (p < N && sub == 0) x[p] = acc;
}

// ---- shared-memory levels of 4, 8 or 16 points per side ----
// The same point operations (and sums, in the same order) as gs_point, resid_point,
// restrict_point and prolong_point, with the size known at compile time: 32-bit indices
// and periodic wraps by masks instead of the general helpers' divisions and 64-bit
// arithmetic, which on one CTA made each pass of these small levels instruction-bound.
template <int N, class S>
__device__ __forceinline__ void sm_smooth(const S* b, S* x, int first_colour, int half_sweeps) {
    constexpr int H = N / 2, M = N - 1, TOT = N * N * H;
    for (int hs = 0; hs < half_sweeps; hs++) {
        const int colour = (first_colour + hs) & 1;
        for (int p = threadIdx.x; p < TOT; p += blockDim.x) {
            const int i = p / (N * H), j = (p / H) % N, kk = p % H;
            const int k = 2 * kk + ((i + j + colour) & 1);
            const int c = (i * N + j) * N + k;
            S s = x[(((i - 1) & M) * N + j) * N + k] + x[(((i + 1) & M) * N + j) * N + k];
            s += x[(i * N + ((j - 1) & M)) * N + k];
            s += x[(i * N + ((j + 1) & M)) * N + k];
            s += x[(i * N + j) * N + ((k - 1) & M)];
            s += x[(i * N + j) * N + ((k + 1) & M)];
            x[c] = (b[c] - s) * neg_sixth<S>();
        }
        __syncthreads();
    }
}
template <int N, class S>
__device__ __forceinline__ void sm_resid(const S* b, const S* x, S* r) {
    constexpr int M = N - 1, TOT = N * N * N;
    for (int p = threadIdx.x; p < TOT; p += blockDim.x) {
        const int i = p / (N * N), j = (p / N) % N, k = p % N;
        S s = x[(((i + 1) & M) * N + j) * N + k] + x[(((i - 1) & M) * N + j) * N + k];
        s += x[(i * N + ((j + 1) & M)) * N + k];
        s += x[(i * N + ((j - 1) & M)) * N + k];
        s += x[(i * N + j) * N + ((k + 1) & M)];
        s += x[(i * N + j) * N + ((k - 1) & M)];
        r[p] = b[p] - (s - S(6) * x[p]);
    }
    __syncthreads();
}
template <int N, class S>
__device__ __forceinline__ void sm_restrict(const S* r, S* bc, S* xc) {
    constexpr int NC = N / 2, M = N - 1, N2 = N * N, TOT = NC * NC * NC;
    for (int p = threadIdx.x; p < TOT; p += blockDim.x) {
        const int I = p / (NC * NC), J = (p / NC) % NC, K = p % NC;
        const int i = 2 * I, j = 2 * J, k = 2 * K;
        const int i0 = i * N2, i1 = ((i + 1) & M) * N2, i2 = ((i - 1) & M) * N2;
        const int j0 = j * N, j1 = ((j + 1) & M) * N, j2 = ((j - 1) & M) * N;
        const int k0 = k, k1 = (k + 1) & M, k2 = (k - 1) & M;
        const S f = r[i2 + j0 + k0] + r[i1 + j0 + k0] + r[i0 + j2 + k0] + r[i0 + j1 + k0] + r[i0 + j0 + k2] +
                        r[i0 + j0 + k1];
        const S e = r[i1 + j0 + k2] + r[i1 + j0 + k1] + r[i2 + j0 + k2] + r[i2 + j0 + k1] + r[i1 + j2 + k0] +
                        r[i1 + j1 + k0] + r[i2 + j2 + k0] + r[i2 + j1 + k0] + r[i0 + j2 + k2] + r[i0 + j2 + k1] +
                        r[i0 + j1 + k2] + r[i0 + j1 + k1];
        const S c = r[i1 + j1 + k2] + r[i1 + j1 + k1] + r[i1 + j2 + k2] + r[i1 + j2 + k1] + r[i2 + j1 + k2] +
                        r[i2 + j1 + k1] + r[i2 + j2 + k2] + r[i2 + j2 + k1];
        const S bv = (S(8) * r[i0 + j0 + k0] + S(4) * f + S(2) * e + c) * (S(0.0625));
        bc[p] = bv;
        xc[p] = ((I + J + K) & 1) == 0 ? bv * neg_sixth<S>() : S(0);
    }
    __syncthreads();
}
template <int N, class S>
__device__ __forceinline__ void sm_prolong(const S* xc, S* x) {
    constexpr int NC = N / 2, MC = NC - 1, NC2 = NC * NC, TOT = N * N * N;
    for (int p = threadIdx.x; p < TOT; p += blockDim.x) {
        const int i = p / (N * N), j = (p / N) % N, k = p % N;
        const int ci = i >> 1, cj = j >> 1, ck = k >> 1;
        const int i0 = ci * NC2, i1 = ((ci + 1) & MC) * NC2;
        const int j0 = cj * NC, j1 = ((cj + 1) & MC) * NC;
        const int k0 = ck, k1 = (ck + 1) & MC;
        const S wi = (i & 1) ? S(0.5) : S(0), wj = (j & 1) ? S(0.5) : S(0), wk = (k & 1) ? S(0.5) : S(0);
        const S a00 = xc[i0 + j0 + k0] * (S(1) - wk) + xc[i0 + j0 + k1] * wk;
        const S a01 = xc[i0 + j1 + k0] * (S(1) - wk) + xc[i0 + j1 + k1] * wk;
        const S a10 = xc[i1 + j0 + k0] * (S(1) - wk) + xc[i1 + j0 + k1] * wk;
        const S a11 = xc[i1 + j1 + k0] * (S(1) - wk) + xc[i1 + j1 + k1] * wk;
        const S b0 = a00 * (S(1) - wj) + a01 * wj, b1 = a10 * (S(1) - wj) + a11 * wj;
        x[p] += b0 * (S(1) - wi) + b1 * wi;
    }
    __syncthreads();
}
__device__ __forceinline__ bool sm_fixed(int n) { return n == 4 || n == 8 || n == 16; }

// Restricts the residual of level lsmall-1 (global) into shared memory, runs the rest of
// the V-cycle there and writes level lsmall's correction back to lev_x[lsmall].
template <class S>
__device__ void small_vcycle(const MixedArgs& a, S* sm, const S* r_above) {
    const int L = a.nlev, ls = a.lsmall;
    auto smooth = [&](int m, int first_colour, int half_sweeps) {
        const int n = a.lev_n[m];
        S* x = small_arr(a, sm, m, 0);
        const S* b = small_arr(a, sm, m, 1);
        if (n == 16) return sm_smooth<16>(b, x, first_colour, half_sweeps);
        if (n == 8) return sm_smooth<8>(b, x, first_colour, half_sweeps);
        if (n == 4) return sm_smooth<4>(b, x, first_colour, half_sweeps);
        for (int h = 0; h < half_sweeps; h++) {
            cta_col(n, (first_colour + h) & 1, [&](int i, int j, int k) { gs_point(n, b, x, i, j, k); });
            __syncthreads();
        }
    };
    S* gsm = small_arr(a, sm, L, 0);  // just past the last level
    if (a.coarse_g != nullptr) {
        const int N = a.lev_n[L - 1] * a.lev_n[L - 1] * a.lev_n[L - 1];
        for (int p = threadIdx.x; p < N; p += blockDim.x) gsm[p] = static_cast<const S*>(a.coarse_g)[p];
    }
    {
        const S* r = r_above;  // red residual of level ls - 1, split layout
        const int nf = a.lev_n[ls - 1], nc = a.lev_n[ls];
        S* bs = small_arr(a, sm, ls, 1);
        S* xs = small_arr(a, sm, ls, 0);
        cta_pts(nc, [&](int I, int J, int K) {
            const S bv = split_restrict_value(nf, r, I, J, K);
            const int cc = (I * nc + J) * nc + K;
            bs[cc] = bv;
            xs[cc] = ((I + J + K) & 1) == 0 ? bv * neg_sixth<S>() : S(0);
        });
        __syncthreads();
    }
    for (int m = ls; m < L - 1; m++) {
        const int n = a.lev_n[m];
        smooth(m, 1, 2 * a.nu1 - 1);
        S* x = small_arr(a, sm, m, 0);
        S* b = small_arr(a, sm, m, 1);
        S* r = small_arr(a, sm, m, 2);
        S* bc = small_arr(a, sm, m + 1, 1);
        S* xc = small_arr(a, sm, m + 1, 0);
        if (sm_fixed(n)) {
            if (n == 16) { sm_resid<16>(b, x, r); sm_restrict<16>(r, bc, xc); }
            else if (n == 8) { sm_resid<8>(b, x, r); sm_restrict<8>(r, bc, xc); }
            else { sm_resid<4>(b, x, r); sm_restrict<4>(r, bc, xc); }
        } else {
            cta_pts(n, [&](int i, int j, int k) { resid_point(n, b, x, r, i, j, k); });
            __syncthreads();
            cta_pts(a.lev_n[m + 1], [&](int I, int J, int K) { restrict_point(n, r, bc, xc, I, J, K); });
            __syncthreads();
        }
    }
    if (a.coarse_g != nullptr) {
        coarse_direct(a.lev_n[L - 1], gsm, small_arr(a, sm, L - 1, 1), small_arr(a, sm, L - 1, 0));
        __syncthreads();
    } else {
        smooth(L - 1, 1, 2 * a.coarse_sweeps - 1);
    }
    for (int m = L - 2; m >= ls; m--) {
        const int n = a.lev_n[m];
        const S* xc = small_arr(a, sm, m + 1, 0);
        S* x = small_arr(a, sm, m, 0);
        if (n == 16) sm_prolong<16>(xc, x);
        else if (n == 8) sm_prolong<8>(xc, x);
        else {
            cta_pts(n, [&](int i, int j, int k) { prolong_point(n, xc, x, i, j, k); });
            __syncthreads();
        }
        smooth(m, 0, 2 * a.nu2);
    }
    const int nl = a.lev_n[ls];
    const S* xs = small_arr(a, sm, ls, 0);
    S* dst = lev_x<S>(a, ls);  // split layout
    cta_pts(nl, [&](int i, int j, int k) { dst[split_idx(nl, i, j, k)] = xs[(i * nl + j) * nl + k]; });
}

// The coarsest level l (n <= kMixedTeamDirectN, rhs in lev_b[l]) solved exactly by the
// whole team: x = G * b, the circular convolution with the pseudo-inverse of the unscaled
// periodic 7-point Laplacian (coarse_g, precomputed on the host), i.e. the zero-mean
// solution of L x = b - mean(b). Every CTA stages G and b in shared memory; a warp forms
// one point's sum, its lanes taking the (j, k) columns r = lane + 32 t of every i plane.
template <class S>
__device__ void team_direct(const MixedArgs& a, const Team& tm, S* sm, int l) {
    const int n = a.lev_n[l], n2 = n * n, N = n2 * n;
    S* gs = sm;
    S* bs = sm + N;
    const S* b = lev_b<S>(a, l);  // split layout
    for (int p = threadIdx.x; p < N; p += blockDim.x) {
        gs[p] = static_cast<const S*>(a.coarse_g)[p];
        const int i = p / n2, j = (p / n) % n, k = p % n;
        bs[p] = b[split_idx(n, i, j, k)];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    constexpr int TM = (kMixedTeamDirectN * kMixedTeamDirectN + 31) / 32;
    S* x = lev_x<S>(a, l);
    for (int p = tm.b * nw + w; p < N; p += tm.nblk * nw) {
        const int pi = p / n2, pj = (p / n) % n, pk = p % n;
        int ro[TM], go[TM];  // b offset (j n + k) and G offset of the lane's columns
#pragma unroll
        for (int t = 0; t < TM; t++) {
            const int r = lane + 32 * t;
            const int qj = r / n, qk = r - qj * n;
            int dj = pj - qj, dk = pk - qk;
            dj += dj < 0 ? n : 0;
            dk += dk < 0 ? n : 0;
            ro[t] = r < n2 ? r : -1;
            go[t] = dj * n + dk;
        }
        S acc = S(0);
        for (int qi = 0; qi < n; qi++) {
            int di = pi - qi;
            di += di < 0 ? n : 0;
            const S* gp = gs + di * n2;
            const S* bp = bs + qi * n2;
#pragma unroll
            for (int t = 0; t < TM; t++)
                if (ro[t] >= 0) acc = fma_s(gp[go[t]], bp[ro[t]], acc);
        }
        acc = warp_sum_s(acc);
        if (lane == 0) x[split_idx(n, pi, pj, pk)] = acc;
    }
}

// ---- the coarse level by FFT (whole team) ----
//
// A coarse level of nc = 32, 64 or 128 points per side is solved exactly, like
// team_direct: x = the zero-mean solution of L x = b - mean(b) for the unscaled periodic
// 7-point Laplacian, whose eigenvalues on the DFT basis are
// lambda(k) = 2 cos(2 pi k1/nc) + 2 cos(2 pi k2/nc) + 2 cos(2 pi k3/nc) - 6. Five passes
// over a half spectrum T[i][j][kk] (kk = 0..nc/2, complex), a team barrier after each:
//   1. rows along k, real to complex, two rows per warp (packed as re + i im);
//   2. lines along j, forward;
//   3. lines along i: forward, times 1/(lambda nc^3) (0 at k = 0), inverse;
//   4. lines along j, inverse;
//   5. rows along k, complex to real, two rows per warp, into x (split layout).
// A warp transforms a line of N = 32 R points, lane t holding points 32 r + t: a length-R
// DFT in registers, twiddles W_N^(t k1), then a length-32 radix-2 decimation in
// frequency across the lanes by shuffles, which leaves X[k1 + R brev5(t)] in lane t,
// register k1. The inverse applies the adjoint of each step in reverse order (the
// transposed butterflies with conjugate twiddles), so forward then inverse is N times
// the identity in any distribution of the frequencies over the lanes.
constexpr int kFftCoarseMax = 128;

template <class S> struct CxT;
template <> struct CxT<float> { using T = float2; };
template <> struct CxT<double> { using T = double2; };
template <class S> using Cx = typename CxT<S>::T;

template <class C> __device__ __forceinline__ C cx(decltype(C::x) re, decltype(C::x) im) { C c; c.x = re; c.y = im; return c; }
template <class C> __device__ __forceinline__ C cadd(C a, C b) { return cx<C>(a.x + b.x, a.y + b.y); }
template <class C> __device__ __forceinline__ C csub(C a, C b) { return cx<C>(a.x - b.x, a.y - b.y); }
template <class C> __device__ __forceinline__ C cmul(C a, C w) { return cx<C>(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x); }
template <class C> __device__ __forceinline__ C cmulc(C a, C w) { return cx<C>(a.x * w.x + a.y * w.y, a.y * w.x - a.x * w.y); }  // a conj(w)
template <class C> __device__ __forceinline__ C cshfl_xor(C a, int m) {
    return cx<C>(__shfl_xor_sync(0xffffffffu, a.x, m), __shfl_xor_sync(0xffffffffu, a.y, m));
}
template <class C> __device__ __forceinline__ C cshfl(C a, int src) {
    return cx<C>(__shfl_sync(0xffffffffu, a.x, src), __shfl_sync(0xffffffffu, a.y, src));
}
__device__ __forceinline__ float fast_div(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double fast_div(double a, double b) { return a / b; }
__device__ __forceinline__ int brev5(int t) { return (int)(__brev((unsigned)t) >> 27); }

// The lane's twiddles of the five across-lane stages: forward, W_{2d}^m on the bottom
// lane of a pair and 1 on the top one (m = t mod d); inverse, +-conj(W_{2d}^m) (+ top,
// - bottom).
template <class C>
struct LaneTw {
    C f[5], i[5];
};
template <int R, class C>
__device__ __forceinline__ LaneTw<C> lane_tw(const C* tw, int t) {
    LaneTw<C> L;
#pragma unroll
    for (int s = 0; s < 5; s++) {
        const int d = 16 >> s;
        const C w = tw[(t & (d - 1)) * (16 / d) * R];
        const bool bottom = (t & d) != 0;
        L.f[s] = bottom ? w : cx<C>(1, 0);
        const int di = 1 << s;
        const C wi = tw[(t & (di - 1)) * (16 / di) * R];
        L.i[s] = (t & di) != 0 ? cx<C>(-wi.x, wi.y) : cx<C>(wi.x, -wi.y);
    }
    return L;
}

// forward DFT of the warp's line: a length-R DFT in registers, twiddles W_N^(t k1)
// (tq[k1 * 32 + t], W_N^e = exp(-2 pi i e / N)), then the across-lane stages d = 16 .. 1, each
// (u, v) -> (u + v, (u - v) W_{2d}^m) on the pair of lanes t, t + d: on either lane
// (+-own + partner) times the lane's twiddle.
template <int R, class C>
__device__ __forceinline__ void wfft_fwd(C (&v)[R], const C* tq, const LaneTw<C>& L, int t) {
    using S = decltype(C::x);
    if constexpr (R == 2) {
        const C a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 4) {
        const C s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]), s13 = cadd(v[1], v[3]), d13 = csub(v[1], v[3]);
        v[0] = cadd(s02, s13);
        v[2] = csub(s02, s13);
        v[1] = cx<C>(d02.x + d13.y, d02.y - d13.x);  // d02 - i d13
        v[3] = cx<C>(d02.x - d13.y, d02.y + d13.x);  // d02 + i d13
    }
#pragma unroll
    for (int k1 = 1; k1 < R; k1++) v[k1] = cmul(v[k1], tq[k1 * 32 + t]);
#pragma unroll
    for (int s = 0; s < 5; s++) {
        const int d = 16 >> s;
        const S sg = (t & d) != 0 ? S(-1) : S(1);
#pragma unroll
        for (int k1 = 0; k1 < R; k1++) {
            const C p = cshfl_xor(v[k1], d);
            v[k1] = cmul(cx<C>(fma_s(sg, v[k1].x, p.x), fma_s(sg, v[k1].y, p.y)), L.f[s]);
        }
    }
}

// N times the inverse of wfft_fwd: the adjoint of each step, last first; the adjoint of a
// stage maps the pair (a, b) on lanes (t, t + d) to (a + conj(w) b, a - conj(w) b).
template <int R, class C>
__device__ __forceinline__ void wfft_inv(C (&v)[R], const C* tq, const LaneTw<C>& L, int t) {
#pragma unroll
    for (int s = 0; s < 5; s++) {
        const int d = 1 << s;
        const bool top = (t & d) == 0;
#pragma unroll
        for (int k1 = 0; k1 < R; k1++) {
            const C p = cshfl_xor(v[k1], d);
            const C a = top ? v[k1] : p, b = top ? p : v[k1];
            const C w = L.i[s];
            v[k1] = cx<C>(fma_s(w.x, b.x, fma_s(-w.y, b.y, a.x)), fma_s(w.x, b.y, fma_s(w.y, b.x, a.y)));
        }
    }
#pragma unroll
    for (int k1 = 1; k1 < R; k1++) v[k1] = cmulc(v[k1], tq[k1 * 32 + t]);
    if constexpr (R == 2) {
        const C a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 4) {
        const C s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]), s13 = cadd(v[1], v[3]), d13 = csub(v[1], v[3]);
        v[0] = cadd(s02, s13);
        v[2] = csub(s02, s13);
        v[1] = cx<C>(d02.x - d13.y, d02.y + d13.x);  // d02 + i d13
        v[3] = cx<C>(d02.x + d13.y, d02.y - d13.x);  // d02 - i d13
    }
}

// Z[N - k] for each register of wfft_fwd's output (lane t, register k1 <-> k = k1 + R brev5(t))
template <int R, class C>
__device__ __forceinline__ C mirror(const C (&v)[R], int k1, int lane, int src0) {
    return k1 == 0 ? cshfl(v[0], src0) : cshfl(v[R - k1], lane ^ 31);
}

template <int R, class S>
__device__ bool team_fft_r(const MixedArgs& a, const Team& tm, unsigned& epoch, int l, Cx<S>* tw, Cx<S>* tq, S* tc,
                           Cx<S>* P, int outer) {
    using C = Cx<S>;
    constexpr int N = 32 * R, H = N / 2 + 1, NH = N * H, NQ = N / 2;
    auto pstamp = [&](int k) { if (outer == 1) stamp(a, 2 + 8 * 8 + k); };
    pstamp(0);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nwc = blockDim.x >> 5;
    const int bl = brev5(lane), src0 = brev5((32 - bl) & 31);
    C* T = static_cast<C*>(a.coarse_spec);
    const S* b = lev_b<S>(a, l);
    S* x = lev_x<S>(a, l);
    for (int e = threadIdx.x; e < N; e += blockDim.x) {
        double sv, cv;
        sincospi(2.0 * e / N, &sv, &cv);
        tw[e] = cx<C>((S)cv, (S)-sv);
    }
    __syncthreads();
    // lane-indexed tables (no bank conflicts): tq[k1][t] = W_N^(t k1), and tc[k1][t] =
    // 2 cos(2 pi ki / N) of the frequency ki = k1 + R brev5(t) a lane holds after wfft_fwd
    for (int e = threadIdx.x; e < 32 * R; e += blockDim.x) {
        const int k1 = e >> 5, t = e & 31;
        tq[e] = tw[t * k1];
        tc[e] = S(2) * tw[k1 + R * brev5(t)].x;
    }
    __syncthreads();
    const LaneTw<C> L = lane_tw<R>(tw, lane);
    pstamp(1);
    // The line tasks of a plane along j: kk = 1 .. N/2 - 1, and task 0 for the DC and Nyquist
    // columns (kk = 0, N/2), both real after the row transforms, as one complex column.
    // A. each CTA takes whole planes i: rows along k (two real rows per warp as one complex
    //    row), then lines along j, in its shared plane P[j][kk]; the plane goes to T[i].
    for (int i = tm.b; i < N; i += tm.nblk) {
        for (int pr = w; pr < N / 2; pr += nwc) {
            const int jA = 2 * pr, jB = jA + 1;
            C v[R];
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int k = 32 * r + lane;
                v[r] = cx<C>(b[split_idx(N, i, jA, k)], b[split_idx(N, i, jB, k)]);
            }
            wfft_fwd<R>(v, tq, L, lane);
#pragma unroll
            for (int k1 = 0; k1 < R; k1++) {  // X_A = (Z[k] + conj Z[N-k]) / 2, X_B = (Z[k] - conj Z[N-k]) / 2i
                const C z = v[k1], zc = mirror(v, k1, lane, src0);
                const int k = k1 + R * bl;
                if (k < H) {
                    P[jA * H + k] = cx<C>(S(0.5) * (z.x + zc.x), S(0.5) * (z.y - zc.y));
                    P[jB * H + k] = cx<C>(S(0.5) * (z.y + zc.y), S(0.5) * (zc.x - z.x));
                }
            }
        }
        __syncthreads();
        for (int kk = w; kk < NQ; kk += nwc) {
            C v[R];
            if (kk == 0) {
#pragma unroll
                for (int r = 0; r < R; r++) {
                    const int j = 32 * r + lane;
                    v[r] = cx<C>(P[j * H].x, P[j * H + NQ].x);
                }
            } else {
#pragma unroll
                for (int r = 0; r < R; r++) v[r] = P[(32 * r + lane) * H + kk];
            }
            wfft_fwd<R>(v, tq, L, lane);
            if (kk == 0) {  // separate the two real columns' spectra (every kj)
                C c0[R], cq[R];
#pragma unroll
                for (int k1 = 0; k1 < R; k1++) {
                    const C z = v[k1], zc = mirror(v, k1, lane, src0);
                    c0[k1] = cx<C>(S(0.5) * (z.x + zc.x), S(0.5) * (z.y - zc.y));
                    cq[k1] = cx<C>(S(0.5) * (z.y + zc.y), S(0.5) * (zc.x - z.x));
                }
#pragma unroll
                for (int k1 = 0; k1 < R; k1++) {
                    P[(k1 + R * bl) * H] = c0[k1];
                    P[(k1 + R * bl) * H + NQ] = cq[k1];
                }
            } else {
#pragma unroll
                for (int k1 = 0; k1 < R; k1++) P[(k1 + R * bl) * H + kk] = v[k1];
            }
        }
        __syncthreads();
        C* Ti = T + (size_t)i * NH;
        for (int e = threadIdx.x; e < NH; e += blockDim.x) Ti[e] = P[e];
        __syncthreads();
    }
    pstamp(2);
    if (!team_sync(tm, epoch)) return false;
    pstamp(3);
    // B. each CTA takes whole planes kj: lines along i forward, times 1/(lambda N^3), inverse.
    //    With more CTAs than planes, the extra CTAs take the lines kk = N/2 of every plane.
    const S inv_n3 = S(1) / (S(N) * S(N) * S(N));
    const bool offload = tm.nblk > N;
    const int kk_end = offload ? NQ : H;
    auto line_i = [&](C (&v)[R], int kj, int kk) {
        wfft_fwd<R>(v, tq, L, lane);
        const S ljk = S(2) * tw[kj].x + S(2) * tw[kk].x - S(6);
#pragma unroll
        for (int k1 = 0; k1 < R; k1++) {
            const int ki = k1 + R * bl;
            const S f = (ki | kj | kk) == 0 ? S(0) : fast_div(inv_n3, tc[k1 * 32 + lane] + ljk);
            v[k1] = cx<C>(v[k1].x * f, v[k1].y * f);
        }
        wfft_inv<R>(v, tq, L, lane);
    };
    for (int kj = tm.b; kj < N; kj += tm.nblk) {
        for (int e = threadIdx.x; e < NH; e += blockDim.x) {
            const int ii = e / H, kk = e - ii * H;
            if (kk < kk_end) P[e] = T[((size_t)ii * N + kj) * H + kk];
        }
        __syncthreads();
        for (int kk = w; kk < kk_end; kk += nwc) {
            C v[R];
#pragma unroll
            for (int r = 0; r < R; r++) v[r] = P[(32 * r + lane) * H + kk];
            line_i(v, kj, kk);
#pragma unroll
            for (int r = 0; r < R; r++) P[(32 * r + lane) * H + kk] = v[r];
        }
        __syncthreads();
        for (int e = threadIdx.x; e < NH; e += blockDim.x) {
            const int ii = e / H, kk = e - ii * H;
            if (kk < kk_end) T[((size_t)ii * N + kj) * H + kk] = P[e];
        }
        __syncthreads();
    }
    if (offload && tm.b >= N) {
        const int nx = (tm.nblk - N) * nwc;
        for (int kj = (tm.b - N) * nwc + w; kj < N; kj += nx) {
            C* line = T + (size_t)kj * H + NQ;
            C v[R];
#pragma unroll
            for (int r = 0; r < R; r++) v[r] = line[(size_t)(32 * r + lane) * NH];
            line_i(v, kj, NQ);
#pragma unroll
            for (int r = 0; r < R; r++) line[(size_t)(32 * r + lane) * NH] = v[r];
        }
    }
    pstamp(4);
    if (!team_sync(tm, epoch)) return false;
    pstamp(5);
    // C. planes i again: lines along j inverse (the DC and Nyquist columns as one complex
    //    column, whose inverse is real in both parts), then rows along k complex to real
    //    (Z = X_A + i X_B, X[k] = conj X[N - k] above N/2) into x
    for (int i = tm.b; i < N; i += tm.nblk) {
        const C* Ti = T + (size_t)i * NH;
        for (int e = threadIdx.x; e < NH; e += blockDim.x) P[e] = Ti[e];
        __syncthreads();
        for (int kk = w; kk < NQ; kk += nwc) {
            C v[R];
            if (kk == 0) {
#pragma unroll
                for (int k1 = 0; k1 < R; k1++) {
                    const C c0 = P[(k1 + R * bl) * H], cq = P[(k1 + R * bl) * H + NQ];
                    v[k1] = cx<C>(c0.x - cq.y, c0.y + cq.x);
                }
            } else {
#pragma unroll
                for (int k1 = 0; k1 < R; k1++) v[k1] = P[(k1 + R * bl) * H + kk];
            }
            wfft_inv<R>(v, tq, L, lane);
            if (kk == 0) {
#pragma unroll
                for (int r = 0; r < R; r++) {
                    const int j = 32 * r + lane;
                    P[j * H] = cx<C>(v[r].x, S(0));
                    P[j * H + NQ] = cx<C>(v[r].y, S(0));
                }
            } else {
#pragma unroll
                for (int r = 0; r < R; r++) P[(32 * r + lane) * H + kk] = v[r];
            }
        }
        __syncthreads();
        for (int pr = w; pr < N / 2; pr += nwc) {
            const int jA = 2 * pr, jB = jA + 1;
            C v[R];
#pragma unroll
            for (int k1 = 0; k1 < R; k1++) {
                const int k = k1 + R * bl;
                const bool up = k >= H;
                const int kr = up ? N - k : k;
                C xa = P[jA * H + kr], xb = P[jB * H + kr];
                if (up) {
                    xa.y = -xa.y;
                    xb.y = -xb.y;
                }
                v[k1] = cx<C>(xa.x - xb.y, xa.y + xb.x);
            }
            wfft_inv<R>(v, tq, L, lane);
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int k = 32 * r + lane;
                x[split_idx(N, i, jA, k)] = v[r].x;
                x[split_idx(N, i, jB, k)] = v[r].y;
            }
        }
        __syncthreads();
    }
    pstamp(6);
    const bool ok = team_sync(tm, epoch);
    pstamp(7);
    return ok;
}

// Shared memory of the FFT-solved coarse level: one plane of the half spectrum.
__host__ __device__ constexpr size_t fft_plane_bytes(int nc, size_t scalar) { return (size_t)nc * (nc / 2 + 1) * 2 * scalar; }

template <class S>
__device__ bool team_fft(const MixedArgs& a, const Team& tm, unsigned& epoch, S* sm, int l, int outer) {
    __shared__ Cx<S> tw[kFftCoarseMax], tq[kFftCoarseMax];
    __shared__ S tc[kFftCoarseMax];
    Cx<S>* P = reinterpret_cast<Cx<S>*>(sm);
    const int n = a.lev_n[l];
    if (n == 128) return team_fft_r<4, S>(a, tm, epoch, l, tw, tq, tc, P, outer);
    if (n == 64) return team_fft_r<2, S>(a, tm, epoch, l, tw, tq, tc, P, outer);
    return team_fft_r<1, S>(a, tm, epoch, l, tw, tq, tc, P, outer);
}

// Grid-wide red-black sweeps of level l: `half_sweeps` colours starting at first_colour,
// a grid barrier after each except (when skip_last_barrier) the last. When esum is not
// null the values written in the last two half-sweeps are summed into it.
template <class T>
__device__ bool grid_smooth(const Team& tm, int n, const T* b, T* x, int first_colour, int half_sweeps,
                            unsigned& epoch, double* esum, bool skip_last_barrier) {
    for (int h = 0; h < half_sweeps; h++) {
        split_gs(tm, n, (first_colour + h) & 1, b, x, esum != nullptr && h >= half_sweeps - 2 ? esum : nullptr);
        if (h == half_sweeps - 1 && skip_last_barrier) break;
        if (!team_sync(tm, epoch)) return false;
    }
    return true;
}

// One V-cycle for the correction x0 of rhs b0 (level 0; r0 is its residual buffer), whose
// first red half-sweep has been done by the residual pass. Level 0 is stored as T0 (S, or
// FP16 for n = 128 and 256 with FP32 levels), the coarser levels as S. Ends after the last
// half-sweep of level 0 without a barrier, with this thread's share of sum(x0) in esum.
template <class S, class T0>
__device__ bool vcycle(const MixedArgs& a, const Team& tm, S* sm, unsigned& epoch, double& esum, int outer,
                       T0* x0, const T0* b0, T0* r0) {
    const int L = a.nlev, ls = a.lsmall, n0 = a.lev_n[0];
    const int lg = ls < L ? ls : L - 1;  // levels 0..lg-1 are smoothed and restricted on the grid
    if (!grid_smooth(tm, n0, b0, x0, 1, 2 * a.nu1 - 1, epoch, nullptr, false)) return false;
    split_resid_red(tm, n0, b0, x0, r0);
    if (!team_sync(tm, epoch)) return false;
    if (1 < ls) {
        split_restrict(tm, n0, r0, lev_b<S>(a, 1), lev_x<S>(a, 1));
        if (!team_sync(tm, epoch)) return false;
    }
    for (int l = 1; l < lg; l++) {
        if (!grid_smooth(tm, a.lev_n[l], lev_b<S>(a, l), lev_x<S>(a, l), 1, 2 * a.nu1 - 1, epoch, nullptr, false))
            return false;
        split_resid_red(tm, a.lev_n[l], lev_b<S>(a, l), lev_x<S>(a, l), lev_r<S>(a, l));
        if (!team_sync(tm, epoch)) return false;
        if (l + 1 < ls) {
            split_restrict(tm, a.lev_n[l], lev_r<S>(a, l), lev_b<S>(a, l + 1), lev_x<S>(a, l + 1));
            if (!team_sync(tm, epoch)) return false;
        }
    }
    stamp_outer(a, outer, 2);
    if (ls < L) {
        if (tm.b == 0) {
            if constexpr (std::is_same<T0, S>::value) small_vcycle(a, sm, ls == 1 ? r0 : lev_r<S>(a, ls - 1));
            else small_vcycle(a, sm, lev_r<S>(a, ls - 1));  // FP16 level 0 implies ls >= 2
        }
        if (!team_sync(tm, epoch)) return false;
    } else if (a.coarse_fft) {
        if (!team_fft<S>(a, tm, epoch, sm, L - 1, outer)) return false;
    } else if (a.coarse_team) {
        team_direct(a, tm, sm, L - 1);
        if (!team_sync(tm, epoch)) return false;
    } else {
        if (!grid_smooth(tm, a.lev_n[L - 1], lev_b<S>(a, L - 1), lev_x<S>(a, L - 1), 1, 2 * a.coarse_sweeps - 1,
                         epoch, nullptr, false))
            return false;
    }
    stamp_outer(a, outer, 3);
    for (int l = lg - 1; l >= 1; l--) {
        split_prolong_black(tm, a.lev_n[l], lev_x<S>(a, l + 1), lev_x<S>(a, l));
        if (!team_sync(tm, epoch)) return false;
        if (!grid_smooth(tm, a.lev_n[l], lev_b<S>(a, l), lev_x<S>(a, l), 0, 2 * a.nu2, epoch, nullptr, false))
            return false;
    }
    split_prolong_black(tm, n0, lev_x<S>(a, 1), x0);
    if (!team_sync(tm, epoch)) return false;
    return grid_smooth(tm, n0, b0, x0, 0, 2 * a.nu2, epoch, &esum, true);
}

// FP64 residual r = B - L X written as the FP32 rhs of the inner solve together with that
// solve's first red half-sweep from e = 0; returns this thread's max |r|. X is 0
// (START_ZERO), X[] (START_X) or the extrapolation 2 X[] - Xp[] (START_EXTRAP); B is c q
// when RHS_Q, else tmp.
enum StartKind { START_ZERO, START_X, START_EXTRAP };
template <int START, bool RHS_Q, class S>
__device__ __forceinline__ double residual_pass(const Team& tm, const MixedArgs& a, const double* X,
                                                const double* Xp, S* e, S* rb) {
    const int n = a.n;
    double rmax = 0.0;
    grid_pts(tm, n, [&](int i, int j, int k) {
        const Nb o = nb_of(n, i, j, k);
        auto x = [&](long q) { return START == START_EXTRAP ? 2 * X[q] - Xp[q] : X[q]; };
        double r;
        if (START == START_ZERO) {
            r = RHS_Q ? a.q[o.c] * a.c : a.tmp[o.c];
        } else {
            double s = x(o.ip) + x(o.im);
            s = s + x(o.jp);
            s = s + x(o.jm);
            s = s + x(o.kp);
            s = s + x(o.km);
            r = (RHS_Q ? a.q[o.c] * a.c : a.tmp[o.c]) - (s - x(o.c) * 6.0);
        }
        const S rf = (S)r;
        const int sx = split_idx(n, i, j, k);
        rb[sx] = rf;
        if (((i + j + k) & 1) == 0) e[sx] = rf * neg_sixth<S>();  // black e: written by the first half-sweep
        rmax = fmax(rmax, fabs(r));
    });
    return rmax;
}

// Vectorised residual pass (n even): a warp covers 64 consecutive k of a row with one
// double2 per lane (the last chunk of a row shorter when 64 does not divide n, its lanes
// past the row idle); k - 1 / k + 1 come from the adjacent lane by a shuffle, from memory
// at the ends of the chunk. Same sums, in the same order, as residual_pass. The rhs and e
// are stored as T (FP32, FP64, or FP16 for level 0 of the mixed form) in units of
// 1 / inv; WRITE false only returns the max |r|.
template <int START, bool RHS_Q, class T, bool WRITE = true>
__device__ __forceinline__ double residual_pass_vec(const Team& tm, const MixedArgs& a, const double* X,
                                                    const double* Xp, T* e, T* rb, double inv) {
    using S = typename Calc<T>::type;
    const int n = a.n, h = n >> 1, lane = threadIdx.x & 31;
    const int hp = h * n * n;
    double rmax = 0.0;
    auto x1 = [&](int q) { return START == START_EXTRAP ? 2 * X[q] - Xp[q] : X[q]; };
    auto x2 = [&](int q) {
        double2 v = *reinterpret_cast<const double2*>(X + q);
        if (START == START_EXTRAP) {
            const double2 p = *reinterpret_cast<const double2*>(Xp + q);
            v.x = 2 * v.x - p.x;
            v.y = 2 * v.y - p.y;
        }
        return v;
    };
    grid_rows(tm, n, [&](int i, int j) {
        const int ip = i + 1 == n ? 0 : i + 1, im = i == 0 ? n - 1 : i - 1;
        const int jp = j + 1 == n ? 0 : j + 1, jm = j == 0 ? n - 1 : j - 1;
        // 32-bit offsets: the mixed solver takes n <= kMixedMaxN (n^3 < 2^31)
        const int row = (i * n + j) * n;
        const int rip = (ip * n + j) * n, rim = (im * n + j) * n;
        const int rjp = (i * n + jp) * n, rjm = (i * n + jm) * n;
        const int cA = (i + j) & 1;  // colour of even k in this row
        const int srow = (i * n + j) * h;
        for (int k0 = 0; k0 < n; k0 += 64) {
            const bool act = k0 + 2 * lane < n;
            const int k = act ? k0 + 2 * lane : n - 2;  // idle lanes read a valid pair, store nothing
            double r0, r1;
            double2 bq;
            if (RHS_Q) {  // q is read only in segments the spreading marked (0 * c elsewhere; n % 64 == 0)
                const int seg = (row >> 6) + (k0 >> 6);
                double2 qv = make_double2(0.0, 0.0);
                if (a.qmask == nullptr || ((a.qmask[seg >> 5] >> (seg & 31)) & 1u))
                    qv = *reinterpret_cast<const double2*>(a.q + row + k);
                bq.x = qv.x * a.c;
                bq.y = qv.y * a.c;
            } else {
                bq = *reinterpret_cast<const double2*>(a.tmp + row + k);
            }
            if (START == START_ZERO) {
                r0 = bq.x;
                r1 = bq.y;
            } else {
                const double2 xip = x2(rip + k), xim = x2(rim + k), xjp = x2(rjp + k), xjm = x2(rjm + k);
                const double2 xc = x2(row + k);
                // the values beside the chunk (lane 0 and the chunk's last lane need them), loaded
                // by every lane ahead of the shuffles so that no load waits on one
                const double xl = x1(row + (k0 == 0 ? n - 1 : k0 - 1));
                const double xr = x1(row + (k + 2 >= n ? 0 : k + 2));
                double km0 = __shfl_sync(0xffffffffu, xc.y, (lane + 31) & 31);
                double kp1 = __shfl_sync(0xffffffffu, xc.x, (lane + 1) & 31);
                if (lane == 0) km0 = xl;
                if (lane == 31 || k + 2 >= n) kp1 = xr;
                double s0 = xip.x + xim.x;
                s0 = s0 + xjp.x;
                s0 = s0 + xjm.x;
                s0 = s0 + xc.y;
                s0 = s0 + km0;
                double s1 = xip.y + xim.y;
                s1 = s1 + xjp.y;
                s1 = s1 + xjm.y;
                s1 = s1 + kp1;
                s1 = s1 + xc.x;
                r0 = bq.x - (s0 - xc.x * 6.0);
                r1 = bq.y - (s1 - xc.y * 6.0);
            }
            if (act) {
                if (WRITE) {
                    const T rf0 = from_calc<T>((S)(r0 * inv)), rf1 = from_calc<T>((S)(r1 * inv));
                    const int p0 = cA * hp + srow + (k >> 1), p1 = (cA ^ 1) * hp + srow + (k >> 1);
                    rb[p0] = rf0;
                    rb[p1] = rf1;
                    // red e only: the first half-sweep (black) writes the black values without reading them
                    if (cA == 0) e[p0] = from_calc<T>(to_calc(rf0) * neg_sixth<S>());
                    else e[p1] = from_calc<T>(to_calc(rf1) * neg_sixth<S>());
                }
                rmax = fmax(rmax, fmax(fabs(r0), fabs(r1)));
            }
        }
    });
    return rmax;
}

template <int START, bool RHS_Q, class T, bool WRITE>
__device__ __forceinline__ double residual_any(const Team& tm, const MixedArgs& a, const double* X,
                                               const double* Xp, T* e, T* rb, double inv) {
    if constexpr (std::is_same<T, __half>::value || !WRITE) {  // FP16: n = 128 or 256
        return residual_pass_vec<START, RHS_Q, T, WRITE>(tm, a, X, Xp, e, rb, inv);
    } else {
        if (a.n % 2 == 0) return residual_pass_vec<START, RHS_Q, T, WRITE>(tm, a, X, Xp, e, rb, inv);
        return residual_pass<START, RHS_Q>(tm, a, X, Xp, e, rb);
    }
}
// the residual pass of refinement start st (rhs c q, or tmp when !rhs_q)
template <bool WRITE, class T>
__device__ __forceinline__ double residual_of(const Team& tm, const MixedArgs& a, int st, bool rhs_q,
                                              const double* X, T* e, T* rb, double inv) {
    if (st == START_ZERO) return residual_any<START_ZERO, true, T, WRITE>(tm, a, X, a.phi_prev, e, rb, inv);
    if (st == START_EXTRAP) return residual_any<START_EXTRAP, true, T, WRITE>(tm, a, X, a.phi_prev, e, rb, inv);
    if (rhs_q) return residual_any<START_X, true, T, WRITE>(tm, a, X, a.phi_prev, e, rb, inv);
    return residual_any<START_X, false, T, WRITE>(tm, a, X, a.phi_prev, e, rb, inv);
}

// home = X + (e - emean) scale with X as residual_pass reads it (0, X[], 2 X[] - phi_prev[])
// and e stored as T in units of 1 / scale.
template <int START, class T>
__device__ __forceinline__ void update_pass(const Team& tm, const MixedArgs& a, const double* X, double* home,
                                            const T* e, double emean, double scale) {
    const int n = a.n;
    if (n % 2 == 0) {  // double2 per lane, e from both colour halves (lanes past the row idle)
        // U chunks of 64 k at a time, all loaded before any is stored (home may be X itself,
        // so a store would otherwise hold the next chunk's loads back)
        constexpr int U = 4;
        const int h = n >> 1, lane = threadIdx.x & 31, hp = h * n * n;
        grid_rows(tm, n, [&](int i, int j) {
            const int row = (i * n + j) * n, srow = (i * n + j) * h;
            const int cA = (i + j) & 1;
            for (int k00 = 0; k00 < n; k00 += 64 * U) {
                double2 xo[U];
                double e0[U], e1[U];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const int k = k00 + 64 * u + 2 * lane;
                    xo[u] = make_double2(0.0, 0.0);
                    e0[u] = e1[u] = 0.0;
                    if (k < n) {
                        if (START != START_ZERO) xo[u] = *reinterpret_cast<const double2*>(X + row + k);
                        if (START == START_EXTRAP) {
                            const double2 p = *reinterpret_cast<const double2*>(a.phi_prev + row + k);
                            xo[u].x = 2 * xo[u].x - p.x;
                            xo[u].y = 2 * xo[u].y - p.y;
                        }
                        e0[u] = to_calc(e[cA * hp + srow + (k >> 1)]);
                        e1[u] = to_calc(e[(cA ^ 1) * hp + srow + (k >> 1)]);
                    }
                }
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const int k = k00 + 64 * u + 2 * lane;
                    if (k < n)
                        *reinterpret_cast<double2*>(home + row + k) =
                            make_double2(xo[u].x + (e0[u] - emean) * scale, xo[u].y + (e1[u] - emean) * scale);
                }
            }
        });
        return;
    }
    grid_pts(tm, n, [&](int i, int j, int k) {
        const long c = ((long)i * n + j) * n + k;
        const double xo = START == START_ZERO ? 0.0 : (START == START_EXTRAP ? 2 * X[c] - a.phi_prev[c] : X[c]);
        home[c] = xo + ((double)to_calc(e[split_idx(n, i, j, k)]) - emean) * scale;
    });
}

template <class T>
__device__ __forceinline__ void update_of(const Team& tm, const MixedArgs& a, int st, const double* X, double* home,
                                          const T* e, double emean, double scale) {
    if (st == START_ZERO) update_pass<START_ZERO>(tm, a, X, home, e, emean, scale);
    else if (st == START_EXTRAP) update_pass<START_EXTRAP>(tm, a, X, home, e, emean, scale);
    else update_pass<START_X>(tm, a, X, home, e, emean, scale);
}

// The refinement loop: r = B - L X in FP64 (checked against tol) -> rhs of the inner solve
// with the correction's first red half-sweep from e = 0; e = V-cycle; X += e - mean(e).
// X starts as Xs (read-only; zero for INIT) and lives in `home` from the first update.
// Level 0 is stored as T0. With FP16 (T0 = __half) its values are kept in units of a scale:
// the max |r| of the first residual (found by a pass that writes nothing), then of the last
// refinement's, so that the rhs stays within [-1, 1] and the correction well inside the
// FP16 range (a residual that leaves [1e-4, 4] times the scale is written again with its own
// max). The first scale is the grid's hint (the last solve's first residual max) when it
// has one, which spares the pass that only measures. The first red half-sweep, the V-cycle
// and the mean of the correction all work in those units; the update multiplies back.
template <class S, class T0>
__device__ __forceinline__ void refine(const MixedArgs& a, const Team& tm, S* sm, unsigned& epoch, int& seq,
                                       int start, bool rhs_q, const double*& Xs, double* home, int& result,
                                       bool& ok) {
    constexpr bool half0 = std::is_same<T0, __half>::value;
    const int n = a.n;
    T0* e = static_cast<T0*>(a.lev_x[0]);
    T0* rb = static_cast<T0*>(a.lev_b[0]);
    T0* r0 = static_cast<T0*>(a.lev_r[0]);
    double scale = 1.0;
    int outer = 0;
    while (ok) {
        stamp_outer(a, outer, 0);
        const int st = outer == 0 ? start : START_X;
        double s0 = 0.0, rmax = 0.0;
        if (half0 && outer == 0) {
            const double hint = a.scale_hint != nullptr ? *a.scale_hint : 0.0;
            if (hint > 0.0) {
                scale = hint;
            } else {
                rmax = residual_of<false>(tm, a, st, rhs_q, Xs, e, rb, 1.0);
                ok = reduce_sum_max(s0, rmax, tm, epoch, seq);
                if (!ok) break;
                if (rmax <= a.tol) {
                    result = 0;
                    break;
                }
                scale = rmax;
                s0 = rmax = 0.0;
            }
        }
        rmax = residual_of<true>(tm, a, st, rhs_q, Xs, e, rb, 1.0 / scale);
        ok = reduce_sum_max(s0, rmax, tm, epoch, seq);
        if (half0 && ok && rmax > a.tol && (rmax > 4.0 * scale || rmax < 1e-4 * scale)) {
            scale = rmax;
            s0 = rmax = 0.0;
            rmax = residual_of<true>(tm, a, st, rhs_q, Xs, e, rb, 1.0 / scale);
            ok = reduce_sum_max(s0, rmax, tm, epoch, seq);
        }
        // every CTA has read the hint before the reductions above
        if (half0 && outer == 0 && ok && a.scale_hint != nullptr && tm.b == 0 && threadIdx.x == 0)
            *a.scale_hint = rmax;
        stamp_outer(a, outer, 1);
        if (a.stamps != nullptr && outer < 8 && tm.b == 0 && threadIdx.x == 0)
            a.stamps[2 + 8 * outer + 7] = (unsigned long long)__double_as_longlong(rmax);
        if (!ok) break;
        if (rmax <= a.tol) {
            result = outer;
            break;
        }
        if (outer >= a.max_outer) break;
        double esum = 0.0, m0 = 0.0;
        ok = vcycle<S, T0>(a, tm, sm, epoch, esum, outer, e, rb, r0);
        if (!ok) break;
        stamp_outer(a, outer, 4);
        // mean of the correction (the periodic Laplacian's null space)
        ok = reduce_sum_max(esum, m0, tm, epoch, seq);
        if (!ok) break;
        stamp_outer(a, outer, 5);
        const double emean = esum / ((double)n * n * n);
        update_of(tm, a, st, Xs, home, e, emean, scale);
        Xs = home;
        ok = team_sync(tm, epoch);
        stamp_outer(a, outer, 6);
        if (half0) scale = rmax;  // the next residual is a fraction of this one
        outer++;
    }
}

// The solve of one system by one team of CTAs, level 0 stored as T0.
template <class S, class T0>
__device__ __forceinline__ void mixed_body(const MixedArgs& a, const Team& tm, S* sm) {
    const int n = a.n;
    unsigned epoch = 0;
    int seq = 0;
    bool ok = true;
    int result = -1;
    if (tm.b == 0) stamp(a, 0);

    // ---- set-up, as the FP64 programs (the unknown X, its start, the rhs B) ----
    // LCG and INIT read the rhs c q on the fly and start from the old field (or 0) without
    // a set-up pass; the MaZe programs keep sigma = L(2 phi - phi_prev) + c q in tmp.
    // (Starting the LCG update from 2 phi - phi_prev instead does not lower the first
    // residual: it is dominated by the local change of the spread charge.)
    double* home = a.phi_new;        // where the solution must end
    const double* X0 = a.phi_old;    // the start (read-only)
    int start = START_X;
    bool rhs_q = true;
    if (a.prog == PROG_INIT_FIELD) {         // y = 0 (later MaZe warm starts), phi = 0 start
        start = START_ZERO;
        grid_pts(tm, n, [&](int i, int j, int k) { a.y[((long)i * n + j) * n + k] = 0.0; });
    } else if (a.prog == PROG_LCG_UPDATE) {  // start from the old phi
    } else if (a.prog == PROG_MG_UPDATE) {   // start from 2 phi - phi_prev
        X0 = a.phi_new;
        grid_pts(tm, n, [&](int i, int j, int k) {
            const long c = ((long)i * n + j) * n + k;
            a.phi_new[c] = 2 * a.phi_old[c] - a.phi_prev[c];
        });
    } else {                                 // MaZe: phi = 2 phi - phi_prev; solve L y = sigma
        home = a.y;
        X0 = a.y;
        rhs_q = false;
        grid_pts(tm, n, [&](int i, int j, int k) {
            const Nb o = nb_of(n, i, j, k);
            auto ex = [&](long q) { return 2 * a.phi_old[q] - a.phi_prev[q]; };
            double s = ex(o.ip) + ex(o.im);
            s = s + ex(o.jp);
            s = s + ex(o.jm);
            s = s + ex(o.kp);
            s = s + ex(o.km);
            a.phi_new[o.c] = ex(o.c);
            a.tmp[o.c] = (s - ex(o.c) * 6.0) + a.c * a.q[o.c];
        });
    }
    if (a.prog != PROG_LCG_UPDATE) ok = team_sync(tm, epoch);
    stamp(a, 1);

    const double* Xs = X0;
    refine<S, T0>(a, tm, sm, epoch, seq, start, rhs_q, Xs, home, result, ok);
    // converged before any update: the solution is the start itself
    if (ok && Xs != home) {
        grid_pts(tm, n, [&](int i, int j, int k) {
            const long c = ((long)i * n + j) * n + k;
            home[c] = start == START_ZERO ? 0.0 : (start == START_EXTRAP ? 2 * Xs[c] - a.phi_prev[c] : Xs[c]);
        });
        ok = team_sync(tm, epoch);
    }
    if (ok && (a.prog == PROG_MAZE_LCG || a.prog == PROG_MAZE_MG)) {  // phi -= y
        grid_pts(tm, n, [&](int i, int j, int k) {
            const long c = ((long)i * n + j) * n + k;
            a.phi_new[c] = a.phi_new[c] + -1.0 * a.y[c];
        });
    }
    if (tm.b == 0 && threadIdx.x == 0) {
        a.result[0] = result;
        a.result[1] = ok ? 0 : 1;
    }
}

// Threads per CTA: 1024 with FP32 levels; 512 with FP64 levels, whose vectorised passes
// hold twice the registers per value (64 registers per thread at 1024 threads would spill).
template <class S> constexpr int threads_of() { return sizeof(S) == 8 ? 512 : kThreads; }

// One kernel per level-0 storage type (S, or FP16 with FP32 levels), each with one
// refinement loop.
template <class S, class T0>
__global__ void __launch_bounds__(threads_of<S>(), 1) mixed_kernel(MixedArgs a) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    const Team tm{(int)gridDim.x, (int)blockIdx.x, a.bar, a.partials};
    mixed_body<S, T0>(a, tm, reinterpret_cast<S*>(sm_raw));
}

// Many systems in one launch (FP32 levels): system r is worked by CTAs [start[r], start[r+1]).
__global__ void __launch_bounds__(kThreads, 1)
    mixed_batch_kernel(const MixedArgs* __restrict__ list, const int* __restrict__ start, int nsys) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    int lo = 0, hi = nsys - 1;  // last r with start[r] <= blockIdx.x
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const int b0 = start[lo], b1 = start[lo + 1];
    if ((int)blockIdx.x >= b1) return;  // CTAs past the last team (none when start[nsys] = gridDim.x)
    __shared__ MixedArgs a;  // this system's arguments, read from shared memory
    for (int w = threadIdx.x; w < (int)(sizeof(MixedArgs) / sizeof(int)); w += blockDim.x)
        reinterpret_cast<int*>(&a)[w] = reinterpret_cast<const int*>(list + lo)[w];
    __syncthreads();
    const Team tm{b1 - b0, (int)blockIdx.x - b0, a.bar, a.partials};
    mixed_body<float, float>(a, tm, reinterpret_cast<float*>(sm_raw));  // level 0 in FP32 (level0_fp16 unused)
}

// Launch configuration of one kernel variant, set up once per device.
struct Variant {
    int device = -1;
    int blocks = 0;
    size_t smem_set = 0;
};
Variant g_mixed_f32, g_mixed_f64, g_mixed_f16;
int g_batch_device = -1;
size_t g_batch_smem_set = 0;

size_t small_smem_bytes(const MixedArgs& a) {
    const size_t w = a.fp64 ? sizeof(double) : sizeof(float);
    if (a.coarse_fft) return fft_plane_bytes(a.lev_n[a.nlev - 1], w);  // one spectrum plane
    if (a.coarse_team) {  // G and b of the coarsest level in every CTA
        const size_t nc = (size_t)a.lev_n[a.nlev - 1];
        return 2 * nc * nc * nc * w;
    }
    size_t v = 0;
    for (int m = a.lsmall; m < a.nlev; m++) v += 3 * (size_t)a.lev_n[m] * a.lev_n[m] * a.lev_n[m];
    if (a.coarse_g != nullptr) v += (size_t)a.lev_n[a.nlev - 1] * a.lev_n[a.nlev - 1] * a.lev_n[a.nlev - 1];
    return v * w;
}

}  // namespace

int mixed_levels(int n, int* sizes) {
    int L = 0;
    int m = n;
    while (L < kMixedMaxLevels) {
        sizes[L++] = m;
        if (m % 2 || (m / 2) % 2 || m / 2 < 4) break;
        m /= 2;
    }
    return L;
}

void mixed_coarse_green(int n, double* g) {
    // g[d] = (1/N) sum_k e^{i w k.d} / lambda(k) over k != 0 (real: 1/lambda is even),
    // as three 1-D inverse transforms of 1/lambda, one axis at a time.
    const int N = n * n * n;
    const double w = 2.0 * 3.14159265358979323846 / n;
    std::vector<double> re((size_t)N), im((size_t)N, 0.0), tr((size_t)N), ti((size_t)N), c(n), sn(n);
    for (int k = 0; k < n; k++) {
        c[k] = cos(w * k);
        sn[k] = sin(w * k);
    }
    for (int k = 0; k < N; k++) {
        const int ki = k / (n * n), kj = (k / n) % n, kk = k % n;
        const double lam = 2 * c[ki] + 2 * c[kj] + 2 * c[kk] - 6.0;
        re[k] = k == 0 ? 0.0 : 1.0 / lam;
    }
    const int stride[3] = {n * n, n, 1};
    for (int ax = 0; ax < 3; ax++) {
        const int st = stride[ax];
        for (int q = 0; q < N; q++) {
            const int pos = (q / st) % n, base = q - pos * st;
            double sr = 0.0, si = 0.0;
            for (int k = 0; k < n; k++) {
                const int m = (k * pos) % n;  // e^{i w k pos}
                const double xr = re[base + k * st], xi = im[base + k * st];
                sr += xr * c[m] - xi * sn[m];
                si += xr * sn[m] + xi * c[m];
            }
            tr[q] = sr;
            ti[q] = si;
        }
        re.swap(tr);
        im.swap(ti);
    }
    for (int d = 0; d < N; d++) g[d] = re[d] / N;
}

void mixed_coarse_green(int n, float* g) {
    std::vector<double> gd((size_t)n * n * n);
    mixed_coarse_green(n, gd.data());
    for (size_t d = 0; d < gd.size(); d++) g[d] = (float)gd[d];
}

int mixed_small_level(int nlev, const int* sizes) {
    for (int l = 0; l < nlev; l++)
        if (sizes[l] <= kMixedSmallN) return l;
    return nlev;
}

size_t mixed_smem_bytes(const MixedArgs& a) { return small_smem_bytes(a); }

int mixed_grid_blocks() {
    int dev = 0, sms = 0;
    MZB_CHECK(cudaGetDevice(&dev));
    MZB_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    return sms;
}

void mixed_batch_launch(const MixedArgs* list, const int* start, int nsys, int nblocks, size_t smem,
                        cudaStream_t stream) {
    int dev;
    MZB_CHECK(cudaGetDevice(&dev));
    if (g_batch_device != dev || smem > g_batch_smem_set) {
        int per_sm = 0, sms = 0;
        if (smem > 48 * 1024)
            MZB_CHECK(cudaFuncSetAttribute(mixed_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        MZB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mixed_batch_kernel, kThreads, smem));
        MZB_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        if (per_sm < 1 || nblocks > per_sm * sms) fatal("batched mixed solver: CTAs cannot be co-resident");
        g_batch_device = dev;
        g_batch_smem_set = smem > g_batch_smem_set ? smem : g_batch_smem_set;
    }
    void* params[] = {(void*)&list, (void*)&start, (void*)&nsys};
    count_launch();
    MZB_CHECK(cudaLaunchCooperativeKernel((const void*)mixed_batch_kernel, dim3(nblocks), dim3(kThreads), params, smem,
                                          stream));
}

namespace {
template <class S, class T0>
void launch_variant(Variant& v, const MixedArgs& a, size_t smem, cudaStream_t stream) {
    const void* fn = (const void*)mixed_kernel<S, T0>;
    constexpr int threads = threads_of<S>();
    int dev;
    MZB_CHECK(cudaGetDevice(&dev));
    if (v.device != dev || smem > v.smem_set) {
        int sms = 0, per_sm = 0;
        if (smem > 48 * 1024)
            MZB_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        MZB_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        MZB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
        if (per_sm < 1) fatal("mixed solver: kernel cannot be resident on this device");
        v.device = dev;
        v.blocks = sms;
        v.smem_set = smem > v.smem_set ? smem : v.smem_set;
    }
    MZB_CHECK(cudaMemsetAsync(a.bar, 0, sizeof(GridBarrier), stream));
    MixedArgs copy = a;
    void* params[] = {&copy};
    count_launch();
    MZB_CHECK(cudaLaunchCooperativeKernel(fn, dim3(v.blocks), dim3(threads), params, smem, stream));
}
}  // namespace

void mixed_launch(const MixedArgs& a, cudaStream_t stream) {
    if (a.lsmall < 1 || a.lsmall > a.nlev || a.nlev < 2 || a.nu1 < 1 || a.nu2 < 1 || a.coarse_sweeps < 1)
        fatal("mixed solver: invalid level plan");
    if (a.level0_fp16 && (a.fp64 || (a.n != 128 && a.n != 256) || a.lsmall < 2))
        fatal("mixed solver: FP16 level 0 needs FP32 levels, n = 128 or 256 and no shared-memory level 1");
    const size_t smem = small_smem_bytes(a);
    if (a.fp64)
        launch_variant<double, double>(g_mixed_f64, a, smem, stream);
    else if (a.level0_fp16)
        launch_variant<float, __half>(g_mixed_f16, a, smem, stream);
    else
        launch_variant<float, float>(g_mixed_f32, a, smem, stream);
}

}  // namespace mzb
