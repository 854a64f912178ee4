// FP64 conjugate-gradient field solves with a TMA-staged 2.5-D stencil (sm_100a).
//
// Serves the CG programs of the solver engine -- conj_grad (library/src/plcg.c:28-90),
// its explicit-Jacobi form (plcg.c:104-166 with precond_jacobi.c:8-14), the LCG field
// init/update (grid_lcg.c:100-149) and the MaZe constraint solve (verlet.c:31-71) -- for
// grids with n % 16 == 0 and 16 <= n <= 256. Arithmetic per point is the reference's
// (same operation order, every product rounded), so single sweeps match bit for bit;
// only the dot products are summed in a different (fixed) order.
//
// One persistent CTA of 1024 threads per SM (cooperative launch). The grid is cut into
// work items (j-block of TJ rows, plane i); CTA c owns a contiguous run of items and
// keeps the same points in every phase. Per CG iteration:
//   phase A: p <- beta p + z(r), Ap = L p, <p, Ap>. The CTA marches along i over its
//     planes: (TJ+2) x n slabs of p_old and r arrive by TMA (one bulk-tensor row copy
//     per row, j wrapped) into a 4-stage mbarrier ring; each thread turns its column
//     into p_new once, keeps p_new(i-1), p_new(i), p_new(i+1) in registers and reads the
//     j+-1 / k+-1 neighbours from a shared p_new plane -- every p_old / r value crosses
//     L2 -> SM about (TJ+2)/TJ x (planes+2)/planes times instead of 7.
//   grid barrier, alpha = <r, z> / <p, Ap>
//   phase B: x += alpha p, r += alpha Ap, <r, r>, max |r| (vectorised streaming).
//   grid barrier, convergence test, beta.
#include <cudaTypedefs.h>

#include "engine.cuh"
#include "tma.cuh"

namespace mzb {

struct CgFastArgs {
    int prog;   // PROG_CG, PROG_INIT_FIELD, PROG_LCG_UPDATE, PROG_MAZE_LCG
    int kind;   // PC_IMPLICIT or PC_JACOBI
    int n, TJ, njb, stages;
    long items;
    double tol, c;
    const double* q;
    const double* phi_old;
    const double* phi_prev;
    double* phi_new;
    double* y;
    const double* b;
    const double* x0;
    double* x;
    double* r;
    double* p0;
    double* p1;
    double* Ap;
    double* tmp;
    double* partials;
    GridBarrier* bar;
    int* result;
    unsigned long long* stamps;  // optional phase timestamps (block 0), see kStampIters
};

namespace {

constexpr int kStampIters = 6;  // iterations whose phase boundaries are time-stamped

constexpr int kCompute = 512;             // compute threads (16 warps)
constexpr int kThreads = kCompute + 32;   // + one TMA producer warp
constexpr int kMaxStages = 6;
constexpr int kMaxElems = 192;  // plane slabs one CTA streams per phase

struct Nbr {
    long c, ip, im, jp, jm, kp, km;
};
__device__ __forceinline__ Nbr nbr_of(int n, int i, int j, int k) {
    const long n2 = (long)n * n;
    Nbr o;
    o.c = ((long)i * n + j) * n + k;
    o.ip = o.c + (i + 1 == n ? -(long)(n - 1) * n2 : n2);
    o.im = o.c + (i == 0 ? (long)(n - 1) * n2 : -n2);
    o.jp = o.c + (j + 1 == n ? -(long)(n - 1) * n : (long)n);
    o.jm = o.c + (j == 0 ? (long)(n - 1) * n : -(long)n);
    o.kp = o.c + (k + 1 == n ? -(long)(n - 1) : 1L);
    o.km = o.c + (k == 0 ? (long)(n - 1) : -1L);
    return o;
}
template <class F>
__device__ __forceinline__ double lap7(const Nbr& o, F&& f) {
    double s = f(o.ip) + f(o.im);
    s = s + f(o.jp);
    s = s + f(o.jm);
    s = s + f(o.kp);
    s = s + f(o.km);
    return s - f(o.c) * 6.0;
}

// Visit the CTA's own points: items [w0, w1), item = jb * n + i, TJ*n points each.
template <class F>
__device__ __forceinline__ void for_own(const CgFastArgs& a, long w0, long w1, F&& f) {
    const int n = a.n, TJ = a.TJ, per = TJ * n;
    for (long w = w0; w < w1; w++) {
        const int jb = (int)(w / n), i = (int)(w - (long)jb * n);
        for (int c = threadIdx.x; c < per; c += blockDim.x) f(i, jb * TJ + c / n, c % n);
    }
}

// NS sums then NM maxima over the grid; deterministic fixed-order gather.
template <int NS, int NM>
__device__ bool reduce(double* s, double* mx, const CgFastArgs& a, unsigned& epoch, int& seq) {
    __shared__ double sh[4 * 32];
    __shared__ double res[4];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const long G = gridDim.x;
#pragma unroll
    for (int q = 0; q < NS; q++) s[q] = warp_sum(s[q]);
#pragma unroll
    for (int q = 0; q < NM; q++) mx[q] = warp_max(mx[q]);
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NS; q++) sh[q * 32 + w] = s[q];
#pragma unroll
        for (int q = 0; q < NM; q++) sh[(NS + q) * 32 + w] = mx[q];
    }
    __syncthreads();
    double* part = a.partials + (long)(seq & 1) * 4 * G;
    if (w == 0) {
#pragma unroll
        for (int q = 0; q < NS + NM; q++) {
            double v = lane < nwarp ? sh[q * 32 + lane] : 0.0;
            v = q < NS ? warp_sum(v) : warp_max(v);
            if (lane == 0) part[q * G + blockIdx.x] = v;
        }
    }
    const bool ok = grid_sync_mono(a.bar, epoch);
    if (w == 0) {
#pragma unroll
        for (int q = 0; q < NS + NM; q++) {
            double v = 0.0;
            for (long b = lane; b < G; b += 32) {
                const double e = __ldcg(part + q * G + b);
                v = q < NS ? v + e : fmax(v, e);
            }
            v = q < NS ? warp_sum(v) : warp_max(v);
            if (lane == 0) res[q] = v;
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NS; q++) s[q] = res[q];
#pragma unroll
    for (int q = 0; q < NM; q++) mx[q] = res[NS + q];
    __syncthreads();
    seq++;
    return ok;
}

// slots 0..3: set-up; 4 + 4 it + {0..3}: phase ends of iteration it < kStampIters;
// 40 + 2 e + {0, 1}: slab e of the first phase A (compute done, next stage landed)
__device__ __forceinline__ void stamp(const CgFastArgs& a, int slot) {
    if (a.stamps != nullptr && blockIdx.x == 0 && threadIdx.x == 0 && slot < 96)
        a.stamps[slot] = global_ns();
}
__device__ __forceinline__ void stamp_it(const CgFastArgs& a, long iter, int k) {
    if (iter < kStampIters) stamp(a, 4 + 4 * (int)iter + k);
}

// z(r): the direction increment of the preconditioned residual, exactly as the
// reference forms it: (1/6) r (conj_grad, plcg.c:342-343,369-370) or
// -1 * (-r / 6) (conj_grad_precond with the Jacobi preconditioner).
template <int KIND>
__device__ __forceinline__ double zf(double r) {
    if (KIND == PC_IMPLICIT) return (1.0 / 6.0) * r;
    return -1.0 * (-r / 6.0);
}


// KIND: PrecondKind; PPT: column pairs per compute thread (1 for n <= 128, else 2). With
// 17 warps one SM sub-partition holds 5 of them, so 96 registers is the most a thread may
// use for the CTA to fit.
template <int KIND, int PPT>
__global__ void __maxnreg__(96)
    cg_fast_kernel(const __grid_constant__ CUtensorMap map_r_row, const __grid_constant__ CUtensorMap map_r_slab,
                   const __grid_constant__ CUtensorMap map_p0_row, const __grid_constant__ CUtensorMap map_p0_slab,
                   const __grid_constant__ CUtensorMap map_p1_row, const __grid_constant__ CUtensorMap map_p1_slab,
                   CgFastArgs a) {
    extern __shared__ __align__(128) unsigned char smraw[];
    const int n = a.n, TJ = a.TJ, R = TJ + 2, S = a.stages, njb = a.njb;
    const long slab = (long)R * n;  // doubles per array per stage
    // TMA destinations must start on 128-byte boundaries of the shared window
    unsigned char* sm0 = smraw + ((128u - (smem_u32(smraw) & 127u)) & 127u);
    double* stg = reinterpret_cast<double*>(sm0);  // [S][2][R][n]: p_old, r slabs
    double* pnb = stg + (long)S * 2 * slab;        // [2][R][n]: p_new planes
    double* wrp = pnb + 2 * slab;                  // [2 sets][S][2][n]: wrapped halo rows
    uint64_t* full = reinterpret_cast<uint64_t*>(wrp + (long)S * 4 * n);
    uint64_t* empty = full + S;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool producer = warp == kCompute / 32;

    if (a.prog != PROG_CG && a.prog != PROG_INIT_FIELD && a.prog != PROG_LCG_UPDATE &&
        a.prog != PROG_MAZE_LCG) {
        if (blockIdx.x == 0 && tid == 0) {
            a.result[0] = -1;
            a.result[1] = 2;
        }
        return;
    }
    __shared__ int abort_sh;
    if (tid == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kCompute / 32);
        }
        fence_mbar_init();
        abort_sh = 0;
    }
    if (producer && lane == 0) {
        prefetch_tensormap(&map_r_row); prefetch_tensormap(&map_r_slab);
        prefetch_tensormap(&map_p0_row); prefetch_tensormap(&map_p0_slab);
        prefetch_tensormap(&map_p1_row); prefetch_tensormap(&map_p1_slab);
    }
    __syncthreads();

    const long G = gridDim.x;
    const long w0 = blockIdx.x * a.items / G, w1 = (blockIdx.x + 1) * a.items / G;
    unsigned epoch = 0;
    int seq = 0;
    bool ok = true;
    int result = -1;

    // ---- set-up of the right-hand side (one pass over own points) ----
    if (a.prog == PROG_INIT_FIELD) {        // y = 0; phi = c q   (grid_lcg.c:108-113)
        for_own(a, w0, w1, [&](int i, int j, int k) {
            const long c = ((long)i * n + j) * n + k;
            a.y[c] = 0.0;
            a.phi_new[c] = a.q[c] * a.c;
        });
    } else if (a.prog == PROG_LCG_UPDATE) { // y = c q            (grid_lcg.c:134-138)
        for_own(a, w0, w1, [&](int i, int j, int k) {
            const long c = ((long)i * n + j) * n + k;
            a.y[c] = a.q[c] * a.c;
        });
    } else if (a.prog == PROG_MAZE_LCG) {   // phi = 2 phi - phi_prev; sigma = L phi + c q
        for_own(a, w0, w1, [&](int i, int j, int k) {
            const Nbr o = nbr_of(n, i, j, k);
            auto ex = [&](long q) { return 2 * a.phi_old[q] - a.phi_prev[q]; };
            a.phi_new[o.c] = ex(o.c);
            a.tmp[o.c] = lap7(o, ex) + a.c * a.q[o.c];
        });
    }
    stamp(a, 0);
    ok = grid_sync_mono(a.bar, epoch);
    stamp(a, 1);
    const double* B = a.prog == PROG_INIT_FIELD ? a.phi_new
                      : a.prog == PROG_LCG_UPDATE ? a.y
                      : a.prog == PROG_MAZE_LCG ? a.tmp : a.b;
    const double* X0 = a.prog == PROG_INIT_FIELD ? a.y
                       : a.prog == PROG_LCG_UPDATE ? a.phi_old
                       : a.prog == PROG_MAZE_LCG ? a.y : a.x0;
    double* X = (a.prog == PROG_INIT_FIELD || a.prog == PROG_LCG_UPDATE) ? a.phi_new
                : a.prog == PROG_MAZE_LCG ? a.y : a.x;

    // ---- r = L x0 - b; x = x0; <r, z(r)> ----
    double rv = 0.0;
    if (ok) {
        double acc[1] = {0.0}, m0[1];
        for_own(a, w0, w1, [&](int i, int j, int k) {
            const Nbr o = nbr_of(n, i, j, k);
            const double x0c = X0[o.c];
            const double rr = lap7(o, [&](long q) { return X0[q]; }) + -1.0 * B[o.c];
            if (X != X0) X[o.c] = x0c;
            a.r[o.c] = rr;
            acc[0] += rr * (KIND == PC_IMPLICIT ? rr * (1.0 / 6.0) : -rr / 6.0);
        });
        ok = reduce<1, 0>(acc, m0, a, epoch, seq);
        rv = KIND == PC_IMPLICIT ? -acc[0] : acc[0];
    }
    stamp(a, 2);

    // ---- plan of plane slabs streamed in phase A (same every iteration) ----
    // For each run of items with the same j-block: planes ia-1, ia, ..., ib+1 (wrapped).
    __shared__ short e_jb[kMaxElems], e_plane[kMaxElems];
    __shared__ unsigned char e_flag[kMaxElems];  // 1: fill p_new plane, 2: emit output, 4: run end
    __shared__ int e_count;
    if (tid == 0) {
        int ne = 0;
        for (long w = w0; w < w1;) {
            const int b = (int)(w / n);
            const long wend = min(w1, (long)(b + 1) * n);
            const int ia = (int)(w - (long)b * n), L = (int)(wend - w) + 2;
            for (int e = 0; e < L && ne < kMaxElems; e++, ne++) {
                e_jb[ne] = (short)b;
                e_plane[ne] = (short)(((ia - 1 + e) % n + n) % n);
                e_flag[ne] = (unsigned char)(((e >= 1 && e <= L - 2) ? 1 : 0) | (e >= 2 ? 2 : 0) |
                                             (e == L - 1 ? 4 : 0));
            }
            w = wend;
        }
        e_count = ne;
    }
    __syncthreads();
    const int nload = e_count;
    const uint32_t stage_bytes = (uint32_t)(2 * slab * sizeof(double));

    // compute threads: column pairs (k, k+1) of the slab, offsets fixed for the kernel
    const int pairs = TJ * n / 2;
    const int ppt = (pairs + kCompute - 1) / kCompute;  // pairs per thread (<= PPT)
    int so[PPT], go[PPT];                    // stage/plane offset, global offset
    bool pv[PPT];
#pragma unroll
    for (int m = 0; m < PPT; m++) {
        const int pr = tid + m * kCompute;
        pv[m] = !producer && m < ppt && pr < pairs;
        const int jl = pv[m] ? (2 * pr) / n : 0, k = pv[m] ? (2 * pr) % n : 0;
        so[m] = (jl + 1) * n + k;
        go[m] = jl * n + k;
    }
    // halo pairs of the p_new plane: row 0 and row R-1, n/2 pairs each
    const bool hv = !producer && tid < n;
    const int hrow = tid < n / 2 ? 0 : R - 1, hk = 2 * (tid % (n / 2 > 0 ? n / 2 : 1));

    const long limit = (long)n * n;
    long iter = 0;
    int ld = 0;  // slab loads issued (CTA lifetime; identical in every thread)
    double beta = 0.0;
    const double* pold = a.p1;
    double* pnew = a.p0;
    while (ok && iter < limit) {
        const bool first = iter == 0;
        const CUtensorMap* mslab = (pold == a.p0) ? &map_p0_slab : &map_p1_slab;
        const CUtensorMap* mrow = (pold == a.p0) ? &map_p0_row : &map_p1_row;
        const int base = ld;
        double pap[1] = {0.0}, m0[1];
        if (producer) {
            // ---- producer warp: stream the slabs through the S-stage ring ----
            if (lane == 0) fence_proxy_async_global();
            for (int e = 0; e < nload; e++) {
                const int sq = base + e, s = sq % S, use = sq / S;
                int good = 1;
                if (lane == 0 && use > 0) {
                    if (abort_sh || !mbar_wait(&empty[s], (uint32_t)((use - 1) & 1))) good = 0;
                }
                good = __shfl_sync(0xffffffffu, good, 0);
                if (!good) {
                    abort_sh = 1;
                    break;
                }
                const int jb = e_jb[e], plane = e_plane[e];
                double* dst = stg + (long)s * 2 * slab;
                double* wdst = wrp + (long)s * 2 * n;
                const bool lo = jb == 0, hi = jb == njb - 1;
                const uint32_t bytes = stage_bytes + ((lo || hi) ? (uint32_t)(2 * n * sizeof(double)) : 0u) +
                                       ((lo && hi) ? (uint32_t)(2 * n * sizeof(double)) : 0u);
                if (lane == 0) mbar_expect_tx(&full[s], bytes);
                __syncwarp();
                // one (n x R) box per array from row j0-1 (rows outside [0,n) are zero-filled);
                // the periodic image of a wrapped row goes to the wrap buffer
                if (lane < 2)
                    tma_load_3d(dst + lane * slab, lane ? &map_r_slab : mslab, 0, jb * TJ - 1, plane, &full[s]);
                if ((lo || hi) && lane >= 2 && lane < 4)
                    tma_load_3d(wdst + (lane - 2) * n, lane == 3 ? &map_r_row : mrow, 0, lo ? n - 1 : 0, plane,
                                &full[s]);
                if (lo && hi && lane >= 4 && lane < 6)
                    tma_load_3d(wdst + (long)S * 2 * n + (lane - 4) * n, lane == 5 ? &map_r_row : mrow, 0, 0,
                                plane, &full[s]);
            }
        } else {
            // ---- compute warps ----
            double2 pprev[PPT], pcur[PPT], pnext[PPT];
#pragma unroll
            for (int m = 0; m < PPT; m++) pprev[m] = pcur[m] = pnext[m] = make_double2(0.0, 0.0);
            int buf = 0;
            for (int e = 0; e < nload; e++) {
                const int sq = base + e, s = sq % S;
                const int jb = e_jb[e], plane = e_plane[e], flag = e_flag[e];
                int good = 1;
                if (lane == 0 && (abort_sh || !mbar_wait(&full[s], (uint32_t)((sq / S) & 1)))) good = 0;
                good = __shfl_sync(0xffffffffu, good, 0);
                if (!good) abort_sh = 1;
                if (first && e < 18 && tid == 0) stamp(a, 40 + 3 * e);
                const double* sp = stg + (long)s * 2 * slab;  // p_old rows
                const double* sr = sp + slab;                 // r rows
                const bool fill = flag & 1;
                double* pb = pnb + (long)buf * slab;
                if (good) {
                    // this slab's p_new on own pairs (and, for planes ia..ib, the shared plane)
#pragma unroll
                    for (int m = 0; m < PPT; m++) {
                        if (!pv[m]) continue;
                        const double2 rr = *reinterpret_cast<const double2*>(sr + so[m]);
                        double2 z = make_double2(zf<KIND>(rr.x), zf<KIND>(rr.y));
                        if (!first) {
                            const double2 po = *reinterpret_cast<const double2*>(sp + so[m]);
                            z.x = po.x * beta + z.x;
                            z.y = po.y * beta + z.y;
                        }
                        pnext[m] = z;
                        if (fill) *reinterpret_cast<double2*>(pb + so[m]) = z;
                    }
                    if (fill && hv) {
                        const bool wrapped = (hrow == 0 && jb == 0) || (hrow == R - 1 && jb == njb - 1);
                        const double* w =
                            wrp + (long)s * 2 * n + ((hrow == R - 1 && njb == 1) ? (long)S * 2 * n : 0);
                        const double* hp = wrapped ? w : sp + hrow * n;
                        const double* hr = wrapped ? w + n : sr + hrow * n;
                        const double2 rr = *reinterpret_cast<const double2*>(hr + hk);
                        double2 z = make_double2(zf<KIND>(rr.x), zf<KIND>(rr.y));
                        if (!first) {
                            const double2 po = *reinterpret_cast<const double2*>(hp + hk);
                            z.x = po.x * beta + z.x;
                            z.y = po.y * beta + z.y;
                        }
                        *reinterpret_cast<double2*>(pb + hrow * n + hk) = z;
                    }
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty[s]);  // this warp is done with stage s
                if (first && e < 18 && tid == 0) stamp(a, 41 + 3 * e);
                if ((flag & 2) && good) {
                    // output plane = plane - 1; its p_new plane is in the other buffer
                    const double* pc = pnb + (long)(buf ^ 1) * slab;
                    const int iout = plane == 0 ? n - 1 : plane - 1;
                    const long plane_off = ((long)iout * n + jb * TJ) * n;
#pragma unroll
                    for (int m = 0; m < PPT; m++) {
                        if (!pv[m]) continue;
                        const int o = so[m], k = o % n;
                        const double2 jp = *reinterpret_cast<const double2*>(pc + o + n);
                        const double2 jm = *reinterpret_cast<const double2*>(pc + o - n);
                        const double km = pc[k == 0 ? o + n - 1 : o - 1];
                        const double kp2 = pc[k + 2 == n ? o + 2 - n : o + 2];
                        double s0 = pnext[m].x + pprev[m].x;
                        s0 = s0 + jp.x;
                        s0 = s0 + jm.x;
                        s0 = s0 + pcur[m].y;
                        s0 = s0 + km;
                        double s1 = pnext[m].y + pprev[m].y;
                        s1 = s1 + jp.y;
                        s1 = s1 + jm.y;
                        s1 = s1 + kp2;
                        s1 = s1 + pcur[m].x;
                        const double2 ap = make_double2(s0 - pcur[m].x * 6.0, s1 - pcur[m].y * 6.0);
                        const long g = plane_off + go[m];
                        *reinterpret_cast<double2*>(pnew + g) = pcur[m];
                        *reinterpret_cast<double2*>(a.Ap + g) = ap;
                        pap[0] += pcur[m].x * ap.x;
                        pap[0] += pcur[m].y * ap.y;
                    }
                }
                if (first && e < 18 && tid == 0) stamp(a, 42 + 3 * e);
                named_bar_sync(1, kCompute);  // p_new planes complete / free again
#pragma unroll
                for (int m = 0; m < PPT; m++) {
                    pprev[m] = pcur[m];
                    pcur[m] = pnext[m];
                }
                if (fill) buf ^= 1;
                if (flag & 4) buf = 0;  // run finished: the next run restarts its window
            }
        }
        ld = base + nload;
        __syncthreads();
        if (abort_sh) {
            ok = false;
            atomicOr(&a.bar->err, 1u);
            break;
        }
        stamp_it(a, iter, 0);
        ok = reduce<1, 0>(pap, m0, a, epoch, seq);
        stamp_it(a, iter, 1);
        if (!ok) break;
        const double alpha = rv / pap[0];

        // phase B: x += alpha p; r += alpha Ap; <r,r>, max|r| (+ <r, P r> for Jacobi).
        // Flattened over the CTA's slabs, two independent double2 per array and thread in
        // flight (~64 KB per SM, past the HBM latency need).
        double sums[2] = {0.0, 0.0}, rmax[1] = {0.0};
        {
            const int per2 = TJ * n / 2;
            const int total = (int)(w1 - w0) * per2;
            const int nt = blockDim.x;
            double* __restrict__ Xr = X;
            double* __restrict__ Rr = a.r;
            const double* __restrict__ Pr = pnew;
            const double* __restrict__ Ar = a.Ap;
            for (int f0 = tid; f0 < total; f0 += 2 * nt) {
                long g[2];
                double2 xx[2], rr[2], pp[2], aa[2];
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    const int f = f0 + u * nt;
                    g[u] = -1;
                    if (f < total) {
                        const int it = f / per2, v = f - it * per2;
                        const long w = w0 + it;
                        const int jb = (int)(w / n), i = (int)(w - (long)jb * n);
                        g[u] = ((long)i * n + jb * TJ) * n + 2L * v;
                        xx[u] = *reinterpret_cast<const double2*>(Xr + g[u]);
                        rr[u] = *reinterpret_cast<const double2*>(Rr + g[u]);
                        pp[u] = *reinterpret_cast<const double2*>(Pr + g[u]);
                        aa[u] = *reinterpret_cast<const double2*>(Ar + g[u]);
                    }
                }
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    if (g[u] < 0) continue;
                    xx[u].x = xx[u].x + alpha * pp[u].x;
                    xx[u].y = xx[u].y + alpha * pp[u].y;
                    rr[u].x = rr[u].x + alpha * aa[u].x;
                    rr[u].y = rr[u].y + alpha * aa[u].y;
                    *reinterpret_cast<double2*>(Xr + g[u]) = xx[u];
                    *reinterpret_cast<double2*>(Rr + g[u]) = rr[u];
                    sums[0] += rr[u].x * rr[u].x;
                    sums[0] += rr[u].y * rr[u].y;
                    if (KIND == PC_JACOBI) {
                        sums[1] += rr[u].x * (-rr[u].x / 6.0);
                        sums[1] += rr[u].y * (-rr[u].y / 6.0);
                    }
                    rmax[0] = fmax(rmax[0], fmax(fabs(rr[u].x), fabs(rr[u].y)));
                }
            }
        }
        stamp_it(a, iter, 2);
        ok = reduce<2, 1>(sums, rmax, a, epoch, seq);
        stamp_it(a, iter, 3);
        if (!ok) break;
        if (rmax[0] <= a.tol) {
            result = (int)iter;
            break;
        }
        const double rnv = KIND == PC_IMPLICIT ? -sums[0] / 6.0 : sums[1];
        beta = rnv / rv;
        rv = rnv;
        iter++;
        pold = pnew;
        pnew = (pnew == a.p0) ? a.p1 : a.p0;
    }

    if (ok && a.prog == PROG_MAZE_LCG) {  // phi -= y (verlet.c:65)
        for_own(a, w0, w1, [&](int i, int j, int k) {
            const long c = ((long)i * n + j) * n + k;
            a.phi_new[c] = a.phi_new[c] + -1.0 * a.y[c];
        });
    }
    if (!ok && producer && lane == 0) {
        // drain copies that may still be in flight into this CTA's shared memory: only the
        // last S issued slabs can be (bounded waits)
        for (int sq = (ld > S ? ld - S : 0); sq < ld; sq++) mbar_wait(&full[sq % S], (uint32_t)((sq / S) & 1));
    }
    if (blockIdx.x == 0 && tid == 0) {
        a.result[0] = result;
        a.result[1] = ok ? 0 : 1;
    }
}

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

}  // namespace

bool encode_grid_map(CUtensorMap* map, const double* base, int n, int bx, int by) {
    if (!g_encode) {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || fn == nullptr)
            return false;
        g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const cuuint64_t dims[3] = {(cuuint64_t)n, (cuuint64_t)n, (cuuint64_t)n};
    const cuuint64_t strides[2] = {(cuuint64_t)n * 8, (cuuint64_t)n * n * 8};
    const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(base), dims,
                                strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// Row-block height TJ for the TMA march: the largest divisor of n not above
// max(8, 1024 / n), so one CTA's plane slab holds about 1024 points.
int cg_fast_rows(int n) {
    int cap = 1024 / n;
    if (cap < 8) cap = 8;
    int best = 1;
    for (int t = 1; t <= cap && t <= n; t++)
        if (n % t == 0) best = t;
    return best;
}

bool cg_fast_supported(int n) { return n % 16 == 0 && n >= 16 && n <= 256; }

int cg_fast_stamp_slots() { return 4 + 4 * kStampIters; }

int cg_fast_stages(int n) {
    const int R = cg_fast_rows(n) + 2;
    const size_t budget = 200 * 1024;  // of the 227 KB a CTA may use
    int s = kMaxStages;
    while (s > 2 && (size_t)(s * 2 + 2) * R * n * sizeof(double) + (size_t)s * 4 * n * sizeof(double) > budget) s--;
    return s;
}

size_t cg_fast_smem(int n) {
    const int R = cg_fast_rows(n) + 2, S = cg_fast_stages(n);
    return (size_t)(S * 2 + 2) * R * n * sizeof(double) + (size_t)S * 4 * n * sizeof(double) +
           2 * S * sizeof(uint64_t) + 128;
}

namespace {
int g_fast_device = -1;
int g_fast_blocks = 0;
}  // namespace

// Launch a CG program on the TMA path. Returns false if the path is unavailable here
// (caller falls back to the general engine).
bool cg_fast_launch(const EngineArgs& e, cudaStream_t stream) {
    static const bool verbose = getenv("MZB_PHASE_TIMING") != nullptr;
    auto no = [&](const char* why) {
        if (verbose) fprintf(stderr, "[cg fast path unavailable: %s]\n", why);
        return false;
    };
    const int n = e.n;
    if (e.pb) return no("Poisson-Boltzmann operator");
    if (!cg_fast_supported(n)) return no("grid size");
    const bool cg_prog = e.prog == PROG_CG || e.prog == PROG_PCG || e.prog == PROG_INIT_FIELD ||
                         e.prog == PROG_LCG_UPDATE || e.prog == PROG_MAZE_LCG;
    if (!cg_prog) return false;
    if ((e.prog == PROG_PCG || e.prog == PROG_MAZE_LCG) && e.precond != PC_IMPLICIT && e.precond != PC_JACOBI)
        return false;
    int dev;
    MZB_CHECK(cudaGetDevice(&dev));
    if (g_fast_device != dev) {
        const int smem_max = (int)cg_fast_smem(256);
        const void* kernels[4] = {(const void*)cg_fast_kernel<PC_IMPLICIT, 1>, (const void*)cg_fast_kernel<PC_IMPLICIT, 2>,
                                  (const void*)cg_fast_kernel<PC_JACOBI, 1>, (const void*)cg_fast_kernel<PC_JACOBI, 2>};
        int sms = 0;
        MZB_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        for (const void* kf : kernels) {
            MZB_CHECK(cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max));
            int per_sm = 0;
            MZB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kf, kThreads, smem_max));
            if (per_sm < 1) {
                if (verbose) {
                    cudaFuncAttributes fa;
                    cudaFuncGetAttributes(&fa, kf);
                    fprintf(stderr, "[cg fast: regs %d static smem %zu max threads %d, dyn smem %d]\n", fa.numRegs,
                            fa.sharedSizeBytes, fa.maxThreadsPerBlock, smem_max);
                }
                return no("occupancy 0");
            }
        }
        g_fast_device = dev;
        g_fast_blocks = sms;
    }
    const int TJ = cg_fast_rows(n);
    CgFastArgs a{};
    a.prog = e.prog == PROG_PCG ? PROG_CG : e.prog;
    a.kind = (e.prog == PROG_PCG || e.prog == PROG_MAZE_LCG) ? e.precond : PC_IMPLICIT;
    a.n = n;
    a.TJ = TJ;
    a.njb = n / TJ;
    a.stages = cg_fast_stages(n);
    a.items = (long)a.njb * n;
    // the per-CTA slab plan must fit kMaxElems
    const long per_cta = (a.items + g_fast_blocks - 1) / g_fast_blocks;
    if (per_cta + 2 * (per_cta / n + 2) > kMaxElems) return no("plan too long");
    a.tol = e.tol;
    a.c = e.c;
    a.q = e.q; a.phi_old = e.phi_old; a.phi_prev = e.phi_prev; a.phi_new = e.phi_new; a.y = e.y;
    a.b = e.b; a.x0 = e.x0; a.x = e.x;
    a.r = e.r; a.p0 = e.p0; a.p1 = e.p1; a.Ap = e.Ap; a.tmp = e.tmp;
    a.partials = e.partials; a.bar = e.bar; a.result = e.result;
    a.stamps = e.stamps;
    CUtensorMap mr, mrs, mp0, mp0s, mp1, mp1s;
    if (!encode_grid_map(&mr, a.r, n, n, 1) || !encode_grid_map(&mp0, a.p0, n, n, 1) ||
        !encode_grid_map(&mp1, a.p1, n, n, 1) || !encode_grid_map(&mrs, a.r, n, n, TJ + 2) ||
        !encode_grid_map(&mp0s, a.p0, n, n, TJ + 2) || !encode_grid_map(&mp1s, a.p1, n, n, TJ + 2))
        return no("tensor map encode");
    MZB_CHECK(cudaMemsetAsync(a.bar, 0, sizeof(GridBarrier), stream));
    const size_t smem = cg_fast_smem(n);
    void* params[] = {&mr, &mrs, &mp0, &mp0s, &mp1, &mp1s, &a};
    count_launch();
    const int ppt = (TJ * n / 2 + kCompute - 1) / kCompute;
    const void* kf = a.kind == PC_JACOBI
                         ? (ppt == 1 ? (const void*)cg_fast_kernel<PC_JACOBI, 1> : (const void*)cg_fast_kernel<PC_JACOBI, 2>)
                         : (ppt == 1 ? (const void*)cg_fast_kernel<PC_IMPLICIT, 1>
                                     : (const void*)cg_fast_kernel<PC_IMPLICIT, 2>);
    if (ppt > 2) return no("more than two column pairs per thread");
    MZB_CHECK(cudaLaunchCooperativeKernel(kf, dim3(g_fast_blocks), dim3(kThreads), params, smem, stream));
    return true;
}

}  // namespace mzb
