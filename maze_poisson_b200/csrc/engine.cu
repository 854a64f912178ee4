// Persistent solver engine (see engine.cuh).
//
// Work decomposition: one warp per grid row (fixed i,j; lanes stride over k), rows
// distributed grid-stride over all warps of the cooperative grid. Every sweep keeps the
// reference's per-point arithmetic (order of the sums, products rounded before adds) so
// single sweeps are bit-identical to the reference; only the global dot products are
// summed in a different (fixed, deterministic) order.
#include <type_traits>
#include <utility>

#include "engine.cuh"

namespace mzb {
namespace {

constexpr int kThreads = 512;
constexpr int kMinBlocksPerSM = 1;

struct Team {
    int lane;
    long gw;
    long nw;
};
__device__ __forceinline__ Team make_team() {
    Team t;
    t.lane = threadIdx.x & 31;
    t.gw = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    t.nw = (long)gridDim.x * (blockDim.x >> 5);
    return t;
}

// Visit every point of an n^3 grid once: warp per (i,j) row, lanes over k.
template <class F>
__device__ __forceinline__ void for_points(const Team& t, int n, F&& f) {
    const long rows = (long)n * n;
    for (long row = t.gw; row < rows; row += t.nw) {
        const int i = (int)(row / n), j = (int)(row - (long)i * n);
        for (int k = t.lane; k < n; k += 32) f(i, j, k);
    }
}
// The same visit for n % 64 == 0 with two points per lane per step, k and k + 32: f(i, j,
// k0, k1) computes both before storing either, so their loads are in flight together; a
// lane still meets its points in ascending k.
template <class F>
__device__ __forceinline__ void for_point_pairs(const Team& t, int n, F&& f) {
    const long rows = (long)n * n;
    for (long row = t.gw; row < rows; row += t.nw) {
        const int i = (int)(row / n), j = (int)(row - (long)i * n);
        for (int k = t.lane; k < n; k += 64) f(i, j, k, k + 32);
    }
}
// Visit the points of one colour ((i+j+k) % 2 == colour) of an n^3 grid (n even).
template <class F>
__device__ __forceinline__ void for_colour(const Team& t, int n, int colour, F&& f) {
    const long rows = (long)n * n;
    for (long row = t.gw; row < rows; row += t.nw) {
        const int i = (int)(row / n), j = (int)(row - (long)i * n);
        for (int k = ((i + j + colour) & 1) + 2 * t.lane; k < n; k += 64) f(i, j, k);
    }
}

// The colour visit for n % 128 == 0 with two points per lane per step, k and k + 64 (the
// same colour, so neither reads the other): f(i, j, k0, k1) computes both before storing.
template <class F>
__device__ __forceinline__ void for_colour_pairs(const Team& t, int n, int colour, F&& f) {
    const long rows = (long)n * n;
    for (long row = t.gw; row < rows; row += t.nw) {
        const int i = (int)(row / n), j = (int)(row - (long)i * n);
        for (int k = ((i + j + colour) & 1) + 2 * t.lane; k < n; k += 128) f(i, j, k, k + 64);
    }
}

struct Nb {
    long c, ip, im, jp, jm, kp, km;
};
__device__ __forceinline__ Nb neighbours(int n, int i, int j, int k) {
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

// 7-point Laplacian in the reference's order: x+1, x-1, y+1, y-1, z+1, z-1, - 6 c
// (library/src/laplace.c:208-216). `f(idx)` yields the operand at a flat index.
template <class F>
__device__ __forceinline__ double lap7(const Nb& o, F&& f) {
    double s = f(o.ip) + f(o.im);
    s = s + f(o.jp);
    s = s + f(o.jm);
    s = s + f(o.kp);
    s = s + f(o.km);
    return s - f(o.c) * 6.0;
}

// The field operators the programs are written over: the reference's Laplacian
// (laplace.c:24-75) and the Poisson-Boltzmann operator (laplace.c:77-145), whose faces
// x+, x-, y+, y-, z+, z- multiply their neighbours in that order before the centre term
// u_c * dg_c, dg = ex_c + ex_{x-1} + ey_c + ey_{y-1} + ez_c + ez_{z-1} + k2_c (the
// reference's inline diagonal, precomputed with the same additions).
struct LapOp {
    template <class F>
    __device__ __forceinline__ double apply(const Nb& o, F&& f) const { return lap7(o, f); }
};
struct PbOp {
    const double *ex, *ey, *ez, *dg;
    template <class F>
    __device__ __forceinline__ double apply(const Nb& o, F&& f) const {
        double s = f(o.ip) * ex[o.c] + f(o.im) * ex[o.im];
        s = s + f(o.jp) * ey[o.c];
        s = s + f(o.jm) * ey[o.jm];
        s = s + f(o.kp) * ez[o.c];
        s = s + f(o.km) * ez[o.km];
        return s - f(o.c) * dg[o.c];
    }
};

// ------------------------------------------------------------------------------------
// Grid-wide reductions: NS sums followed by NM maxima. Results land in every thread.
// Partials are double-buffered by a sequence number so a fast block writing reduction
// k+1 never overwrites values a slow block is still gathering for reduction k.
// ------------------------------------------------------------------------------------
template <int NS, int NM>
__device__ bool grid_reduce(double* s, double* mx, const EngineArgs& a, int& seq) {
    __shared__ double sh[8 * 32];
    __shared__ double res[8];
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
    double* part = a.partials + (long)(seq & 1) * 8 * G;
    if (w == 0) {
#pragma unroll
        for (int q = 0; q < NS + NM; q++) {
            double v = lane < nwarp ? sh[q * 32 + lane] : 0.0;
            v = q < NS ? warp_sum(v) : warp_max(v);
            if (lane == 0) part[q * G + blockIdx.x] = v;
        }
    }
    const bool ok = grid_sync(a.bar);
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

// ------------------------------------------------------------------------------------
// Multigrid sweeps (library/src/multigrid.c)
// ------------------------------------------------------------------------------------

// One red-black Gauss-Seidel iteration: red ((i+j+k) even) then black
// (multigrid.c:636-729). Neighbour sum order i-1, i+1, j-1, j+1, k-1, k+1.
__device__ bool rbgs(const Team& t, const double* rhs, double* x, int n, const EngineArgs& a) {
    const double inv_diag = -1.0 / 6.0;
    for (int colour = 0; colour < 2; colour++) {
        for_colour(t, n, colour, [&](int i, int j, int k) {
            const Nb o = neighbours(n, i, j, k);
            double s = x[o.im] + x[o.ip];
            s = s + x[o.jm];
            s = s + x[o.jp];
            s = s + x[o.km];
            s = s + x[o.kp];
            x[o.c] = (rhs[o.c] - s) * inv_diag;
        });
        if (!grid_sync(a.bar)) return false;
    }
    return true;
}

// One red-black iteration of the PB smoother (multigrid_pb.c:544-640): x_c = (faces x+,
// x-, y+, y-, z+, z- times their neighbours, minus rhs_c) / max(dg_c, 1e-14).
__device__ bool rbgs_pb(const Team& t, const double* rhs, double* x, int n, const PbOp& op,
                        const EngineArgs& a) {
    auto value = [&](const Nb& o) {
        double d = op.dg[o.c];
        if (d < 1e-14) d = 1e-14;
        double s = op.ex[o.c] * x[o.ip] + op.ex[o.im] * x[o.im];
        s = s + op.ey[o.c] * x[o.jp];
        s = s + op.ey[o.jm] * x[o.jm];
        s = s + op.ez[o.c] * x[o.kp];
        s = s + op.ez[o.km] * x[o.km];
        s = s - rhs[o.c];
        return s / d;
    };
    for (int colour = 0; colour < 2; colour++) {
        if (n % 128 == 0) {
            for_colour_pairs(t, n, colour, [&](int i, int j, int k0, int k1) {
                const Nb o0 = neighbours(n, i, j, k0), o1 = neighbours(n, i, j, k1);
                const double v0 = value(o0), v1 = value(o1);
                x[o0.c] = v0;
                x[o1.c] = v1;
            });
        } else {
            for_colour(t, n, colour, [&](int i, int j, int k) {
                const Nb o = neighbours(n, i, j, k);
                x[o.c] = value(o);
            });
        }
        if (!grid_sync(a.bar)) return false;
    }
    return true;
}

// 27-point full weighting, coarse (I,J,K) <- fine (2I,2J,2K) (multigrid.c:523-594).
__device__ void restrict27(const Team& t, const double* in, double* out, int n) {
    const int nc = n / 2;
    const long n2 = (long)n * n;
    for_points(t, nc, [&](int I, int J, int K) {
        const int i = 2 * I, j = 2 * J, k = 2 * K;
        const long i0 = (long)i * n2, i1 = (long)(i + 1 == n ? 0 : i + 1) * n2,
                   i2 = (long)(i == 0 ? n - 1 : i - 1) * n2;
        const long j0 = (long)j * n, j1 = (long)(j + 1 == n ? 0 : j + 1) * n,
                   j2 = (long)(j == 0 ? n - 1 : j - 1) * n;
        const long k0 = k, k1 = (k + 1 == n ? 0 : k + 1), k2 = (k == 0 ? n - 1 : k - 1);
        double f = in[i2 + j0 + k0] + in[i1 + j0 + k0];
        f = f + in[i0 + j2 + k0];
        f = f + in[i0 + j1 + k0];
        f = f + in[i0 + j0 + k2];
        f = f + in[i0 + j0 + k1];
        double e = in[i1 + j0 + k2] + in[i1 + j0 + k1];
        e = e + in[i2 + j0 + k2];
        e = e + in[i2 + j0 + k1];
        e = e + in[i1 + j2 + k0];
        e = e + in[i1 + j1 + k0];
        e = e + in[i2 + j2 + k0];
        e = e + in[i2 + j1 + k0];
        e = e + in[i0 + j2 + k2];
        e = e + in[i0 + j2 + k1];
        e = e + in[i0 + j1 + k2];
        e = e + in[i0 + j1 + k1];
        double c = in[i1 + j1 + k2] + in[i1 + j1 + k1];
        c = c + in[i1 + j2 + k2];
        c = c + in[i1 + j2 + k1];
        c = c + in[i2 + j1 + k2];
        c = c + in[i2 + j1 + k1];
        c = c + in[i2 + j2 + k2];
        c = c + in[i2 + j2 + k1];
        double v = 8.0 * in[i0 + j0 + k0] + 4.0 * f;
        v = v + 2.0 * e;
        v = v + c;
        out[((long)I * nc + J) * nc + K] = v * (1.0 / 64.0);
    });
}

// Trilinear prolongation value at fine (i,j,k) from an nc^3 coarse grid
// (multigrid.c:393-463): weights (1,0) on even fine indices, (0.5,0.5) on odd.
__device__ __forceinline__ double prolong_at(const double* in, int nc, int i, int j, int k) {
    const double wi0 = (i & 1) ? 0.5 : 1.0, wi1 = (i & 1) ? 0.5 : 0.0;
    const double wj0 = (j & 1) ? 0.5 : 1.0, wj1 = (j & 1) ? 0.5 : 0.0;
    const double wk0 = (k & 1) ? 0.5 : 1.0, wk1 = (k & 1) ? 0.5 : 0.0;
    const long n2 = (long)nc * nc;
    const int ci = i >> 1, cj = j >> 1, ck = k >> 1;
    const long i0 = (long)ci * n2, i1 = (long)(ci + 1 == nc ? 0 : ci + 1) * n2;
    const long j0 = (long)cj * nc, j1 = (long)(cj + 1 == nc ? 0 : cj + 1) * nc;
    const long k0 = ck, k1 = (ck + 1 == nc ? 0 : ck + 1);
    double s = in[i0 + j0 + k0] * wi0 * wj0 * wk0 + in[i1 + j0 + k0] * wi1 * wj0 * wk0;
    s = s + in[i0 + j1 + k0] * wi0 * wj1 * wk0;
    s = s + in[i1 + j1 + k0] * wi1 * wj1 * wk0;
    s = s + in[i0 + j0 + k1] * wi0 * wj0 * wk1;
    s = s + in[i1 + j0 + k1] * wi1 * wj0 * wk1;
    s = s + in[i0 + j1 + k1] * wi0 * wj1 * wk1;
    s = s + in[i1 + j1 + k1] * wi1 * wj1 * wk1;
    return s;
}

// ------------------------------------------------------------------------------------
// Conjugate gradients on A x = b (plcg.c:28-238, multigrid.c:13-96, multigrid_pb.c:16-97).
// ------------------------------------------------------------------------------------
struct CgSpec {
    int n;
    const double* b;
    const double* x0;
    double* x;
    double* r;
    double* p0;
    double* p1;
    double* Ap;
    double* v;      // PC_MG: preconditioner output (warm-started)
    int kind;       // PrecondKind
    bool coarse;    // cg_coarse semantics (relative stop, denominator guard, count)
    double tol;     // absolute stop (conj_grad*)
    double rtol;    // relative stop (cg_coarse)
    long limit;     // iteration cap
};

__device__ bool vcycle(const Team& t, const double* rhs, double* x, int n, int sm, const EngineArgs& a,
                       int& seq);

// Points of the hyperplane i + j + k = s of an n^3 grid, spread over every warp.
template <class F>
__device__ __forceinline__ void for_hyperplane(const Team& t, int n, int s, F&& f) {
    const int ilo = s - 2 * (n - 1) > 0 ? s - 2 * (n - 1) : 0, ihi = s < n - 1 ? s : n - 1;
    if (ilo > ihi) return;
    const long pairs = (long)(ihi - ilo + 1) * n;
    for (long q = t.gw * 32 + t.lane; q < pairs; q += t.nw * 32) {
        const int i = ilo + (int)(q / n), j = (int)(q % n), k = s - i - j;
        if (k >= 0 && k < n) f(i, j, k);
    }
}

// SSOR preconditioner (precond_ssor.c:1240-1252, omega = 1.75): v = r; a forward solve in
// index order, v_c = (v_c + the neighbours of smaller flat index in the order x+1, x-1,
// y+1, y-1, z+1, z-1) / (6/omega); v *= -6; a backward solve in reverse index order over
// the neighbours of larger index; v *= (2-omega)/omega. Every smaller-index neighbour lies
// on an earlier hyperplane i+j+k (the periodic x+1 neighbour of i = n-1 sits n-1 planes
// back), so each solve is a wavefront of 3n-2 hyperplanes with a grid barrier between
// them. The copy and the -6 scaling are folded into the solves' reads of v_c.
__device__ bool ssor_apply(const Team& t, const double* r, double* v, int n, const EngineArgs& a) {
    const double omega = 1.75, dc = 6.0 / omega;
    for (int dir = 0; dir < 2; dir++) {
        const bool fwd = dir == 0;
        for (int h = 0; h <= 3 * (n - 1); h++) {
            const int s = fwd ? h : 3 * (n - 1) - h;
            for_hyperplane(t, n, s, [&](int i, int j, int k) {
                const Nb o = neighbours(n, i, j, k);
                double x = fwd ? r[o.c] : v[o.c] * -6.0;
                const long nb[6] = {o.ip, o.im, o.jp, o.jm, o.kp, o.km};
#pragma unroll
                for (int q = 0; q < 6; q++)
                    if (fwd ? nb[q] < o.c : nb[q] > o.c) x = x + v[nb[q]];
                v[o.c] = x / dc;
            });
            if (!grid_sync(a.bar)) return false;
        }
    }
    const double fin = (2 - omega) / omega;
    for_points(t, n, [&](int i, int j, int k) {
        const long c = ((long)i * n + j) * n + k;
        v[c] = v[c] * fin;
    });
    return grid_sync(a.bar);
}

// Block-Jacobi preconditioner (precond_blockjacobi.c:173-206): the (n/10)^3 blocks as
// rows of 1000 values in (i, j, k) order times the block inverse, C = R Ainv, the
// reference's dgemm with every output summed over l in increasing order (linalg.c:170-181)
// and every product rounded. A CTA computes 64 x 64 tiles of C from 8-deep slices of R
// (gathered straight from the grid, so no reorder pass) and Ainv staged in shared memory;
// each thread holds a 4 x 2 block of C.
__device__ __forceinline__ long bj_point(int n, int nb, int blk, int l) {
    const int bk = blk % nb, bj = (blk / nb) % nb, bi = blk / (nb * nb);
    const int ii = l / 100, jj = (l / 10) % 10, kk = l % 10;
    return ((long)(bi * kBlockJacobiB + ii) * n + (bj * kBlockJacobiB + jj)) * n + bk * kBlockJacobiB + kk;
}

__device__ bool bj_apply(const Team& t, const double* r, double* v, int n, const EngineArgs& a) {
    constexpr int T = 64, K = 8;
    static_assert(kThreads == 512, "the tile map assumes 512 threads");
    __shared__ double As[K][T];
    __shared__ double Bs[K][T];
    const int nb = n / kBlockJacobiB, nblk = nb * nb * nb;
    const int rt = (nblk + T - 1) / T, ct = (kBlockJacobiB3 + T - 1) / T;
    const int tr = threadIdx.x >> 5, tc = threadIdx.x & 31;       // rows 4 tr.., cols 2 tc..
    const int lk = threadIdx.x / T, lr = threadIdx.x % T;          // loader slot
    for (int tile = blockIdx.x; tile < rt * ct; tile += gridDim.x) {
        const int row0 = (tile / ct) * T, col0 = (tile % ct) * T;
        double acc[4][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
        for (int k0 = 0; k0 < kBlockJacobiB3; k0 += K) {
            const int blk = row0 + lr, col = col0 + lr;
            As[lk][lr] = blk < nblk ? r[bj_point(n, nb, blk, k0 + lk)] : 0.0;
            Bs[lk][lr] = col < kBlockJacobiB3 ? a.bj_inv[(long)(k0 + lk) * kBlockJacobiB3 + col] : 0.0;
            __syncthreads();
#pragma unroll
            for (int kk = 0; kk < K; kk++) {
                const double b0 = Bs[kk][2 * tc], b1 = Bs[kk][2 * tc + 1];
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const double av = As[kk][4 * tr + i];
                    acc[i][0] = acc[i][0] + av * b0;
                    acc[i][1] = acc[i][1] + av * b1;
                }
            }
            __syncthreads();
        }
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const int blk = row0 + 4 * tr + i, col = col0 + 2 * tc + j;
                if (blk < nblk && col < kBlockJacobiB3) v[bj_point(n, nb, blk, col)] = acc[i][j];
            }
    }
    return grid_sync(a.bar);
}

// v = M^-1 r for the explicit preconditioners of conj_grad_precond
template <int KIND>
__device__ bool precond_apply(const Team& t, const double* r, double* v, int n, const EngineArgs& a, int& seq) {
    if (KIND == PC_SSOR) return ssor_apply(t, r, v, n, a);
    if (KIND == PC_BLOCKJACOBI) return bj_apply(t, r, v, n, a);
    return vcycle(t, r, v, n, 5, a, seq);
}

// Returns the reference's value: conj_grad* -> 0-based iteration at convergence or -1;
// cg_coarse* -> number of iterations run. `ok` turns false on a barrier failure.
// KIND is the PrecondKind; COARSE selects the cg_coarse variant (implicit Jacobi for the
// Laplacian, none for PB; never an MG preconditioner, so the V-cycle -> coarse CG call
// chain is not recursive). OP is the operator A (LapOp or PbOp).
template <int KIND, bool COARSE, class OP>
__device__ int cg_run(const Team& t, const CgSpec& s, const OP& op, const EngineArgs& a, int& seq, bool& ok) {
    static_assert(!(COARSE && KIND != PC_IMPLICIT && KIND != PC_NONE), "coarse CG has no MG preconditioner");
    const int n = s.n;
    // r = L x0 - b; x = x0; v = 0 (PC_MG)
    double acc[2] = {0.0, 0.0}, mx[1] = {0.0};
    for_points(t, n, [&](int i, int j, int k) {
        const Nb o = neighbours(n, i, j, k);
        const double x0c = s.x0[o.c];
        const double rr = op.apply(o, [&](long q) { return s.x0[q]; }) + -1.0 * s.b[o.c];
        if (s.x != s.x0) s.x[o.c] = x0c;
        s.r[o.c] = rr;
        if (KIND == PC_IMPLICIT) acc[0] += rr * (rr * (1.0 / 6.0));
        else if (KIND == PC_JACOBI) acc[0] += rr * (-rr / 6.0);
        else if (KIND == PC_NONE) acc[0] += rr * rr;
        else s.v[o.c] = 0.0;
        mx[0] = fmax(mx[0], fabs(rr));
    });
    ok = grid_reduce<1, 1>(acc, mx, a, seq);
    if (!ok) return -1;
    double rv;
    if (KIND == PC_IMPLICIT) rv = -acc[0];
    else if (KIND == PC_JACOBI || KIND == PC_NONE) rv = acc[0];
    else {
        ok = precond_apply<KIND>(t, s.r, s.v, n, a, seq);
        if (!ok) return -1;
        double d[1] = {0.0}, m0[1];
        for_points(t, n, [&](int i, int j, int k) {
            const long c = ((long)i * n + j) * n + k;
            d[0] += s.r[c] * s.v[c];
        });
        ok = grid_reduce<1, 0>(d, m0, a, seq);
        if (!ok) return -1;
        rv = d[0];
    }
    const double r0 = mx[0];
    if (COARSE && r0 == 0.0) return 0;

    long iter = 0;
    int res = COARSE ? (int)s.limit : -1;
    double beta = 0.0;
    const double* pold = s.p1;
    double* pnew = s.p0;
    while (iter < s.limit) {
        const bool first = (iter == 0);
        // phase A: p <- beta p + z(r); Ap = L p; <p, Ap>
        auto zf = [&](long q) {
            if (KIND == PC_IMPLICIT) return (1.0 / 6.0) * s.r[q];
            if (KIND == PC_JACOBI) return -1.0 * (-s.r[q] / 6.0);
            if (KIND == PC_NONE) return -1.0 * s.r[q];
            return -1.0 * s.v[q];
        };
        auto pf = [&](long q) { return first ? zf(q) : pold[q] * beta + zf(q); };
        double pap[1] = {0.0}, m0[1];
        if (n % 64 == 0) {
            for_point_pairs(t, n, [&](int i, int j, int k0, int k1) {
                const Nb o0 = neighbours(n, i, j, k0), o1 = neighbours(n, i, j, k1);
                const double pc0 = pf(o0.c), pc1 = pf(o1.c);
                const double ap0 = op.apply(o0, pf), ap1 = op.apply(o1, pf);
                pnew[o0.c] = pc0;
                s.Ap[o0.c] = ap0;
                pnew[o1.c] = pc1;
                s.Ap[o1.c] = ap1;
                pap[0] += pc0 * ap0;
                pap[0] += pc1 * ap1;
            });
        } else {
            for_points(t, n, [&](int i, int j, int k) {
                const Nb o = neighbours(n, i, j, k);
                const double pc = pf(o.c);
                const double ap = op.apply(o, pf);
                pnew[o.c] = pc;
                s.Ap[o.c] = ap;
                pap[0] += pc * ap;
            });
        }
        ok = grid_reduce<1, 0>(pap, m0, a, seq);
        if (!ok) return -1;
        if (COARSE && fabs(pap[0]) < 1e-300) { res = (int)iter; break; }
        const double alpha = rv / pap[0];
        // phase B: x += alpha p; r += alpha Ap; <r,r>, |r|_inf (+ <r, P r> for Jacobi)
        double sums[2] = {0.0, 0.0}, rmax[1] = {0.0};
        auto upd = [&](double rn) {
            sums[0] += rn * rn;
            if (KIND == PC_JACOBI) sums[1] += rn * (-rn / 6.0);
            rmax[0] = fmax(rmax[0], fabs(rn));
        };
        if (n % 64 == 0) {
            for_point_pairs(t, n, [&](int i, int j, int k0, int k1) {
                const long c0 = ((long)i * n + j) * n + k0, c1 = c0 + (k1 - k0);
                const double x0 = s.x[c0] + alpha * pnew[c0], x1 = s.x[c1] + alpha * pnew[c1];
                const double rn0 = s.r[c0] + alpha * s.Ap[c0], rn1 = s.r[c1] + alpha * s.Ap[c1];
                s.x[c0] = x0;
                s.x[c1] = x1;
                s.r[c0] = rn0;
                s.r[c1] = rn1;
                upd(rn0);
                upd(rn1);
            });
        } else {
            for_points(t, n, [&](int i, int j, int k) {
                const long c = ((long)i * n + j) * n + k;
                s.x[c] = s.x[c] + alpha * pnew[c];
                const double rn = s.r[c] + alpha * s.Ap[c];
                s.r[c] = rn;
                upd(rn);
            });
        }
        ok = grid_reduce<2, 1>(sums, rmax, a, seq);
        if (!ok) return -1;
        if (COARSE) {
            if (rmax[0] <= s.rtol * r0) { res = (int)iter + 1; break; }
        } else if (rmax[0] <= s.tol) {
            res = (int)iter;
            break;
        }
        double rnv;
        if (KIND == PC_IMPLICIT) rnv = -sums[0] / 6.0;
        else if (KIND == PC_JACOBI) rnv = sums[1];
        else if (KIND == PC_NONE) rnv = sums[0];
        else {
            ok = precond_apply<KIND>(t, s.r, s.v, n, a, seq);
            if (!ok) return -1;
            double d[1] = {0.0}, m1[1];
            for_points(t, n, [&](int i, int j, int k) {
                const long c = ((long)i * n + j) * n + k;
                d[0] += s.r[c] * s.v[c];
            });
            ok = grid_reduce<1, 0>(d, m1, a, seq);
            if (!ok) return -1;
            rnv = d[0];
        }
        beta = rnv / rv;
        rv = rnv;
        iter++;
        pold = pnew;
        pnew = (pnew == s.p0) ? s.p1 : s.p0;
    }
    return res;
}

// One V-cycle as the reference runs it (recursion bottoms out at depth 1): sm RBGS
// iterations, residual rf = -(L x) + rhs, 27-pt restriction, coarse CG (50 it, rtol
// 1e-5) from zero, x += P e, sm RBGS iterations (multigrid.c:99-168).
__device__ bool vcycle(const Team& t, const double* rhs, double* x, int n, int sm, const EngineArgs& a,
                       int& seq) {
    const int nc = n / 2;
    for (int it = 0; it < sm; it++)
        if (!rbgs(t, rhs, x, n, a)) return false;
    for_points(t, n, [&](int i, int j, int k) {
        const Nb o = neighbours(n, i, j, k);
        const double lx = lap7(o, [&](long q) { return x[q]; });
        a.rf[o.c] = -lx + 1.0 * rhs[o.c];
    });
    if (!grid_sync(a.bar)) return false;
    restrict27(t, a.rf, a.rc, n);
    for_points(t, nc, [&](int i, int j, int k) { a.ec[((long)i * nc + j) * nc + k] = 0.0; });
    if (!grid_sync(a.bar)) return false;
    CgSpec cs;
    cs.n = nc; cs.b = a.rc; cs.x0 = a.ec; cs.x = a.ec; cs.r = a.cr; cs.p0 = a.cp0; cs.p1 = a.cp1;
    cs.Ap = a.cAp; cs.v = nullptr; cs.kind = PC_IMPLICIT; cs.coarse = true; cs.tol = 0.0;
    cs.rtol = 1e-5; cs.limit = 50;
    bool ok = true;
    cg_run<PC_IMPLICIT, true>(t, cs, LapOp{}, a, seq, ok);
    if (!ok) return false;
    for_points(t, n, [&](int i, int j, int k) {
        const long c = ((long)i * n + j) * n + k;
        x[c] = x[c] + 1.0 * prolong_at(a.ec, nc, i, j, k);
    });
    if (!grid_sync(a.bar)) return false;
    for (int it = 0; it < sm; it++)
        if (!rbgs(t, rhs, x, n, a)) return false;
    return true;
}

// One PB V-cycle (multigrid_pb.c:270-328): sm PB smoother iterations, residual
// rf = -(A x) + rhs, 27-pt restriction, coarse PB CG (unpreconditioned, 50 it, rtol
// 1e-5) from zero on the restricted coefficients, x += P e, sm iterations.
__device__ bool vcycle_pb(const Team& t, const double* rhs, double* x, int n, int sm, const EngineArgs& a,
                          int& seq) {
    const int nc = n / 2;
    const PbOp fine{a.ex, a.ey, a.ez, a.dg}, coarse{a.cex, a.cey, a.cez, a.cdg};
    for (int it = 0; it < sm; it++)
        if (!rbgs_pb(t, rhs, x, n, fine, a)) return false;
    auto res = [&](const Nb& o) { return -fine.apply(o, [&](long q) { return x[q]; }) + 1.0 * rhs[o.c]; };
    if (n % 64 == 0) {
        for_point_pairs(t, n, [&](int i, int j, int k0, int k1) {
            const Nb o0 = neighbours(n, i, j, k0), o1 = neighbours(n, i, j, k1);
            const double r0 = res(o0), r1 = res(o1);
            a.rf[o0.c] = r0;
            a.rf[o1.c] = r1;
        });
    } else {
        for_points(t, n, [&](int i, int j, int k) {
            const Nb o = neighbours(n, i, j, k);
            a.rf[o.c] = res(o);
        });
    }
    if (!grid_sync(a.bar)) return false;
    restrict27(t, a.rf, a.rc, n);
    for_points(t, nc, [&](int i, int j, int k) { a.ec[((long)i * nc + j) * nc + k] = 0.0; });
    if (!grid_sync(a.bar)) return false;
    CgSpec cs;
    cs.n = nc; cs.b = a.rc; cs.x0 = a.ec; cs.x = a.ec; cs.r = a.cr; cs.p0 = a.cp0; cs.p1 = a.cp1;
    cs.Ap = a.cAp; cs.v = nullptr; cs.kind = PC_NONE; cs.coarse = true; cs.tol = 0.0;
    cs.rtol = 1e-5; cs.limit = 50;
    bool ok = true;
    cg_run<PC_NONE, true>(t, cs, coarse, a, seq, ok);
    if (!ok) return false;
    if (n % 64 == 0) {
        for_point_pairs(t, n, [&](int i, int j, int k0, int k1) {
            const long c0 = ((long)i * n + j) * n + k0, c1 = c0 + (k1 - k0);
            const double v0 = x[c0] + 1.0 * prolong_at(a.ec, nc, i, j, k0);
            const double v1 = x[c1] + 1.0 * prolong_at(a.ec, nc, i, j, k1);
            x[c0] = v0;
            x[c1] = v1;
        });
    } else {
        for_points(t, n, [&](int i, int j, int k) {
            const long c = ((long)i * n + j) * n + k;
            x[c] = x[c] + 1.0 * prolong_at(a.ec, nc, i, j, k);
        });
    }
    if (!grid_sync(a.bar)) return false;
    for (int it = 0; it < sm; it++)
        if (!rbgs_pb(t, rhs, x, n, fine, a)) return false;
    return true;
}

// max |A x - b| over the grid (the reference's residual check after each V-cycle).
template <class OP>
__device__ bool resid_max(const Team& t, const double* x, const double* b, int n, const OP& op,
                          const EngineArgs& a, int& seq, double& out) {
    double s0[1], mx[1] = {0.0};
    for_points(t, n, [&](int i, int j, int k) {
        const Nb o = neighbours(n, i, j, k);
        const double lx = op.apply(o, [&](long q) { return x[q]; });
        mx[0] = fmax(mx[0], fabs(lx + -1.0 * b[o.c]));
    });
    const bool ok = grid_reduce<0, 1>(s0, mx, a, seq);
    out = mx[0];
    return ok;
}

// The programs over operator OP. With the PB operator the solves follow the reference's
// PB branches: conj_grad_pb (plcg.c:169-238, implicit Jacobi whatever the grid's
// preconditioner), verlet_poisson_pb (verlet.c:152-193), and the PB V-cycle with 4
// smoother iterations (MG_SOLVE_SM_PB, grid_multigrid.c:151-177, verlet.c:212-271).
template <class OP>
__device__ void engine_body(const Team& t, const EngineArgs& a, const OP& op, int& result, bool& ok) {
    constexpr bool PB = !std::is_same<OP, LapOp>::value;
    int seq = 0;
    const int n = a.n;
    auto mg_cycle = [&](const double* rhs, double* x, int sm) {
        if constexpr (PB) return vcycle_pb(t, rhs, x, n, sm, a, seq);
        else return vcycle(t, rhs, x, n, sm, a, seq);
    };

    switch (a.prog) {
    case PROG_LAPLACE:
        for_points(t, n, [&](int i, int j, int k) {
            const Nb o = neighbours(n, i, j, k);
            a.out[o.c] = op.apply(o, [&](long q) { return a.u[q]; });
        });
        break;

    case PROG_CG:
    case PROG_PCG:
    case PROG_CG_COARSE: {
        CgSpec s;
        s.n = n; s.b = a.b; s.x0 = a.x0; s.x = a.x; s.r = a.r; s.p0 = a.p0; s.p1 = a.p1; s.Ap = a.Ap;
        s.v = a.v; s.kind = a.prog == PROG_PCG ? a.precond : PC_IMPLICIT;
        s.coarse = a.prog == PROG_CG_COARSE; s.tol = a.tol; s.rtol = a.rtol;
        s.limit = s.coarse ? a.maxit : (long)n * n;
        if constexpr (PB) {
            if (s.coarse) result = cg_run<PC_NONE, true>(t, s, op, a, seq, ok);
            else result = cg_run<PC_IMPLICIT, false>(t, s, op, a, seq, ok);
        } else {
            if (s.coarse) result = cg_run<PC_IMPLICIT, true>(t, s, op, a, seq, ok);
            else if (s.kind == PC_JACOBI) result = cg_run<PC_JACOBI, false>(t, s, op, a, seq, ok);
            else if (s.kind == PC_MG) result = cg_run<PC_MG, false>(t, s, op, a, seq, ok);
            else if (s.kind == PC_SSOR) result = cg_run<PC_SSOR, false>(t, s, op, a, seq, ok);
            else if (s.kind == PC_BLOCKJACOBI) result = cg_run<PC_BLOCKJACOBI, false>(t, s, op, a, seq, ok);
            else result = cg_run<PC_IMPLICIT, false>(t, s, op, a, seq, ok);
        }
        break;
    }

    case PROG_SMOOTH:
        for (int it = 0; it < a.sm && ok; it++) {
            if constexpr (PB) ok = rbgs_pb(t, a.b, a.x, n, op, a);
            else ok = rbgs(t, a.b, a.x, n, a);
        }
        break;

    case PROG_RESTRICT:
        restrict27(t, a.u, a.out, n);
        break;

    case PROG_SSOR:
        ok = ssor_apply(t, a.u, a.out, n, a);
        break;

    case PROG_BLOCKJACOBI:
        ok = bj_apply(t, a.u, a.out, n, a);
        break;

    case PROG_PROLONG:  // n is the coarse size here
        for_points(t, 2 * n, [&](int i, int j, int k) {
            a.out[((long)i * 2 * n + j) * 2 * n + k] = prolong_at(a.u, n, i, j, k);
        });
        break;

    case PROG_MG_APPLY:
        ok = mg_cycle(a.b, a.x, a.sm);
        break;

    case PROG_INIT_FIELD:
    case PROG_LCG_UPDATE: {
        // INIT:   y = 0; phi = c q; CG(b = phi, x0 = y, x = phi)   (grid_lcg.c:100-124)
        // UPDATE: y = c q; CG(b = y, x0 = phi_prev, x = phi)      (grid_lcg.c:126-149)
        const bool init = a.prog == PROG_INIT_FIELD;
        for_points(t, n, [&](int i, int j, int k) {
            const long c = ((long)i * n + j) * n + k;
            const double bq = a.q[c] * a.c;
            if (init) { a.y[c] = 0.0; a.phi_new[c] = bq; }
            else a.y[c] = bq;
        });
        ok = grid_sync(a.bar);
        if (!ok) break;
        CgSpec s;
        s.n = n; s.b = init ? a.phi_new : a.y; s.x0 = init ? a.y : a.phi_old; s.x = a.phi_new;
        s.r = a.r; s.p0 = a.p0; s.p1 = a.p1; s.Ap = a.Ap; s.v = a.v; s.kind = PC_IMPLICIT;
        s.coarse = false; s.tol = a.tol; s.rtol = 0.0; s.limit = (long)n * n;
        result = cg_run<PC_IMPLICIT, false>(t, s, op, a, seq, ok);
        break;
    }

    case PROG_MAZE_LCG:
    case PROG_MAZE_MG:
    case PROG_MG_UPDATE: {
        // phi_new = 2 phi - phi_prev (verlet.c:46-51). MaZe: tmp = A phi_new + c q,
        // the constraint sigma_p (verlet.c:54-55,108-110,174-179). MULTIGRID: tmp = c q.
        const bool maze = a.prog != PROG_MG_UPDATE;
        for_points(t, n, [&](int i, int j, int k) {
            const Nb o = neighbours(n, i, j, k);
            auto ex = [&](long q) { return 2 * a.phi_old[q] - a.phi_prev[q]; };
            const double pc = ex(o.c);
            a.phi_new[o.c] = pc;
            if (maze) a.tmp[o.c] = op.apply(o, ex) + a.c * a.q[o.c];
            else a.tmp[o.c] = a.q[o.c] * a.c;
        });
        ok = grid_sync(a.bar);
        if (!ok) break;
        double* sol = maze ? a.y : a.phi_new;
        if (a.prog == PROG_MAZE_LCG) {
            CgSpec s;
            s.n = n; s.b = a.tmp; s.x0 = a.y; s.x = a.y; s.r = a.r; s.p0 = a.p0; s.p1 = a.p1;
            s.Ap = a.Ap; s.v = a.v; s.kind = PB ? PC_IMPLICIT : a.precond; s.coarse = false; s.tol = a.tol;
            s.rtol = 0.0; s.limit = (long)n * n;
            if (PB || s.kind == PC_IMPLICIT) result = cg_run<PC_IMPLICIT, false>(t, s, op, a, seq, ok);
            else if constexpr (!PB) {
                if (s.kind == PC_JACOBI) result = cg_run<PC_JACOBI, false>(t, s, op, a, seq, ok);
                else if (s.kind == PC_SSOR) result = cg_run<PC_SSOR, false>(t, s, op, a, seq, ok);
                else if (s.kind == PC_BLOCKJACOBI) result = cg_run<PC_BLOCKJACOBI, false>(t, s, op, a, seq, ok);
                else result = cg_run<PC_MG, false>(t, s, op, a, seq, ok);
            }
            if (!ok) break;
        } else {
            // repeat V-cycles until |A sol - tmp|_inf <= tol, at most 1000
            // (grid_multigrid.c:151-206, verlet.c:121-136, 236-262)
            result = -1;
            int it = 0;
            while (it < 1000) {
                ok = mg_cycle(a.tmp, sol, PB ? 4 : 3);
                if (!ok) break;
                double rmax;
                ok = resid_max(t, sol, a.tmp, n, op, a, seq, rmax);
                if (!ok) break;
                it++;
                if (rmax <= a.tol) { result = it; break; }
            }
            if (!ok) break;
        }
        if (maze) {
            for_points(t, n, [&](int i, int j, int k) {
                const long c = ((long)i * n + j) * n + k;
                a.phi_new[c] = a.phi_new[c] + -1.0 * a.y[c];
            });
        }
        break;
    }
    default:
        ok = false;
        break;
    }
}

__global__ void __launch_bounds__(kThreads, kMinBlocksPerSM) engine_kernel(EngineArgs a) {
    const Team t = make_team();
    bool ok = true;
    int result = 0;
    if (a.pb) engine_body(t, a, PbOp{a.ex, a.ey, a.ez, a.dg}, result, ok);
    else engine_body(t, a, LapOp{}, result, ok);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.result[0] = result;
        a.result[1] = ok ? 0 : 1;
    }
}

struct EngineShape {
    int device = -1;
    int blocks = 0;
};
EngineShape g_shape;

void ensure_shape() {
    int dev;
    MZB_CHECK(cudaGetDevice(&dev));
    if (g_shape.device == dev) return;
    int sms = 0, per_sm = 0;
    MZB_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MZB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, engine_kernel, kThreads, 0));
    if (per_sm < 1) fatal("solver engine: kernel cannot be resident on this device");
    g_shape.device = dev;
    g_shape.blocks = sms * (per_sm < kMinBlocksPerSM ? per_sm : kMinBlocksPerSM);
}

}  // namespace

// Gauss-Jordan elimination with partial pivoting on the block's Laplacian (the LU-based
// inverse LAPACK's dgetrf + dgetri give the reference, linalg.c:16-35), in plain FP64 on
// the host; computed on first use and kept.
const std::vector<double>& block_jacobi_inverse() {
    static std::vector<double> inv;
    if (!inv.empty()) return inv;
    const int B = kBlockJacobiB, n = kBlockJacobiB3;
    std::vector<double> m((size_t)n * n, 0.0), x((size_t)n * n, 0.0);
    for (int i = 0; i < B; i++)
        for (int j = 0; j < B; j++)
            for (int k = 0; k < B; k++) {
                const long r = (i * B + j) * B + k;
                m[r * n + r] = -6.0;
                if (i > 0) m[r * n + r - B * B] = 1.0;
                if (i < B - 1) m[r * n + r + B * B] = 1.0;
                if (j > 0) m[r * n + r - B] = 1.0;
                if (j < B - 1) m[r * n + r + B] = 1.0;
                if (k > 0) m[r * n + r - 1] = 1.0;
                if (k < B - 1) m[r * n + r + 1] = 1.0;
            }
    for (long r = 0; r < n; r++) x[r * n + r] = 1.0;
    for (long c = 0; c < n; c++) {
        long piv = c;
        for (long r = c + 1; r < n; r++)
            if (fabs(m[r * n + c]) > fabs(m[piv * n + c])) piv = r;
        if (piv != c)
            for (long q = 0; q < n; q++) {
                std::swap(m[c * n + q], m[piv * n + q]);
                std::swap(x[c * n + q], x[piv * n + q]);
            }
        const double d = m[c * n + c];
        for (long q = 0; q < n; q++) {
            m[c * n + q] /= d;
            x[c * n + q] /= d;
        }
        for (long r = 0; r < n; r++) {
            const double f = m[r * n + c];
            if (r == c || f == 0.0) continue;
            for (long q = 0; q < n; q++) {
                m[r * n + q] -= f * m[c * n + q];
                x[r * n + q] -= f * x[c * n + q];
            }
        }
    }
    inv.swap(x);
    return inv;
}

int engine_grid_blocks() {
    ensure_shape();
    return g_shape.blocks;
}

void engine_launch(const EngineArgs& a, cudaStream_t stream) {
    ensure_shape();
    MZB_CHECK(cudaMemsetAsync(a.bar, 0, sizeof(GridBarrier), stream));
    EngineArgs copy = a;
    void* params[] = {&copy};
    count_launch();
    MZB_CHECK(cudaLaunchCooperativeKernel((const void*)engine_kernel, dim3(g_shape.blocks),
                                          dim3(kThreads), params, 0, stream));
}

}  // namespace mzb
