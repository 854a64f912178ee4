// Poisson-Boltzmann implicit solvent (see pb.cuh). FP64, compiled with --fmad=false.
//
// Coefficients. The reference scales eps_x/y/z and k2 ion by ion (grid_general.c:
// 138-301, a serial loop): a grid point covered by several solvation shells gets their
// factors multiplied in ion order. Here each CTA owns an 8^3 tile of points and streams
// the ions in index order through shared memory, keeping only those whose box
// (+-(floor((r_s+w)/h)+1) points around floor(pos/h), periodic) reaches the tile; every
// thread applies the factors of its point in that order, so the products round exactly
// as the reference's do. pow(x, 2) is x * x (what glibc returns for it); pow(x, 3) is the
// correctly rounded cube, which glibc's pow misses by one ulp in ~0.08 % of inputs.
//
// Forces. particles_compute_forces_pb (particles.c:420-775) walks each ion's box of
// +-(floor((r_s+w)/h)+2) points. Here CTA (slab, ion) takes the points with one x offset,
// each thread sums the terms of its points, and the 9 sums (dielectric boundary, ionic
// boundary, non-polar; x, y, z) are reduced in a fixed order over threads and then over
// slabs: deterministic, within a few ulps of the reference's serial sum.
#include "pb.cuh"

namespace mzb {
namespace {

constexpr int kTile = 8;                          // coefficient tile side
constexpr int kTileThreads = kTile * kTile * kTile;
constexpr int kForceThreads = 256;

// An ion's box: position, solvation radius, shell bounds (r_s +- w)^2, base point
// floor(pos/h) and half-width `range` in points.
struct IonBox {
    double px, py, pz, rs, rp2, rm2;
    int ix, iy, iz, range;
};

__device__ __forceinline__ IonBox ion_box(const double* pos, const double* radii, int p, double h,
                                          double w, int extra) {
    IonBox b;
    b.px = pos[3 * p];
    b.py = pos[3 * p + 1];
    b.pz = pos[3 * p + 2];
    b.rs = radii[p];
    const double a = b.rs + w, c = b.rs - w;
    b.rp2 = a * a;
    b.rm2 = c * c;
    b.range = (int)floor(a / h) + extra;
    b.ix = (int)floor(b.px / h);
    b.iy = (int)floor(b.py / h);
    b.iz = (int)floor(b.pz / h);
    return b;
}

__device__ __forceinline__ int wrapn(int a, int n) {
    a %= n;
    return a < 0 ? a + n : a;
}

// Does the periodic range {base + d : |d| <= range} meet [lo, hi)?
__device__ __forceinline__ bool axis_hits(int base, int range, int lo, int hi, int n) {
    if (2 * range + 1 >= n) return true;
    const int b = wrapn(base, n);
    if (b >= lo && b < hi) return true;
    return wrapn(lo - b, n) <= range || wrapn(b - (hi - 1), n) <= range;
}

// The offsets d (|d| <= range, ascending) with base + d == g (mod n): at most two since
// range < n. Returns their count.
__device__ __forceinline__ int images(int g, int base, int range, int n, int (&d)[2]) {
    int c = 0;
#pragma unroll
    for (int m = -1; m <= 2; m++) {
        const int v = g - base + m * n;
        if (v >= -range && v <= range && c < 2) d[c++] = v;
    }
    return c;
}

// Transition switch -(1/(4 w^3)) a^3 + (3/(4 w^2)) a^2 (grid_general.c:213-216); c1 =
// 1/(4 w^3), c2 = 3/(4 w^2).
__device__ __forceinline__ double pb_switch(double a, double c1, double c2) {
    return -c1 * cube_rn(a) + c2 * (a * a);
}

// One coefficient at squared distance r2 from the ion (grid_general.c:207-222).
__device__ __forceinline__ void pb_scale(double& v, double r2, const IonBox& b, double w, double c1,
                                         double c2) {
    if (r2 >= b.rp2) return;
    if (r2 > b.rm2) v = v * pb_switch(sqrt(r2) - b.rs + w, c1, c2);
    else v = 0.0;
}

struct CoefArgs {
    int n;
    double h, w, base, kbar2, eps_int;
    double *ex, *ey, *ez, *k2;
};

__global__ void __launch_bounds__(kTileThreads) k_pb_coefficients(CoefArgs A, const double* pos,
                                                                  const double* radii, int np) {
    __shared__ IonBox cand[kTileThreads];
    __shared__ int wcount[kTileThreads / 32];
    const int n = A.n, nt = (n + kTile - 1) / kTile;
    int tb = blockIdx.x;
    const int tz = tb % nt;
    tb /= nt;
    const int ty = tb % nt, tx = tb / nt;
    const int x0 = tx * kTile, y0 = ty * kTile, z0 = tz * kTile;
    const int x1 = min(x0 + kTile, n), y1 = min(y0 + kTile, n), z1 = min(z0 + kTile, n);
    const int gi = x0 + (threadIdx.x >> 6), gj = y0 + ((threadIdx.x >> 3) & 7), gk = z0 + (threadIdx.x & 7);
    const bool mine = gi < n && gj < n && gk < n;
    const double h = A.h, w = A.w, w2 = w * w, w3 = w2 * w, hd2 = h / 2.0;
    const double c1 = 1 / (4 * w3), c2 = 3 / (4 * w2);
    double vx = A.base, vy = A.base, vz = A.base, vk = A.kbar2;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;

    for (int p0 = 0; p0 < np; p0 += kTileThreads) {
        const int p = p0 + threadIdx.x;
        bool hit = false;
        IonBox b;
        if (p < np) {
            b = ion_box(pos, radii, p, h, w, 1);
            hit = axis_hits(b.ix, b.range, x0, x1, n) && axis_hits(b.iy, b.range, y0, y1, n) &&
                  axis_hits(b.iz, b.range, z0, z1, n);
        }
        // keep the hits in ion order: warp-ballot ranks plus the counts of earlier warps
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (lane == 0) wcount[wid] = __popc(m);
        __syncthreads();
        int off = 0, total = 0;
        for (int q = 0; q < kTileThreads / 32; q++) {
            const int c = wcount[q];
            off += q < wid ? c : 0;
            total += c;
        }
        if (hit) cand[off + __popc(m & ((1u << lane) - 1u))] = b;
        __syncthreads();
        if (mine) {
            for (int c = 0; c < total; c++) {
                const IonBox& e = cand[c];
                int di[2], dj[2], dk[2];
                const int ni = images(gi, e.ix, e.range, n, di);
                const int nj = images(gj, e.iy, e.range, n, dj);
                const int nk = images(gk, e.iz, e.range, n, dk);
                for (int a = 0; a < ni; a++) {
                    const double dx = e.px - (e.ix + di[a]) * h, dx2 = dx * dx, ax = dx - hd2;
                    for (int bq = 0; bq < nj; bq++) {
                        const double dy = e.py - (e.iy + dj[bq]) * h, dy2 = dy * dy, ay = dy - hd2;
                        for (int cq = 0; cq < nk; cq++) {
                            const double dz = e.pz - (e.iz + dk[cq]) * h, dz2 = dz * dz, az = dz - hd2;
                            pb_scale(vk, dx2 + dy2 + dz2, e, w, c1, c2);
                            pb_scale(vx, ax * ax + dy2 + dz2, e, w, c1, c2);
                            pb_scale(vy, dx2 + ay * ay + dz2, e, w, c1, c2);
                            pb_scale(vz, dx2 + dy2 + az * az, e, w, c1, c2);
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
    if (mine) {
        const long c = ((long)gi * n + gj) * n + gk;
        A.ex[c] = vx + A.eps_int;
        A.ey[c] = vy + A.eps_int;
        A.ez[c] = vz + A.eps_int;
        A.k2[c] = vk;
    }
}

// dg_c = ex_c + ex_{x-1} + ey_c + ey_{y-1} + ez_c + ez_{z-1} + k2_c (laplace.c:131-140)
__global__ void k_pb_diag(int n, const double* ex, const double* ey, const double* ez, const double* k2,
                          double* dg) {
    const long m = (long)n * n * n;
    for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < m; c += (long)gridDim.x * blockDim.x) {
        const int i = (int)(c / ((long)n * n)), j = (int)((c / n) % n), k = (int)(c % n);
        const long xm = ((long)wrap_dec(i, n) * n + j) * n + k;
        const long ym = ((long)i * n + wrap_dec(j, n)) * n + k;
        const long zm = ((long)i * n + j) * n + wrap_dec(k, n);
        double d = ex[c] + ex[xm];
        d = d + ey[c];
        d = d + ey[ym];
        d = d + ez[c];
        d = d + ez[zm];
        dg[c] = d + k2[c];
    }
}

// Coarse coefficients (multigrid_pb.c:330-527, one process: n_start = 0): faces are the
// mean of the 2x2 fine faces of their axis; k2 the mean of the fine cube at
// i in {2I+1, 2I+2}, j in {2J, 2J+1}, k in {2K, 2K+1}.
__global__ void k_pb_restrict(int n, const double* ex, const double* ey, const double* ez, const double* k2,
                              double* cex, double* cey, double* cez, double* ck2) {
    const int nc = n / 2;
    const long mc = (long)nc * nc * nc;
    for (long C = blockIdx.x * (long)blockDim.x + threadIdx.x; C < mc; C += (long)gridDim.x * blockDim.x) {
        const int I = (int)(C / ((long)nc * nc)), J = (int)((C / nc) % nc), K = (int)(C % nc);
        const int i = 2 * I, j = 2 * J, k = 2 * K;
        const int i1 = wrap_inc(i, n), j1 = wrap_inc(j, n), k1 = wrap_inc(k, n);
        auto at = [&](const double* a, int x, int y, int z) { return a[((long)x * n + y) * n + z]; };
        cex[C] = (at(ex, i, j, k) + at(ex, i, j, k1) + at(ex, i, j1, k) + at(ex, i, j1, k1)) * 0.25;
        cey[C] = (at(ey, i, j, k) + at(ey, i, j, k1) + at(ey, i1, j, k) + at(ey, i1, j, k1)) * 0.25;
        cez[C] = (at(ez, i, j, k) + at(ez, i1, j, k) + at(ez, i, j1, k) + at(ez, i1, j1, k)) * 0.25;
        const int a0 = i + 1, a1 = wrap_inc(a0, n);
        const double s = at(k2, a0, j, k) + at(k2, a0, j, k1) + at(k2, a0, j1, k) + at(k2, a0, j1, k1) +
                         at(k2, a1, j, k) + at(k2, a1, j, k1) + at(k2, a1, j1, k) + at(k2, a1, j1, k1);
        ck2[C] = (1.0 / 8.0) * s;
    }
}

// d(switch)/da / switch (particles.c:407-418)
__device__ __forceinline__ double h_ratio(double rad, double w2, double w3) {
    const double r2 = rad * rad;
    return (-(3 / (4 * w3)) * r2 + (3 / (2 * w2)) * rad) / (-(1 / (4 * w3)) * cube_rn(rad) + (3 / (4 * w2)) * r2);
}

struct ForceArgs {
    int n, np, slabs, nonpolar;
    double h, w, eps_int;
    const double *phi, *ex, *ey, *ez, *k2, *pos, *radii;
    double* part;
};

__global__ void __launch_bounds__(kForceThreads) k_pb_forces(ForceArgs A) {
    __shared__ double sh[9][kForceThreads / 32];
    const int p = blockIdx.y, slab = blockIdx.x, n = A.n;
    const double h = A.h, w = A.w, w2 = w * w, w3 = w2 * w, hd2 = h / 2.0, ei = A.eps_int;
    const IonBox b = ion_box(A.pos, A.radii, p, h, w, 2);
    const int R = b.range, side = 2 * R + 1;
    double acc[9];
#pragma unroll
    for (int q = 0; q < 9; q++) acc[q] = 0.0;
    if (slab < side) {
        const int ii = b.ix + slab - R;
        const double dx = b.px - ii * h, dx2 = dx * dx;
        const int i = wrapn(ii, n), ip = wrap_inc(i, n), im = wrap_dec(i, n);
        for (int q = threadIdx.x; q < side * side; q += blockDim.x) {
            const int jj = b.iy + q / side - R, kk = b.iz + q % side - R;
            const double dy = b.py - jj * h, dy2 = dy * dy;
            const double dz = b.pz - kk * h, dz2 = dz * dz;
            const int j = wrapn(jj, n), k = wrapn(kk, n);
            const int jp = wrap_inc(j, n), jm = wrap_dec(j, n), kp = wrap_inc(k, n), km = wrap_dec(k, n);
            auto idx = [&](int x, int y, int z) { return ((long)x * n + y) * n + z; };
            const long c = idx(i, j, k);
            const double exc = A.ex[c], eyc = A.ey[c], ezc = A.ez[c];
            const double exb = A.ex[idx(im, j, k)], eyb = A.ey[idx(i, jm, k)], ezb = A.ez[idx(i, j, km)];
            const double ddx = exc - exb, ddy = eyc - eyb, ddz = ezc - ezb;
            const double dn = sqrt(ddx * ddx + ddy * ddy + ddz * ddz) / h;
            const double ig = (dn > 0.0) ? 1.0 / dn : 0.0;
            const double pc = A.phi[c];
            double r2 = dx2 + dy2 + dz2;
            if (r2 < b.rp2 && r2 > b.rm2) {  // ionic boundary at the point
                const double r1 = sqrt(r2) + 1E-12;
                const double hr = h_ratio(r1 - b.rs + w, w2, w3);
                const double a = A.k2[c] * pc * pc * hr;
                acc[3] += a * (dx / r1);
                acc[4] += a * (dy / r1);
                acc[5] += a * (dz / r1);
            }
            // faces x-, x+, y-, y+, z-, z+ (particles.c:579-765)
#pragma unroll
            for (int f = 0; f < 6; f++) {
                const int axis = f >> 1;
                const bool fwd = f & 1;
                const double o = fwd ? -hd2 : hd2;
                double ux = dx, uy = dy, uz = dz, g;
                if (axis == 0) { ux = dx + o; r2 = ux * ux + dy2 + dz2; g = ig * ddx; }
                else if (axis == 1) { uy = dy + o; r2 = dx2 + uy * uy + dz2; g = ig * ddy; }
                else { uz = dz + o; r2 = dx2 + dy2 + uz * uz; g = ig * ddz; }
                if (!(r2 < b.rp2 && r2 > b.rm2)) continue;
                const double r1 = sqrt(r2) + 1E-12;
                const double rx = ux / r1, ry = uy / r1, rz = uz / r1;
                const double hr = h_ratio(r1 - b.rs + w, w2, w3);
                const double ef = axis == 0 ? (fwd ? exc : exb) : axis == 1 ? (fwd ? eyc : eyb) : (fwd ? ezc : ezb);
                const long nb = axis == 0 ? idx(fwd ? ip : im, j, k)
                                          : axis == 1 ? idx(i, fwd ? jp : jm, k) : idx(i, j, fwd ? kp : km);
                const double a = (ef - ei) * hr;
                const double t = a * (A.phi[nb] - pc) * pc;
                acc[0] -= t * rx;
                acc[1] -= t * ry;
                acc[2] -= t * rz;
                if (A.nonpolar) {
                    const double ag = a * g;
                    if (fwd) { acc[6] += ag * rx; acc[7] += ag * ry; acc[8] += ag * rz; }
                    else { acc[6] -= ag * rx; acc[7] -= ag * ry; acc[8] -= ag * rz; }
                }
            }
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 9; q++) {
        const double v = warp_sum(acc[q]);
        if (lane == 0) sh[q][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 9) {
        double s = 0.0;
        for (int q = 0; q < kForceThreads / 32; q++) s += sh[threadIdx.x][q];
        A.part[((long)p * A.slabs + slab) * 9 + threadIdx.x] = s;
    }
}

// Sum each ion's slab partials in slab order and scale (particles.c:770-774).
__global__ void k_pb_forces_final(int np, int slabs, double cdb, double cnp, const double* part, double* fdb,
                                  double* fib, double* fnp) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= np * 9) return;
    const int p = t / 9, q = t % 9;
    double s = 0.0;
    for (int sl = 0; sl < slabs; sl++) s += part[((long)p * slabs + sl) * 9 + q];
    const int d = q % 3;
    if (q < 3) fdb[3 * p + d] = s * cdb;
    else if (q < 6) fib[3 * p + d] = s * cdb;
    else fnp[3 * p + d] = s * cnp;
}

int grid_blocks(long m) {
    const long b = (m + 255) / 256;
    return (int)(b < 148 * 16 ? (b < 1 ? 1 : b) : 148 * 16);
}

}  // namespace

void pb_derive(const PbGrid& G, cudaStream_t s) {
    const int n = G.n;
    const long m = (long)n * n * n;
    count_launch();
    k_pb_diag<<<grid_blocks(m), 256, 0, s>>>(n, G.ex, G.ey, G.ez, G.k2, G.dg);
    MZB_CHECK(cudaGetLastError());
    if (G.cex) {
        const int nc = n / 2;
        const long mc = (long)nc * nc * nc;
        count_launch();
        k_pb_restrict<<<grid_blocks(mc), 256, 0, s>>>(n, G.ex, G.ey, G.ez, G.k2, G.cex, G.cey, G.cez, G.ck2);
        count_launch();
        k_pb_diag<<<grid_blocks(mc), 256, 0, s>>>(nc, G.cex, G.cey, G.cez, G.ck2, G.cdg);
        MZB_CHECK(cudaGetLastError());
    }
}

void pb_update_coefficients(const PbGrid& G, const double* pos, const double* radii, int np,
                            cudaStream_t s) {
    CoefArgs A;
    A.n = G.n;
    A.h = G.h;
    A.w = G.w;
    A.base = G.eps_s - G.eps_int;
    A.kbar2 = G.kbar2;
    A.eps_int = G.eps_int;
    A.ex = G.ex; A.ey = G.ey; A.ez = G.ez; A.k2 = G.k2;
    const int nt = (G.n + kTile - 1) / kTile;
    count_launch();
    k_pb_coefficients<<<nt * nt * nt, kTileThreads, 0, s>>>(A, pos, radii, np);
    MZB_CHECK(cudaGetLastError());
    pb_derive(G, s);
}

void pb_forces(const PbGrid& G, const double* phi, const double* pos, const double* radii, int np,
               int range_max, double cdb, double cnp, double* part, double* fdb, double* fib,
               double* fnp, cudaStream_t s) {
    if (np == 0) return;
    ForceArgs A;
    A.n = G.n;
    A.np = np;
    A.slabs = 2 * range_max + 1;
    A.nonpolar = G.nonpolar;
    A.h = G.h;
    A.w = G.w;
    A.eps_int = G.eps_int;
    A.phi = phi; A.ex = G.ex; A.ey = G.ey; A.ez = G.ez; A.k2 = G.k2; A.pos = pos; A.radii = radii;
    A.part = part;
    count_launch();
    k_pb_forces<<<dim3(A.slabs, np), kForceThreads, 0, s>>>(A);
    count_launch();
    k_pb_forces_final<<<(np * 9 + 255) / 256, 256, 0, s>>>(np, A.slabs, cdb, cnp, part, fdb, fib, fnp);
    MZB_CHECK(cudaGetLastError());
}

}  // namespace mzb
