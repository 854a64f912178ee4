// Shifted-force pair forces -- Tosi-Fumi (Born-Mayer-Huggins), Lennard-Jones and soft-core
// repulsion -- warp per 32 cell-sorted ions (reference: library/src/forces.c:112-337,
// parameters particles.c:181-295). Every potential is summed over both orders of each
// pair and the energy halved, which for the soft-core potential equals the reference's
// sum over i < j with Newton's third law.
//
// Compiled with --fmad=true: this kernel is bound by the FP64 pipe, and its results are
// already ulp-level (exp and inverse powers) rather than bit-level equal to the
// reference, which uses glibc exp/pow.
//
// Layout: ions are sorted by cell (linked cells, particles.cu). Warp w takes the 32
// consecutive ions of block w / split in that order (every lane holds an ion) and the
// w % split-th contiguous chunk of partner cells; partner ions are broadcast loads.
// Partner cells whose minimum-image distance to the bounding box of the warp's ions
// exceeds r_cut = L/2 are skipped (with a 1e-9 relative margin), which removes ~40% of
// the N^2 pair work; pruning is turned off when any coordinate lies outside [0, L).
// 1/r comes from one FP64 rsqrt and r = r2 (1/r); the cutoff is tested on r^2. Partial
// forces per chunk are summed in chunk order.
#include "particles.cuh"

namespace mzb {

constexpr int kTfWarps = 4;

// min-image gap along one axis between the interval [lo, hi] and the cell [c0, c0 + cl]
__device__ __forceinline__ double axis_gap(double lo, double hi, double c0, double cl, double L) {
    double best = 1e300;
#pragma unroll
    for (int s = -1; s <= 1; s++) {
        const double a = c0 + s * L, b = a + cl;
        const double g = fmax(0.0, fmax(a - hi, lo - b));
        best = fmin(best, g);
    }
    return best;
}

// Shifted-force pair force (times 1/r, to be multiplied by the separation vector) and
// pair energy of one pair at r^2 with 1/r = ir, from the type pair's constants t.
template <int POT>
__device__ __forceinline__ void pair_terms(const double* t, double r2, double ir, double& fr, double& vm) {
    const double r = r2 * ir;
    if (POT == POT_TF) {  // forces.c:112-186
        const double a = t[0], b = t[1], c = t[2], d = t[3], sg = t[4], al = t[5], be = t[6];
        const double ir2 = ir * ir, ir6 = ir2 * ir2 * ir2;
        const double ir7 = ir6 * ir, ir8 = ir6 * ir2, ir9 = ir8 * ir;
        const double ex = exp(b * (sg - r));
        const double fm = b * a * ex - 6 * c * ir7 - 8 * d * ir9 - al;
        vm = a * ex - c * ir6 - d * ir8 + al * r + be;
        fr = fm * ir;
    } else if (POT == POT_LJ) {  // forces.c:199-271
        const double sg = t[0], ep = t[1], al = t[2], be = t[3];
        const double s = sg * ir, s2 = s * s, s6 = s2 * s2 * s2, s12 = s6 * s6;
        const double fm = 4 * ep * (12 * s12 - 6 * s6) * ir - al;
        vm = 4 * ep * (s12 - s6) + al * r + be;
        fr = fm * ir;
    } else {  // forces.c:283-337
        const double nu = t[0], d = t[1], B = t[2], al = t[3], be = t[4];
        const double p = pow(d * ir, nu);
        const double fm = B * nu * p * ir - al;
        vm = B * p + al * r + be;
        fr = fm * ir;
    }
}

template <int POT>
__global__ void __launch_bounds__(kTfWarps * 32) k_tf(ParticleDev P) {
    __shared__ double tab[64 * 7];
    for (int x = threadIdx.x; x < P.ntyp * P.ntyp * 7; x += blockDim.x) tab[x] = P.tab[x];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const long gw = (long)blockIdx.x * kTfWarps + (threadIdx.x >> 5);
    const int nblk = (P.np + 31) / 32;
    const long total = (long)nblk * P.tf_split;
    if (gw >= total) return;
    const int blk = (int)(gw / P.tf_split), chunk = (int)(gw % P.tf_split);
    const int cj0 = (int)((long)chunk * P.ncell / P.tf_split);
    const int cj1 = (int)((long)(chunk + 1) * P.ncell / P.tf_split);
    const int nc = P.nc;
    const double L = P.L, invL = 1.0 / L, rcut = P.rcut;
    const double cl = L / nc;
    const double prune2 = rcut * rcut * (1.0 + 1e-9);
    const double rc2 = rcut * rcut;
    const bool prune = P.flags[1] == 0;
    const int ntyp = P.ntyp;

    const int si = blk * 32 + lane;
    const bool valid = si < P.np;
    const int sl = valid ? si : blk * 32;  // invalid lanes mirror lane 0 for the bounding box
    const double xi = P.spos[3 * sl], yi = P.spos[3 * sl + 1], zi = P.spos[3 * sl + 2];
    const int ti = P.stype[sl];
    double lx = xi, hx = xi, ly = yi, hy = yi, lz = zi, hz = zi;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lx = fmin(lx, __shfl_xor_sync(0xffffffffu, lx, o));
        hx = fmax(hx, __shfl_xor_sync(0xffffffffu, hx, o));
        ly = fmin(ly, __shfl_xor_sync(0xffffffffu, ly, o));
        hy = fmax(hy, __shfl_xor_sync(0xffffffffu, hy, o));
        lz = fmin(lz, __shfl_xor_sync(0xffffffffu, lz, o));
        hz = fmax(hz, __shfl_xor_sync(0xffffffffu, hz, o));
    }
    double fx = 0.0, fy = 0.0, fz = 0.0, e_acc = 0.0;
    for (int cj = cj0; cj < cj1; cj++) {
        if (prune) {
            const int cjx = cj / (nc * nc), cjy = (cj / nc) % nc, cjz = cj % nc;
            const double gx = axis_gap(lx, hx, cjx * cl, cl, L), gy = axis_gap(ly, hy, cjy * cl, cl, L);
            const double gz = axis_gap(lz, hz, cjz * cl, cl, L);
            if (gx * gx + gy * gy + gz * gz > prune2) continue;
        }
        const int jb = P.cell_start[cj], je = P.cell_start[cj + 1];
        for (int sj = jb; sj < je; sj++) {
            const double xj = P.spos[3 * sj], yj = P.spos[3 * sj + 1], zj = P.spos[3 * sj + 2];
            const int tj = P.stype[sj];
            if (!valid || sj == si) continue;
            double dx = xi - xj, dy = yi - yj, dz = zi - zj;
            dx -= L * round(dx * invL);
            dy -= L * round(dy * invL);
            dz -= L * round(dz * invL);
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 > rc2) continue;
            double fr, vm;
            pair_terms<POT>(tab + 7 * (ti * ntyp + tj), r2, rsqrt(r2), fr, vm);
            fx += fr * dx;
            fy += fr * dy;
            fz += fr * dz;
            e_acc += vm;
        }
    }
    if (valid) {
        double* o = P.fpart + ((long)chunk * P.np + si) * 3;
        o[0] = fx;
        o[1] = fy;
        o[2] = fz;
    }
    e_acc = warp_sum(e_acc);
    if (lane == 0) P.epart[gw] = e_acc;
}

// Sum the chunk partials in chunk order, scatter back to ion order.
__global__ void k_tf_gather(ParticleDev P) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P.np) return;
    const int s = P.srank[p];
    double f[3] = {0.0, 0.0, 0.0};
    for (int c = 0; c < P.tf_split; c++) {
        const double* o = P.fpart + ((long)c * P.np + s) * 3;
        f[0] += o[0];
        f[1] += o[1];
        f[2] += o[2];
    }
    P.fn[3 * p] = f[0];
    P.fn[3 * p + 1] = f[1];
    P.fn[3 * p + 2] = f[2];
}

__global__ void k_tf_energy(ParticleDev P) {
    const long m = (long)((P.np + 31) / 32) * P.tf_split;
    double v[1] = {0.0};
    for (long x = threadIdx.x; x < m; x += blockDim.x) v[0] += P.epart[x];
    __shared__ double sh[4 * 32];
    block_sum<1>(v, sh);
    if (threadIdx.x == 0) P.red[1] = v[0] / 2;
}

void tf_forces(ParticleDev& P, cudaStream_t s) {
    if (P.np == 0) {
        MZB_CHECK(cudaMemsetAsync(P.red + 1, 0, sizeof(double), s));
        return;
    }
    if (P.ntyp * P.ntyp > 64) fatal("pair forces: more than 8 particle types");
    const long warps = (long)((P.np + 31) / 32) * P.tf_split;
    count_launch();
    const unsigned nb = (unsigned)((warps + kTfWarps - 1) / kTfWarps);
    if (P.pot == POT_LJ)
        k_tf<POT_LJ><<<nb, kTfWarps * 32, 0, s>>>(P);
    else if (P.pot == POT_SC)
        k_tf<POT_SC><<<nb, kTfWarps * 32, 0, s>>>(P);
    else
        k_tf<POT_TF><<<nb, kTfWarps * 32, 0, s>>>(P);
    count_launch();
    k_tf_gather<<<(P.np + 127) / 128, 128, 0, s>>>(P);
    count_launch();
    k_tf_energy<<<1, 1024, 0, s>>>(P);
    MZB_CHECK(cudaGetLastError());
}

}  // namespace mzb
