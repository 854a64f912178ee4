// Shifted-force pair forces -- Tosi-Fumi (Born-Mayer-Huggins), Lennard-Jones and soft-core
// repulsion (reference: library/src/forces.c:112-337, parameters particles.c:181-295). The
// reference sums every potential over both orders of each pair and halves the energy;
// here each pair inside r_cut = L/2 is evaluated once and its force applied to both ions
// with opposite signs (for the soft-core potential this is the reference's own i < j
// loop with Newton's third law).
//
// Compiled with --fmad=true: this kernel is bound by the FP64 pipe, and its results are
// already ulp-level (exp and inverse powers) rather than bit-level equal to the
// reference, which uses glibc exp/pow.
//
// Layout. Ions are sorted by linked cell (particles.cu), cut into blocks of 32 and the
// blocks into super-blocks of 8 (256 ions). A CTA of 8 warps takes one super-block pair
// (SI, SJ) of a half shell (SJ = SI + d, d = 0 .. nsb/2, the middle distance only once):
// warp w owns block I = 8 SI + w -- one ion per lane, its forces in registers -- and
// walks the J blocks of SJ; in step s (0..15) lane l pairs its ion with ions (l + s) and
// (l + s + 16) mod 32 of the J block, two independent chains, so the 32 lanes touch 32
// distinct J ions at a time and add the reactions into a warp-private shared array
// (structure of arrays, conflict-free) without atomics, with a __syncwarp between the two
// halves. On the diagonal super-tile each unordered block pair is taken once (and each
// pair inside a block once, 16 steps of one partner). A tile whose bounding
// boxes are farther apart than r_cut (minimum image, 1e-9 relative margin) is skipped;
// pruning is off when a coordinate lies outside [0, L). Inside a tile, a step in which no
// lane's two partners lie inside r_cut skips the pair terms (a warp vote). 1/r is an FP32
// seed refined by two FP64 Newton steps; types sit in the shared position arrays as integer
// bits; the pair-constant rows have an odd stride (no bank conflicts between type pairs).
//
// Determinism. Registers and warp arrays accumulate in step order; the warps' J partials
// are summed in warp order; each ion's force is the sum of its super-tile partials in a
// fixed order (k_tf_gather over a host-built list), the energy the sum of the CTAs'
// energies in CTA order.
#include <algorithm>
#include <vector>

#include "particles.cuh"

namespace mzb {

constexpr int kTfSb = 8;                  // blocks of 32 ions per super-block
constexpr int kTfThreads = kTfSb * 32;    // one warp per I block of a super-block
// Pair-constant table in shared memory, up to 8 types, one row of kTfTabStride doubles per
// type pair: the odd stride puts the rows a warp reads at once (lanes of different type
// pairs) on different banks.
constexpr int kTfTabStride = kPairConsts + 1;
constexpr int kTfTab = 64 * kTfTabStride;
constexpr size_t kTfSmem =
    sizeof(double) * (kTfTab + 2 * kTfSb * 32 * 4 + kTfSb * kTfSb * 32 * 3);

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
        const double ex = r2 < t[7] ? exp(b * (sg - r)) : 0.0;  // negligible beyond (tf_exp_r2_limit)
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

// Bounding box of each block of 32 cell-ordered ions: [lo x, lo y, lo z, hi x, hi y, hi z].
__device__ __forceinline__ void k_tf_boxes_body(const ParticleDev& P, int bx) {
    const int lane = threadIdx.x & 31;
    const int b = (int)((bx * (long)blockDim.x + threadIdx.x) >> 5);
    const int nblk = (P.np + 31) / 32;
    if (b >= nblk) return;
    const int s = b * 32 + lane < P.np ? b * 32 + lane : b * 32;  // idle lanes mirror lane 0
    double lo[3], hi[3];
#pragma unroll
    for (int d = 0; d < 3; d++) lo[d] = hi[d] = P.spos[3 * s + d];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int d = 0; d < 3; d++) {
            lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
            hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
        }
    if (lane < 3) {
        P.tf_box[6 * b + lane] = lo[lane];
        P.tf_box[6 * b + 3 + lane] = hi[lane];
    }
}
__global__ void k_tf_boxes(ParticleDev P) { k_tf_boxes_body(P, blockIdx.x); }

// The ion type stored in a double slot of the shared position arrays as its integer bits
// (read back without a conversion).
__device__ __forceinline__ double type_bits(int t) { return __longlong_as_double((long long)t); }
__device__ __forceinline__ int type_of(double v) { return (int)__double_as_longlong(v); }

// One pair (i, partner j at x, y, z of type tj) for the lane's ion: whether it is inside
// r_cut (and both ions exist), and its force times the separation and energy.
// 1/sqrt(x) for x in the range of squared pair distances (normal FP32 numbers): an FP32
// seed (relative error below 2^-22) refined by two Newton-Raphson steps for x^(-1/2),
// y <- y (3/2 - x y^2 / 2), each of which squares the relative error, so the result is
// within a few ulp of the FP64 value.
__device__ __forceinline__ double rsqrt_nr(double x) {
    double y = (double)rsqrtf((float)x);
    const double h = 0.5 * x;
    y = y * fma(-h * y, y, 1.5);
    y = y * fma(-h * y, y, 1.5);
    return y;
}

struct PairSep {
    double dx, dy, dz, r2;
    bool in;
};
__device__ __forceinline__ PairSep pair_sep(double L, double invL, double rc2, double xi, double yi, double zi, int ti,
                                            double xj, double yj, double zj, int tj) {
    PairSep p;
    p.dx = xi - xj;
    p.dy = yi - yj;
    p.dz = zi - zj;
    p.dx -= L * round(p.dx * invL);
    p.dy -= L * round(p.dy * invL);
    p.dz -= L * round(p.dz * invL);
    p.r2 = p.dx * p.dx + p.dy * p.dy + p.dz * p.dz;
    p.in = ti >= 0 && tj >= 0 && p.r2 <= rc2;
    return p;
}
template <int POT>
__device__ __forceinline__ void pair_force(const double* tab, int ntyp, double rc2, int ti, int tj, const PairSep& p,
                                           double& ax, double& ay, double& az, double& vm) {
    const double r2s = p.in ? p.r2 : rc2;  // a harmless value for lanes whose pair is not taken
    double fr;
    pair_terms<POT>(tab + kTfTabStride * ((p.in ? ti : 0) * ntyp + (p.in ? tj : 0)), r2s, rsqrt_nr(r2s), fr, vm);
    ax = fr * p.dx;
    ay = fr * p.dy;
    az = fr * p.dz;
}
template <int POT>
__device__ __forceinline__ bool pair_eval(const double* tab, int ntyp, double L, double invL, double rc2, double xi,
                                          double yi, double zi, int ti, double xj, double yj, double zj, int tj,
                                          double& ax, double& ay, double& az, double& vm) {
    const PairSep p = pair_sep(L, invL, rc2, xi, yi, zi, ti, xj, yj, zj, tj);
    pair_force<POT>(tab, ntyp, rc2, ti, tj, p, ax, ay, az, vm);
    return p.in;
}

template <int POT>
__device__ __forceinline__ void k_tf_body(const ParticleDev& P, int bx) {
    extern __shared__ double sm[];
    double* tab = sm;                              // [64][kTfTabStride]
    double* ipos = tab + kTfTab;                   // [4][256]: x, y, z, type (structure of arrays)
    double* jpos = ipos + kTfSb * 32 * 4;          // [4][256]
    double* fjw = jpos + kTfSb * 32 * 4;           // [8 warps][8 J blocks][3][32]
    constexpr int NQ = kTfSb * 32;
    const int st = bx;
    const int SI = P.tf_st[2 * st], SJ = P.tf_st[2 * st + 1];
    const bool diag = SI == SJ;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int np = P.np, nblk = (np + 31) / 32, ntyp = P.ntyp;
    const double L = P.L, invL = 1.0 / L, rc2 = P.rcut * P.rcut;
    const double prune2 = rc2 * (1.0 + 1e-9);
    const bool prune = P.flags[1] == 0;

    for (int x = threadIdx.x; x < ntyp * ntyp * kPairConsts; x += blockDim.x)
        tab[(x / kPairConsts) * kTfTabStride + x % kPairConsts] = P.tab[x];
    for (int q = threadIdx.x; q < NQ; q += blockDim.x) {
        const int gi = SI * NQ + q, gj = SJ * NQ + q;
        const bool vi = gi < np, vj = gj < np;
        ipos[q] = vi ? P.spos[3 * gi] : 0.0;
        ipos[NQ + q] = vi ? P.spos[3 * gi + 1] : 0.0;
        ipos[2 * NQ + q] = vi ? P.spos[3 * gi + 2] : 0.0;
        ipos[3 * NQ + q] = type_bits(vi ? P.stype[gi] : -1);
        jpos[q] = vj ? P.spos[3 * gj] : 0.0;
        jpos[NQ + q] = vj ? P.spos[3 * gj + 1] : 0.0;
        jpos[2 * NQ + q] = vj ? P.spos[3 * gj + 2] : 0.0;
        jpos[3 * NQ + q] = type_bits(vj ? P.stype[gj] : -1);
    }
    for (int x = threadIdx.x; x < kTfSb * kTfSb * 32 * 3; x += blockDim.x) fjw[x] = 0.0;
    __syncthreads();

    double fx = 0.0, fy = 0.0, fz = 0.0, e_acc = 0.0;
    const int I = SI * kTfSb + w;
    if (I < nblk) {
        const int me = w * 32 + lane;
        const double xi = ipos[me], yi = ipos[NQ + me], zi = ipos[2 * NQ + me];
        const int ti = type_of(ipos[3 * NQ + me]);  // -1: no ion in this lane
        const double* bI = P.tf_box + 6 * I;
        for (int t = 0; t < kTfSb; t++) {
            const int d = (t - w) & (kTfSb - 1);
            if (diag && (d > kTfSb / 2 || (d == kTfSb / 2 && w >= kTfSb / 2))) continue;
            const int J = SJ * kTfSb + t;
            if (J >= nblk) continue;
            const bool self = diag && d == 0;
            if (prune && !self) {
                const double* bJ = P.tf_box + 6 * J;
                const double gx = axis_gap(bI[0], bI[3], bJ[0], bJ[3] - bJ[0], L);
                const double gy = axis_gap(bI[1], bI[4], bJ[1], bJ[4] - bJ[1], L);
                const double gz = axis_gap(bI[2], bI[5], bJ[2], bJ[5] - bJ[2], L);
                if (gx * gx + gy * gy + gz * gz > prune2) continue;
            }
            const double* jx = jpos + t * 32;
            const double* jy = jx + NQ;
            const double* jz = jx + 2 * NQ;
            const double* jt = jx + 3 * NQ;
            double* fjx = fjw + (w * kTfSb + t) * 3 * 32;
            double* fjy = fjx + 32;
            double* fjz = fjx + 64;
            if (self) {
                // partners (l + s) mod 32 for s = 1..16, the last step by half the lanes, so
                // every pair inside the block comes once
                for (int s = 1; s <= 16; s++) {
                    const int jj = (lane + s) & 31;
                    double ax, ay, az, vm;
                    const bool in = pair_eval<POT>(tab, ntyp, L, invL, rc2, xi, yi, zi, ti, jx[jj], jy[jj], jz[jj],
                                                   type_of(jt[jj]), ax, ay, az, vm);
                    if (in && !(s == 16 && lane >= 16)) {
                        fx += ax;
                        fy += ay;
                        fz += az;
                        fjx[jj] -= ax;
                        fjy[jj] -= ay;
                        fjz[jj] -= az;
                        e_acc += vm;
                    }
                    __syncwarp();
                }
                continue;
            }
            // two partners per step, (l + s) and (l + s + 16) mod 32, as two independent
            // chains; their reactions go in one after the other (each a permutation of the
            // 32 entries)
            for (int s = 0; s < 16; s++) {
                const int ja = (lane + s) & 31, jb = (lane + s + 16) & 31;
                double ax, ay, az, va, bx, by, bz, vb;
                const int tja = type_of(jt[ja]), tjb = type_of(jt[jb]);
                const PairSep pa = pair_sep(L, invL, rc2, xi, yi, zi, ti, jx[ja], jy[ja], jz[ja], tja);
                const PairSep pb = pair_sep(L, invL, rc2, xi, yi, zi, ti, jx[jb], jy[jb], jz[jb], tjb);
                if (!__any_sync(0xffffffffu, pa.in || pb.in)) continue;  // no pair of this step inside r_cut
                pair_force<POT>(tab, ntyp, rc2, ti, tja, pa, ax, ay, az, va);
                pair_force<POT>(tab, ntyp, rc2, ti, tjb, pb, bx, by, bz, vb);
                const bool ina = pa.in, inb = pb.in;
                if (ina) {
                    fx += ax;
                    fy += ay;
                    fz += az;
                    fjx[ja] -= ax;
                    fjy[ja] -= ay;
                    fjz[ja] -= az;
                    e_acc += va;
                }
                __syncwarp();
                if (inb) {
                    fx += bx;
                    fy += by;
                    fz += bz;
                    fjx[jb] -= bx;
                    fjy[jb] -= by;
                    fjz[jb] -= bz;
                    e_acc += vb;
                }
                __syncwarp();
            }
        }
    }
    // I side: this warp's block; J side: the warps' arrays summed in warp order
    double* out = P.fpart + (size_t)st * 2 * kTfSb * 32 * 3;
    if (I < nblk) {
        double* o = out + (w * 32 + lane) * 3;
        o[0] = fx;
        o[1] = fy;
        o[2] = fz;
    }
    __shared__ double esh[kTfSb];
    e_acc = warp_sum(e_acc);
    if (lane == 0) esh[w] = e_acc;
    __syncthreads();
    for (int x = threadIdx.x; x < kTfSb * 32 * 3; x += blockDim.x) {
        const int t = x / 96, jj = (x / 3) % 32, dd = x % 3;  // out layout [J block][32][3]
        const int y = (t * 3 + dd) * 32 + jj;                  // warp arrays [J block][3][32]
        double v = 0.0;
        for (int q = 0; q < kTfSb; q++) v += fjw[q * kTfSb * 32 * 3 + y];
        out[kTfSb * 32 * 3 + x] = v;
    }
    if (threadIdx.x == 0) {
        double e = 0.0;
        for (int q = 0; q < kTfSb; q++) e += esh[q];
        P.epart[st] = e;
    }
}
template <int POT>
__global__ void __launch_bounds__(kTfThreads, 3) k_tf(ParticleDev P) { k_tf_body<POT>(P, blockIdx.x); }

// Each ion's force: its super-tile partials in list order, scattered back to ion order.
// A warp per block of 32 cell-ordered ions: the block's list is walked once for all 32
// lanes (one ion each), whose partials lie side by side.
__device__ __forceinline__ void k_tf_gather_body(const ParticleDev& P, int bx) {
    const int b = (int)((bx * (long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (b >= (P.np + 31) / 32) return;
    double f[3] = {0.0, 0.0, 0.0};
    const int e1 = P.tf_gstart[b + 1];
#pragma unroll 4
    for (int e = P.tf_gstart[b]; e < e1; e++) {
        const int ent = P.tf_gent[e];
        const int st = ent >> 4, side = (ent >> 3) & 1, slot = ent & 7;
        const double* o = P.fpart + (((size_t)st * 2 + side) * kTfSb + slot) * 32 * 3 + lane * 3;
        f[0] += o[0];
        f[1] += o[1];
        f[2] += o[2];
    }
    const int s = b * 32 + lane;
    if (s >= P.np) return;
    const int p = P.cell_ions[s];
    P.fn[3 * p] = f[0];
    P.fn[3 * p + 1] = f[1];
    P.fn[3 * p + 2] = f[2];
}
__global__ void k_tf_gather(ParticleDev P) { k_tf_gather_body(P, blockIdx.x); }

__device__ __forceinline__ void k_tf_energy_body(const ParticleDev& P, int bx) {
    double v[1] = {0.0};
    for (int x = threadIdx.x; x < P.tf_nst; x += blockDim.x) v[0] += P.epart[x];
    __shared__ double sh[4 * 32];
    block_sum<1>(v, sh);
    if (threadIdx.x == 0) P.red[1] = v[0];
}
__global__ void k_tf_energy(ParticleDev P) { k_tf_energy_body(P, blockIdx.x); }

void tf_plan(ParticleDev& P) {
    dev_free(P.tf_st);
    dev_free(P.tf_gstart);
    dev_free(P.tf_gent);
    dev_free(P.tf_box);
    dev_free(P.fpart);
    dev_free(P.epart);
    const int nblk = (P.np + 31) / 32 > 0 ? (P.np + 31) / 32 : 1;
    const int nsb = (nblk + kTfSb - 1) / kTfSb;
    std::vector<int> st;
    for (int si = 0; si < nsb; si++) {
        st.push_back(si);
        st.push_back(si);
        for (int d = 1; 2 * d <= nsb; d++) {
            if (2 * d == nsb && si >= nsb / 2) continue;  // the middle distance once
            st.push_back(si);
            st.push_back((si + d) % nsb);
        }
    }
    P.tf_nst = (int)st.size() / 2;
    std::vector<std::vector<int>> lists(nblk);
    for (int k = 0; k < P.tf_nst; k++)
        for (int side = 0; side < 2; side++)
            for (int slot = 0; slot < kTfSb; slot++) {
                const int b = st[2 * k + side] * kTfSb + slot;
                if (b < nblk) lists[b].push_back((k << 4) | (side << 3) | slot);
            }
    std::vector<int> gstart(nblk + 1, 0), gent;
    for (int b = 0; b < nblk; b++) {
        gent.insert(gent.end(), lists[b].begin(), lists[b].end());
        gstart[b + 1] = (int)gent.size();
    }
    auto up = [](void** d, const void* h, size_t bytes) {
        *d = dev_alloc(bytes);
        MZB_CHECK(cudaMemcpy(*d, h, bytes, cudaMemcpyHostToDevice));
        MZB_CHECK(cudaStreamSynchronize(cudaStreamLegacy));  // landed before any later kernel
    };
    up((void**)&P.tf_st, st.data(), sizeof(int) * st.size());
    up((void**)&P.tf_gstart, gstart.data(), sizeof(int) * gstart.size());
    up((void**)&P.tf_gent, gent.data(), sizeof(int) * gent.size());
    P.tf_box = static_cast<double*>(dev_alloc(sizeof(double) * 6 * nblk));
    P.fpart = static_cast<double*>(dev_alloc(sizeof(double) * (size_t)P.tf_nst * 2 * kTfSb * 32 * 3));
    P.epart = static_cast<double*>(dev_alloc(sizeof(double) * P.tf_nst));
    static unsigned long long attr_done = 0;  // devices whose kernels allow kTfSmem
    int dev = 0;
    MZB_CHECK(cudaGetDevice(&dev));
    if (!(attr_done >> (dev & 63) & 1ull)) {
        MZB_CHECK(cudaFuncSetAttribute(k_tf<POT_TF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTfSmem));
        MZB_CHECK(cudaFuncSetAttribute(k_tf<POT_LJ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTfSmem));
        MZB_CHECK(cudaFuncSetAttribute(k_tf<POT_SC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTfSmem));
        attr_done |= 1ull << (dev & 63);
    }
}

void tf_forces(ParticleDev& P, cudaStream_t s) {
    if (P.np == 0) {
        MZB_CHECK(cudaMemsetAsync(P.red + 1, 0, sizeof(double), s));
        return;
    }
    if (P.ntyp * P.ntyp > 64) fatal("pair forces: more than 8 particle types");
    if (!P.tf_st) fatal("pair forces: no plan (tf_plan)");
    const int nblk = (P.np + 31) / 32;
    count_launch();
    k_tf_boxes<<<(nblk * 32 + 255) / 256, 256, 0, s>>>(P);
    count_launch();
    if (P.pot == POT_LJ)
        k_tf<POT_LJ><<<P.tf_nst, kTfThreads, kTfSmem, s>>>(P);
    else if (P.pot == POT_SC)
        k_tf<POT_SC><<<P.tf_nst, kTfThreads, kTfSmem, s>>>(P);
    else
        k_tf<POT_TF><<<P.tf_nst, kTfThreads, kTfSmem, s>>>(P);
    count_launch();
    k_tf_gather<<<(nblk * 32 + 127) / 128, 128, 0, s>>>(P);
    count_launch();
    k_tf_energy<<<1, 1024, 0, s>>>(P);
    MZB_CHECK(cudaGetLastError());
}

// The pair-force stages of a batched step over a replica table (particles.cuh): boxes,
// pair forces (one launch per potential present), gather, energy.
namespace {
__global__ void __launch_bounds__(256) kt_tfbox(const StageArgs* __restrict__ A, const int* __restrict__ start,
                                                int nsys) {
    table_run(A, start, nsys, [&](const StageArgs& a, int b) { k_tf_boxes_body(a.P, b); });
}
template <int POT>
__global__ void __launch_bounds__(kTfThreads, 3) kt_tf(const StageArgs* __restrict__ A, const int* __restrict__ start,
                                                       int nsys) {
    table_run(A, start, nsys, [&](const StageArgs& a, int b) { k_tf_body<POT>(a.P, b); });
}
__global__ void __launch_bounds__(128) kt_tfg(const StageArgs* __restrict__ A, const int* __restrict__ start,
                                              int nsys) {
    table_run(A, start, nsys, [&](const StageArgs& a, int b) { k_tf_gather_body(a.P, b); });
}
__global__ void __launch_bounds__(1024) kt_tfe(const StageArgs* __restrict__ A, const int* __restrict__ start,
                                               int nsys) {
    table_run(A, start, nsys, [&](const StageArgs& a, int b) { k_tf_energy_body(a.P, b); });
}
void tf_tlaunch(const StageTable& t, int k, void (*kernel)(const StageArgs*, const int*, int), int threads,
                size_t smem, cudaStream_t s) {
    if (t.total[k] <= 0) return;
    count_launch();
    kernel<<<t.total[k], threads, smem, s>>>(t.args, t.start + k * (t.nsys + 1), t.nsys);
    MZB_CHECK(cudaGetLastError());
}
}  // namespace

void tf_stages(const StageTable& t, cudaStream_t s) {
    static unsigned long long attr_done = 0;  // devices whose table kernels allow kTfSmem
    int dev = 0;
    MZB_CHECK(cudaGetDevice(&dev));
    if (!(attr_done >> (dev & 63) & 1ull)) {
        MZB_CHECK(cudaFuncSetAttribute(kt_tf<POT_TF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTfSmem));
        MZB_CHECK(cudaFuncSetAttribute(kt_tf<POT_LJ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTfSmem));
        MZB_CHECK(cudaFuncSetAttribute(kt_tf<POT_SC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTfSmem));
        attr_done |= 1ull << (dev & 63);
    }
    tf_tlaunch(t, SK_TFBOX, kt_tfbox, 256, 0, s);
    tf_tlaunch(t, SK_TF_TF, kt_tf<POT_TF>, kTfThreads, kTfSmem, s);
    tf_tlaunch(t, SK_TF_LJ, kt_tf<POT_LJ>, kTfThreads, kTfSmem, s);
    tf_tlaunch(t, SK_TF_SC, kt_tf<POT_SC>, kTfThreads, kTfSmem, s);
    tf_tlaunch(t, SK_TFG, kt_tfg, 128, 0, s);
    tf_tlaunch(t, SK_TFE, kt_tfe, 1024, 0, s);
}

}  // namespace mzb
