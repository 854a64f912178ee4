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
//                                   Laplacian, trilinear prolongation, levels down to
//                                   4^3, coarse levels <= 32^3 worked by one CTA)
//           x += e - mean(e)       (FP64; the periodic Laplacian's null space is the
//                                   constants, and dropping e's mean keeps x's mean
//                                   where it started, as CG does)
//
// Each V-cycle moves ~10 FP64-equivalent passes of the fine grid instead of the ~10 per
// CG iteration of the reference's solver, and a warm-started MD step needs a few cycles
// where CG needs hundreds of iterations.
#include "engine.cuh"
#include "mixed.cuh"
#include "tma.cuh"

namespace mzb {
namespace {

constexpr int kThreads = 1024;
constexpr int kSmallN = 32;  // levels with n <= kSmallN are worked by CTA 0 alone

// warp-per-row point loops over an n^3 grid, either over the whole grid (all CTAs) or
// inside CTA 0 only (small levels)
template <class F>
__device__ __forceinline__ void for_pts(bool single, int n, F&& f) {
    const int lane = threadIdx.x & 31;
    long gw, nw;
    if (single) {
        gw = threadIdx.x >> 5;
        nw = blockDim.x >> 5;
    } else {
        gw = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
        nw = (long)gridDim.x * (blockDim.x >> 5);
    }
    const long rows = (long)n * n;
    for (long row = gw; row < rows; row += nw) {
        const int i = (int)(row / n), j = (int)(row - (long)i * n);
        for (int k = lane; k < n; k += 32) f(i, j, k);
    }
}
template <class F>
__device__ __forceinline__ void for_col(bool single, int n, int colour, F&& f) {
    const int lane = threadIdx.x & 31;
    long gw, nw;
    if (single) {
        gw = threadIdx.x >> 5;
        nw = blockDim.x >> 5;
    } else {
        gw = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
        nw = (long)gridDim.x * (blockDim.x >> 5);
    }
    const long rows = (long)n * n;
    for (long row = gw; row < rows; row += nw) {
        const int i = (int)(row / n), j = (int)(row - (long)i * n);
        for (int k = ((i + j + colour) & 1) + 2 * lane; k < n; k += 64) f(i, j, k);
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

// block-level barrier for single-CTA work, grid barrier otherwise
__device__ __forceinline__ bool sync_level(bool single, GridBarrier* bar, unsigned& epoch) {
    if (single) {
        __syncthreads();
        return true;
    }
    return grid_sync_mono(bar, epoch);
}

// Grid reduction of one sum and one max (deterministic fixed-order gather).
__device__ bool reduce_sum_max(double& s, double& mx, const MixedArgs& a, unsigned& epoch, int& seq) {
    __shared__ double sh[2][32];
    __shared__ double res[2];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const long G = gridDim.x;
    s = warp_sum(s);
    mx = warp_max(mx);
    if (lane == 0) {
        sh[0][w] = s;
        sh[1][w] = mx;
    }
    __syncthreads();
    double* part = a.partials + (long)(seq & 1) * 2 * G;
    if (w == 0) {
        double v0 = lane < nwarp ? sh[0][lane] : 0.0, v1 = lane < nwarp ? sh[1][lane] : 0.0;
        v0 = warp_sum(v0);
        v1 = warp_max(v1);
        if (lane == 0) {
            part[blockIdx.x] = v0;
            part[G + blockIdx.x] = v1;
        }
    }
    const bool ok = grid_sync_mono(a.bar, epoch);
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

// ---- FP32 multigrid pieces ----

__device__ void rbgs32(bool single, int n, const float* b, float* x, int colour) {
    for_col(single, n, colour, [&](int i, int j, int k) {
        const Nb o = nb_of(n, i, j, k);
        float s = x[o.im] + x[o.ip];
        s += x[o.jm];
        s += x[o.jp];
        s += x[o.km];
        s += x[o.kp];
        x[o.c] = (b[o.c] - s) * (-1.0f / 6.0f);
    });
}

__device__ void resid32(bool single, int n, const float* b, const float* x, float* r) {
    for_pts(single, n, [&](int i, int j, int k) {
        const Nb o = nb_of(n, i, j, k);
        float s = x[o.ip] + x[o.im];
        s += x[o.jp];
        s += x[o.jm];
        s += x[o.kp];
        s += x[o.km];
        r[o.c] = b[o.c] - (s - 6.0f * x[o.c]);
    });
}

// coarse b = 4 * R27(r), coarse x = 0
__device__ void restrict32(bool single, int n, const float* r, float* bc, float* xc) {
    const int nc = n / 2;
    const long n2 = (long)n * n;
    for_pts(single, nc, [&](int I, int J, int K) {
        const int i = 2 * I, j = 2 * J, k = 2 * K;
        const long i0 = (long)i * n2, i1 = (long)(i + 1 == n ? 0 : i + 1) * n2, i2 = (long)(i == 0 ? n - 1 : i - 1) * n2;
        const long j0 = (long)j * n, j1 = (long)(j + 1 == n ? 0 : j + 1) * n, j2 = (long)(j == 0 ? n - 1 : j - 1) * n;
        const long k0 = k, k1 = (k + 1 == n ? 0 : k + 1), k2 = (k == 0 ? n - 1 : k - 1);
        const float f = r[i2 + j0 + k0] + r[i1 + j0 + k0] + r[i0 + j2 + k0] + r[i0 + j1 + k0] + r[i0 + j0 + k2] +
                        r[i0 + j0 + k1];
        const float e = r[i1 + j0 + k2] + r[i1 + j0 + k1] + r[i2 + j0 + k2] + r[i2 + j0 + k1] + r[i1 + j2 + k0] +
                        r[i1 + j1 + k0] + r[i2 + j2 + k0] + r[i2 + j1 + k0] + r[i0 + j2 + k2] + r[i0 + j2 + k1] +
                        r[i0 + j1 + k2] + r[i0 + j1 + k1];
        const float c = r[i1 + j1 + k2] + r[i1 + j1 + k1] + r[i1 + j2 + k2] + r[i1 + j2 + k1] + r[i2 + j1 + k2] +
                        r[i2 + j1 + k1] + r[i2 + j2 + k2] + r[i2 + j2 + k1];
        const long cc = ((long)I * nc + J) * nc + K;
        bc[cc] = (8.0f * r[i0 + j0 + k0] + 4.0f * f + 2.0f * e + c) * (4.0f / 64.0f);
        xc[cc] = 0.0f;
    });
}

// fine x += P(coarse x), trilinear
__device__ void prolong32(bool single, int n, const float* xc, float* x) {
    const int nc = n / 2;
    const long n2c = (long)nc * nc;
    for_pts(single, n, [&](int i, int j, int k) {
        const int ci = i >> 1, cj = j >> 1, ck = k >> 1;
        const long i0 = (long)ci * n2c, i1 = (long)(ci + 1 == nc ? 0 : ci + 1) * n2c;
        const long j0 = (long)cj * nc, j1 = (long)(cj + 1 == nc ? 0 : cj + 1) * nc;
        const long k0 = ck, k1 = (ck + 1 == nc ? 0 : ck + 1);
        const float wi = (i & 1) ? 0.5f : 0.0f, wj = (j & 1) ? 0.5f : 0.0f, wk = (k & 1) ? 0.5f : 0.0f;
        const float a00 = xc[i0 + j0 + k0] * (1.0f - wk) + xc[i0 + j0 + k1] * wk;
        const float a01 = xc[i0 + j1 + k0] * (1.0f - wk) + xc[i0 + j1 + k1] * wk;
        const float a10 = xc[i1 + j0 + k0] * (1.0f - wk) + xc[i1 + j0 + k1] * wk;
        const float a11 = xc[i1 + j1 + k0] * (1.0f - wk) + xc[i1 + j1 + k1] * wk;
        const float b0 = a00 * (1.0f - wj) + a01 * wj, b1 = a10 * (1.0f - wj) + a11 * wj;
        x[((long)i * n + j) * n + k] += b0 * (1.0f - wi) + b1 * wi;
    });
}

// One V-cycle: x[0] improved in place for rhs b[0]. Levels with n > kSmallN use all
// CTAs with grid barriers between sweeps; the smaller ones, and the coarsest solve, run
// in CTA 0 with block barriers while the other CTAs wait at the next grid barrier.
__device__ bool vcycle32(const MixedArgs& a, unsigned& epoch) {
    const int L = a.nlev;
    int lsmall = L;
    for (int l = 0; l < L; l++)
        if (a.lev_n[l] <= kSmallN) {
            lsmall = l;
            break;
        }
    const int lbig = lsmall < L - 1 ? lsmall : L - 1;  // big levels below the coarsest
    auto smooth = [&](bool single, int l, int sweeps) -> bool {
        for (int s = 0; s < sweeps; s++)
            for (int c = 0; c < 2; c++) {
                rbgs32(single, a.lev_n[l], a.lev_b[l], a.lev_x[l], c);
                if (!sync_level(single, a.bar, epoch)) return false;
            }
        return true;
    };
    for (int l = 0; l < lbig; l++) {
        if (!smooth(false, l, a.nu1)) return false;
        resid32(false, a.lev_n[l], a.lev_b[l], a.lev_x[l], a.lev_r[l]);
        if (!grid_sync_mono(a.bar, epoch)) return false;
        restrict32(false, a.lev_n[l], a.lev_r[l], a.lev_b[l + 1], a.lev_x[l + 1]);
        if (!grid_sync_mono(a.bar, epoch)) return false;
    }
    if (lsmall < L) {
        if (blockIdx.x == 0) {
            for (int m = lsmall; m < L - 1; m++) {
                smooth(true, m, a.nu1);
                resid32(true, a.lev_n[m], a.lev_b[m], a.lev_x[m], a.lev_r[m]);
                __syncthreads();
                restrict32(true, a.lev_n[m], a.lev_r[m], a.lev_b[m + 1], a.lev_x[m + 1]);
                __syncthreads();
            }
            smooth(true, L - 1, a.coarse_sweeps);
            for (int m = L - 2; m >= lsmall; m--) {
                prolong32(true, a.lev_n[m], a.lev_x[m + 1], a.lev_x[m]);
                __syncthreads();
                smooth(true, m, a.nu2);
            }
        }
        if (!grid_sync_mono(a.bar, epoch)) return false;
    } else {
        if (!smooth(false, L - 1, a.coarse_sweeps)) return false;
    }
    for (int l = lbig - 1; l >= 0; l--) {
        prolong32(false, a.lev_n[l], a.lev_x[l + 1], a.lev_x[l]);
        if (!grid_sync_mono(a.bar, epoch)) return false;
        if (!smooth(false, l, a.nu2)) return false;
    }
    return true;
}

__global__ void __launch_bounds__(kThreads, 1) mixed_kernel(MixedArgs a) {
    const int n = a.n;
    unsigned epoch = 0;
    int seq = 0;
    bool ok = true;
    int result = -1;

    // ---- set-up: right-hand side B and solution X (FP64), as the FP64 programs ----
    double* X = a.phi_new;
    const double* B = a.tmp;
    if (a.prog == PROG_INIT_FIELD) {         // y = 0, phi = 0 start, b = c q
        for_pts(false, n, [&](int i, int j, int k) {
            const long c = ((long)i * n + j) * n + k;
            a.y[c] = 0.0;
            a.phi_new[c] = 0.0;
            a.tmp[c] = a.q[c] * a.c;
        });
    } else if (a.prog == PROG_LCG_UPDATE) {  // y = c q; start from phi_prev (old phi)
        for_pts(false, n, [&](int i, int j, int k) {
            const long c = ((long)i * n + j) * n + k;
            const double bq = a.q[c] * a.c;
            a.y[c] = bq;
            a.tmp[c] = bq;
            a.phi_new[c] = a.phi_old[c];
        });
    } else if (a.prog == PROG_MG_UPDATE) {   // phi = 2 phi - phi_prev (start), b = c q
        for_pts(false, n, [&](int i, int j, int k) {
            const long c = ((long)i * n + j) * n + k;
            a.phi_new[c] = 2 * a.phi_old[c] - a.phi_prev[c];
            a.tmp[c] = a.q[c] * a.c;
        });
    } else {                                 // MaZe: phi = 2 phi - phi_prev; sigma = L phi + c q
        X = a.y;
        for_pts(false, n, [&](int i, int j, int k) {
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
    ok = grid_sync_mono(a.bar, epoch);

    float* e = a.lev_x[0];
    float* rb = a.lev_b[0];
    int outer = 0;
    while (ok) {
        // r = B - L X in FP64 -> FP32 rhs of the inner solve; |r|_inf
        double s0 = 0.0, rmax = 0.0;
        for_pts(false, n, [&](int i, int j, int k) {
            const Nb o = nb_of(n, i, j, k);
            double s = X[o.ip] + X[o.im];
            s = s + X[o.jp];
            s = s + X[o.jm];
            s = s + X[o.kp];
            s = s + X[o.km];
            const double r = B[o.c] - (s - X[o.c] * 6.0);
            rb[o.c] = (float)r;
            e[o.c] = 0.0f;
            rmax = fmax(rmax, fabs(r));
        });
        ok = reduce_sum_max(s0, rmax, a, epoch, seq);
        if (!ok) break;
        if (rmax <= a.tol) {
            result = outer;
            break;
        }
        if (outer >= a.max_outer) break;
        for (int c = 0; c < a.cycles; c++) {
            ok = vcycle32(a, epoch);
            if (!ok) break;
        }
        if (!ok) break;
        // mean of the correction (the periodic Laplacian's null space)
        double esum = 0.0, m0 = 0.0;
        for_pts(false, n, [&](int i, int j, int k) { esum += (double)e[((long)i * n + j) * n + k]; });
        ok = reduce_sum_max(esum, m0, a, epoch, seq);
        if (!ok) break;
        const double emean = esum / ((double)n * n * n);
        for_pts(false, n, [&](int i, int j, int k) {
            const long c = ((long)i * n + j) * n + k;
            X[c] = X[c] + ((double)e[c] - emean);
        });
        ok = grid_sync_mono(a.bar, epoch);
        outer++;
    }
    if (ok && (a.prog == PROG_MAZE_LCG || a.prog == PROG_MAZE_MG)) {  // phi -= y
        for_pts(false, n, [&](int i, int j, int k) {
            const long c = ((long)i * n + j) * n + k;
            a.phi_new[c] = a.phi_new[c] + -1.0 * a.y[c];
        });
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.result[0] = result;
        a.result[1] = ok ? 0 : 1;
    }
}

int g_mixed_device = -1;
int g_mixed_blocks = 0;

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

void mixed_launch(const MixedArgs& a, cudaStream_t stream) {
    int dev;
    MZB_CHECK(cudaGetDevice(&dev));
    if (g_mixed_device != dev) {
        int sms = 0, per_sm = 0;
        MZB_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        MZB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mixed_kernel, kThreads, 0));
        if (per_sm < 1) fatal("mixed solver: kernel cannot be resident on this device");
        g_mixed_device = dev;
        g_mixed_blocks = sms;
    }
    MZB_CHECK(cudaMemsetAsync(a.bar, 0, sizeof(GridBarrier), stream));
    MixedArgs copy = a;
    void* params[] = {&copy};
    count_launch();
    MZB_CHECK(cudaLaunchCooperativeKernel((const void*)mixed_kernel, dim3(g_mixed_blocks), dim3(kThreads), params,
                                          0, stream));
}

}  // namespace mzb
