// Particle-side kernels (see particles.cuh). FP64, compiled with --fmad=false.
#include <climits>

#include "particles.cuh"

namespace mzb {

__device__ __forceinline__ int wrapi(int a, int n) {
    a %= n;
    return a < 0 ? a + n : a;
}

// CIC weight with the minimum image over L = n*h (library/src/charges.c:8-14).
__device__ __forceinline__ double w_cic(double x, double L, double h) {
    x = fabs(x - round(x / L) * L);
    if (x >= h) return 0.0;
    return 1.0 - x / h;
}

// Assignment weight of scheme CAS with the minimum image over L (charges.c:8-38).
template <int CAS>
__device__ __forceinline__ double w_cas(double x, double L, double h) {
    if (CAS == CAS_CIC) return w_cic(x, L, h);
    x = fabs(x - round(x / L) * L) / h;
    if (CAS == CAS_SPL_QUADR) {
        if (x < 0.5) return 0.75 - x * x;
        if (x < 1.5) {
            const double y = 1.5 - x;
            return 0.5 * (y * y);
        }
        return 0.0;
    }
    if (x < 1) return (4.0 - 6.0 * (x * x) + 3.0 * cube_rn(x)) / 6.0;
    if (x < 2) return cube_rn(2 - x) / 6.0;
    return 0.0;
}

// Stencil point o of scheme CAS around base cell b, in the reference's neighbour order
// (CIC: particles.c:323-344; splines: particles.c:366-381, a/b/c = -1..2 nested).
template <int CAS>
__device__ __forceinline__ void stencil_point(int o, const int* b, int n, int& i, int& j, int& k) {
    if (CAS == CAS_CIC) {
        const int di = (o == 1 || o == 4 || o == 5 || o == 7);
        const int dj = (o == 2 || o == 4 || o == 6 || o == 7);
        const int dk = (o == 3 || o == 5 || o == 6 || o == 7);
        i = di ? (b[0] + 1 == n ? 0 : b[0] + 1) : b[0];
        j = dj ? (b[1] + 1 == n ? 0 : b[1] + 1) : b[1];
        k = dk ? (b[2] + 1 == n ? 0 : b[2] + 1) : b[2];
    } else {
        i = (b[0] + o / 16 - 1 + n) % n;
        j = (b[1] + (o / 4) % 4 - 1 + n) % n;
        k = (b[2] + o % 4 - 1 + n) % n;
    }
}
template <int CAS>
constexpr int stencil_size() { return CAS == CAS_CIC ? 8 : 64; }

// CIC corner c (0..7) in the reference's order (particles.c:323-344):
// (0,0,0) (1,0,0) (0,1,0) (0,0,1) (1,1,0) (1,0,1) (0,1,1) (1,1,1)
__device__ __forceinline__ void corner_offsets(int c, int& di, int& dj, int& dk) {
    di = (c == 1 || c == 4 || c == 5 || c == 7);
    dj = (c == 2 || c == 4 || c == 6 || c == 7);
    dk = (c == 3 || c == 5 || c == 6 || c == 7);
}

// part[0] + part[1] + ... + part[n-1], added from 0 in index order, by one whole warp: the
// lanes load 32 values at a time and lane 0's running sum takes them in turn by shuffles
// (the result of a serial loop, without its chain of dependent loads). Every lane
// returns the sum.
__device__ __forceinline__ double warp_ordered_sum(const double* part, int n) {
    const int lane = threadIdx.x & 31;
    double s = 0.0;
    for (int c = 0; c < n; c += 32) {
        const double v = c + lane < n ? part[c + lane] : 0.0;
        const int k = min(32, n - c);
        for (int y = 0; y < k; y++) s += __shfl_sync(0xffffffffu, v, y);
    }
    return s;
}

// ------------------------------------------------------------------------------------
// Exclusive scan of count[0..m) into start[0..m] (start[m] = total); start is also copied
// into fill[0..m) as a scatter cursor. One block of 1024 threads: thread t takes the
// contiguous chunk [t C, (t + 1) C) (C a multiple of 4, read as int4 where the chunk is
// whole), so every load is issued before the one block-wide scan of the chunk totals.
// Optionally sums `part[0..np_part)` in index order into *sum_out.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ void k_scan_body(const int32_t* __restrict__ count, int m, int32_t* __restrict__ start, int32_t* __restrict__ fill, const double* __restrict__ part, int np_part, double* __restrict__ sum_out, int bx) {
    __shared__ int32_t wsum[32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5, nw = blockDim.x >> 5;
    const int C = (((m + (int)blockDim.x - 1) / (int)blockDim.x) + 3) & ~3;
    const int lo = min(m, t * C), hi = min(m, lo + C);
    const int hv = lo + ((hi - lo) & ~3);  // end of the whole int4 groups
    int32_t tot = 0;
    for (int x = lo; x < hv; x += 4) {
        const int4 v = *reinterpret_cast<const int4*>(count + x);
        tot += v.x + v.y + v.z + v.w;
    }
    for (int x = hv; x < hi; x++) tot += count[x];
    int32_t incl = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
        int32_t y = lane < nw ? wsum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t u = __shfl_up_sync(0xffffffffu, y, o);
            if (lane >= o) y += u;
        }
        wsum[lane] = y;
    }
    __syncthreads();
    int32_t run = incl - tot + (w > 0 ? wsum[w - 1] : 0);
    for (int x = lo; x < hv; x += 4) {
        const int4 v = *reinterpret_cast<const int4*>(count + x);
        int4 o;
        o.x = run;
        o.y = o.x + v.x;
        o.z = o.y + v.y;
        o.w = o.z + v.z;
        run = o.w + v.w;
        *reinterpret_cast<int4*>(start + x) = o;
        *reinterpret_cast<int4*>(fill + x) = o;
    }
    for (int x = hv; x < hi; x++) {
        const int32_t v = count[x];
        start[x] = run;
        fill[x] = run;
        run += v;
    }
    if (t == (int)blockDim.x - 1) start[m] = run;
    if (sum_out != nullptr && w == 0) {
        const double s = warp_ordered_sum(part, np_part);
        if (lane == 0) *sum_out = s;
    }
}
__global__ void __launch_bounds__(1024) k_scan(const int32_t* __restrict__ count, int m,
                                               int32_t* __restrict__ start, int32_t* __restrict__ fill,
                                               const double* __restrict__ part, int np_part,
                                               double* __restrict__ sum_out) { k_scan_body(count, m, start, fill, part, np_part, sum_out, blockIdx.x); }

// The same scan over many blocks (large m): k_scan_reduce sums the counts of each block
// of 1024, k_scan_apply scans each block from the sum of the blocks before it (read in
// block order), coalesced, one count per thread.
__device__ __forceinline__ void k_scan_reduce_body(const int32_t* __restrict__ count, int m, int32_t* __restrict__ blk, int bx) {
    __shared__ int32_t wsum[32];
    const int x = bx * 1024 + threadIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int32_t v = x < m ? count[x] : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) wsum[w] = v;
    __syncthreads();
    if (w == 0) {
        int32_t y = wsum[lane];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
        if (lane == 0) blk[bx] = y;
    }
}
__global__ void __launch_bounds__(1024) k_scan_reduce(const int32_t* __restrict__ count, int m,
                                                      int32_t* __restrict__ blk) { k_scan_reduce_body(count, m, blk, blockIdx.x); }

__device__ __forceinline__ void k_scan_apply_body(const int32_t* __restrict__ count, int m, const int32_t* __restrict__ blk, int32_t* __restrict__ start, int32_t* __restrict__ fill, const double* __restrict__ part, int np_part, double* __restrict__ sum_out, int bx) {
    __shared__ int32_t wsum[32];
    __shared__ int32_t base_s;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int x = bx * 1024 + t;
    if (w == 0) {
        int32_t b = 0;
        for (int u = lane; u < (int)bx; u += 32) b += blk[u];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) b += __shfl_xor_sync(0xffffffffu, b, o);
        if (lane == 0) base_s = b;
    }
    const int32_t v = x < m ? count[x] : 0;
    int32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
        int32_t y = wsum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t u = __shfl_up_sync(0xffffffffu, y, o);
            if (lane >= o) y += u;
        }
        wsum[lane] = y;
    }
    __syncthreads();
    const int32_t excl = base_s + incl - v + (w > 0 ? wsum[w - 1] : 0);
    if (x < m) {
        start[x] = excl;
        fill[x] = excl;
    }
    if (x == m - 1) start[m] = excl + v;
    if (m == 0 && bx == 0 && t == 0) start[0] = 0;
    if (sum_out != nullptr && bx == 0 && w == 0) {
        const double s = warp_ordered_sum(part, np_part);
        if (lane == 0) *sum_out = s;
    }
}
__global__ void __launch_bounds__(1024) k_scan_apply(const int32_t* __restrict__ count, int m,
                                                     const int32_t* __restrict__ blk, int32_t* __restrict__ start,
                                                     int32_t* __restrict__ fill, const double* __restrict__ part,
                                                     int np_part, double* __restrict__ sum_out) { k_scan_apply_body(count, m, blk, start, fill, part, np_part, sum_out, blockIdx.x); }

// Exclusive scan of count[0..m) into start (and fill): one block for small m, else the
// two-kernel form with per-block totals in blk ([ceil(m / 1024)]).
void scan_counts(const int32_t* count, int m, int32_t* start, int32_t* fill, int32_t* blk, const double* part,
                 int np_part, double* sum_out, cudaStream_t s) {
    if (m <= 4096 || blk == nullptr) {
        count_launch();
        k_scan<<<1, 1024, 0, s>>>(count, m, start, fill, part, np_part, sum_out);
        return;
    }
    const int nblk = (m + 1023) / 1024;
    count_launch(2);
    k_scan_reduce<<<nblk, 1024, 0, s>>>(count, m, blk);
    k_scan_apply<<<nblk, 1024, 0, s>>>(count, m, blk, start, fill, part, np_part, sum_out);
}

// ------------------------------------------------------------------------------------
// Charge spreading
// ------------------------------------------------------------------------------------

// Per ion: base cell floor(pos/h) (wrapped), tile histogram and the ion's total spread
// charge (block partial, summed later in block order). With q_old non-null (a CIC grid
// whose only nonzeros are the corners of the bases being replaced) the ion first zeroes
// the 8 corners of its old base cell.
template <int CAS>
__device__ __forceinline__ void k_spread_bin_body(const ParticleDev& P, int n, double h, double* __restrict__ part, double* __restrict__ q_old, int bx) {
    const int p = bx * blockDim.x + threadIdx.x;
    double u = 0.0;
    if (p < P.np) {
        if (q_old != nullptr) {
            const int o0 = P.base[3 * p], o1 = P.base[3 * p + 1], o2 = P.base[3 * p + 2];
            const long n2 = (long)n * n;
#pragma unroll
            for (int o = 0; o < 8; o++) {
                const int i = o0 + (o >> 2) == n ? 0 : o0 + (o >> 2);
                const int j = o1 + ((o >> 1) & 1) == n ? 0 : o1 + ((o >> 1) & 1);
                const int k = o2 + (o & 1) == n ? 0 : o2 + (o & 1);
                q_old[(long)i * n2 + (long)j * n + k] = 0.0;
            }
        }
        int b[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            b[d] = wrapi((int)floor(P.pos[3 * p + d] / h), n);
            P.base[3 * p + d] = b[d];
        }
        const int tile = ((b[0] / kTileI) * P.ntj + b[1] / kTileJ) * P.ntk + b[2] / kTileK;
        atomicAdd(&P.tile_count[tile], 1);
        const double L = n * h, q = P.chg[p];
        for (int o = 0; o < stencil_size<CAS>(); o++) {
            int a, bb, e;
            stencil_point<CAS>(o, b, n, a, bb, e);
            double w = w_cas<CAS>(P.pos[3 * p] - a * h, L, h) * w_cas<CAS>(P.pos[3 * p + 1] - bb * h, L, h);
            w = w * w_cas<CAS>(P.pos[3 * p + 2] - e * h, L, h);
            u += q * w;
        }
    }
    __shared__ double sh[4 * 32];
    double v[1] = {u};
    block_sum<1>(v, sh);
    if (threadIdx.x == 0) part[bx] = v[0];
}
template <int CAS>
__global__ void k_spread_bin(ParticleDev P, int n, double h, double* __restrict__ part, double* __restrict__ q_old) { k_spread_bin_body<CAS>(P, n, h, part, q_old, blockIdx.x); }

__device__ __forceinline__ void k_spread_fill_body(const ParticleDev& P, int bx) {
    const int p = bx * blockDim.x + threadIdx.x;
    if (p >= P.np) return;
    const int* b = P.base + 3 * p;
    const int tile = ((b[0] / kTileI) * P.ntj + b[1] / kTileJ) * P.ntk + b[2] / kTileK;
    const int slot = atomicAdd(&P.tile_fill[tile], 1);
    P.tile_ions[slot] = p;
}
__global__ void k_spread_fill(ParticleDev P) { k_spread_fill_body(P, blockIdx.x); }

// Is grid index g one of the stencil's indices along an axis with base index b (wrapped)?
// CIC: b, b+1; splines: b-1 .. b+2 (particles.c:297-385).
template <int CAS>
__device__ __forceinline__ bool in_stencil(int g, int b, int n) {
    if (CAS == CAS_CIC) return g == b || g == (b + 1 == n ? 0 : b + 1);
    const int d = g - b + 1;
    return (d >= 0 && d <= 3) || (d + n >= 0 && d + n <= 3) || (d - n >= 0 && d - n <= 3);
}

// Spline spreading (CIC takes k_spread_ions below). One warp per tile (grid-stride over
// warps): gather the ions whose stencil can reach the tile (base cell in this tile or the
// 7 tiles below it for CIC, whose +1 corners reach up; in the 27 tiles around it for the
// splines, whose offsets run -1..2), sort them by
// ion index (beyond kTileCap candidates, take them in the same order by repeated warp
// minima over the source tiles' lists instead), and let every lane sum the contributions of its TI x TJ points (one k column)
// over those ions in ascending ion order -- for each point the order of the reference's
// serial scatter (charges.c:123-141), with the same weight expression -- then write the
// tile, zeros included, 32 consecutive k per store. q is written once; no atomics touch
// it, and the warps of a CTA never wait on one another.
constexpr int kSpreadWarps = 4;
constexpr int kSpreadStage = 32;  // staged candidates per round (one per lane)

template <int CAS>
__global__ void __launch_bounds__(kSpreadWarps * 32) k_spread_tiles(ParticleDev P, double* __restrict__ q, int n,
                                                                    double h) {
    constexpr int NSRC = CAS == CAS_CIC ? 8 : 27;
    __shared__ int cand_all[kSpreadWarps][kTileCap];
    __shared__ int sorted_all[kSpreadWarps][kTileCap];
    __shared__ double spos_all[kSpreadWarps][kSpreadStage][4];  // x, y, z, charge (rank order)
    __shared__ int sbase_all[kSpreadWarps][kSpreadStage][3];
    __shared__ int srcs_all[kSpreadWarps][32];
    __shared__ int lfirst_all[kSpreadWarps][32], lcnt_all[kSpreadWarps][32];  // source lists (overflow path)
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int* cand = cand_all[w];
    int* sorted = sorted_all[w];
    double (*spos)[4] = spos_all[w];
    int (*sbase)[3] = sbase_all[w];
    int* srcs = srcs_all[w];
    int* lfirst = lfirst_all[w];
    int* lcnt = lcnt_all[w];
    const double L = n * h;
    const long n2 = (long)n * n;
    const long nwarps = (long)gridDim.x * kSpreadWarps;
    for (long tile = (long)blockIdx.x * kSpreadWarps + w; tile < P.ntiles; tile += nwarps) {
        const int ti = (int)(tile / (P.ntj * P.ntk)), tj = (int)((tile / P.ntk) % P.ntj), tk = (int)(tile % P.ntk);
        int s = -1;
        if (lane < NSRC) {
            int si, sj, sk;
            if (CAS == CAS_CIC) {
                si = wrapi(ti - ((lane >> 2) & 1), P.nti);
                sj = wrapi(tj - ((lane >> 1) & 1), P.ntj);
                sk = wrapi(tk - (lane & 1), P.ntk);
            } else {
                si = wrapi(ti + lane / 9 - 1, P.nti);
                sj = wrapi(tj + (lane / 3) % 3 - 1, P.ntj);
                sk = wrapi(tk + lane % 3 - 1, P.ntk);
            }
            s = (si * P.ntj + sj) * P.ntk + sk;
            srcs[lane] = s;
        }
        __syncwarp();
        int cnt = 0, first = 0;
        if (lane < NSRC) {
            bool dup = false;
            for (int d = 0; d < lane; d++) dup |= (srcs[d] == s);
            if (!dup) {
                first = P.tile_start[s];
                cnt = P.tile_start[s + 1] - first;
            }
        }
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
        }
        const int nc = __shfl_sync(0xffffffffu, incl, 31);
        const int i0 = ti * kTileI, j0 = tj * kTileJ, k = tk * kTileK + lane;
        double acc[kTileI][kTileJ];
#pragma unroll
        for (int a = 0; a < kTileI; a++)
#pragma unroll
            for (int r = 0; r < kTileJ; r++) acc[a][r] = 0.0;
        // one round: lane l stages ion p (or nothing, p < 0), then every lane adds the
        // round's cn ions, in lane order, to its points
        auto stage_and_add = [&](int p, int cn) {
            if (p >= 0) {
                spos[lane][0] = P.pos[3 * p];
                spos[lane][1] = P.pos[3 * p + 1];
                spos[lane][2] = P.pos[3 * p + 2];
                spos[lane][3] = P.chg[p];
                sbase[lane][0] = P.base[3 * p];
                sbase[lane][1] = P.base[3 * p + 1];
                sbase[lane][2] = P.base[3 * p + 2];
            }
            __syncwarp();
            if (k < n) {
                for (int x = 0; x < cn; x++) {
                    if (!in_stencil<CAS>(k, sbase[x][2], n)) continue;
                    const double zk = w_cas<CAS>(spos[x][2] - k * h, L, h);
                    const double cq = spos[x][3];
#pragma unroll
                    for (int a = 0; a < kTileI; a++) {
                        const int i = i0 + a;
                        if (i >= n || !in_stencil<CAS>(i, sbase[x][0], n)) continue;
                        const double wx = w_cas<CAS>(spos[x][0] - i * h, L, h);
#pragma unroll
                        for (int r = 0; r < kTileJ; r++) {
                            const int j = j0 + r;
                            if (j < n && in_stencil<CAS>(j, sbase[x][1], n)) {
                                double wgt = wx * w_cas<CAS>(spos[x][1] - j * h, L, h);
                                wgt = wgt * zk;
                                acc[a][r] += cq * wgt;
                            }
                        }
                    }
                }
            }
            __syncwarp();
        };
        if (nc <= kTileCap) {
            for (int x = 0; x < cnt; x++) cand[incl - cnt + x] = P.tile_ions[first + x];
            __syncwarp();
            for (int x = lane; x < nc; x += 32) {
                const int me = cand[x];
                int rank = 0;
                for (int y = 0; y < nc; y++) rank += (cand[y] < me);
                sorted[rank] = me;
            }
            __syncwarp();
            for (int c0 = 0; c0 < nc; c0 += kSpreadStage) {
                const int cn = min(kSpreadStage, nc - c0);
                stage_and_add(lane < cn ? sorted[c0 + lane] : -1, cn);
            }
        } else {
            // more candidates than the shared lists hold (crowded ions, or small grids
            // whose 27 source tiles cover much of the box): the same rounds in the same
            // ascending ion order, each ion found as the warp minimum of the source lists
            // above the last one taken (an ion lies in one tile, so the indices differ)
            lfirst[lane] = first;
            lcnt[lane] = cnt;
            __syncwarp();
            int last = -1;
            for (int c0 = 0; c0 < nc; c0 += kSpreadStage) {
                const int cn = min(kSpreadStage, nc - c0);
                int mine = -1;
                for (int t = 0; t < cn; t++) {
                    int best = INT_MAX;
                    for (int src = 0; src < NSRC; src++) {
                        const int f = lfirst[src], c = lcnt[src];
                        for (int x = lane; x < c; x += 32) {
                            const int id = P.tile_ions[f + x];
                            if (id > last && id < best) best = id;
                        }
                    }
                    best = __reduce_min_sync(0xffffffffu, best);
                    if (lane == t) mine = best;
                    last = best;
                }
                stage_and_add(mine, cn);
            }
        }
        if (k < n) {
#pragma unroll
            for (int a = 0; a < kTileI; a++)
#pragma unroll
                for (int r = 0; r < kTileJ; r++) {
                    const int i = i0 + a, j = j0 + r;
                    if (i < n && j < n) q[(long)i * n2 + (long)j * n + k] = acc[a][r];
                }
        }
        __syncwarp();
    }
}

// CIC spreading by ion, into a q that is zero away from the corners written here. Ion
// p's stencil covers the corners P = b + o, o in {0,1}^3, of its base cell b; the ions
// that contribute to a corner are those whose base cell is P - {0,1}^3, so every
// contributor to any of p's corners has its base within one cell of b, in the (at most
// eight) tiles around b. For each corner the contributor of lowest index writes the
// corner's value: the contributions summed from 0 in ascending ion order -- the order of
// the reference's serial scatter (charges.c:123-141), with the same weight expression as
// k_spread_tiles -- so each point is written once and no atomics touch q.
//
// Eight lanes per ion: lane l scans tile l for near ions (base within one cell of b along
// every axis; usually p alone) into the ion's list in shared memory, then handles corner
// l. A crowd of more than kNear near ions takes a slower exact path that scans the tiles
// for each corner.
constexpr int kNear = 16;
constexpr int kIonLanes = 8;
constexpr int kSpreadIonThreads = 128;
constexpr int kIonsPerCta = kSpreadIonThreads / kIonLanes;

__device__ __forceinline__ int wrap_delta(int d, int n) {  // d in (-n, n) -> (-n/2, n/2]
    if (2 * d > n) return d - n;
    if (2 * d <= -n) return d + n;
    return d;
}

__device__ __forceinline__ double cic_contrib(const ParticleDev& P, int c, int i, int j, int k, double L, double h) {
    const double wx = w_cas<CAS_CIC>(P.pos[3 * c] - i * h, L, h);
    double wgt = wx * w_cas<CAS_CIC>(P.pos[3 * c + 1] - j * h, L, h);
    wgt = wgt * w_cas<CAS_CIC>(P.pos[3 * c + 2] - k * h, L, h);
    return P.chg[c] * wgt;
}

__device__ __forceinline__ void k_spread_ions_body(const ParticleDev& P, double* __restrict__ q, uint32_t* __restrict__ qmask, int n, double h, int bx) {
    __shared__ int near_id_s[kIonsPerCta][kNear];
    __shared__ int near_o_s[kIonsPerCta][kNear];  // offset code (di+1)*9 + (dj+1)*3 + (dk+1)
    __shared__ int near_n_s[kIonsPerCta];
    const int g = threadIdx.x / kIonLanes, sub = threadIdx.x % kIonLanes;
    const int p = bx * kIonsPerCta + g;
    if (p >= P.np) return;  // whole groups of eight lanes leave together
    const unsigned gmask = 0xffu << (threadIdx.x & 24);
    const double L = n * h;
    const int b0 = P.base[3 * p], b1 = P.base[3 * p + 1], b2 = P.base[3 * p + 2];
    // the distinct tiles holding the cells b - 1 .. b + 1 (at most two per axis)
    int ts[2][3], nt[3];
    {
        const int bb[3] = {b0, b1, b2}, tsz[3] = {kTileI, kTileJ, kTileK}, ntl[3] = {P.nti, P.ntj, P.ntk};
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const int lo = wrapi(bb[d] - 1, n) / tsz[d], hi = wrapi(bb[d] + 1, n) / tsz[d];
            ts[0][d] = lo;
            ts[1][d] = hi;
            nt[d] = lo == hi || ntl[d] == 1 ? 1 : 2;
        }
    }
    auto near_code = [&](int c) {  // offset code of ion c, or -1 if its base is not within one cell
        const int di = wrap_delta(P.base[3 * c] - b0, n), dj = wrap_delta(P.base[3 * c + 1] - b1, n),
                  dk = wrap_delta(P.base[3 * c + 2] - b2, n);
        if (di < -1 || di > 1 || dj < -1 || dj > 1 || dk < -1 || dk > 1) return -1;
        return (di + 1) * 9 + (dj + 1) * 3 + (dk + 1);
    };
    auto tile_of = [&](int l) { return (ts[l >> 2][0] * P.ntj + ts[(l >> 1) & 1][1]) * P.ntk + ts[l & 1][2]; };
    auto tile_valid = [&](int l) { return (l >> 2) < nt[0] && ((l >> 1) & 1) < nt[1] && (l & 1) < nt[2]; };
    if (sub == 0) near_n_s[g] = 0;
    __syncwarp(gmask);
    if (tile_valid(sub)) {
        const int tile = tile_of(sub);
        for (int x = P.tile_start[tile], e1 = P.tile_start[tile + 1]; x < e1; x++) {
            const int c = P.tile_ions[x];
            const int code = near_code(c);
            if (code < 0) continue;
            const int slot = atomicAdd(&near_n_s[g], 1);
            if (slot < kNear) {
                near_id_s[g][slot] = c;
                near_o_s[g][slot] = code;
            }
        }
    }
    __syncwarp(gmask);
    const int nn_all = near_n_s[g];
    const bool crowd = nn_all > kNear;
    const int nn = crowd ? kNear : nn_all;
    const int* near_id = near_id_s[g];
    const int* near_o = near_o_s[g];
    // corner o = sub; c contributes to it iff o - (base_c - b) is in {0,1}^3
    const int oi = sub >> 2, oj = (sub >> 1) & 1, ok = sub & 1;
    const int i = b0 + oi == n ? 0 : b0 + oi, j = b1 + oj == n ? 0 : b1 + oj, k = b2 + ok == n ? 0 : b2 + ok;
    auto contributes = [&](int code) {
        const int ei = oi - (code / 9 - 1), ej = oj - ((code / 3) % 3 - 1), ek = ok - (code % 3 - 1);
        return ei >= 0 && ei <= 1 && ej >= 0 && ej <= 1 && ek >= 0 && ek <= 1;
    };
    double acc = 0.0;
    if (!crowd) {
        int owner = p, m = 0;
        for (int x = 0; x < nn; x++)
            if (contributes(near_o[x])) {
                owner = min(owner, near_id[x]);
                m++;
            }
        if (owner != p) return;
        int last = -1;
        for (int t = 0; t < m; t++) {  // contributors in ascending ion order
            int next = INT_MAX;
            for (int x = 0; x < nn; x++)
                if (near_id[x] > last && near_id[x] < next && contributes(near_o[x])) next = near_id[x];
            acc += cic_contrib(P, next, i, j, k, L, h);
            last = next;
        }
    } else {  // the same, scanning the tiles for every contributor
        auto for_contrib = [&](auto&& f) {
            for (int l = 0; l < 8; l++) {
                if (!tile_valid(l)) continue;
                const int tile = tile_of(l);
                for (int x = P.tile_start[tile]; x < P.tile_start[tile + 1]; x++) {
                    const int c = P.tile_ions[x];
                    const int code = near_code(c);
                    if (code >= 0 && contributes(code)) f(c);
                }
            }
        };
        int owner = p;
        for_contrib([&](int c) { owner = min(owner, c); });
        if (owner != p) return;
        int last = -1;
        while (true) {
            int next = INT_MAX;
            for_contrib([&](int c) {
                if (c > last && c < next) next = c;
            });
            if (next == INT_MAX) break;
            acc += cic_contrib(P, next, i, j, k, L, h);
            last = next;
        }
    }
    q[((long)i * n + j) * n + k] = acc;
    if (qmask != nullptr) {
        const long seg = ((long)i * n + j) * (n >> 6) + (k >> 6);
        atomicOr(qmask + (seg >> 5), 1u << (seg & 31));
    }
}
__global__ void __launch_bounds__(kSpreadIonThreads) k_spread_ions(ParticleDev P, double* __restrict__ q,
                                                                   uint32_t* __restrict__ qmask, int n, double h) { k_spread_ions_body(P, q, qmask, n, h, blockIdx.x); }

void spread_charges(ParticleDev& P, double* q, uint32_t* qmask, int n, double h, cudaStream_t s) {
    const int nb = (P.np + 127) / 128;
    MZB_CHECK(cudaMemsetAsync(P.tile_count, 0, sizeof(int32_t) * P.ntiles, s));
    // CIC: q keeps zeros away from the ions' corners, so only the old corners need
    // clearing when q holds the last CIC spreading of these ions; otherwise clear it all
    const bool sparse = P.cas == CAS_CIC && P.q_sparse == q;
    if (P.cas == CAS_CIC && !sparse) MZB_CHECK(cudaMemsetAsync(q, 0, sizeof(double) * (size_t)n * n * n, s));
    count_launch();
    if (P.cas == CAS_CIC)
        k_spread_bin<CAS_CIC><<<nb > 0 ? nb : 1, 128, 0, s>>>(P, n, h, P.partial, sparse ? q : nullptr);
    else if (P.cas == CAS_SPL_QUADR)
        k_spread_bin<CAS_SPL_QUADR><<<nb > 0 ? nb : 1, 128, 0, s>>>(P, n, h, P.partial, nullptr);
    else
        k_spread_bin<CAS_SPL_CUBIC><<<nb > 0 ? nb : 1, 128, 0, s>>>(P, n, h, P.partial, nullptr);
    scan_counts(P.tile_count, P.ntiles, P.tile_start, P.tile_fill, P.tile_part, P.partial, nb > 0 ? nb : 1,
                P.red + 0, s);
    if (nb > 0) count_launch();
    if (nb > 0) k_spread_fill<<<nb, 128, 0, s>>>(P);
    const size_t mask_bytes = qmask != nullptr ? sizeof(uint32_t) * (((size_t)n * n * (n >> 6) + 31) / 32) : 0;
    if (P.cas == CAS_CIC) {  // the corners the ions reach (q is zero elsewhere)
        if (qmask != nullptr) MZB_CHECK(cudaMemsetAsync(qmask, 0, mask_bytes, s));
        if (P.np > 0) {
            count_launch();
            k_spread_ions<<<(P.np + kIonsPerCta - 1) / kIonsPerCta, kSpreadIonThreads, 0, s>>>(P, q, qmask, n, h);
        }
        MZB_CHECK(cudaGetLastError());
        P.q_sparse = q;
        return;
    }
    P.q_sparse = nullptr;  // the tile kernel writes every point
    if (qmask != nullptr) MZB_CHECK(cudaMemsetAsync(qmask, 0xff, mask_bytes, s));
    int dev, sms;
    MZB_CHECK(cudaGetDevice(&dev));
    MZB_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int ctas = (P.ntiles + kSpreadWarps - 1) / kSpreadWarps;
    const int grid = ctas < sms * 12 ? ctas : sms * 12;
    count_launch();
    if (P.cas == CAS_SPL_QUADR)
        k_spread_tiles<CAS_SPL_QUADR><<<grid, kSpreadWarps * 32, 0, s>>>(P, q, n, h);
    else
        k_spread_tiles<CAS_SPL_CUBIC><<<grid, kSpreadWarps * 32, 0, s>>>(P, q, n, h);
    MZB_CHECK(cudaGetLastError());
}

// ------------------------------------------------------------------------------------
// Field forces: central differences of phi at the stencil points (forces.c:26-100).
// ------------------------------------------------------------------------------------
// Eight lanes per ion: lane l takes the stencil points c = l, l + 8, ... (one for CIC, 8
// for the splines) and the ion's sums are then formed from 0 in the stencil's order c = 0,
// 1, 2, ... by shuffling each term to the lanes in turn -- the reference's order, so the
// forces are bit-exact -- and written by the first lane.
constexpr int kForceLanes = 8;

template <int CAS>
__device__ __forceinline__ void k_field_forces_body(const ParticleDev& P, const double* __restrict__ phi, int n, double h, int bx) {
    constexpr int S = stencil_size<CAS>(), T = S / kForceLanes;
    const int p = (bx * blockDim.x + threadIdx.x) / kForceLanes, sub = threadIdx.x % kForceLanes;
    if (p >= P.np) return;  // whole groups of eight lanes leave together
    const unsigned gmask = 0xffu << (threadIdx.x & 24);
    const int g0 = threadIdx.x & 31 & ~(kForceLanes - 1);
    const double L = n * h, h2 = 2.0 * h;
    const long n2 = (long)n * n;
    const int* b = P.base + 3 * p;
    const double px = P.pos[3 * p], py = P.pos[3 * p + 1], pz = P.pos[3 * p + 2], chg = P.chg[p];
    double tx[T], ty[T], tz[T];
#pragma unroll
    for (int u = 0; u < T; u++) {
        int i, j, k;
        stencil_point<CAS>(u * kForceLanes + sub, b, n, i, j, k);
        double qc = chg * w_cas<CAS>(px - i * h, L, h);
        qc = qc * w_cas<CAS>(py - j * h, L, h);
        qc = qc * w_cas<CAS>(pz - k * h, L, h);
        const long i0 = i * n2, j0 = (long)j * n;
        const long ip = (long)wrap_inc(i, n) * n2, im = (long)wrap_dec(i, n) * n2;
        const long jp = (long)wrap_inc(j, n) * n, jm = (long)wrap_dec(j, n) * n;
        const int kp = wrap_inc(k, n), km = wrap_dec(k, n);
        tx[u] = qc * ((phi[im + j0 + k] - phi[ip + j0 + k]) / h2);
        ty[u] = qc * ((phi[i0 + jm + k] - phi[i0 + jp + k]) / h2);
        tz[u] = qc * ((phi[i0 + j0 + km] - phi[i0 + j0 + kp]) / h2);
    }
    double fx = 0.0, fy = 0.0, fz = 0.0;
#pragma unroll
    for (int u = 0; u < T; u++)
#pragma unroll
        for (int l = 0; l < kForceLanes; l++) {
            fx += __shfl_sync(gmask, tx[u], g0 + l);
            fy += __shfl_sync(gmask, ty[u], g0 + l);
            fz += __shfl_sync(gmask, tz[u], g0 + l);
        }
    if (sub == 0) {
        P.fe[3 * p] = fx;
        P.fe[3 * p + 1] = fy;
        P.fe[3 * p + 2] = fz;
    }
}
template <int CAS>
__global__ void __launch_bounds__(128) k_field_forces(ParticleDev P, const double* __restrict__ phi, int n, double h) { k_field_forces_body<CAS>(P, phi, n, h, blockIdx.x); }

void field_forces(ParticleDev& P, const double* phi, int n, double h, cudaStream_t s) {
    if (P.np == 0) return;
    count_launch();
    const int nb = (P.np * kForceLanes + 127) / 128;
    if (P.cas == CAS_CIC)
        k_field_forces<CAS_CIC><<<nb, 128, 0, s>>>(P, phi, n, h);
    else if (P.cas == CAS_SPL_QUADR)
        k_field_forces<CAS_SPL_QUADR><<<nb, 128, 0, s>>>(P, phi, n, h);
    else
        k_field_forces<CAS_SPL_CUBIC><<<nb, 128, 0, s>>>(P, phi, n, h);
    MZB_CHECK(cudaGetLastError());
}

// ------------------------------------------------------------------------------------
// Linked cells by counting sort, stable in ion index: cell (IX,IY,IZ) with
// IX = int((nc/L) * x) (maze_poisson/linkedcell.py:18-26), clamped into the box.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ void k_cell_count_body(const ParticleDev& P, int bx) {
    const int p = bx * blockDim.x + threadIdx.x;
    if (p >= P.np) return;
    const double rel = P.nc / P.L;
    int c[3];
    bool inside = true;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double x = P.pos[3 * p + d];
        inside &= (x >= 0.0 && x < P.L);
        int v = (int)(rel * x);
        if (!(rel * x >= 0.0)) v = 0;
        c[d] = v < 0 ? 0 : (v >= P.nc ? P.nc - 1 : v);
    }
    if (!inside) atomicOr(&P.flags[1], 1);
    const int cell = (c[0] * P.nc + c[1]) * P.nc + c[2];
    P.cell_of[p] = cell;
    atomicAdd(&P.cell_count[cell], 1);
}
__global__ void k_cell_count(ParticleDev P) { k_cell_count_body(P, blockIdx.x); }

__device__ __forceinline__ void k_cell_fill_body(const ParticleDev& P, int bx) {
    const int p = bx * blockDim.x + threadIdx.x;
    if (p >= P.np) return;
    const int slot = atomicAdd(&P.cell_fill[P.cell_of[p]], 1);
    P.cell_ions[slot] = p;
}
__global__ void k_cell_fill(ParticleDev P) { k_cell_fill_body(P, blockIdx.x); }

// One warp per cell: restore ascending ion order inside the cell (the scatter above is
// unordered) by ranking each ion against the cell's others (ion indices are distinct, so
// the ranks are a permutation; a cell of more than kCellStage ions is insertion-sorted by
// one lane), then gather positions/types into cell order and record each ion's rank.
constexpr int kCellStage = 256;

__device__ __forceinline__ void k_cell_sort_gather_body(const ParticleDev& P, int bx) {
    __shared__ int stage_all[4][kCellStage];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cell = bx * 4 + w;
    if (cell >= P.ncell) return;
    const int b = P.cell_start[cell], e = P.cell_start[cell + 1], m = e - b;
    int* st = stage_all[w];
    if (m <= kCellStage) {
        for (int x = lane; x < m; x += 32) st[x] = P.cell_ions[b + x];
        __syncwarp();
        for (int x = lane; x < m; x += 32) {
            const int v = st[x];
            int r = 0;
            for (int y = 0; y < m; y++) r += st[y] < v;
            P.cell_ions[b + r] = v;
        }
    } else if (lane == 0) {
        for (int x = b + 1; x < e; x++) {
            const int v = P.cell_ions[x];
            int y = x - 1;
            while (y >= b && P.cell_ions[y] > v) {
                P.cell_ions[y + 1] = P.cell_ions[y];
                y--;
            }
            P.cell_ions[y + 1] = v;
        }
    }
    __syncwarp();
    for (int x = b + lane; x < e; x += 32) {
        const int p = P.cell_ions[x];
        P.spos[3 * x] = P.pos[3 * p];
        P.spos[3 * x + 1] = P.pos[3 * p + 1];
        P.spos[3 * x + 2] = P.pos[3 * p + 2];
        P.stype[x] = P.types[p];
        P.srank[p] = x;
    }
}
__global__ void __launch_bounds__(128) k_cell_sort_gather(ParticleDev P) { k_cell_sort_gather_body(P, blockIdx.x); }

void build_cells(ParticleDev& P, cudaStream_t s) {
    MZB_CHECK(cudaMemsetAsync(P.cell_count, 0, sizeof(int32_t) * P.ncell, s));
    MZB_CHECK(cudaMemsetAsync(P.flags + 1, 0, sizeof(int), s));
    if (P.np > 0) count_launch();
    if (P.np > 0) k_cell_count<<<(P.np + 127) / 128, 128, 0, s>>>(P);
    count_launch();
    k_scan<<<1, 1024, 0, s>>>(P.cell_count, P.ncell, P.cell_start, P.cell_fill, nullptr, 0, nullptr);
    if (P.np > 0) count_launch();
    if (P.np > 0) k_cell_fill<<<(P.np + 127) / 128, 128, 0, s>>>(P);
    count_launch();
    k_cell_sort_gather<<<(P.ncell + 3) / 4, 128, 0, s>>>(P);
    MZB_CHECK(cudaGetLastError());
}

// ------------------------------------------------------------------------------------
// fcs_tot = (0 + 1*fcs_elec) + 1*fcs_noel (particles.c:777-795)
// ------------------------------------------------------------------------------------
__device__ __forceinline__ void k_total_forces_body(const ParticleDev& P, int bx) {
    const int t = bx * blockDim.x + threadIdx.x;
    if (t >= 3 * P.np) return;
    double v = 0.0;
    v += 1.0 * P.fe[t];
    v += 1.0 * P.fn[t];
    if (P.fdb) {
        v += 1.0 * P.fdb[t];
        v += 1.0 * P.fib[t];
        v += 1.0 * P.fnp[t];
    }
    P.ft[t] = v;
}
__global__ void k_total_forces(ParticleDev P) { k_total_forces_body(P, blockIdx.x); }

void total_forces(ParticleDev& P, cudaStream_t s) {
    if (P.np == 0) return;
    count_launch();
    k_total_forces<<<(3 * P.np + 255) / 256, 256, 0, s>>>(P);
    MZB_CHECK(cudaGetLastError());
}

// ------------------------------------------------------------------------------------
// Kinetic energy, momentum, temperature (particles.c:798-839). Block partials are summed
// in block order by one thread: deterministic for a given N.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ void k_ke_partial_body(const ParticleDev& P, int bx) {
    const int p = bx * blockDim.x + threadIdx.x;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (p < P.np) {
        const double m = P.mass[p], vx = P.vel[3 * p], vy = P.vel[3 * p + 1], vz = P.vel[3 * p + 2];
        double a = 0.0;
        a += vx * vx;
        a += vy * vy;
        a += vz * vz;
        v[0] = m * a;
        v[1] = m * vx;
        v[2] = m * vy;
        v[3] = m * vz;
    }
    __shared__ double sh[4 * 32];
    block_sum<4>(v, sh);
    if (threadIdx.x == 0)
        for (int q = 0; q < 4; q++) P.partial[4 * bx + q] = v[q];
}
__global__ void k_ke_partial(ParticleDev P) { k_ke_partial_body(P, blockIdx.x); }

// red[2] = KE, red[3..5] = momentum, red[6] = T, red[7] = sqrt(T_target / T)
__device__ __forceinline__ void k_ke_final_body(const ParticleDev& P, int nblocks, double T_target, int bx) {
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int b = 0; b < nblocks; b++)
        for (int q = 0; q < 4; q++) s[q] += P.partial[4 * b + q];
    const double ke = 0.5 * s[0];
    P.red[2] = ke;
    P.red[3] = s[1];
    P.red[4] = s[2];
    P.red[5] = s[3];
    const double T = 2 * ke / (3 * P.np * kBoltzmannHartree);
    P.red[6] = T;
    P.red[7] = sqrt(T_target / T);
}
__global__ void k_ke_final(ParticleDev P, int nblocks, double T_target) { k_ke_final_body(P, nblocks, T_target, blockIdx.x); }

static void ke_reduce(ParticleDev& P, double T_target, cudaStream_t s) {
    const int nb = P.np > 0 ? (P.np + 255) / 256 : 1;
    count_launch();
    k_ke_partial<<<nb, 256, 0, s>>>(P);
    count_launch();
    k_ke_final<<<1, 1, 0, s>>>(P, nb, T_target);
    MZB_CHECK(cudaGetLastError());
}

void kinetic_and_momentum(ParticleDev& P, cudaStream_t s) { ke_reduce(P, 1.0, s); }

// ------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) and Box-Muller normals.
// Counter = (ion, draw, call_lo, call_hi), key = (seed_lo, seed_hi); each draw gives two
// normals from two 53-bit uniforms in (0,1).
// ------------------------------------------------------------------------------------
__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const uint32_t lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
        const uint32_t lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

__device__ __forceinline__ double u53(uint32_t hi, uint32_t lo) {
    const uint64_t a = ((uint64_t)hi << 32) | lo;
    return ((double)(a >> 11) + 0.5) * 0x1.0p-53;
}

__device__ void philox_normal3(uint64_t seed, uint64_t call, uint32_t ion, double z[3]) {
    for (uint32_t draw = 0; draw < 2; draw++) {
        uint32_t c[4] = {ion, draw, (uint32_t)call, (uint32_t)(call >> 32)};
        philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
        const double u1 = u53(c[0], c[1]), u2 = u53(c[2], c[3]);
        const double rad = sqrt(-2.0 * log(u1));
        double sn, cs;
        sincospi(2.0 * u2, &sn, &cs);
        z[2 * draw] = rad * cs;
        if (draw == 0) z[1] = rad * sn;
    }
}

__global__ void k_philox(uint64_t seed, uint64_t call, int np, double* out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    double z[3];
    philox_normal3(seed, call, (uint32_t)p, z);
    out[3 * p] = z[0];
    out[3 * p + 1] = z[1];
    out[3 * p + 2] = z[2];
}

void philox_normals(uint64_t seed, uint64_t call, int np, double* out, cudaStream_t s) {
    if (np == 0) return;
    count_launch();
    k_philox<<<(np + 127) / 128, 128, 0, s>>>(seed, call, np, out);
    MZB_CHECK(cudaGetLastError());
}

// ------------------------------------------------------------------------------------
// Integrators (integrator_verlet.c, integrator_ovrvo.c)
// ------------------------------------------------------------------------------------
__device__ __forceinline__ double wrap_box(double a, double L) {
    if (a < 0) return a + L;
    if (a >= L) return a - L;
    return a;
}

// Velocity Verlet part 1: optional rescale to the target T, half kick, drift, wrap.
__device__ __forceinline__ void k_verlet1_body(const ParticleDev& P, double dt, int rescale, int bx) {
    const int t = bx * blockDim.x + threadIdx.x;
    if (t >= 3 * P.np) return;
    const int p = t / 3;
    double v = P.vel[t];
    if (rescale) v *= P.red[7];
    v += 0.5 * dt * P.ft[t] / P.mass[p];
    P.vel[t] = v;
    P.pos[t] = wrap_box(P.pos[t] + dt * v, P.L);
}
__global__ void k_verlet1(ParticleDev P, double dt, int rescale) { k_verlet1_body(P, dt, rescale, blockIdx.x); }
__device__ __forceinline__ void k_verlet2_body(const ParticleDev& P, double dt, int bx) {
    const int t = bx * blockDim.x + threadIdx.x;
    if (t >= 3 * P.np) return;
    P.vel[t] += 0.5 * dt * P.ft[t] / P.mass[t / 3];
}
__global__ void k_verlet2(ParticleDev P, double dt) { k_verlet2_body(P, dt, blockIdx.x); }

// OVRVO: part1 = [O] V R, part2 = V [O]; O uses Philox normals for call `call`.
__device__ __forceinline__ void k_ovrvo_body(const ParticleDev& P, const IntegratorDev& I, int part, uint64_t call, int bx) {
    const int p = bx * blockDim.x + threadIdx.x;
    if (p >= P.np) return;
    if (I.ocalls_d != nullptr) call = *I.ocalls_d;
    const double m = P.mass[p];
    double v[3] = {P.vel[3 * p], P.vel[3 * p + 1], P.vel[3 * p + 2]};
    auto o_block = [&]() {
        const double c1s = sqrt(I.c1), var2 = (1 - I.c1) * kBoltzmannHartree * I.T;
        const double var1 = sqrt(var2 / m);
        double z[3];
        philox_normal3(I.seed, call, (uint32_t)p, z);
        for (int d = 0; d < 3; d++) {
            v[d] *= c1s;
            v[d] += var1 * z[d];
        }
    };
    auto v_block = [&]() {
        for (int d = 0; d < 3; d++) v[d] += 0.5 * I.dt * I.c2 * P.ft[3 * p + d] / m;
    };
    if (part == 1) {
        if (I.enabled) o_block();
        v_block();
        for (int d = 0; d < 3; d++) P.pos[3 * p + d] = wrap_box(P.pos[3 * p + d] + I.c2 * I.dt * v[d], P.L);
    } else {
        v_block();
        if (I.enabled) o_block();
    }
    for (int d = 0; d < 3; d++) P.vel[3 * p + d] = v[d];
}
__global__ void k_ovrvo(ParticleDev P, IntegratorDev I, int part, uint64_t call) { k_ovrvo_body(P, I, part, call, blockIdx.x); }

__device__ __forceinline__ void k_advance_counter_body(uint64_t* c, int bx) { *c += 1; }
__global__ void k_advance_counter(uint64_t* c) { k_advance_counter_body(c, blockIdx.x); }

static void advance_ocalls(IntegratorDev& I, cudaStream_t s) {
    if (!I.enabled) return;
    I.ocalls++;
    if (I.ocalls_d != nullptr) {
        count_launch();
        k_advance_counter<<<1, 1, 0, s>>>(I.ocalls_d);
    }
}

void integrator_part1(ParticleDev& P, IntegratorDev& I, cudaStream_t s) {
    if (P.np == 0) return;
    if (I.type == 1) {
        if (I.enabled) ke_reduce(P, I.T, s);
        count_launch();
        k_verlet1<<<(3 * P.np + 255) / 256, 256, 0, s>>>(P, I.dt, I.enabled);
    } else {
        count_launch();
        k_ovrvo<<<(P.np + 127) / 128, 128, 0, s>>>(P, I, 1, I.ocalls);
        advance_ocalls(I, s);
    }
    MZB_CHECK(cudaGetLastError());
}

void integrator_part2(ParticleDev& P, IntegratorDev& I, cudaStream_t s) {
    if (P.np == 0) return;
    if (I.type == 1) {
        count_launch();
        k_verlet2<<<(3 * P.np + 255) / 256, 256, 0, s>>>(P, I.dt);
    } else {
        count_launch();
        k_ovrvo<<<(P.np + 127) / 128, 128, 0, s>>>(P, I, 2, I.ocalls);
        advance_ocalls(I, s);
    }
    MZB_CHECK(cudaGetLastError());
}

// rescale_velocities (particles.c:841-857): per-type velocity sums accumulated serially
// in ion order (one thread per type and component), then v -= 2*sum/N.
__global__ void k_rescale_sum(ParticleDev P, double* iv) {
    const int t = threadIdx.x;
    if (t >= 3 * P.ntyp) return;
    const int typ = t / 3, d = t % 3;
    double s = 0.0;
    for (int p = 0; p < P.np; p++)
        if (P.types[p] == typ) s += P.vel[3 * p + d];
    iv[t] = s;
}
__global__ void k_rescale_apply(ParticleDev P, const double* iv) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * P.np) return;
    const int p = t / 3, d = t % 3;
    P.vel[t] -= 2 * iv[P.types[p] * 3 + d] / P.np;
}

void rescale_velocities(ParticleDev& P, cudaStream_t s) {
    if (P.np == 0) return;
    if (3 * P.ntyp > 1024) fatal("rescale_velocities: too many particle types");
    count_launch();
    k_rescale_sum<<<1, 3 * P.ntyp, 0, s>>>(P, P.partial);
    count_launch();
    k_rescale_apply<<<(3 * P.np + 255) / 256, 256, 0, s>>>(P, P.partial);
    MZB_CHECK(cudaGetLastError());
}

// ------------------------------------------------------------------------------------
// Replica tables (particles.cuh): the particle stages of a batched MD step, one launch per
// stage over all systems, each CTA running the per-system kernel's body for its system.
// ------------------------------------------------------------------------------------
namespace {

// The step's zeroing for one system, over one run of units: tile counts, the charge
// bitmap, cell counts, the bad-cell flag and the field solve's barrier words (and the whole
// charge grid when it does not hold only the last corners) -- what the per-system path
// clears with memsets.
constexpr int kZeroThreads = 256;
long zero_units(const StageArgs& a) {
    return (long)a.P.ntiles + a.mask_words + a.P.ncell + 1 + 4 + (a.q_sparse ? 0 : (long)a.n * a.n * a.n);
}
__device__ __forceinline__ void zero_body(const StageArgs& a, int bx) {
    long u = (long)bx * blockDim.x + threadIdx.x;
    const ParticleDev& P = a.P;
    if (u < P.ntiles) {
        P.tile_count[u] = 0;
        return;
    }
    u -= P.ntiles;
    if (u < a.mask_words) {
        a.qmask[u] = 0u;
        return;
    }
    u -= a.mask_words;
    if (u < P.ncell) {
        P.cell_count[u] = 0;
        return;
    }
    u -= P.ncell;
    if (u == 0) {
        P.flags[1] = 0;
        return;
    }
    u -= 1;
    if (u < 4) {
        reinterpret_cast<unsigned int*>(a.bar)[u] = 0u;
        return;
    }
    u -= 4;
    if (!a.q_sparse && u < (long)a.n * a.n * a.n) a.q[u] = 0.0;
}

__device__ __forceinline__ int blocks_of(long units, int per) { return (int)((units + per - 1) / per); }
// CTAs of the per-ion spreading kernel (their partial charge sums are summed by the scan)
__device__ __forceinline__ int spread_bin_blocks(const StageArgs& a) { return a.P.np > 0 ? blocks_of(a.P.np, 128) : 1; }

// CTAs of every stage for system a (the per-system launches' grids), into c[SK_COUNT]
void stage_blocks(const StageArgs& a, int* c) {
    const ParticleDev& P = a.P;
    const long np = P.np, nblk32 = (np + 31) / 32;
    const bool verlet = a.I.type == 1, has = np > 0;
    auto cdiv = [](long u, long per) { return (int)((u + per - 1) / per); };
    for (int k = 0; k < SK_COUNT; k++) c[k] = 0;
    c[SK_ZERO] = cdiv(zero_units(a), kZeroThreads);
    c[SK_KE] = has && verlet && a.I.enabled ? cdiv(np, 256) : 0;
    c[SK_KEF] = has && verlet && a.I.enabled ? 1 : 0;
    c[SK_INT1] = c[SK_INT2] = has ? cdiv(verlet ? 3 * np : np, 128) : 0;
    c[SK_ADV1] = c[SK_ADV2] = has && !verlet && a.I.enabled ? 1 : 0;
    c[SK_BIN] = has ? cdiv(np, 128) : 1;  // spread_bin_blocks
    c[SK_SCANR] = c[SK_SCANA] = cdiv(P.ntiles, 1024);
    c[SK_FILL] = has ? cdiv(np, 128) : 0;
    c[SK_IONS] = has ? cdiv(np, kIonsPerCta) : 0;
    c[SK_QCHK] = c[SK_SCHK] = 1;
    c[SK_FF] = has ? cdiv(8 * np, 128) : 0;
    c[SK_CCOUNT] = c[SK_CFILL] = has ? cdiv(np, 128) : 0;
    c[SK_CSCAN] = 1;
    c[SK_CSORT] = cdiv(P.ncell, 4);
    c[SK_TFBOX] = has ? cdiv(32 * nblk32, 256) : 0;
    c[SK_TF_TF] = has && P.pot == POT_TF ? P.tf_nst : 0;
    c[SK_TF_LJ] = has && P.pot == POT_LJ ? P.tf_nst : 0;
    c[SK_TF_SC] = has && P.pot == POT_SC ? P.tf_nst : 0;
    c[SK_TFG] = has ? cdiv(32 * nblk32, 128) : 0;
    c[SK_TFE] = 1;
    c[SK_TOT] = has ? cdiv(3 * np, 256) : 0;
}

#define MZB_TABLE_KERNEL(name, threads, ...)                                                                \
    __global__ void __launch_bounds__(threads) name(const StageArgs* __restrict__ A,                        \
                                                    const int* __restrict__ start, int nsys) {               \
        table_run(A, start, nsys, [&](const StageArgs& a, int b) { __VA_ARGS__; });                         \
    }

MZB_TABLE_KERNEL(kt_zero, kZeroThreads, zero_body(a, b))
MZB_TABLE_KERNEL(kt_ke, 256, k_ke_partial_body(a.P, b))
MZB_TABLE_KERNEL(kt_kef, 32, if (threadIdx.x == 0) k_ke_final_body(a.P, blocks_of(a.P.np, 256), a.I.T, b))
MZB_TABLE_KERNEL(kt_int1, 128,
                 if (a.I.type == 1) k_verlet1_body(a.P, a.I.dt, a.I.enabled, b);
                 else k_ovrvo_body(a.P, a.I, 1, a.I.ocalls, b))
MZB_TABLE_KERNEL(kt_int2, 128,
                 if (a.I.type == 1) k_verlet2_body(a.P, a.I.dt, b);
                 else k_ovrvo_body(a.P, a.I, 2, a.I.ocalls, b))
MZB_TABLE_KERNEL(kt_adv, 32, if (threadIdx.x == 0) k_advance_counter_body(a.I.ocalls_d, b))
MZB_TABLE_KERNEL(kt_bin, 128, k_spread_bin_body<CAS_CIC>(a.P, a.n, a.h, a.P.partial, a.q_sparse ? a.q : nullptr, b))
MZB_TABLE_KERNEL(kt_scanr, 1024, k_scan_reduce_body(a.P.tile_count, a.P.ntiles, a.P.tile_part, b))
MZB_TABLE_KERNEL(kt_scana, 1024,
                 k_scan_apply_body(a.P.tile_count, a.P.ntiles, a.P.tile_part, a.P.tile_start, a.P.tile_fill,
                                   a.P.partial, spread_bin_blocks(a), a.P.red + 0, b))
MZB_TABLE_KERNEL(kt_fill, 128, k_spread_fill_body(a.P, b))
MZB_TABLE_KERNEL(kt_ions, kSpreadIonThreads, k_spread_ions_body(a.P, a.q, a.qmask, a.n, a.h, b))
// the charge check of solver_update_charges (solver_md.c:98-102) and the solve's status,
// kept on the device and read after the call
MZB_TABLE_KERNEL(kt_qchk, 32, if (threadIdx.x == 0) {
    const double q = a.P.red[0];
    if (fabs(*a.qtot - q) > 1e-6) a.err[0] = 1;
    *a.qtot = q;
})
MZB_TABLE_KERNEL(kt_schk, 32, if (threadIdx.x == 0 && (a.result[0] < 0 || a.result[1] != 0)) a.err[2] = 1)
MZB_TABLE_KERNEL(kt_ff, 128, k_field_forces_body<CAS_CIC>(a.P, a.phi, a.n, a.h, b))
MZB_TABLE_KERNEL(kt_ccount, 128, k_cell_count_body(a.P, b))
MZB_TABLE_KERNEL(kt_cscan, 1024,
                 k_scan_body(a.P.cell_count, a.P.ncell, a.P.cell_start, a.P.cell_fill, nullptr, 0, nullptr, b))
MZB_TABLE_KERNEL(kt_cfill, 128, k_cell_fill_body(a.P, b))
MZB_TABLE_KERNEL(kt_csort, 128, k_cell_sort_gather_body(a.P, b))
MZB_TABLE_KERNEL(kt_tot, 256, k_total_forces_body(a.P, b))

#undef MZB_TABLE_KERNEL

void tlaunch(const StageTable& t, int k, void (*kernel)(const StageArgs*, const int*, int), int threads,
             cudaStream_t s) {
    if (t.total[k] <= 0) return;
    count_launch();
    kernel<<<t.total[k], threads, 0, s>>>(t.args, t.start + k * (t.nsys + 1), t.nsys);
    MZB_CHECK(cudaGetLastError());
}

}  // namespace

bool stage_table_ok(const StageArgs& a) { return a.P.cas == CAS_CIC && a.P.fdb == nullptr; }

StageTable stage_table_build(const std::vector<StageArgs>& a) {
    StageTable t;
    t.nsys = (int)a.size();
    const int w = t.nsys + 1;
    std::vector<int> start((size_t)SK_COUNT * w, 0);
    int c[SK_COUNT];
    for (int r = 0; r < t.nsys; r++) {
        stage_blocks(a[r], c);
        for (int k = 0; k < SK_COUNT; k++) start[(size_t)k * w + r + 1] = start[(size_t)k * w + r] + c[k];
    }
    for (int k = 0; k < SK_COUNT; k++) t.total[k] = start[(size_t)k * w + t.nsys];
    t.args = static_cast<StageArgs*>(dev_alloc(sizeof(StageArgs) * a.size()));
    t.start = static_cast<int*>(dev_alloc(sizeof(int) * start.size()));
    MZB_CHECK(cudaMemcpy(t.args, a.data(), sizeof(StageArgs) * a.size(), cudaMemcpyHostToDevice));
    MZB_CHECK(cudaMemcpy(t.start, start.data(), sizeof(int) * start.size(), cudaMemcpyHostToDevice));
    return t;
}

void stage_table_free(StageTable& t) {
    dev_free(t.args);
    dev_free(t.start);
    t = StageTable{};
}

void stages_before_solve(const StageTable& t, cudaStream_t s) {
    tlaunch(t, SK_ZERO, kt_zero, kZeroThreads, s);
    tlaunch(t, SK_KE, kt_ke, 256, s);
    tlaunch(t, SK_KEF, kt_kef, 32, s);
    tlaunch(t, SK_INT1, kt_int1, 128, s);
    tlaunch(t, SK_ADV1, kt_adv, 32, s);
    tlaunch(t, SK_BIN, kt_bin, 128, s);
    tlaunch(t, SK_SCANR, kt_scanr, 1024, s);
    tlaunch(t, SK_SCANA, kt_scana, 1024, s);
    tlaunch(t, SK_FILL, kt_fill, 128, s);
    tlaunch(t, SK_IONS, kt_ions, kSpreadIonThreads, s);
    tlaunch(t, SK_QCHK, kt_qchk, 32, s);
}

void stages_after_solve(const StageTable& t, cudaStream_t s) {
    tlaunch(t, SK_SCHK, kt_schk, 32, s);
    tlaunch(t, SK_FF, kt_ff, 128, s);
    tlaunch(t, SK_CCOUNT, kt_ccount, 128, s);
    tlaunch(t, SK_CSCAN, kt_cscan, 1024, s);
    tlaunch(t, SK_CFILL, kt_cfill, 128, s);
    tlaunch(t, SK_CSORT, kt_csort, 128, s);
    tf_stages(t, s);
    tlaunch(t, SK_TOT, kt_tot, 256, s);
    tlaunch(t, SK_INT2, kt_int2, 128, s);
    tlaunch(t, SK_ADV2, kt_adv, 32, s);
}

}  // namespace mzb
