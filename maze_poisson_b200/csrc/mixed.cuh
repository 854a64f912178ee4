// Multigrid field solve with FP64 refinement (see mixed.cu): FP32 levels (the
// mixed-precision form) or FP64 levels (the FP64 multigrid form).
#pragma once

#include "mzb_common.cuh"

namespace mzb {

constexpr int kMixedMaxLevels = 10;
constexpr int kMixedSmallN = 16;     // levels with n <= this live in CTA 0's shared memory
constexpr int kMixedMaxN = 1024;     // largest grid of the mixed solver (32-bit offsets in a level)
constexpr int kMixedStampSlots = 2 + 8 * 8 + 8;  // + coarse-FFT pass stamps of refinement 1

struct MixedArgs {
    int prog;           // PROG_INIT_FIELD, PROG_LCG_UPDATE, PROG_MAZE_LCG, PROG_MG_UPDATE, PROG_MAZE_MG
    int n;
    double tol;         // absolute inf-norm tolerance on the FP64 residual
    double c;           // right-hand-side constant (as the FP64 programs)
    int max_outer;      // refinement steps before giving up (-1 returned)
    int nu1, nu2;       // red-black GS sweeps before / after the coarse correction (>= 1)
    int coarse_sweeps;  // sweeps on the coarsest level (>= 1) when coarse_g is null
    int fp64;               // 1: level arrays and V-cycle in FP64, 0: in FP32
    const void* coarse_g;   // Green's function of the coarsest level (mixed_coarse_green), stored
                            // like the levels (float or double), or null
    int coarse_team;        // 1: the coarsest level is solved by every CTA of the team with coarse_g
    int coarse_fft;         // 1: the coarsest level (32, 64 or 128 per side) is solved by every CTA
                            // of the team by FFT, in coarse_spec
    void* coarse_spec;      // n (n/2 + 1) n complex values (float2, or double2 when fp64)
    int level0_fp16;        // 1 (FP32 levels, n = 128 or 256): level 0's x, b and r are stored as
                            // FP16 in units of the last residual's max (lev_x/b/r[0] hold n^3 halves)
    double* scale_hint;     // device: the first residual max of the last solve of this grid (0:
                            // none yet), the first scale of an FP16 level 0; or null
    int nlev;
    int lsmall;         // first level held in shared memory (nlev if none; >= 1)
    int lev_n[kMixedMaxLevels];
    void* lev_x[kMixedMaxLevels];  // level arrays: float, or double when fp64
    void* lev_b[kMixedMaxLevels];
    void* lev_r[kMixedMaxLevels];
    const double* q;
    const uint32_t* qmask;  // segments of 64 k where q may be nonzero (spread_charges), or null
    const double* phi_old;
    const double* phi_prev;
    double* phi_new;
    double* y;
    double* tmp;        // FP64 right-hand side (MaZe programs)
    double* partials;   // >= 4 x gridDim.x doubles
    GridBarrier* bar;
    int* result;        // [0] refinement steps taken or -1, [1] status (0 ok)
    unsigned long long* stamps;  // optional phase time stamps (kMixedStampSlots) or null
};

// Level sizes n, n/2, ... while the next size is even and >= 4; returns the count.
int mixed_levels(int n, int* sizes);
// First level with n <= kMixedSmallN (nlev if none).
int mixed_small_level(int nlev, const int* sizes);
// Largest coarsest level solved directly in CTA 0's shared memory (n^3 values of its
// Green's function).
constexpr int kMixedDirectN = 6;
// The hierarchy stops at the first level of at most this many points per side, which
// every CTA of the team solves directly: a slice of the convolution with its Green's
// function each (see mixed.cu).
constexpr int kMixedTeamDirectN = 16;
// Coarse levels the team solves by FFT (mixed_fft_coarse_ok): 32, 64 or 128 points per side.
inline bool mixed_fft_coarse_ok(int nc) { return nc == 32 || nc == 64 || nc == 128; }
// Pseudo-inverse kernel of the unscaled periodic 7-point Laplacian on an n^3 grid:
// g[d] = (1/n^3) sum_{k != 0} cos(2 pi k.d / n) / lambda(k),
// lambda(k) = 2 cos(2 pi k1/n) + 2 cos(2 pi k2/n) + 2 cos(2 pi k3/n) - 6.
void mixed_coarse_green(int n, double* g);
void mixed_coarse_green(int n, float* g);
void mixed_launch(const MixedArgs& a, cudaStream_t stream);
// Dynamic shared memory one system's solve needs.
size_t mixed_smem_bytes(const MixedArgs& a);
// CTAs of a full (one per SM) launch on the current device.
int mixed_grid_blocks();
// Solve nsys systems (FP32 levels) in one cooperative launch of nblocks CTAs: system r (list[r], in
// device memory) is worked by CTAs [start[r], start[r+1]), start[nsys] = nblocks, each
// team on its own barrier (zeroed by the caller) and partials. smem is the largest
// mixed_smem_bytes of the list.
void mixed_batch_launch(const MixedArgs* list, const int* start, int nsys, int nblocks, size_t smem,
                        cudaStream_t stream);

}  // namespace mzb
