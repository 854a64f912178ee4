// Mixed-precision field solve (see mixed.cu).
#pragma once

#include "mzb_common.cuh"

namespace mzb {

constexpr int kMixedMaxLevels = 10;

struct MixedArgs {
    int prog;           // PROG_INIT_FIELD, PROG_LCG_UPDATE, PROG_MAZE_LCG, PROG_MG_UPDATE, PROG_MAZE_MG
    int n;
    double tol;         // absolute inf-norm tolerance on the FP64 residual
    double c;           // right-hand-side constant (as the FP64 programs)
    int max_outer;      // refinement steps before giving up (-1 returned)
    int cycles;         // V-cycles per refinement step
    int nu1, nu2;       // red-black GS sweeps before / after the coarse correction
    int coarse_sweeps;  // sweeps on the coarsest level
    int nlev;
    int lev_n[kMixedMaxLevels];
    float* lev_x[kMixedMaxLevels];
    float* lev_b[kMixedMaxLevels];
    float* lev_r[kMixedMaxLevels];
    const double* q;
    const double* phi_old;
    const double* phi_prev;
    double* phi_new;
    double* y;
    double* tmp;        // FP64 right-hand side
    double* partials;   // >= 4 x gridDim.x doubles
    GridBarrier* bar;
    int* result;        // [0] refinement steps taken or -1, [1] status (0 ok)
};

// Level sizes n, n/2, ... while the next size is even and >= 4; returns the count.
int mixed_levels(int n, int* sizes);
void mixed_launch(const MixedArgs& a, cudaStream_t stream);

}  // namespace mzb
