// Persistent "solver engine": one cooperative launch runs a whole field solve (CG, PCG,
// V-cycles, MaZe constraint solve) with grid barriers between the sweeps, so no solve
// pays a launch or a host round trip per iteration.
#pragma once

#include <vector>

#include "mzb_common.cuh"

namespace mzb {

enum EngineProg : int {
    PROG_LAPLACE = 1,     // out = L u
    PROG_CG = 2,          // conj_grad(b, x0 -> x)                      plcg.c:28-90
    PROG_PCG = 3,         // conj_grad_precond(b, x0 -> x, precond)     plcg.c:104-166
    PROG_SMOOTH = 4,      // x <- RBGS^sm (rhs=b, x)                    multigrid.c:636-729
    PROG_RESTRICT = 5,    // out(coarse) = R27 u(fine)                  multigrid.c:523-594
    PROG_PROLONG = 6,     // out(fine) = P u(coarse)                    multigrid.c:393-463
    PROG_CG_COARSE = 7,   // cg_coarse(b, x) on n^3                     multigrid.c:13-96
    PROG_MG_APPLY = 8,    // one V-cycle: x <- MG(b, x)                 multigrid.c:99-168
    PROG_INIT_FIELD = 9,  // y=0; phi_prev=phi; phi = CG(c*q, 0)        grid_lcg.c:100-124
    PROG_LCG_UPDATE = 10, // phi_prev=phi; phi = CG(c*q, phi_prev)      grid_lcg.c:126-149
    PROG_MAZE_LCG = 11,   // verlet_poisson                             verlet.c:31-71
    PROG_MG_UPDATE = 12,  // multigrid_grid_update_field                grid_multigrid.c:110-212
    PROG_MAZE_MG = 13,    // verlet_poisson_multigrid                   verlet.c:86-149
    PROG_SSOR = 14,       // out = SSOR^-1 u                            precond_ssor.c:1240-1252
    PROG_BLOCKJACOBI = 15,// out = block-Jacobi^-1 u                    precond_blockjacobi.c:173-206
};

// The reference's preconditioner numbers (grid_general.c:16) for IMPLICIT (its NONE: the
// implicit 1/6 scaling of conj_grad), JACOBI, MG and SSOR; PC_NONE is an unpreconditioned
// CG, p = -r (the PB coarse solve, multigrid_pb.c:16-97).
enum PrecondKind : int { PC_IMPLICIT = 0, PC_JACOBI = 1, PC_MG = 2, PC_SSOR = 3, PC_BLOCKJACOBI = 4, PC_NONE = 5 };

// Block-Jacobi blocks: 10^3 points (precond_blockjacobi.c:10)
constexpr int kBlockJacobiB = 10, kBlockJacobiB3 = 1000;

struct EngineArgs {
    int prog;
    int n;          // fine grid points per side
    int precond;    // PrecondKind for PROG_PCG / PROG_MAZE_LCG
    int sm;         // RBGS sweeps per V-cycle half (PROG_SMOOTH / PROG_MG_APPLY)
    int maxit;      // PROG_CG_COARSE
    double tol;     // absolute inf-norm tolerance
    double rtol;    // PROG_CG_COARSE
    double c;       // right-hand-side constant applied to q

    // field state (PROG_INIT_FIELD .. PROG_MAZE_MG)
    const double* q;
    const double* phi_old;   // phi at entry
    const double* phi_prev;  // phi_prev at entry
    double* phi_new;         // phi at exit (never aliases phi_old / phi_prev)
    double* y;

    // kernel-level programs
    const double* b;
    const double* x0;
    double* x;
    const double* u;
    double* out;

    // fine work arrays (n^3)
    double* r;
    double* p0;
    double* p1;
    double* Ap;
    double* v;
    double* rf;
    double* tmp;
    // coarse work arrays ((n/2)^3)
    double* rc;
    double* ec;
    double* cr;
    double* cp0;
    double* cp1;
    double* cAp;

    // Poisson-Boltzmann operator (pb != 0, laplace.c:77-145): +x/+y/+z face coefficients
    // and the diagonal (six faces + k2) of the n^3 grid, and the same for the (n/2)^3
    // grid of the PB V-cycle (multigrid_pb.c:270-328)
    int pb;
    const double *ex, *ey, *ez, *dg;
    const double *cex, *cey, *cez, *cdg;

    // inverse of one 10^3 block's Laplacian (1000 x 1000, row-major), PC_BLOCKJACOBI
    const double* bj_inv;

    double* partials;  // 2 sets x 8 values x gridDim.x
    GridBarrier* bar;
    int* result;       // [0] program return value, [1] engine status (0 ok)
    unsigned long long* stamps;  // optional phase timestamps of the CG kernel (or null)
};

// Launch the engine for `a` on `stream` (cooperative; shapes chosen once per device).
void engine_launch(const EngineArgs& a, cudaStream_t stream);
// Launch a CG program (PROG_CG, PROG_PCG with Jacobi, PROG_INIT_FIELD, PROG_LCG_UPDATE,
// PROG_MAZE_LCG without MG) on the TMA-staged kernel of cg_fast.cu; false when the grid
// size or device does not allow it (the caller then uses engine_launch).
bool cg_fast_launch(const EngineArgs& a, cudaStream_t stream);
int cg_fast_stamp_slots();
// The inverse of the 7-point Laplacian of one 10^3 block with Dirichlet edges
// (precond_blockjacobi.c:14-69), row-major 1000 x 1000, computed once on the host.
const std::vector<double>& block_jacobi_inverse();
// Bytes of partials the engine needs and its grid size on this device.
int engine_grid_blocks();

}  // namespace mzb
