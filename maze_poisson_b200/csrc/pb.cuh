// Poisson-Boltzmann implicit solvent: the face dielectric coefficients and screening term
// built from the solvation shells of the ions, the coefficients the PB operator and its
// V-cycle read, and the dielectric-boundary, ionic-boundary and non-polar forces.
#pragma once

#include "mzb_common.cuh"

namespace mzb {

struct PbGrid {
    int n = 0;
    double h = 0, w = 0, eps_s = 1, eps_int = 1, kbar2 = 0;
    int nonpolar = 0;
    // n^3: +x/+y/+z face coefficients of each point, its screening term, and the
    // operator diagonal dg = ex_c + ex_{x-1} + ey_c + ey_{y-1} + ez_c + ez_{z-1} + k2_c
    double *ex = nullptr, *ey = nullptr, *ez = nullptr, *k2 = nullptr, *dg = nullptr;
    // (n/2)^3 coefficients of the PB V-cycle's coarse grid (null on non-multigrid grids)
    double *cex = nullptr, *cey = nullptr, *cez = nullptr, *ck2 = nullptr, *cdg = nullptr;
};

// grid_update_eps_and_k2 (grid_general.c:138-301) for ions at pos (n_p x 3, bohr) with
// solvation radii `radii`, then the diagonal and, when allocated, the coarse coefficients
// (restriction_eps / restriction_k2screen, multigrid_pb.c:330-527).
void pb_update_coefficients(const PbGrid& G, const double* pos, const double* radii, int np,
                            cudaStream_t s);
// Diagonal and coarse coefficients of G from its ex/ey/ez/k2 (kernel-level entry points).
void pb_derive(const PbGrid& G, cudaStream_t s);

// particles_compute_forces_pb (particles.c:420-775): fdb, fib, fnp (n_p x 3) from phi.
// `part` holds n_p * (2 range_max + 1) * 9 doubles; range_max bounds
// floor((r_s + w)/h) + 2 over the ions. cdb = h / (8 pi), cnp = -gamma_np h / (eps_s - eps_int).
void pb_forces(const PbGrid& G, const double* phi, const double* pos, const double* radii, int np,
               int range_max, double cdb, double cnp, double* part, double* fdb, double* fib,
               double* fnp, cudaStream_t s);

}  // namespace mzb
