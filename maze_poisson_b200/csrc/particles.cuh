// Particle-side kernels of the MD step: CIC charge spreading, linked cells, field-force
// interpolation, Tosi-Fumi pair forces, integrators and reductions.
#pragma once

#include "mzb_common.cuh"

namespace mzb {

// Spreading tile: TI x TJ x TK grid points written by one warp (one k column of TI x TJ
// points per lane); TI >= 2 so the splines' -1..2 stencils reach at most one tile either
// way.
constexpr int kTileI = 2, kTileJ = 8, kTileK = 32;
constexpr int kTileCap = 1024;  // candidate ions one tile's warp can hold (see spread_tiles)

// Charge assignment schemes (particles.c:28): CIC (8 points), quadratic and cubic
// B-splines (4 x 4 x 4 = 64 points, offsets -1..2 around floor(pos/h)).
enum CasType { CAS_CIC = 0, CAS_SPL_QUADR = 1, CAS_SPL_CUBIC = 2 };
// Pair potentials (particles.c:17): Tosi-Fumi, Lennard-Jones, soft-core repulsion.
enum PotType { POT_TF = 0, POT_LJ = 1, POT_SC = 2 };

// Pair-potential constants per type pair in ParticleDev::tab: Tosi-Fumi [A, B, C, D,
// sigma, alpha, beta, r^2 beyond which the exponential terms are dropped], Lennard-Jones
// [sigma, epsilon, alpha, beta], soft core [nu, d, B, alpha, beta].
constexpr int kPairConsts = 8;

struct ParticleDev {
    int np = 0, ntyp = 0, n = 0;
    double L = 0, h = 0, rcut = 0;
    int32_t* types = nullptr;
    double* pos = nullptr;
    double* vel = nullptr;
    double* fe = nullptr;
    double* fn = nullptr;
    double* ft = nullptr;
    double* mass = nullptr;
    double* chg = nullptr;
    double* tab = nullptr;   // [ntyp*ntyp][kPairConsts] pair-potential constants per type pair
    int32_t* base = nullptr; // [np][3] base cell floor(pos/h) (wrapped)
    int cas = CAS_CIC;       // charge assignment scheme
    // the charge grid whose only nonzeros are the CIC corners of `base` (left by the last
    // CIC spreading into it), or null: the next CIC spreading into it zeroes those corners
    // instead of the whole grid
    const double* q_sparse = nullptr;
    int pot = POT_TF;        // pair potential

    // spreading bins
    int ntiles = 0, nti = 0, ntj = 0, ntk = 0;
    int32_t* tile_count = nullptr;   // [ntiles]
    int32_t* tile_start = nullptr;   // [ntiles+1]
    int32_t* tile_fill = nullptr;    // [ntiles]
    int32_t* tile_ions = nullptr;    // [np]
    int32_t* tile_part = nullptr;    // [ceil(ntiles / 1024)] per-block totals of the tile scan

    // linked cells (Tosi-Fumi)
    int nc = 0, ncell = 0;
    int32_t* cell_of = nullptr;      // [np]
    int32_t* cell_count = nullptr;   // [ncell]
    int32_t* cell_start = nullptr;   // [ncell+1]
    int32_t* cell_fill = nullptr;    // [ncell]
    int32_t* cell_ions = nullptr;    // [np]
    int32_t* srank = nullptr;        // [np] position of ion p in cell order
    double* spos = nullptr;          // [np][3] positions in cell order
    int32_t* stype = nullptr;        // [np]
    // pair-force plan (tf_forces.cu): super-tiles of 8 x 8 blocks of 32 cell-ordered ions
    int tf_nst = 0;                  // super-tiles (CTAs of the pair-force kernel)
    int* tf_st = nullptr;            // [tf_nst][2] (I super-block, J super-block)
    int* tf_gstart = nullptr;        // [nblk + 1] gather-list offsets per block
    int* tf_gent = nullptr;          // gather entries (super-tile << 4 | side << 3 | slot)
    double* tf_box = nullptr;        // [nblk][6] bounding boxes of the blocks
    double* fpart = nullptr;         // [tf_nst][2][8][32][3] force partials
    double* epart = nullptr;         // [tf_nst] energy partials

    // Poisson-Boltzmann (solver_initialize_particles_pois_boltz, particles.c:111-127);
    // fdb/fib/fnp are null unless it was called
    double* radii = nullptr;         // [np] solvation radii
    double* fdb = nullptr;           // [np][3] dielectric-boundary forces
    double* fib = nullptr;           // [np][3] ionic-boundary forces
    double* fnp = nullptr;           // [np][3] non-polar forces
    double* pb_part = nullptr;       // [np][2 pb_range + 1][9] force partials
    int pb_range = 0;                // largest floor((r_s + w)/h) + 2 (0: not sized yet)
    double gamma_np = 0, beta_np = 0;

    // scalars
    double* red = nullptr;           // reduction outputs (device)
    int* flags = nullptr;            // [0] spread overflow, [1] bad cell index
    double* partial = nullptr;       // block partials
};

// Build the CIC base cells, the tile bins and q (bit-identical to the reference's serial
// update_charges). Writes the spread total charge to red[0].
// qmask (n % 64 == 0, else null): one bit per run of 64 consecutive k of a grid row, set
// where the spreading may have written a nonzero charge (readers may skip the others).
void spread_charges(ParticleDev& P, double* q, uint32_t* qmask, int n, double h, cudaStream_t s);
// Forces from -grad(phi) at the 8 CIC corners (forces.c:26-100) into P.fe.
void field_forces(ParticleDev& P, const double* phi, int n, double h, cudaStream_t s);
// Linked cells (counting sort, stable by ion index) + Tosi-Fumi forces into P.fn;
// pair energy / 2 into red[1].
void build_cells(ParticleDev& P, cudaStream_t s);
// Super-tile list, gather lists and partial buffers of the pair-force kernel for P.np.
void tf_plan(ParticleDev& P);
void tf_forces(ParticleDev& P, cudaStream_t s);
// fcs_tot = fcs_elec + fcs_noel (+ fcs_db + fcs_ib + fcs_np when set; particles.c:777-795)
void total_forces(ParticleDev& P, cudaStream_t s);
// Kinetic energy into red[2] and momentum into red[3..5] (particles.c:798-839).
void kinetic_and_momentum(ParticleDev& P, cudaStream_t s);

struct IntegratorDev {
    int type = 1;      // 0 OVRVO, 1 VERLET
    int enabled = 0;
    double dt = 0, T = 0, c1 = 1, c2 = 1;
    uint64_t seed = 0x5eedULL;
    uint64_t ocalls = 0;  // O-blocks applied so far (Philox counter)
    // When set (batched steps replayed from a CUDA graph), the Philox counter lives in
    // device memory: k_ovrvo reads it and a one-thread kernel advances it.
    uint64_t* ocalls_d = nullptr;
};

void integrator_part1(ParticleDev& P, IntegratorDev& I, cudaStream_t s);
void integrator_part2(ParticleDev& P, IntegratorDev& I, cudaStream_t s);
void rescale_velocities(ParticleDev& P, cudaStream_t s);

// Philox4x32-10 standard normals of the O-block (O-block call `call`, ion `ion`,
// components 0..2) written to out[3*ion + d] for ion < np.
void philox_normals(uint64_t seed, uint64_t call, int np, double* out, cudaStream_t s);

}  // namespace mzb
