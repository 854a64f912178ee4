// Particle-side kernels of the MD step: CIC charge spreading, linked cells, field-force
// interpolation, Tosi-Fumi pair forces, integrators and reductions.
#pragma once

#include <vector>

#include "mzb_common.cuh"

namespace mzb {

// Spreading tile: TI x TJ x TK grid points written by one warp (one k column of TI x TJ
// points per lane); TI >= 2 so the splines' -1..2 stencils reach at most one tile either
// way.
constexpr int kTileI = 2, kTileJ = 8, kTileK = 32;
constexpr int kTileCap = 1024;  // candidate ions one tile's warp sorts in shared memory (more take a slower path)

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
    int* flags = nullptr;            // [0] unused, [1] a coordinate outside [0, L) (cell clamping)
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

// ------------------------------------------------------------------------------------
// Replica tables: each particle stage of the batched MD step as ONE launch over all the
// systems of the batch. The launch's CTAs are the systems' own grids of that stage laid
// end to end (start[r] .. start[r + 1] for system r, per stage); every CTA finds its
// system, stages that system's StageArgs in shared memory and runs the stage's kernel
// body with its block index inside the system's grid -- the same body, block for block,
// as the per-system launch, so the results are the same.
// ------------------------------------------------------------------------------------
struct StageArgs {
    ParticleDev P;
    IntegratorDev I;            // ocalls_d set: the Philox counter lives on the device
    double* q = nullptr;        // charge grid (n^3)
    uint32_t* qmask = nullptr;  // its bitmap of runs of 64 k (n % 64 == 0), or null
    int mask_words = 0;
    int n = 0;
    double h = 0;
    int q_sparse = 1;           // q holds only the CIC corners of the ions' base cells (else cleared whole)
    const double* phi = nullptr;  // the field the step's solve writes
    double* qtot = nullptr;       // device charge total of the last step
    int* err = nullptr;           // device error words ([0] charge drift, [2] solve failure)
    const int* result = nullptr;  // the solve's result words
    GridBarrier* bar = nullptr;   // the solve team's barrier (zeroed at the start of the step)
};

// The system of this CTA in a launch over a replica table (the last r with start[r] <=
// blockIdx.x: systems without CTAs in the launch have start[r] == start[r + 1]), its
// arguments staged in shared memory, and f(args, block index inside the system's grid).
template <class F>
__device__ __forceinline__ void table_run(const StageArgs* __restrict__ A, const int* __restrict__ start, int nsys,
                                          F&& f) {
    // raw storage: StageArgs has default member initialisers, and a __shared__ object of it
    // would have every thread store them at its declaration, racing with the copy below
    __shared__ __align__(16) unsigned char a_raw[sizeof(StageArgs)];
    StageArgs& a = *reinterpret_cast<StageArgs*>(a_raw);
    int lo = 0, hi = nsys - 1;
    const int b = (int)blockIdx.x;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    const int* src = reinterpret_cast<const int*>(A + lo);
    int* dst = reinterpret_cast<int*>(a_raw);
    for (int w = threadIdx.x; w < (int)(sizeof(StageArgs) / sizeof(int)); w += blockDim.x) dst[w] = src[w];
    __syncthreads();
    f(a, b - start[lo]);
}

enum StageKind {
    SK_ZERO, SK_KE, SK_KEF, SK_INT1, SK_ADV1, SK_BIN, SK_SCANR, SK_SCANA, SK_FILL, SK_IONS, SK_QCHK,
    SK_SCHK, SK_FF, SK_CCOUNT, SK_CSCAN, SK_CFILL, SK_CSORT, SK_TFBOX, SK_TF_TF, SK_TF_LJ, SK_TF_SC, SK_TFG,
    SK_TFE, SK_TOT, SK_INT2, SK_ADV2, SK_COUNT
};

struct StageTable {
    int nsys = 0;
    StageArgs* args = nullptr;  // device [nsys]
    int* start = nullptr;       // device [SK_COUNT][nsys + 1]
    int total[SK_COUNT] = {};   // CTAs of each stage's launch (0: not launched)
};

// Whether a system can be stepped through the tables (CIC charge assignment).
bool stage_table_ok(const StageArgs& a);
// Per-stage CTA counts of every system and the device copies of the table.
StageTable stage_table_build(const std::vector<StageArgs>& a);
void stage_table_free(StageTable& t);
// The stages before the field solve (integrator part 1, charge spreading, charge check,
// zeroing of the step's counters and the solve's barriers), and after it (solve check,
// field forces, linked cells, pair forces, total forces, integrator part 2).
void stages_before_solve(const StageTable& t, cudaStream_t s);
void stages_after_solve(const StageTable& t, cudaStream_t s);
// The pair-force stages (tf_forces.cu): boxes, pair forces, gather, energy.
void tf_stages(const StageTable& t, cudaStream_t s);

}  // namespace mzb
