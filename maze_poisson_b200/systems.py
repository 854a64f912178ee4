"""Seeded synthetic molten-salt (Na+/Cl-) systems.

The reference measures on no public dataset; its runs start from lattice or restart
files (examples/). These systems follow that recipe:

* ncell^3 cubic cells of side a = L/ncell, each with a Na+ at the corner and a Cl- at
  the body centre (the 2-ion cell of maze_poisson/cli/utilities/bcc_generate.py:17-32),
  so N = 2 ncell^3 (250 / 2000 / 16000 for ncell = 5 / 10 / 20);
* uniform jitter U(-0.1 a, 0.1 a) per coordinate from numpy.random.default_rng(seed),
  wrapped into [0, L);
* L from the mass density: L[A] = ((N/2) * 58.443 / N_A / rho)^(1/3) * 1e8;
* Maxwell-Boltzmann velocities at T (a.u.), centre-of-mass drift removed;
* Tosi-Fumi NaCl parameters (kJ/mol, A) converted to atomic units exactly as
  maze_poisson/solver.py:198-202 does.

Units are atomic (bohr, Hartree, electron mass, a.u. of time), constants from
maze_poisson/constants.py.
"""
import dataclasses
import os

import numpy as np

A0 = 0.529177210903            # A per bohr
T_AU_FS = 2.4188843265857e-2   # fs per a.u. of time
AMU_TO_KG = 1.66054e-27
M_E = 9.1093837e-31
CONV_MASS = AMU_TO_KG / M_E
KB = 3.1668e-6                 # Hartree / K
KJMOL_TO_HARTREE = 0.0003808798
N_AVOGADRO = 6.02214076e23
NACL_MOLAR_MASS = 58.443       # g/mol

SPECIES = (("Na", 1.0, 22.99), ("Cl", -1.0, 35.453))  # type, charge, mass [amu]
# Tosi-Fumi NaCl: (type1, type2, A [kJ/mol], B [1/A], C [kJ/mol A^6], D [kJ/mol A^8], sigma [A])
TOSI_FUMI = (
    ("Na", "Na", 25.4435, 3.1546, 101.1719, 48.1771, 2.340),
    ("Na", "Cl", 20.3548, 3.1546, 674.4793, 837.0770, 2.755),
    ("Cl", "Cl", 15.2661, 3.1546, 6985.6786, 14031.5785, 3.170),
)


def box_length_ang(n_ions, density):
    """Cubic box side [A] holding n_ions/2 NaCl formula units at `density` g/cm^3."""
    return ((n_ions / 2) * NACL_MOLAR_MASS / N_AVOGADRO / density) ** (1.0 / 3.0) * 1e8


def tf_params_au():
    """[2][2][A,B,C,D,sigma] in a.u., flattened (the pot_params of solver_initialize_particles)."""
    names = [s[0] for s in SPECIES]
    arr = np.full((2, 2, 5), np.nan)
    for t1, t2, A, B, C, D, s in TOSI_FUMI:
        v = np.array([A, B, C, D, s], dtype=np.float64)
        i, j = names.index(t1), names.index(t2)
        arr[i, j] = v
        arr[j, i] = v
    arr[:, :, 0] *= KJMOL_TO_HARTREE
    arr[:, :, 1] *= A0
    arr[:, :, 2] *= KJMOL_TO_HARTREE / A0 ** 6
    arr[:, :, 3] *= KJMOL_TO_HARTREE / A0 ** 8
    arr[:, :, 4] /= A0
    return np.ascontiguousarray(arr.reshape(-1), dtype=np.float64)


@dataclasses.dataclass
class MoltenSalt:
    ncell: int
    n_grid: int
    density: float
    T: float
    seed: int
    L: float                 # bohr
    h: float                 # bohr
    types: np.ndarray        # int32 [N]
    pos: np.ndarray          # float64 [N, 3] bohr
    vel: np.ndarray          # float64 [N, 3] a.u.
    mass: np.ndarray         # float64 [N] a.u.
    charges: np.ndarray      # float64 [N]
    pot_params: np.ndarray   # float64 [2*2*5]

    @property
    def n_ions(self):
        return len(self.types)

    def copy(self):
        return dataclasses.replace(self, types=self.types.copy(), pos=self.pos.copy(),
                                   vel=self.vel.copy(), mass=self.mass.copy(),
                                   charges=self.charges.copy(), pot_params=self.pot_params.copy())


def make_system(ncell, n_grid, density=1.379, T=1200.0, seed=0, jitter=0.1):
    """Build the jittered 2-ion-cell NaCl lattice with MB velocities (see module doc)."""
    rng = np.random.default_rng(seed)
    n = 2 * ncell ** 3
    L = box_length_ang(n, density) / A0
    a = L / ncell
    cells = np.stack(np.meshgrid(np.arange(ncell), np.arange(ncell), np.arange(ncell),
                                 indexing="ij"), axis=-1).reshape(-1, 3).astype(np.float64)
    pos = np.empty((n, 3))
    pos[0::2] = cells * a
    pos[1::2] = (cells + 0.5) * a
    pos += rng.uniform(-jitter * a, jitter * a, size=pos.shape)
    pos = np.mod(pos, L)
    pos = np.where(pos >= L, pos - L, pos)
    types = np.tile(np.array([0, 1], dtype=np.int32), ncell ** 3)
    charges = np.array([SPECIES[t][1] for t in types], dtype=np.float64)
    mass = np.array([SPECIES[t][2] for t in types], dtype=np.float64) * CONV_MASS
    vel = rng.normal(0.0, 1.0, size=(n, 3)) * np.sqrt(KB * T / mass)[:, None]
    vel -= (mass[:, None] * vel).sum(axis=0) / mass.sum()
    return MoltenSalt(ncell=ncell, n_grid=n_grid, density=density, T=T, seed=seed, L=L,
                      h=L / n_grid, types=np.ascontiguousarray(types),
                      pos=np.ascontiguousarray(pos), vel=np.ascontiguousarray(vel),
                      mass=np.ascontiguousarray(mass), charges=np.ascontiguousarray(charges),
                      pot_params=tf_params_au())


def make_melt(n_ions, n_grid, density=1.379, T=1200.0, seed=0, jitter=0.1):
    """A +-1 ionic melt of any even n_ions: the 2-ion cells of the smallest cubic lattice
    that holds n_ions/2 of them, n_ions/2 cells drawn at random (seeded), each with its Na+
    at the corner and Cl- at the body centre, jittered as make_system; the box holds the
    n_ions at `density`."""
    if n_ions < 2 or n_ions % 2:
        raise ValueError("n_ions must be even and positive")
    rng = np.random.default_rng(seed)
    pairs = n_ions // 2
    ncell = int(np.ceil(pairs ** (1.0 / 3.0) - 1e-9))
    L = box_length_ang(n_ions, density) / A0
    a = L / ncell
    cells = np.stack(np.meshgrid(np.arange(ncell), np.arange(ncell), np.arange(ncell),
                                 indexing="ij"), axis=-1).reshape(-1, 3).astype(np.float64)
    cells = cells[np.sort(rng.choice(len(cells), size=pairs, replace=False))]
    pos = np.empty((n_ions, 3))
    pos[0::2] = cells * a
    pos[1::2] = (cells + 0.5) * a
    pos += rng.uniform(-jitter * a, jitter * a, size=pos.shape)
    pos = np.mod(pos, L)
    pos = np.where(pos >= L, pos - L, pos)
    types = np.tile(np.array([0, 1], dtype=np.int32), pairs)
    charges = np.array([SPECIES[t][1] for t in types], dtype=np.float64)
    mass = np.array([SPECIES[t][2] for t in types], dtype=np.float64) * CONV_MASS
    vel = rng.normal(0.0, 1.0, size=(n_ions, 3)) * np.sqrt(KB * T / mass)[:, None]
    vel -= (mass[:, None] * vel).sum(axis=0) / mass.sum()
    return MoltenSalt(ncell=ncell, n_grid=n_grid, density=density, T=T, seed=seed, L=L,
                      h=L / n_grid, types=np.ascontiguousarray(types),
                      pos=np.ascontiguousarray(pos), vel=np.ascontiguousarray(vel),
                      mass=np.ascontiguousarray(mass), charges=np.ascontiguousarray(charges),
                      pot_params=tf_params_au())


def replica_set(count=64, seed=2026, n_min=128, n_max=4000, densities=(1.329, 1.379), grids=(32, 64, 96, 128),
                spacing_ang=0.3):
    """The replicas of the batched configuration: N log-uniform in [n_min, n_max] rounded to
    an even count, density drawn from `densities`, grid from `grids` closest to a spacing
    of `spacing_ang`; returns (n_ions, n_grid, density, seed) per replica."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(round(np.exp(rng.uniform(np.log(n_min), np.log(n_max))) / 2)) * 2
        rho = float(rng.choice(densities))
        target = box_length_ang(n, rho) / spacing_ang
        g = min(grids, key=lambda x: abs(x - target))
        out.append((n, g, rho, int(rng.integers(1 << 30))))
    return out


# Lennard-Jones Na+/Cl- pairs: (type1, type2, sigma [A], epsilon [kJ/mol])
LENNARD_JONES = (("Na", "Na", 2.350, 0.544), ("Na", "Cl", 3.370, 0.477), ("Cl", "Cl", 4.400, 0.418))


def lj_params_au():
    """[sigma, epsilon] per type pair in a.u. (the conversion of solver.py:266-269), laid out
    so that both readers see the same table: the pairs (0,0), (0,1), (1,0), (1,1) sit at
    doubles 0, 2, 4, 6 (stride 2, the layout solver.py passes and this build reads) and at
    doubles 0, 4, 8, 12 (stride 4, the reference's read, particles.c:241)."""
    names = [s[0] for s in SPECIES]
    tab = {}
    for t1, t2, sg, ep in LENNARD_JONES:
        v = (sg / A0, ep * KJMOL_TO_HARTREE)
        tab[(names.index(t1), names.index(t2))] = v
        tab[(names.index(t2), names.index(t1))] = v
    out = np.zeros(14)
    for k, pair in enumerate([(0, 0), (0, 1), (1, 0), (1, 1)]):
        out[2 * k:2 * k + 2] = tab[pair]
        out[4 * k:4 * k + 2] = tab[pair]
    assert np.array_equal(out[:8].reshape(4, 2), out[[0, 1, 4, 5, 8, 9, 12, 13]].reshape(4, 2))
    return np.ascontiguousarray(out, dtype=np.float64)


def sc_params_au(nu=8.0, d_ang=2.8):
    """[nu, d, B] of the soft-core repulsion in a.u., B = 1.74 / (6 nu d) as
    solver.py:207-233 derives it."""
    d = d_ang / A0
    return np.ascontiguousarray([nu, d, 1.74 / (6 * nu * d)], dtype=np.float64)


def make_lj_system(ncell, n_grid, density=1.379, T=1200.0, seed=0, jitter=0.1):
    """The NaCl melt of make_system with Lennard-Jones pairs instead of Tosi-Fumi."""
    s = make_system(ncell, n_grid, density=density, T=T, seed=seed, jitter=jitter)
    s.pot_params = lj_params_au()
    return s


def make_sc_system(ncell, n_grid, density=1.379, T=1200.0, seed=0, jitter=0.1):
    """The NaCl melt of make_system with the soft-core repulsion instead of Tosi-Fumi."""
    s = make_system(ncell, n_grid, density=density, T=T, seed=seed, jitter=jitter)
    s.pot_params = sc_params_au()
    return s


def pair_system(ncell, n_grid, pot="TF", density=1.379, T=1200.0, seed=0):
    """make_system with the pair potential's parameters (TF, LJ or SC)."""
    if pot == "LJ":
        return make_lj_system(ncell, n_grid, density=density, T=T, seed=seed)
    if pot == "SC":
        return make_sc_system(ncell, n_grid, density=density, T=T, seed=seed)
    return make_system(ncell, n_grid, density=density, T=T, seed=seed)


# Poisson-Boltzmann implicit solvent (maze_poisson/solver.py:145-163, 346-356). The
# reference passes each ion's solvation radius (its species radius plus the probe radius,
# in bohr), the shell half-width w and the screening term kbar^2 h^2 to the library.
ION_RADII_ANG = (1.02, 1.81)     # Na+, Cl- ionic radii [A]
PROBE_RADIUS_ANG = 1.4           # maze_poisson/myio/input/base_file_input.py:129
EC_SI, EPS0_SI, KB_SI, BOHR_M = 1.602176634e-19, 8.854187817e-12, 1.380649e-23, 5.29177210903e-11


@dataclasses.dataclass
class PBSettings:
    """Arguments of solver_initialize_grid_pois_boltz / _particles_pois_boltz."""
    w: float                 # shell half-width [bohr]
    kbar2: float             # kbar^2 h^2
    nonpolar: int            # 1: non-polar forces on
    gamma_np: float          # a.u.
    beta_np: float
    radii: np.ndarray        # float64 [N] solvation radii [bohr]


def pb_kbar2(ionic_strength, T, eps_s, h):
    """kbar^2 h^2 of the linearised screening term, formed as solver.py:149-153 does
    (ionic strength in mol/L, h in bohr)."""
    return ((8 * np.pi * N_AVOGADRO * EC_SI ** 2 * ionic_strength * 1e3)
            / (eps_s * EPS0_SI * KB_SI * T) * BOHR_M ** 2 * h ** 2)


def pb_settings(system, eps_s=78.4, ionic_strength=0.15, w=1.0, nonpolar=1, gamma_np=0.005,
                beta_np=0.0):
    """PB arguments for `system`: solvation radius = ionic radius + probe (as solver.py:349-352
    forms it), gamma_np in kcal/mol/A^2 converted as base_file_input.py:145-147 does."""
    radii = (np.array([ION_RADII_ANG[t] for t in system.types]) + PROBE_RADIUS_ANG) / A0
    return PBSettings(w=w, kbar2=pb_kbar2(ionic_strength, system.T, eps_s, system.h),
                      nonpolar=nonpolar, gamma_np=gamma_np * 0.0065934, beta_np=beta_np,
                      radii=np.ascontiguousarray(radii, dtype=np.float64))


def make_pb_system(n_ions, n_grid, box_ang, T=300.0, seed=0, cluster_ang=None, min_sep_ang=2.7):
    """A solute of n_ions alternating Na+/Cl- ions at random positions inside a sphere of
    radius cluster_ang (default a quarter of the box) around the box centre, at least
    min_sep_ang apart, in implicit solvent; MB velocities at T, Tosi-Fumi pairs."""
    rng = np.random.default_rng(seed)
    L = box_ang / A0
    R = (cluster_ang if cluster_ang is not None else box_ang / 4) / A0
    sep = min_sep_ang / A0
    pos = []
    while len(pos) < n_ions:
        p = rng.uniform(-R, R, size=3)
        if np.linalg.norm(p) > R:
            continue
        if all(np.linalg.norm(p - q) >= sep for q in pos):
            pos.append(p)
    pos = np.mod(np.array(pos) + L / 2, L)
    types = np.array([k % 2 for k in range(n_ions)], dtype=np.int32)
    charges = np.array([SPECIES[t][1] for t in types], dtype=np.float64)
    mass = np.array([SPECIES[t][2] for t in types], dtype=np.float64) * CONV_MASS
    vel = rng.normal(0.0, 1.0, size=(n_ions, 3)) * np.sqrt(KB * T / mass)[:, None]
    return MoltenSalt(ncell=0, n_grid=n_grid, density=0.0, T=T, seed=seed, L=L, h=L / n_grid,
                      types=types, pos=np.ascontiguousarray(pos), vel=np.ascontiguousarray(vel),
                      mass=np.ascontiguousarray(mass), charges=np.ascontiguousarray(charges),
                      pot_params=tf_params_au())


# Workloads of the reference's configurations (sizes only; solver settings in md.py)
WORKLOADS = {
    "nacl250_64": dict(ncell=5, n_grid=64, density=1.379),
    "nacl2000_128": dict(ncell=10, n_grid=128, density=1.329),
    "nacl16000_256": dict(ncell=20, n_grid=256, density=1.379),
}


def write_reference_inputs(system, directory, name="input.csv"):
    """Write species.csv, tosi_fumi.csv and a positions/velocities CSV (A, a.u.) that the
    reference's SolverMD reads (maze_poisson/solver.py:165-205, 276-330)."""
    os.makedirs(directory, exist_ok=True)
    with open(os.path.join(directory, "species.csv"), "w") as f:
        f.write("type,charge,mass,radius\n")
        for t, q, m in SPECIES:
            f.write(f"{t},{q},{m},1.0\n")
    with open(os.path.join(directory, "tosi_fumi.csv"), "w") as f:
        f.write("type1,type2,A,B,C,D,sigma\n")
        for row in TOSI_FUMI:
            f.write(",".join(str(x) for x in row) + "\n")
    names = [s[0] for s in SPECIES]
    with open(os.path.join(directory, name), "w") as f:
        f.write("type,x,y,z,vx,vy,vz\n")
        for t, p, v in zip(system.types, system.pos * A0, system.vel):
            vals = ",".join(repr(float(x)) for x in (*p, *v))  # shortest round-trip decimal
            f.write(f"{names[t]},{vals}\n")
