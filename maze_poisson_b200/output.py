"""Output and restart path of the MD loop, in the reference's file formats.

The reference writes, every `stride` steps, energy.csv (iter, K, V_notelec), momentum.csv
(iter, Px, Py, Pz), temperature.csv (iter, T), tot_force.csv (iter, Fx, Fy, Fz: the sum
over ions), solute.csv (per ion: charge, iter, particle, x, y, z, vx, vy, vz, fx_elec,
fy_elec, fz_elec) and, at `restart_step`, restart.csv (type, x, y, z [A], vx, vy, vz) and
restart_field.csv (phi_prev, phi), each read through the blocking getters
(maze_poisson/myio/output/csv.py:45-183, base_out.py:136-152). A restart reads the
particles from restart.csv as the input file and the fields through solver_set_field /
solver_set_field_prev (solver.py:276-330, 371-409).

`Outputs` writes the same files with the same columns. On this build's library it takes
the values from asynchronous snapshots (mzb_snapshot_begin / _fetch: staged on the
device, copied to pinned memory while the next steps run) and writes a snapshot's rows
when its slot is needed again or at close; on any other library with the reference's ABI
(the oracle, the reference itself) it calls the getters, as the reference does.
"""
import os

import numpy as np
import pandas as pd

from .systems import A0

SNAP_POS, SNAP_VEL, SNAP_FORCES, SNAP_SCALARS, SNAP_FIELDS = 1, 2, 4, 8, 16

HEADERS = {
    "energy": ["iter", "K", "V_notelec"],
    "momentum": ["iter", "Px", "Py", "Pz"],
    "temperature": ["iter", "T"],
    "tot_force": ["iter", "Fx", "Fy", "Fz"],
    "solute": ["charge", "iter", "particle", "x", "y", "z", "vx", "vy", "vz", "fx_elec", "fy_elec", "fz_elec"],
    "restart": ["type", "x", "y", "z", "vx", "vy", "vz"],
    "restart_field": ["phi_prev", "phi"],
}
PER_STRIDE = ("energy", "momentum", "temperature", "tot_force", "solute")


class _Frame:
    """One output instant's values: own arrays (getters) or views into a snapshot's
    pinned host buffer (`host`, a flat float64 array)."""

    def __init__(self, it, n_ions, n_grid, with_fields, host=None):
        self.it = it
        self.restart = with_fields
        if host is None:
            self.pos, self.vel, self.fe, self.fn, self.ft = (np.empty((n_ions, 3)) for _ in range(5))
            self.scalars = np.zeros(8)
            self.phi = np.empty((n_grid,) * 3) if with_fields else None
            self.phi_prev = np.empty((n_grid,) * 3) if with_fields else None
            return
        v = 3 * n_ions
        self.pos, self.vel, self.fe, self.fn, self.ft = (host[k * v:(k + 1) * v].reshape(n_ions, 3)
                                                         for k in range(5))
        self.scalars = host[5 * v:5 * v + 8]
        m = n_grid ** 3
        f0 = 5 * v + 8
        self.phi = host[f0:f0 + m].reshape((n_grid,) * 3) if with_fields else None
        self.phi_prev = host[f0 + m:f0 + 2 * m].reshape((n_grid,) * 3) if with_fields else None


class Outputs:
    """The reference's per-stride and restart outputs of one system (see module doc)."""

    def __init__(self, capi, path, type_names, n_grid, stride=1, restart_step=None, files=PER_STRIDE,
                 use_snapshots=None, write=True):
        self.capi = capi
        self.write = write  # False: collect the values but write no file (times the transfers)
        self.path = path
        self.type_names = list(type_names)
        self.n_grid = n_grid
        self.stride = stride
        self.restart_step = restart_step
        self.files = [f for f in files if f in PER_STRIDE]
        if use_snapshots is None:
            use_snapshots = "mzb_snapshot_begin" in getattr(capi, "functions", {})
        self.async_ = use_snapshots
        self.pending = []   # (frame, slot) in queue order
        self.last = -1
        os.makedirs(path, exist_ok=True)
        self.n_ions = None
        self.charges = None
        self.types = None
        for name in self.files if write else ():
            with open(self._file(name), "w") as f:
                pd.DataFrame(columns=HEADERS[name]).to_csv(f, index=False)

    def _file(self, name):
        return os.path.join(self.path, f"{name}.csv")

    def _static(self):
        """Types and charges, which do not change during a run."""
        if self.charges is None:
            c = self.capi
            types = np.empty(self._n(), dtype=np.int32)
            c.get_types(types)
            charges = np.empty(self._n())
            c.get_charges(charges)
            self.types, self.charges = types, charges

    def _n(self):
        if self.n_ions is None:
            raise RuntimeError("Outputs.bind(n_ions) has not been called")
        return self.n_ions

    def bind(self, n_ions):
        self.n_ions = n_ions
        return self

    # -- the reference's OutputFiles.output(itr, solver, force) -------------------------
    def output(self, it, potential_notelec=None, force=False):
        """Queue the outputs due at step `it` (per-stride files; restart files at
        restart_step). potential_notelec is the last solver_compute_forces_noel value
        (used by the getter path; snapshots carry it)."""
        self._static()
        if (force or it % self.stride == 0) and self.last != it and self.files:
            self.last = it
            self._queue(it, False, potential_notelec)
        if self.restart_step == it:
            self._queue(it, True, potential_notelec)

    def _queue(self, it, restart, v_notelec):
        c = self.capi
        if self.async_:
            what = SNAP_POS | SNAP_VEL | SNAP_FORCES | SNAP_SCALARS | (SNAP_FIELDS if restart else 0)
            slot = c.mzb_snapshot_begin(what)
            if slot < 0:  # both slots hold unwritten snapshots: write the oldest first
                self._write_oldest()
                slot = c.mzb_snapshot_begin(what)
            self.pending.append((it, restart, slot))
        else:
            frame = _Frame(it, self._n(), self.n_grid, restart)
            c.get_pos(frame.pos)
            c.get_vel(frame.vel)
            c.get_fcs_elec(frame.fe)
            c.get_fcs_noel(frame.fn)
            c.get_fcs_tot(frame.ft)
            mom = np.empty(3)
            c.get_momentum(mom)
            frame.scalars[:] = [0.0, v_notelec if v_notelec is not None else np.nan, c.get_kinetic_energy(),
                                mom[0], mom[1], mom[2], c.get_temperature(), 0.0]
            if restart:
                c.get_field(frame.phi)
                c.get_field_prev(frame.phi_prev)
            self._write(frame)

    def _write_oldest(self):
        """Write the oldest queued snapshot from its pinned buffer in place, then release
        its slot."""
        it, restart, slot = self.pending.pop(0)
        c = self.capi
        buf = c.mzb_snapshot_host(slot)
        if not buf:
            raise RuntimeError("snapshot slot held no snapshot")
        n = self._n()
        size = 15 * n + 8 + (2 * self.n_grid ** 3 if restart else 0)
        host = np.ctypeslib.as_array(buf, shape=(size,))
        self._write(_Frame(it, n, self.n_grid, restart, host=host))
        del host
        c.mzb_snapshot_fetch(slot, *([None] * 8))

    def _write(self, fr):
        if not self.write:
            return
        s = fr.scalars
        if fr.restart:
            df = pd.DataFrame({"type": [self.type_names[t] for t in self.types]})
            df[["x", "y", "z"]] = fr.pos * A0
            df[["vx", "vy", "vz"]] = fr.vel
            with open(self._file("restart"), "w") as f:
                df.to_csv(f, columns=HEADERS["restart"], index=False)
            with open(self._file("restart_field"), "w") as f:
                pd.DataFrame({"phi": fr.phi.ravel(), "phi_prev": fr.phi_prev.ravel()}).to_csv(
                    f, columns=HEADERS["restart_field"], index=False)
            return
        rows = {
            "energy": pd.DataFrame({"iter": [fr.it], "K": [s[2]], "V_notelec": [s[1]]}),
            "momentum": pd.DataFrame({"iter": [fr.it], "Px": [s[3]], "Py": [s[4]], "Pz": [s[5]]}),
            "temperature": pd.DataFrame({"iter": [fr.it], "T": [s[6]]}),
        }
        tf = pd.DataFrame(fr.ft.sum(axis=0).reshape(1, 3), columns=["Fx", "Fy", "Fz"])
        tf["iter"] = fr.it
        rows["tot_force"] = tf
        sol = pd.DataFrame()
        sol[["x", "y", "z"]] = fr.pos
        sol[["vx", "vy", "vz"]] = fr.vel
        sol[["fx_elec", "fy_elec", "fz_elec"]] = fr.fe
        sol["charge"] = self.charges
        sol["iter"] = fr.it
        sol["particle"] = range(len(fr.pos))
        rows["solute"] = sol
        for name in self.files:
            with open(self._file(name), "a") as f:
                rows[name].to_csv(f, columns=HEADERS[name], header=False, index=False)

    def close(self):
        while self.pending:
            self._write_oldest()


def read_restart(path, type_names):
    """Particles of a restart.csv (or any input CSV with type, x, y, z [A] and optional
    vx, vy, vz): int32 types, positions in bohr, velocities (a.u. or None)."""
    df = pd.read_csv(path)
    lut = {name: k for k, name in enumerate(type_names)}
    types = np.ascontiguousarray([lut[t] for t in df["type"]], dtype=np.int32)
    pos = np.ascontiguousarray(df[["x", "y", "z"]].values / A0, dtype=np.float64)
    vel = np.ascontiguousarray(df[["vx", "vy", "vz"]].values, dtype=np.float64) if "vx" in df.columns else None
    return types, pos, vel


def read_restart_field(path, n_grid):
    """phi and phi_prev of a restart_field.csv, as (n, n, n) arrays."""
    df = pd.read_csv(path)
    phi = np.ascontiguousarray(df["phi"].values).reshape((n_grid,) * 3)
    phi_prev = np.ascontiguousarray(df["phi_prev"].values).reshape((n_grid,) * 3)
    return phi, phi_prev
