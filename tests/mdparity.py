"""Helpers of the MD parity tests: one MD run through the product library and the same
run through the CPU oracle, driven by the reference's call sequence (MDRun), compared
after the bootstrap and after every step."""
import numpy as np

from maze_poisson_b200.md import MDRun


def rel(a, b):
    """Max-norm ratio |a - b|_inf / |b|_inf."""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def rms_rel(a, b):
    """RMS of a - b over RMS of b."""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2)) / max(np.sqrt(np.mean(b ** 2)), 1e-300))


def inject_noise(prod, system, steps):
    """Feed the product's Philox O-block draws for the bootstrap and `steps` OVRVO steps
    into the oracle (each integrator part draws once per call when the thermostat is on)."""
    from oracle.loader import load_kernels
    calls = 2 + 2 * steps
    z = np.empty((calls, system.n_ions, 3))
    for c in range(calls):
        prod.mzb_philox_normals(c, z[c])
    load_kernels().orc_set_noise(np.ascontiguousarray(z.reshape(-1)), z.size)


def run_pair(prod, orc, system, steps, check_each=True, noise=False, bound=1e-10, bounds=None, **kw):
    """Run the same MD on product and oracle; compare after init and every step
    (max-norm ratio below `bound` for fields, forces, positions and velocities; kinetic
    energy to `bound`; solver iteration counts within 1); `bounds` overrides the bound of
    single quantities. `kw` are MDRun's settings. Returns the last states and the
    largest error seen per quantity."""
    a = MDRun(prod, system.copy(), **kw)
    b = MDRun(orc, system.copy(), **kw)
    worst = {}

    def note(key, err, where):
        worst[key] = max(worst.get(key, 0.0), err)
        assert err < (bounds or {}).get(key, bound), (where, key, err)

    a.initialize()
    if noise:
        inject_noise(prod, system, steps)
    b.initialize()
    try:
        sa, sb = a.state(), b.state()
        note("q", rel(sa["q"], sb["q"]), "init")
        note("field", rel(sa["field"], sb["field"]), "init")
        for key in ("fcs_elec", "fcs_noel", "fcs_tot", "pos", "vel"):
            note(key, rel(sa[key], sb[key]), "init")
        note("potential_notelec", abs(sa["potential_notelec"] - sb["potential_notelec"]) /
             abs(sb["potential_notelec"]), "init")
        for s in range(steps):
            a.step()
            b.step()
            if check_each or s == steps - 1:
                sa, sb = a.state(), b.state()
                assert abs(sa["n_iters"] - sb["n_iters"]) <= 1, (s, sa["n_iters"], sb["n_iters"])
                for key in ("field", "fcs_tot", "pos", "vel"):
                    note(key, rel(sa[key], sb[key]), s)
                note("kinetic", abs(sa["kinetic"] - sb["kinetic"]) / sb["kinetic"], s)
        return sa, sb, worst
    finally:
        a.finalize()
        b.finalize()


def restart(run, pos, vel, field, field_prev):
    """Start `run` from a given state the way the reference's restart path does
    (maze_poisson/solver.py:371-409 with a restart field), then compute that state's
    forces (MDRun.restart)."""
    run.restart(pos, vel, field, field_prev)


def oracle_floor(orc, system, steps, keys=("field", "fcs_elec", "fcs_tot", "pos", "vel"), pert=1e-15, **kw):
    """Sensitivity of the reference's algorithm itself: the largest max-norm change of each
    quantity over `steps` MD steps of the oracle when the initial positions are scaled by
    (1 + pert)."""
    runs = []
    for p in (0.0, pert):
        s = system.copy()
        s.pos = np.ascontiguousarray(s.pos * (1 + p))
        r = MDRun(orc, s, **kw)
        r.initialize()
        try:
            states = []
            for _ in range(steps):
                r.step()
                st = r.state()
                states.append({k: st[k].copy() for k in keys})
            runs.append(states)
        finally:
            r.finalize()
    return {k: max(rel(b[k], a[k]) for a, b in zip(*runs)) for k in keys}
