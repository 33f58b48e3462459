"""Mixed precision against FP64 at the benchmark configurations, per result:
relative L2 of each field, the drift of the global charge Q (conserved in
exact arithmetic), the kinetic energy E_kin of the boundary superflow, the
deviation of its energy spectrum, and the vortex count.  The FP64 GPU path
these runs compare against is itself pinned to the oracle
(``test_gpu_parity_long.py``).

* driven 301x301x21 (L = 100, mu = 6, dt = 0.02, A_y(z=0) = 2*pi*7/20,
  winding removal), 100 and 1000 steps;
* vortex lattice 512x512x25 (L = 128, 400 vortices of charge +-1 at uniform
  positions, seed 1, no winding removal) at dt = 0.01, 100 and 4000 steps
  (t = 40; at dt = 0.02 the scheme is unstable at this spacing).

Bar: every field within 1e-6 relative L2 after 100 steps (A_x and A_y, which
start at zero without a drive, on the scale of the gauge field A_t).  Over
the long runs the flow is chaotic, so a difference of any origin grows; the
yardstick there is the spread between two FP64 runs that differ only in the
summation order of their line transforms (another transform engine): the
mixed run's field and spectrum deviations must stay within 10x of that
spread or 1e-6, whichever is larger.  All figures are printed, and written
as JSON lines to the file named by HQT_PRECISION_REPORT when it is set.
"""
import importlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VY7 = -2 * np.pi * 7 / 20


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def run(hqt, state, cfg, prec, marks, engine=None):
    """Step to each count in `marks`; per mark: fields, observables, counts,
    spectrum.  `engine` forces a line-transform engine (HQT_LINE_ENGINE)."""
    api = importlib.import_module(hqt.__name__ + ".api")
    old = os.environ.get("HQT_LINE_ENGINE")
    if engine:
        os.environ["HQT_LINE_ENGINE"] = engine
    try:
        sim = hqt.Simulation(cfg["nx"], cfg["nx"], cfg["nz"], Lx=cfg["L"], mu=6.0,
                             vy=cfg["vy"], dt=cfg["dt"], remove_winding=cfg["rw"],
                             precision=prec)
    finally:
        if engine:
            if old is None:
                os.environ.pop("HQT_LINE_ENGINE", None)
            else:
                os.environ["HQT_LINE_ENGINE"] = old
    out = {}
    with sim:
        t = [api.to_device(a) for a in state]
        obs0 = sim.observables_device(t[0], t[4])
        done = 0
        for m in marks:
            info = sim.step_device(*t, nsteps=m - done)
            assert info.nonfinite_step == -1
            done = m
            O = sim.order_parameter_device(t[0])
            out[m] = dict(fields=[api.from_device(x) for x in t],
                          obs=sim.observables_device(t[0], t[4]),
                          counts=list(sim.count_vortices_device(O)),
                          spec=sim.energy_spectrum_device(O))
        del t
    return obs0, out


def compare(a, b, gauge_fields):
    """Deviation of run a from run b (both dicts of one mark)."""
    fa, fb = a["fields"], b["fields"]
    gauge = np.linalg.norm(fb[1].ravel())
    names = ("Z1", "Z2", "Z3", "Z4", "rhoi")
    field = {}
    for i, n in enumerate(names):
        if n in gauge_fields:
            field[n] = float(np.linalg.norm((fa[i] - fb[i]).ravel()) / gauge)
        else:
            field[n] = rel_l2(fa[i], fb[i])
    return {"field": field,
            "Q_rel": (a["obs"]["Q"] - b["obs"]["Q"]) / abs(b["obs"]["Q"]),
            "E_kin_rel": (a["obs"]["E_kin"] - b["obs"]["E_kin"]) / abs(b["obs"]["E_kin"]),
            "N_O_rel": (a["obs"]["N_O"] - b["obs"]["N_O"]) / abs(b["obs"]["N_O"]),
            "spectrum_rel_l2": {k: rel_l2(a["spec"][i], b["spec"][i])
                                for i, k in ((1, "E"), (2, "E_c"), (3, "E_i"))},
            "counts": [a["counts"], b["counts"]]}


def report(hqt, name, state, cfg, marks, alt_engine, gauge_fields):
    q0f, f = run(hqt, state, cfg, "fp64", marks)
    q0m, m = run(hqt, state, cfg, "mixed", marks)
    _, g = run(hqt, state, cfg, "fp64", marks, engine=alt_engine)
    rows = []
    for k in marks:
        r = {"config": name, "steps": k,
             "mixed_vs_fp64": compare(m[k], f[k], gauge_fields),
             "fp64_engine_spread": compare(g[k], f[k], gauge_fields),
             "charge_drift": {"fp64": (f[k]["obs"]["Q"] - q0f["Q"]) / abs(q0f["Q"]),
                              "mixed": (m[k]["obs"]["Q"] - q0m["Q"]) / abs(q0m["Q"])},
             "alt_engine": alt_engine}
        rows.append(r)
        print(json.dumps(r))
        path = os.environ.get("HQT_PRECISION_REPORT")
        if path:
            with open(path, "a") as fh:
                fh.write(json.dumps(r) + "\n")
    return rows


def check(rows):
    """The 1e-6 field bar after 100 steps; fields and E_kin at every mark
    within 10x of the FP64 engine spread or 1e-6, whichever is larger.  The
    spectrum is that of the fluctuations about the mean flow, so its relative
    deviation is the field's divided by their relative size (about 1e-3 in
    the driven run): it is reported, with a loose bar of 1e-4."""
    short = rows[0]
    assert max(short["mixed_vs_fp64"]["field"].values()) <= 1e-6, short["mixed_vs_fp64"]["field"]
    for r in rows:
        mv, sp = r["mixed_vs_fp64"], r["fp64_engine_spread"]
        bar = max(1e-6, 10 * max(sp["field"].values()))
        assert max(mv["field"].values()) <= bar, (r["steps"], mv["field"], sp["field"])
        # spectra: reported; bounded by the field deviation times the ratio of
        # the mean flow to its fluctuations, so only a loose sanity bar here
        assert max(mv["spectrum_rel_l2"].values()) <= max(1e-4, 10 * max(
            sp["spectrum_rel_l2"].values())), (r["steps"], mv, sp)
        ebar = max(1e-6, 10 * abs(sp["E_kin_rel"]))
        assert abs(mv["E_kin_rel"]) <= ebar
        # the charge is conserved to roundoff in both precisions
        assert abs(r["charge_drift"]["fp64"]) <= 1e-12
        assert abs(r["charge_drift"]["mixed"]) <= 1e-6


def test_mixed_precision_driven301(hqt, cuda):
    cfg = dict(nx=301, nz=21, L=100.0, vy=VY7, dt=0.02, rw=True)
    prof = hqt.seed.stationary_profile(6.0, VY7)
    state = hqt.seed.init_driven(301, 301, 21, prof, noise="complex", amplitude=1e-3, seed=0)
    rows = report(hqt, "driven301", state, cfg, (100, 1000), "stockham", ("Z3",))
    check(rows)
    assert rows[-1]["mixed_vs_fp64"]["counts"][0] == rows[-1]["mixed_vs_fp64"]["counts"][1]


def test_mixed_precision_lattice512(hqt, cuda):
    """dt = 0.01: at dt = 0.02 the reference scheme is unstable at this
    spacing (the run turns non-finite after ~1350 steps in FP64 and mixed
    alike; the oracle shows the same on a 128x128 cut,
    test_gpu_parity_long.py::test_lattice_instability_matches_the_oracle).
    4000 steps cover the configuration's t = 40."""
    nx, nz, L, nv = 512, 25, 128.0, 400
    cfg = dict(nx=nx, nz=nz, L=L, vy=0.0, dt=0.01, rw=False)
    prof = hqt.seed.stationary_profile(6.0, 0.0)
    rng = np.random.default_rng(1)
    xs, ys = rng.uniform(0, L, nv), rng.uniform(0, L, nv)
    q = np.r_[np.ones(nv // 2), -np.ones(nv // 2)]
    state = hqt.seed.init_lattice(nx, nx, nz, prof, L, L, xs, ys, q, periodic_images=0)
    rows = report(hqt, "lattice512", state, cfg, (100, 4000), "runtime", ("Z3", "Z4"))
    check(rows)
