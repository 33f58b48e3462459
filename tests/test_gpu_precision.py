"""Mixed precision against FP64 over the full step counts of the benchmark
configurations, per result: relative L2 of each field, the drift of the
global charge Q (conserved in exact arithmetic), the kinetic energy E_kin of
the boundary superflow, the deviation of its energy spectrum, and the vortex
count.  The FP64 GPU path these runs compare against is itself pinned to the
oracle (``test_gpu_parity_long.py``).

* driven 301x301x21 (L = 100, mu = 6, dt = 0.02, A_y(z=0) = 2*pi*7/20,
  winding removal), 1000 steps;
* vortex lattice 512x512x25 (L = 128, 400 vortices of charge +-1 at uniform
  positions, seed 1, no winding removal), 2000 steps.

Bar (the task's): every field within 1e-6 relative L2 after the run; A_x and
A_y, which start at zero without a drive, on the scale of the gauge field
A_t.  The per-result figures are printed, and written as JSON to the file
named by the environment variable HQT_PRECISION_REPORT when it is set.
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


def run(hqt, state, cfg, prec, nsteps):
    api = importlib.import_module(hqt.__name__ + ".api")
    t = [api.to_device(a) for a in state]
    with hqt.Simulation(cfg["nx"], cfg["nx"], cfg["nz"], Lx=cfg["L"], mu=6.0, vy=cfg["vy"],
                        dt=cfg["dt"], remove_winding=cfg["rw"], precision=prec) as sim:
        obs0 = sim.observables_device(t[0], t[4])
        info = sim.step_device(*t, nsteps=nsteps)
        assert info.steps_done == nsteps and info.nonfinite_step == -1
        obs1 = sim.observables_device(t[0], t[4])
        O = sim.order_parameter_device(t[0])
        counts = sim.count_vortices_device(O)
        k, E, Ec, Ei = sim.energy_spectrum_device(O)
    fields = [api.from_device(x) for x in t]
    return fields, obs0, obs1, counts, (k, E, Ec, Ei)


def report(hqt, name, state, cfg, nsteps):
    f, fo0, fo1, fc, fs = run(hqt, state, cfg, "fp64", nsteps)
    m, mo0, mo1, mc, ms = run(hqt, state, cfg, "mixed", nsteps)
    gauge = np.linalg.norm(f[1].ravel())
    r = {"config": name, "steps": nsteps,
         "field_rel_l2": {"Z1": rel_l2(m[0], f[0]), "Z2": rel_l2(m[1], f[1]),
                          "Z3": rel_l2(m[2], f[2]), "Z4": rel_l2(m[3], f[3]),
                          "rhoi": rel_l2(m[4], f[4])},
         "gauge_scale_l2": {"Z3": float(np.linalg.norm((m[2] - f[2]).ravel()) / gauge),
                            "Z4": float(np.linalg.norm((m[3] - f[3]).ravel()) / gauge)},
         "charge_drift": {"fp64": (fo1["Q"] - fo0["Q"]) / abs(fo0["Q"]),
                          "mixed": (mo1["Q"] - mo0["Q"]) / abs(mo0["Q"]),
                          "mixed_vs_fp64": (mo1["Q"] - fo1["Q"]) / abs(fo1["Q"])},
         "E_kin_rel": (mo1["E_kin"] - fo1["E_kin"]) / abs(fo1["E_kin"]),
         "N_O_rel": (mo1["N_O"] - fo1["N_O"]) / abs(fo1["N_O"]),
         "spectrum_rel_l2": {"E": rel_l2(ms[1], fs[1]), "E_c": rel_l2(ms[2], fs[2]),
                             "E_i": rel_l2(ms[3], fs[3])},
         "counts": {"fp64": list(fc), "mixed": list(mc)}}
    print(json.dumps(r))
    path = os.environ.get("HQT_PRECISION_REPORT")
    if path:
        with open(path, "a") as fh:
            fh.write(json.dumps(r) + "\n")
    return r


def check(r, gauge_fields):
    errs = dict(r["field_rel_l2"])
    for k in gauge_fields:
        errs[k] = r["gauge_scale_l2"][k]
    assert max(errs.values()) <= 1e-6, errs
    assert abs(r["charge_drift"]["mixed_vs_fp64"]) <= 1e-6
    assert abs(r["E_kin_rel"]) <= 1e-6
    assert max(r["spectrum_rel_l2"].values()) <= 1e-6


def test_mixed_precision_driven301_1000_steps(hqt, cuda):
    cfg = dict(nx=301, nz=21, L=100.0, vy=VY7, dt=0.02, rw=True)
    prof = hqt.seed.stationary_profile(6.0, VY7)
    state = hqt.seed.init_driven(301, 301, 21, prof, noise="complex", amplitude=1e-3, seed=0)
    r = report(hqt, "driven301", state, cfg, 1000)
    check(r, ["Z3"])
    assert r["counts"]["fp64"] == r["counts"]["mixed"]


def test_mixed_precision_lattice512_2000_steps(hqt, cuda):
    nx, nz, L, nv = 512, 25, 128.0, 400
    cfg = dict(nx=nx, nz=nz, L=L, vy=0.0, dt=0.02, rw=False)
    prof = hqt.seed.stationary_profile(6.0, 0.0)
    rng = np.random.default_rng(1)
    xs, ys = rng.uniform(0, L, nv), rng.uniform(0, L, nv)
    q = np.r_[np.ones(nv // 2), -np.ones(nv // 2)]
    state = hqt.seed.init_lattice(nx, nx, nz, prof, L, L, xs, ys, q, periodic_images=0)
    r = report(hqt, "lattice512", state, cfg, 2000)
    check(r, ["Z3", "Z4"])
