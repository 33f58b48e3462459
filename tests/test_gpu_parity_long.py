"""Step-level parity over many steps at the benchmark configurations.

* ``64x64x21`` (L = 50, mu = 6, dt = 0.02, zero flow, noise 1e-3, seed 0):
  the CPU-runnable configuration, 200 steps against the oracle run here.
* ``64x64x21`` with the drive A_y(z=0) = 2*pi*7/20 and a phase winding of 2
  imprinted along y, so the winding removal acts: 100 steps against the
  oracle, and the per-step winding sequence of one-step calls equal to the
  oracle's.
* ``301x301x21`` driven (the benchmark's workload): 100 steps against the
  oracle's stored run (``tests/golden/driven301_fp64.npz``, made by
  ``tests/golden/make_driven_golden.py``; the oracle needs seconds per step at
  this size).  Whole fields are compared through Rademacher sketches at steps
  1, 10, 50 and 100, the planes next to the AdS boundary value by value at
  step 100, and the per-step windings exactly.

Bar: relative L2 <= 1e-10 per field (A_x, which starts at zero, on the scale
of the gauge field A_t); windings and vortex counts are integers: exact.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
if str(GOLDEN) not in sys.path:
    sys.path.insert(0, str(GOLDEN))

VY7 = -2 * np.pi * 7 / 20
BAR = 1e-10


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def oracle_run(oracle, state, nx, ny, nz, L, nsteps, mu, vy, rw=True, dt=0.02):
    op = oracle.build_operators(nx, ny, nz, L)
    s = oracle.OracleState(*[a.copy() for a in state])
    ws = []
    for _ in range(nsteps):
        s, w = oracle.rk4_step(op, s, dt, mu, vy, rw)
        ws.append(w)
    return op, s, ws


def field_errors(got, ref):
    g1, g2, g3, g4, gr = got
    scale = np.linalg.norm(ref.Z2.ravel())
    return {"Z1": rel_l2(g1, ref.Z1), "Z2": rel_l2(g2, ref.Z2), "Z4": rel_l2(g4, ref.Z4),
            "rhoi": rel_l2(gr, ref.rhoi),
            "Z3_gauge": float(np.linalg.norm((g3 - ref.Z3).ravel()) / scale)}


def test_c1_200_steps_fp64(hqt, oracle, cuda):
    """64x64x21, L=50, mu=6, dt=0.02, 200 steps, zero flow: one 200-step call."""
    nx, nz, L = 64, 21, 50.0
    prof = hqt.seed.stationary_profile(6.0, 0.0)
    state = hqt.seed.init_driven(nx, nx, nz, prof, noise="complex", amplitude=1e-3, seed=0)
    _, ref, ws = oracle_run(oracle, state, nx, nx, nz, L, 200, 6.0, 0.0)
    with hqt.Simulation(nx, nx, nz, Lx=L, mu=6.0, vy=0.0, dt=0.02) as sim:
        got, info = sim.step(*state, nsteps=200)
    errs = field_errors(got, ref)
    print("c1 200 steps:", errs)
    assert info.steps_done == 200 and info.nonfinite_step == -1
    assert max(errs.values()) < BAR, errs
    assert info.last_winding == ws[-1]


def test_driven64_100_steps_with_winding_removal(hqt, oracle, cuda, dev):
    """The drive and the winding removal over 100 steps: one 100-step call,
    and 100 one-step calls whose windings must be the oracle's, step by step."""
    to_d, from_d = dev
    nx, nz, L = 64, 21, 50.0
    prof = hqt.seed.stationary_profile(6.0, VY7)
    state = list(hqt.seed.init_driven(nx, nx, nz, prof, noise="complex", amplitude=1e-3,
                                      seed=0))
    state[0] = state[0] * np.exp(2j * np.pi * 2 * np.arange(nx) / nx)[None, :, None]
    _, ref, ws = oracle_run(oracle, state, nx, nx, nz, L, 100, 6.0, VY7)
    assert ws[0] == 2
    with hqt.Simulation(nx, nx, nz, Lx=L, mu=6.0, vy=VY7, dt=0.02) as sim:
        got, info = sim.step(*state, nsteps=100)
        errs = field_errors(got, ref)
        print("driven 64 x 100 steps:", errs)
        assert max(errs.values()) < BAR, errs
        t = [to_d(a) for a in state]
        gw = [sim.step_device(*t, nsteps=1).last_winding for _ in range(100)]
    assert gw == ws
    errs1 = field_errors([from_d(x) for x in t], ref)
    assert max(errs1.values()) < BAR, errs1


@pytest.fixture(scope="module")
def golden301():
    d = np.load(GOLDEN / "driven301_fp64.npz")
    return {k: d[k] for k in d.files}


def sketch_errors(gs, got, sk_ref):
    """Sketch estimates of the relative L2 error of each field (A_x on the
    scale of A_t's sketch)."""
    sk = gs.state_sketches(*got)
    names = ("Z1", "Z2", "Z3", "Z4", "rho")
    out = {}
    for i, n in enumerate(names):
        ref = sk_ref[i]
        num = np.linalg.norm(sk[n] - ref)
        den = np.linalg.norm(sk_ref[1] if n == "Z3" else ref)
        out[n] = float(num / den)
    return out


def test_driven301_100_steps_against_stored_oracle(hqt, cuda, dev, golden301):
    import golden_state as gs
    to_d, from_d = dev
    w = gs.DRIVEN301
    fx = golden301
    nx, ny, nz = w["nx"], w["ny"], w["nz"]
    state = gs.initial_state(fx, nx, ny, w["amp"], w["seed"])
    # the initial state is rebuilt exactly (the sketch's dot products may sum
    # in another order on another host's BLAS)
    init = sketch_errors(gs, state, fx["sk0"])
    assert max(init.values()) < 1e-13, init
    t = [to_d(a) for a in state]
    done = 0
    with hqt.Simulation(nx, ny, nz, Lx=w["L"], mu=w["mu"], vy=w["vy"], dt=w["dt"],
                        remove_winding=w["remove_winding"]) as sim:
        for cp in w["checkpoints"]:
            info = sim.step_device(*t, nsteps=cp - done)
            assert info.nonfinite_step == -1
            done = cp
            host = [from_d(x) for x in t]
            errs = sketch_errors(gs, host, fx[f"sk{cp}"])
            print(f"driven301 step {cp}:", errs)
            assert max(errs.values()) < BAR, (cp, errs)
        # planes next to the AdS boundary, value by value, at the last step
        lev = int(fx["plane_level"])
        g1, g2, g3, g4, gr = host
        scale = np.max(np.abs(fx["plane_Z2"]))
        assert rel_l2(g1[:, :, lev], fx["plane_Z1"]) < BAR
        assert rel_l2(g2[:, :, lev], fx["plane_Z2"]) < BAR
        assert rel_l2(g4[:, :, lev], fx["plane_Z4"]) < BAR
        assert rel_l2(gr[:, :, -1], fx["plane_rho"]) < BAR
        assert np.max(np.abs(g3[:, :, lev] - fx["plane_Z3"])) < BAR * scale
        # vortex counts of O at the stored steps
        O = sim.order_parameter_device(t[0])
        last = fx["counts"][-1]
        assert tuple(sim.count_vortices_device(O)) == tuple(int(v) for v in last[1:])
        # per-step windings of one-step calls
        t2 = [to_d(a) for a in state]
        gw = [sim.step_device(*t2, nsteps=1).last_winding for _ in range(done)]
    assert gw == [int(v) for v in fx["windings"]]
    errs = sketch_errors(gs, [from_d(x) for x in t2], fx[f"sk{done}"])
    assert max(errs.values()) < BAR, errs


def test_lattice_instability_matches_the_oracle(hqt, cuda, dev):
    """At the spacing of the 512x512x25 lattice configuration (L/nx = 0.25) and
    dt = 0.02 the reference scheme is unstable.  The C + OpenMP oracle's run
    of a 128x128x25 cut (``tests/golden/lattice128_dt002.json``, made by
    ``tests/golden/make_lattice_golden.py``) turns non-finite after some 1800
    steps; the GPU must follow it (max|Psi|, max|A_y| every 50 steps) and
    stop within a few dozen steps of it."""
    import json
    import golden_state as gs
    to_d, from_d = dev
    d = json.loads((GOLDEN / "lattice128_dt002.json").read_text())
    w = d["config"]
    state = gs.lattice_state(gs.profile_from(d["profile"]), w)
    t = [to_d(a) for a in state]
    want = {r[0]: r[1:] for r in d["maxima"]}
    bad, done = 0, 0
    with hqt.Simulation(w["nx"], w["nx"], w["nz"], Lx=w["L"], mu=w["mu"], vy=0.0, dt=w["dt"],
                        remove_winding=False) as sim:
        while done < w["max_steps"]:
            try:
                sim.step_device(*t, nsteps=w["every"])
            except hqt.NonfiniteEvolution as e:
                bad = done + e.info.nonfinite_step
                break
            done += w["every"]
            if done in want and done <= 1000:
                z1 = float(t[0].abs().max())
                z4 = float(t[3].abs().max())
                assert abs(z1 - want[done][0]) <= 1e-8 * want[done][0], (done, z1, want[done])
                assert abs(z4 - want[done][1]) <= 1e-8 * want[done][1], (done, z4, want[done])
    assert d["nonfinite_step"] > 0
    print("non-finite at step", bad, "oracle", d["nonfinite_step"])
    assert bad > 0 and abs(bad - d["nonfinite_step"]) <= 100
