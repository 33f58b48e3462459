"""Generate ``driven301_fp64.npz``: the CPU oracle's 100-step run of the driven
301x301x21 configuration (L = 100, mu = 6, dt = 0.02, A_y(z=0) = 2*pi*7/20,
winding removal and filter on, complex noise 1e-3 from ``default_rng(0)``).

The oracle takes seconds per step at this size, too slow to rerun inside the
GPU tests, so its results are stored once here (format: ``golden_state.py``).
Run from the repository root (about 15-20 minutes on 8 cores):

    python tests/golden/make_driven_golden.py
"""
import importlib
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path[:0] = [str(ROOT), str(ROOT / "oracle"), str(HERE)]

import golden_state as gs  # noqa: E402
import hqt_oracle as oracle  # noqa: E402


def main() -> None:
    w = gs.DRIVEN301
    seed_mod = importlib.import_module("ads4-holographic-quantum-turbulence_b200.seed")
    prof = seed_mod.stationary_profile(w["mu"], w["vy"])
    cols = gs.profile_arrays(prof, w["nz"])
    state = gs.initial_state(cols, w["nx"], w["ny"], w["amp"], w["seed"])
    op = oracle.build_operators(w["nx"], w["ny"], w["nz"], w["L"])
    s = oracle.OracleState(*state)
    out = dict(cols)
    out["sk0"] = np.stack(list(gs.state_sketches(*state).values()))
    windings, counts = [], {}
    last = max(w["checkpoints"])
    t0 = time.time()
    for step in range(1, last + 1):
        s, wind = oracle.rk4_step(op, s, w["dt"], w["mu"], w["vy"], w["remove_winding"])
        windings.append(wind)
        if step in w["checkpoints"]:
            sk = gs.state_sketches(s.Z1, s.Z2, s.Z3, s.Z4, s.rhoi)
            out[f"sk{step}"] = np.stack(list(sk.values()))
            out[f"norm{step}"] = np.array([np.linalg.norm(a) for a in
                                           (s.Z1, s.Z2, s.Z3, s.Z4, s.rhoi[:, :, -1])])
            O = oracle.boundary_order_parameter(op, s.Z1)
            counts[step] = oracle.countN(O)
            print(f"step {step}: {time.time() - t0:.0f} s, winding {wind}, "
                  f"countN {counts[step]}", flush=True)
    lev = w["nz"] - 2
    out["plane_Z1"] = s.Z1[:, :, lev]
    out["plane_Z2"] = s.Z2[:, :, lev]
    out["plane_Z3"] = s.Z3[:, :, lev]
    out["plane_Z4"] = s.Z4[:, :, lev]
    out["plane_rho"] = s.rhoi[:, :, -1]
    out["plane_level"] = np.int64(lev)
    out["windings"] = np.array(windings, dtype=np.int64)
    out["counts"] = np.array([[k, *v] for k, v in sorted(counts.items())], dtype=np.int64)
    meta = {k: (list(v) if isinstance(v, tuple) else v) for k, v in w.items()}
    meta["sketch_rows"] = gs.SKETCH_ROWS
    meta["sketch_seed"] = gs.SKETCH_SEED
    out["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(HERE / "driven301_fp64.npz", **out)


if __name__ == "__main__":
    main()
