"""Generate ``lattice128_dt002.json``: the C + OpenMP oracle's run of a
vortex lattice at the grid spacing of the 512x512x25 lattice configuration
(L/nx = 0.25) on a 128x128x25 cut (L = 32, 26 vortices of charge +-1 at
uniform positions from default_rng(1), bare atan2 imprint of
tevol_lattice.m:109-135, no winding removal, dt = 0.02).  At this spacing
and step the reference scheme is unstable: the run turns non-finite after
some 1800 steps.  The fixture records the stationary profile it starts from
(so the GPU test rebuilds the same initial fields), max|Psi| and max|A_y|
every 50 steps, and the first non-finite step.  About 10-15 minutes on 8
cores:

    python tests/golden/make_lattice_golden.py
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
    w = gs.LATTICE128
    seed_mod = importlib.import_module("ads4-holographic-quantum-turbulence_b200.seed")
    prof = seed_mod.stationary_profile(w["mu"], 0.0)
    state = gs.lattice_state(prof, w)
    op = oracle.build_operators(w["nx"], w["nx"], w["nz"], w["L"])
    s = oracle.OracleState(*state)
    rows, bad, done, t0 = [], 0, 0, time.time()
    while done < w["max_steps"] and not bad:
        s, _, b = oracle.omp_run(op, s, w["every"], w["dt"], w["mu"], 0.0, False)
        if b:
            bad = done + b
            break
        done += w["every"]
        rows.append([done, float(np.abs(s.Z1).max()), float(np.abs(s.Z4).max())])
        print(done, f"{time.time() - t0:.0f} s", rows[-1][1:], flush=True)
    out = {"config": w, "profile": {"z": prof.z.tolist(), "Z1": prof.Z1.tolist(),
                                    "Z2": prof.Z2.tolist(), "Vy1": prof.Vy1.tolist(),
                                    "rhoi": prof.rhoi.tolist()},
           "maxima": rows, "nonfinite_step": bad}
    (HERE / "lattice128_dt002.json").write_text(json.dumps(out))


if __name__ == "__main__":
    main()
