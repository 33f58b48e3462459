"""The stored oracle run of the driven 301x301x21 configuration
(``tests/golden/driven301_fp64.npz``) is consistent with the oracle in this
checkout: the initial state rebuilt from the fixture matches its stored
sketch exactly, and one oracle step from it reproduces the stored step-1
sketches (the same code; BLAS threading may change the last bits only)."""
import sys
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"
if str(GOLDEN) not in sys.path:
    sys.path.insert(0, str(GOLDEN))


def test_fixture_step_one_matches_the_oracle(oracle):
    import golden_state as gs
    d = np.load(GOLDEN / "driven301_fp64.npz")
    w = gs.DRIVEN301
    state = gs.initial_state(d, w["nx"], w["ny"], w["amp"], w["seed"])
    assert np.array_equal(np.stack(list(gs.state_sketches(*state).values())), d["sk0"])
    op = oracle.build_operators(w["nx"], w["ny"], w["nz"], w["L"])
    s, wind = oracle.rk4_step(op, oracle.OracleState(*state), w["dt"], w["mu"], w["vy"],
                              w["remove_winding"])
    assert wind == int(d["windings"][0])
    sk = gs.state_sketches(s.Z1, s.Z2, s.Z3, s.Z4, s.rhoi)
    for i, k in enumerate(("Z1", "Z2", "Z3", "Z4", "rho")):
        ref = d["sk1"][i]
        den = np.linalg.norm(d["sk1"][1] if k == "Z3" else ref)
        assert np.linalg.norm(sk[k] - ref) <= 1e-13 * den, k


def test_fixture_records_the_configuration():
    import json
    import golden_state as gs
    d = np.load(GOLDEN / "driven301_fp64.npz")
    meta = json.loads(str(d["meta"]))
    for k in ("nx", "ny", "nz", "L", "mu", "vy", "dt", "seed", "amp"):
        assert meta[k] == gs.DRIVEN301[k], k
    assert len(d["windings"]) == max(gs.DRIVEN301["checkpoints"])
