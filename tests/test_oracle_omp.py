"""The C + OpenMP restatement of the step (``oracle/hqt_step_omp.c``, the
timed CPU baseline) against the NumPy oracle on the same inputs: the same
arithmetic in another order, so they agree to roundoff (bar 1e-13 relative
L2 after a few steps; windings identical)."""
import numpy as np
import pytest

VY7 = -2 * np.pi * 7 / 20


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


@pytest.fixture(scope="module")
def omp(oracle):
    import subprocess
    from pathlib import Path
    root = Path(oracle.__file__).resolve().parent
    subprocess.run(["make", "-C", str(root), "-s"], check=True)
    return oracle


@pytest.mark.parametrize("nx,ny,nz,L,vy,rw,filt,nsteps", [
    (33, 33, 10, 16.0, VY7, True, True, 5),      # driven, winding imprinted
    (48, 40, 12, 20.0, 0.0, False, True, 3),     # lattice script, non-square
    (30, 22, 8, 12.0, VY7, True, False, 3),      # without the filter
])
def test_omp_step_matches_numpy_oracle(hqt, omp, nx, ny, nz, L, vy, rw, filt, nsteps):
    oracle = omp
    prof = hqt.seed.stationary_profile(6.0, vy)
    st = list(hqt.seed.init_driven(nx, ny, nz, prof, noise="complex", amplitude=1e-2, seed=4))
    st[0] = st[0] * np.exp(2j * np.pi * 2 * np.arange(ny) / ny)[None, :, None]
    op = oracle.build_operators(nx, ny, nz, L)
    s = oracle.OracleState(*[a.copy() for a in st])
    ws = []
    for _ in range(nsteps):
        s, w = oracle.rk4_step(op, s, 0.02, 6.0, vy, rw, filt)
        ws.append(w)
    c, cw, bad = oracle.omp_run(op, oracle.OracleState(*st), nsteps, 0.02, 6.0, vy, rw, filt)
    assert bad == 0 and cw == ws
    for got, want in ((c.Z1, s.Z1), (c.Z2, s.Z2), (c.Z4, s.Z4), (c.rhoi, s.rhoi)):
        assert rel_l2(got, want) < 1e-13
    assert np.max(np.abs(c.Z3 - s.Z3)) < 1e-13 * np.max(np.abs(s.Z2))


def test_omp_step_stops_at_nan(hqt, omp):
    oracle = omp
    prof = hqt.seed.stationary_profile(6.0, 0.0)
    st = list(hqt.seed.init_driven(16, 16, 6, prof))
    st[2] = st[2].copy()
    st[2][3, 4, 2] = np.nan
    op = oracle.build_operators(16, 16, 6, 8.0)
    _, ws, bad = oracle.omp_run(op, oracle.OracleState(*st), 5, 0.02, 6.0, 0.0)
    assert bad == 1 and len(ws) == 1
