"""The line-pass autotuner (hqt_params.autotune): it times every engine
pairing the build has for the grid (prime-factor tensor-core, compile-time
Stockham, runtime-plan) and the runtime engine's lines per block, keeps the
fastest, caches the choice per process and in the HQT_TUNE_CACHE file, and
leaves the context as created: a tuned run gives the untuned run's fields to
roundoff (different engines sum in different orders)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VY7 = -2 * np.pi * 7 / 20


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


@pytest.mark.parametrize("nx,ny,nz", [(64, 64, 21), (301, 40, 8), (48, 36, 12)])
def test_autotuned_run_matches_default_run(hqt, cuda, nx, ny, nz, tmp_path, monkeypatch):
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("HQT_TUNE_CACHE", str(cache))
    prof = hqt.seed.stationary_profile(6.0, VY7)
    state = hqt.seed.init_driven(nx, ny, nz, prof, noise="complex", amplitude=1e-2, seed=5)
    kw = dict(Lx=0.5 * nx, Ly=0.5 * ny, mu=6.0, vy=VY7, dt=0.02)
    with hqt.Simulation(nx, ny, nz, **kw) as sim:
        want, _ = sim.step(*state, nsteps=3)
        assert sim.config_report()["autotuned"] is False
    with hqt.Simulation(nx, ny, nz, autotune=True, **kw) as sim:
        rep = sim.config_report()
        got, info = sim.step(*state, nsteps=3)
    assert rep["autotuned"] is True
    if not rep["cached"]:
        cands = rep["candidates"]
        assert len(cands) >= 2
        best = min(cands, key=lambda c: c["ms_per_step"])
        assert best["geometry"] == rep["chosen"]
        assert cache.exists() and rep["key"] in cache.read_text()
    assert info.steps_done == 3
    for g, w in zip(got, want):
        assert rel_l2(g, w) < 1e-12
    # a second context of the same configuration takes the cached choice
    with hqt.Simulation(nx, ny, nz, autotune=True, **kw) as sim:
        rep2 = sim.config_report()
    assert rep2["cached"] is True and rep2["chosen"] == rep["chosen"]
