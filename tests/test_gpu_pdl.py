"""Programmatic dependent launch (the step's kernels wait in
griddepcontrol.wait for the kernel before them): the fields must be the same
bits with it on and off (HQT_PDL=0, read when a context is created), on every
line engine, in mixed precision and in an ensemble; the context reports
whether its step graph carries it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VY7 = -2 * np.pi * 7 / 20


def run(hqt, monkeypatch, pdl, nx, ny, nz, nsteps=4, engine=None, mixed=False):
    monkeypatch.setenv("HQT_PDL", "1" if pdl else "0")
    if engine:
        monkeypatch.setenv("HQT_LINE_ENGINE", engine)
    else:
        monkeypatch.delenv("HQT_LINE_ENGINE", raising=False)
    prof = hqt.seed.stationary_profile(6.0, VY7)
    state = hqt.seed.init_driven(nx, ny, nz, prof, noise="complex", amplitude=1e-2, seed=3)
    kw = dict(Lx=0.5 * nx, Ly=0.5 * ny, mu=6.0, vy=VY7, dt=0.02)
    if mixed:
        kw["precision"] = "mixed"
    with hqt.Simulation(nx, ny, nz, **kw) as sim:
        fields, info = sim.step(*state, nsteps=nsteps)
        rep = sim.config_report()
    assert info.steps_done == nsteps
    return fields, rep


@pytest.mark.parametrize("nx,ny,nz,engine", [(301, 301, 9, None), (64, 48, 21, None),
                                             (64, 48, 25, "runtime"), (40, 36, 33, None)])
def test_pdl_bit_identical(hqt, cuda, monkeypatch, nx, ny, nz, engine):
    on, rep_on = run(hqt, monkeypatch, True, nx, ny, nz, engine=engine)
    off, rep_off = run(hqt, monkeypatch, False, nx, ny, nz, engine=engine)
    assert rep_off["pdl"] is False
    assert isinstance(rep_on["pdl"], bool)
    for a, b in zip(on, off):
        assert np.array_equal(a, b)


def test_pdl_bit_identical_mixed(hqt, cuda, monkeypatch):
    on, _ = run(hqt, monkeypatch, True, 301, 301, 9, mixed=True)
    off, _ = run(hqt, monkeypatch, False, 301, 301, 9, mixed=True)
    for a, b in zip(on, off):
        assert np.array_equal(a, b)


def test_pdl_bit_identical_ensemble(hqt, cuda, monkeypatch):
    api = __import__(hqt.__name__ + ".api", fromlist=["to_device"])
    members = [(64, 64, 21, "fp64"), (48, 40, 25, "mixed")]

    def ens_run(pdl):
        monkeypatch.setenv("HQT_PDL", "1" if pdl else "0")
        monkeypatch.delenv("HQT_LINE_ENGINE", raising=False)
        sims, states = [], []
        for k, (nx, ny, nz, prec) in enumerate(members):
            prof = hqt.seed.stationary_profile(6.0, VY7)
            st = hqt.seed.init_driven(nx, ny, nz, prof, noise="complex", amplitude=1e-3, seed=k)
            sims.append(hqt.Simulation(nx, ny, nz, Lx=0.5 * nx, Ly=0.5 * ny, mu=6.0, vy=VY7,
                                       dt=0.02, precision=prec))
            states.append([api.to_device(a) for a in st])
        with hqt.Ensemble(sims) as ens:
            info = ens.step_device(states, nsteps=5)
        for s in sims:
            s.close()
        assert [i.steps_done for i in info] == [5, 5]
        return [[api.from_device(x) for x in st] for st in states]

    on, off = ens_run(True), ens_run(False)
    for a, b in zip(on, off):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
