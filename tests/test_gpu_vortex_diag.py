"""Vortex positions (find_vortices) and vortex structure factors
(compute_vortex_structure_factor) on the GPU against the oracle.  Charges,
find order and refined positions are exact (integer sums and one division);
spectra agree to FFT roundoff."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def smoke_phi():
    g = np.arange(33) * 2 * np.pi / 33
    x, y = np.meshgrid(g, g, indexing="ij")
    return np.sin(x + 0.271) + 1j * np.sin(y + 0.613)


def vortex_plane(nx, ny, nv, seed):
    rng = np.random.default_rng(seed)
    x = np.arange(nx)[:, None] * 2 * np.pi / nx
    y = np.arange(ny)[None, :] * 2 * np.pi / ny
    psi = np.ones((nx, ny), dtype=complex)
    for _ in range(nv):
        kx, ky = rng.integers(1, 5, size=2)
        psi *= (np.sin(kx * x + rng.uniform(0, 6)) + 1j * np.sin(ky * y + rng.uniform(0, 6))
                + rng.uniform(-0.3, 0.3))
    return psi


CASES = [("smoke", 33, 33), ("v64", 64, 64), ("v301", 301, 301), ("v53x48", 53, 48)]


def field(name, nx, ny):
    return smoke_phi() if name == "smoke" else vortex_plane(nx, ny, 4, seed=nx + ny)


@pytest.mark.parametrize("name,nx,ny", CASES)
def test_find_vortices_parity(hqt, oracle, cuda, name, nx, ny):
    api = importlib.import_module(hqt.__name__ + ".api")
    O = field(name, nx, ny)
    want_v, want_a = oracle.find_vortices(O, 0.4, 2)
    with hqt.Simulation(nx, ny, 5, Lx=10.0) as sim:
        v, a = sim.find_vortices_device(api.to_device(O[:, :, None])[0], 0.4, 2)
    assert v.shape == want_v.shape and a.shape == want_a.shape
    assert np.array_equal(v, want_v) and np.array_equal(a, want_a)


@pytest.mark.parametrize("name,nx,ny", CASES)
def test_structure_factor_parity(hqt, oracle, cuda, name, nx, ny):
    api = importlib.import_module(hqt.__name__ + ".api")
    O = field(name, nx, ny)
    Lx, Ly = 2 * np.pi, 1.7 * np.pi
    k, Sc, Sn, vort, sp = oracle.vortex_structure_factor(O, Lx, Ly)
    with hqt.Simulation(nx, ny, 5, Lx=10.0) as sim:
        gk, gSc, gSn, gv, gsp = sim.vortex_structure_factor_device(
            api.to_device(O[:, :, None])[0], Lx, Ly)
    assert np.array_equal(gv, vort)
    assert len(gk) == len(k) and np.array_equal(gk, k)
    for got, want in ((gSc, Sc), (gSn, Sn)):
        assert np.max(np.abs(got - want)) <= 1e-10 * max(np.max(np.abs(want)), 1.0)
    for key in sp:
        assert abs(gsp[key] - sp[key]) <= 1e-12 * abs(sp[key])


def test_vortex_diagnostics_without_vortices(hqt, cuda):
    api = importlib.import_module(hqt.__name__ + ".api")
    O = np.ones((24, 20), complex) * (1 + 0.5j)
    with hqt.Simulation(24, 20, 5, Lx=10.0) as sim:
        t = api.to_device(O[:, :, None])[0]
        v, a = sim.find_vortices_device(t, 0.4, 2)
        k, Sc, Sn, vort, sp = sim.vortex_structure_factor_device(t, 1.0, 1.0)
    assert v.shape == (0, 2) and a.shape == (0, 2)
    assert k.size == 0 and vort.shape == (0, 3) and sp is None
