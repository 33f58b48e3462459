"""Boundary-field extraction on the GPU (hqt_boundary_velocity_device and the
checkpoint -> driven_*.mat pipeline) against the oracle.  The weighted
velocity is bounded at vortex cores, so it is compared relative to its
maximum; vortex counts are bit-exact."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def vortex_field(nx, ny, nz, nv, seed):
    rng = np.random.default_rng(seed)
    x = np.arange(nx)[:, None] * 2 * np.pi / nx
    y = np.arange(ny)[None, :] * 2 * np.pi / ny
    psi = np.ones((nx, ny), dtype=complex)
    for _ in range(nv):
        kx, ky = rng.integers(1, 4, size=2)
        psi *= (np.sin(kx * x + rng.uniform(0, 6)) + 1j * np.sin(ky * y + rng.uniform(0, 6)) + 0.2)
    z = np.linspace(1, 0, nz)
    return psi[:, :, None] * (z * (1.5 - z))[None, None, :]


def relmax(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("nx,ny,nz", [(64, 64, 9), (301, 301, 9), (53, 48, 8)])
def test_boundary_velocity_parity(hqt, oracle, cuda, nx, ny, nz):
    api = importlib.import_module(hqt.__name__ + ".api")
    Lx, Ly = 0.4 * nx, 0.35 * ny
    Z1 = vortex_field(nx, ny, nz, 4, seed=nx + 1)
    op = oracle.build_operators(nx, ny, nz, Lx, Ly)
    O = oracle.boundary_order_parameter(op, Z1)
    vx, vy = oracle.boundary_velocity(O, Lx, Ly)
    with hqt.Simulation(nx, ny, nz, Lx=Lx, Ly=Ly) as sim:
        gx, gy = sim.boundary_velocity_device(api.to_device(O[:, :, None])[0])
    assert relmax(api.from_device(gx), vx) < 1e-10
    assert relmax(api.from_device(gy), vy) < 1e-10


def test_extract_boundary_fields_from_checkpoints(hqt, oracle, cuda, tmp_path):
    ck = importlib.import_module(hqt.__name__ + ".checkpoint")
    nx, ny, nz, L = 48, 40, 9, 20.0
    op = oracle.build_operators(nx, ny, nz, L, L)
    paths, want = [], []
    for t, seed in ((10, 1), (20, 2), (30, 3)):
        Z1 = vortex_field(nx, ny, nz, 3, seed)
        z = np.zeros((nx, ny, nz))
        paths.append(ck.save_checkpoint(tmp_path / ck.checkpoint_name(t), Z1, z, z, z, z))
        want.append(oracle.boundary_fields(op, Z1))
    with hqt.Simulation(nx, ny, nz, Lx=L, Ly=L) as sim:
        NofV, O, vx, vy = ck.extract_boundary_fields(sim, paths)
    assert NofV.shape == (1, 3) and O.shape == (nx, ny, 3)
    for i, (o, wx, wy, n) in enumerate(want):
        assert NofV[0, i] == n
        assert relmax(O[:, :, i], o) < 1e-12
        assert relmax(vx[:, :, i], wx) < 1e-10
        assert relmax(vy[:, :, i], wy) < 1e-10
    out = ck.save_boundary_fields(tmp_path / ck.driven_name(6, -2 * np.pi * 7 / 20),
                                  NofV, O, vx, vy)
    a, b, c, d = ck.load_boundary_fields(out)
    assert np.array_equal(a, NofV) and np.array_equal(b, O)
