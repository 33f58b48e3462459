"""Boundary-field extraction (scripts/analysis/plots_cluster.m:77-99) on the
CPU: the oracle's velocity observable, MATLAB's column-wise max, the output
file name and the MAT v5 file."""
import importlib

import numpy as np
import pytest


@pytest.fixture(scope="module")
def ckpt(hqt):
    return importlib.import_module(hqt.__name__ + ".checkpoint")


def test_velocity_normalised_per_y_column(oracle):
    # O(x, y) = c(y) g(x): band-limited g, so the spectral derivative is exact.
    # MATLAB's max(abs(O)) of the nx x ny slice is the row of column maxima:
    # each y column is divided by its own maximum, so vx does not depend on c.
    nx, ny = 32, 8
    x = np.arange(nx) * 2 * np.pi / nx
    g = 1.5 * np.exp(1j * x) + 0.25 * np.exp(2j * x) + 0.25
    dg = 1.5j * np.exp(1j * x) + 0.5j * np.exp(2j * x)
    c = 1.0 + np.arange(ny)
    O = g[:, None] * c[None, :]
    vx, vy = oracle.boundary_velocity(O, 2 * np.pi, 2 * np.pi)
    want = np.abs(g) / np.abs(g).max() * np.imag(dg / g)
    for j in range(ny):
        assert np.max(np.abs(vx[:, j] - want)) < 1e-12
    assert np.max(np.abs(vy)) < 1e-12


def test_boundary_fields_frame(oracle):
    nx, ny, nz = 24, 20, 7
    rng = np.random.default_rng(3)
    x = np.arange(nx)[:, None] * 2 * np.pi / nx
    y = np.arange(ny)[None, :] * 2 * np.pi / ny
    psi = (np.sin(x + 0.3) + 1j * np.sin(y + 1.1) + 0.2) * (np.sin(2 * x) + 1j * np.sin(y) - 0.1)
    Z1 = psi[:, :, None] * np.linspace(1, 0, nz)[None, None, :] * (1 + 0.01 * rng.standard_normal(nz))
    op = oracle.build_operators(nx, ny, nz, 10.0, 9.0)
    O, vx, vy, n = oracle.boundary_fields(op, Z1)
    assert np.allclose(O, oracle.boundary_order_parameter(op, Z1), rtol=0, atol=0)
    assert n == oracle.countN(O)[0]
    wx, wy = oracle.boundary_velocity(O, 10.0, 9.0)
    assert np.array_equal(vx, wx) and np.array_equal(vy, wy)


def test_num2str_and_driven_name(ckpt):
    assert ckpt.num2str(6) == "6"
    assert ckpt.num2str(6.0) == "6"
    assert ckpt.num2str(np.pi) == "3.1416"
    assert ckpt.num2str(-2.5) == "-2.5"
    assert ckpt.num2str(0.05) == "0.05"
    assert ckpt.num2str(123.456) == "123.456"
    vy_load = -2 * np.pi * 7 / 20
    assert ckpt.driven_name(6, vy_load) == "driven_mu=6,v=7_20.mat"
    assert ckpt.driven_name(4.5, -2 * np.pi * 3 / 20) == "driven_mu=4.5,v=3_20.mat"


def test_boundary_field_file_roundtrip(ckpt, tmp_path):
    rng = np.random.default_rng(0)
    nx, ny, nt = 6, 5, 3
    NofV = np.arange(nt, dtype=np.float64).reshape(1, nt)
    O = rng.standard_normal((nx, ny, nt)) + 1j * rng.standard_normal((nx, ny, nt))
    vx, vy = rng.standard_normal((2, nx, ny, nt))
    p = ckpt.save_boundary_fields(tmp_path / ckpt.driven_name(6, -2 * np.pi * 7 / 20),
                                  NofV, O, vx, vy)
    a, b, c, d = ckpt.load_boundary_fields(p)
    assert a.shape == (1, nt) and np.array_equal(a, NofV)
    assert np.array_equal(b, O) and np.array_equal(c, vx) and np.array_equal(d, vy)
