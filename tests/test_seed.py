"""Host-side seeding: Newton stationary solve, spline regrid, initial fields.

The reference ships three stationary seeds (``data/reference/mu=6,nz=30,
vy=7_20.mat``, ``mu=5,...,vy=3.8_20.mat``, ``mu=8,...,vy=13.5_20.mat``);
``tests/golden/make_golden.py`` stores them as the ``seed_*.npz`` fixtures.
Each must be a fixed point of the restated Newton solver and be reached by
its continuation from an analytic guess."""
import numpy as np
import pytest

from conftest import GOLDEN

VY7 = -2 * np.pi * 7 / 20
SHIPPED = [("seed_mu6_nz30_vy7", 6.0, 7.0), ("seed_mu5_nz30_vy3.8", 5.0, 3.8),
           ("seed_mu8_nz30_vy13.5", 8.0, 13.5)]


def load_seed(stem):
    d = np.load(GOLDEN / f"{stem}.npz")
    return {k: d[k] for k in d.files}


@pytest.mark.parametrize("stem,mu,n", SHIPPED)
def test_shipped_seed_is_newton_fixed_point(hqt, stem, mu, n):
    # the reference's own shipped profile satisfies the restated equations
    s = load_seed(stem)
    assert float(s["mu"]) == mu
    Z1, Z2, V, it, err = hqt.seed.NewtonRaphson_vy(30, s["Z1"], s["Z2"], s["Vy1"],
                                                   -2 * np.pi * n / 20)
    assert it == 0 and err < 1e-6
    assert np.max(np.abs(Z1 - s["Z1"])) < 1e-6


@pytest.mark.parametrize("stem,mu,n", SHIPPED)
def test_continuation_reproduces_shipped_seed(hqt, stem, mu, n):
    prof = hqt.seed.stationary_profile(mu, -2 * np.pi * n / 20)
    s = load_seed(stem)
    assert np.max(np.abs(prof.Z1 - s["Z1"])) < 1e-6
    assert np.max(np.abs(prof.Z2 - s["Z2"])) < 1e-6
    assert np.max(np.abs(prof.Vy1 - s["Vy1"])) < 1e-6
    assert np.max(np.abs(prof.rhoi - s["rhoi"])) < 1e-5


def test_smoke_test_newton_cases(hqt, shipped_seed):
    # hqt_smoke_test.m:180-183: vy = -2*pi*7/20 and vy = 0 from the seed
    s = shipped_seed
    for vy in (VY7, 0.0):
        Z1, Z2, V, it, err = hqt.seed.NewtonRaphson_vy(30, s["Z1"], s["Z2"],
                                                       s["Vy1"], vy)
        assert np.all(np.isfinite(np.r_[Z1, Z2, V])) and it < 1000
        assert np.isfinite(err)


@pytest.mark.parametrize("stem,mu,n", SHIPPED)
def test_rhoi_is_minus_lz_z2(hqt, stem, mu, n):
    _, Lz = hqt.seed.radial_grid(30)
    s = load_seed(stem)
    assert np.max(np.abs(-(Lz @ s["Z2"]) - s["rhoi"])) < 1e-9


def test_chebdif_matches_oracle(hqt, oracle):
    for n in (10, 17, 21, 33):
        x1, D1 = hqt.seed.chebdif(n)
        x2, DM = oracle.chebdif(n, 1)
        assert np.array_equal(x1, x2)
        assert np.max(np.abs(D1 - DM[0])) < 1e-12 * np.max(np.abs(DM[0]))


@pytest.mark.parametrize("mu", [4.5, 8.0])
def test_condensed_branch_over_mu(hqt, mu):
    p = hqt.seed.stationary_profile(mu, 0.0)
    assert p.Z1[0] > 0.1 and abs(p.Z2[-1] - mu) < 1e-9


def test_regrid_keeps_endpoints(hqt, shipped_seed):
    prof = hqt.seed.stationary_profile(6.0, VY7)
    z, (Z1, Z2, V, rho) = hqt.seed.regrid(prof, 21)
    assert z[0] == 1.0 and z[-1] == 0.0
    assert abs(Z2[-1] - 6.0) < 1e-9 and abs(V[-1] - VY7) < 1e-6


def test_init_driven_layout(hqt):
    prof = hqt.seed.stationary_profile(6.0, VY7)
    Z1, Z2, Z3, Z4, rhoi = hqt.seed.init_driven(16, 12, 9, prof, seed=3)
    assert Z1.shape == (16, 12, 9) and Z1.dtype == np.complex128
    assert np.allclose(Z4[:, :, -1], -VY7)       # A_y(z=0) = -vy
    assert np.allclose(Z2[:, :, -1], 6.0)
    assert np.all(Z3 == 0)
    assert np.ptp(rhoi) == 0.0
    # deterministic in the seed
    again = hqt.seed.init_driven(16, 12, 9, prof, seed=3)[0]
    assert np.array_equal(Z1, again)


def test_init_lattice_vortex_count(hqt, oracle):
    prof = hqt.seed.stationary_profile(6.0, 0.0)
    L = 64.0
    xs, ys, q = hqt.seed.random_vortices(8, L, L, seed=1)
    Z1, *_ = hqt.seed.init_lattice(64, 64, 9, prof, L, L, xs, ys, q, sigma=2.0)
    op = oracle.build_operators(64, 64, 9, L)
    O = oracle.boundary_order_parameter(op, Z1)
    n, npos, nneg = oracle.countN(O)
    assert (n, npos, nneg) == (8, 4, 4)
