"""The full-size configurations, through size-independent properties.

The oracle cannot step these grids in test time, so at full size the checks
are: mixed precision against the FP64 path (itself pinned to the oracle on
smaller grids) within the mixed-precision bar of 1e-6 (relative L2; A_x, A_y
on the gauge scale max|A_t|), finite fields, vortex counts of the
GPU's boundary order parameter bit-exact against the oracle's countN of the
same field, and the energy spectrum of that field against the oracle.

- 512x512x25, L = 128, mu = 6, dt = 0.02, 400 vortices (+-1, equal numbers,
  uniform positions, seed 1) imprinted on the stationary profile, no winding
  removal (the vortex-lattice decay run);
- 1024x1024x33, L = 256, mu = 6, dt = 0.01: a seeded vortex tangle (unit
  modulus phase field of a smoothed complex Gaussian field, seed 2) on the
  stationary profile (the large single run).
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def mixed_vs_fp64(hqt, state, nx, nz, L, dt, nsteps, remove_winding):
    api = importlib.import_module(hqt.__name__ + ".api")
    out, O = {}, None
    for prec in ("fp64", "mixed"):
        t = [api.to_device(a) for a in state]
        with hqt.Simulation(nx, nx, nz, Lx=L, mu=6.0, vy=0.0, dt=dt,
                            remove_winding=remove_winding, precision=prec) as sim:
            sim.step_device(*t, nsteps=nsteps)
            if prec == "fp64":
                Od = sim.order_parameter_device(t[0])
                counts = sim.count_vortices_device(Od)
                O = api.from_device(Od)
                k, E, Ec, Ei = sim.energy_spectrum_device(Od)
        out[prec] = [api.from_device(x) for x in t]
        del t
    m, f = out["mixed"], out["fp64"]
    scale = np.max(np.abs(f[1]))
    errs = {"Z1": rel_l2(m[0], f[0]), "Z2": rel_l2(m[1], f[1]), "rhoi": rel_l2(m[4], f[4]),
            "Z3_abs": float(np.max(np.abs(m[2] - f[2])) / scale),
            "Z4_abs": float(np.max(np.abs(m[3] - f[3])) / scale)}
    for a in f:
        assert np.all(np.isfinite(a))
    return errs, O, counts, (k, E, Ec, Ei)


def test_lattice_512x25(hqt, oracle, cuda):
    nx, nz, L, nv = 512, 25, 128.0, 400
    prof = hqt.seed.stationary_profile(6.0, 0.0)
    rng = np.random.default_rng(1)
    xs, ys = rng.uniform(0, L, nv), rng.uniform(0, L, nv)
    q = np.r_[np.ones(nv // 2), -np.ones(nv // 2)]
    state = hqt.seed.init_lattice(nx, nx, nz, prof, L, L, xs, ys, q, periodic_images=0)
    errs, O, counts, spec = mixed_vs_fp64(hqt, state, nx, nz, L, 0.02, 20, False)
    print("512^2x25 lattice, mixed vs fp64 after 20 steps:", errs, "counts", counts)
    # vortex cores and phase windings: ~2.5e-8 after 20 steps (FP32 rounding
    # of the line derivatives accumulates roughly linearly in the step count)
    assert max(errs.values()) < 1e-6, errs
    assert counts == oracle.countN(O)
    # the imprint's bare phase (no periodic images) adds windings at the seams
    assert counts[0] >= nv // 2


def test_large_1024x33(hqt, oracle, cuda):
    nx, nz, L = 1024, 33, 256.0
    prof = hqt.seed.stationary_profile(6.0, 0.0)
    z, (Z1p, Z2p, Vy1p, rhop) = hqt.seed.regrid(prof, nz)
    rng = np.random.default_rng(2)
    noise = rng.standard_normal((nx, nx)) + 1j * rng.standard_normal((nx, nx))
    k = np.fft.fftfreq(nx)
    u = np.fft.ifft2(np.fft.fft2(noise) * np.exp(-(k[:, None] ** 2 + k[None, :] ** 2) * 20.0 ** 2))
    a = np.abs(u)
    plane = u / a * np.tanh(a / (0.5 * np.sqrt(np.mean(a ** 2))))
    psi = Z1p * np.exp(1j * hqt.seed._theta_profile(z, Z2p))
    Z1 = plane[:, :, None] * psi[None, None, :]
    Z2 = np.broadcast_to(Z2p[None, None, :], (nx, nx, nz)).copy()
    Z3 = np.zeros((nx, nx, nz))
    Z4 = np.broadcast_to(-Vy1p[None, None, :], (nx, nx, nz)).copy()
    rhoi = np.full((nx, nx, nz), float(rhop[-1]))
    errs, O, counts, (kk, E, Ec, Ei) = mixed_vs_fp64(hqt, (Z1, Z2, Z3, Z4, rhoi), nx, nz, L,
                                                     0.01, 2, True)
    print("1024^2x33 tangle, mixed vs fp64 after 2 steps:", errs, "counts", counts)
    assert max(errs.values()) < 1e-6, errs
    assert counts == oracle.countN(O)
    assert counts[0] > 100
    k2, E2, Ec2, Ei2 = oracle.energy_spectrum(O, L, L)
    assert len(kk) == len(k2)
    for got, want in ((E, E2), (Ec, Ec2), (Ei, Ei2)):
        assert np.max(np.abs(got - want)) < 1e-9 * E2.max()
