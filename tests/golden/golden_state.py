"""Helpers shared by the golden-fixture generator and the tests that read it.

The fixture of the driven 301x301x21 run (``driven301_fp64.npz``) is too
large to hold as whole fields (76 MB per state), so it stores:

* the radial profiles the initial state is built from, so that the initial
  fields are rebuilt bit for bit from the fixture plus the seeded noise
  (no Newton solve, no LAPACK rounding differences between machines);
* Rademacher sketches of every field at a few step counts: ``K`` projections
  ``s_k = sum_i r_k(i) a(i)`` with ``r_k(i) = +-1`` drawn from
  ``numpy.random.default_rng(SKETCH_SEED)`` over the MATLAB (column-major)
  linear index.  ``E||S d||^2 = K ||d||^2``, so ``||S(a-b)|| / ||S b||``
  estimates the relative L2 difference of the whole field (relative spread
  about ``sqrt(2/K)``);
* exact planes of every field at the last step (the level next to the AdS
  boundary and the boundary charge), compared value by value.
"""
from __future__ import annotations

import numpy as np

SKETCH_ROWS = 32
SKETCH_SEED = 20240601

DRIVEN301 = dict(nx=301, ny=301, nz=21, L=100.0, mu=6.0, vy=-2 * np.pi * 7 / 20,
                 dt=0.02, remove_winding=True, noise="complex", amp=1e-3, seed=0,
                 checkpoints=(1, 10, 50, 100))


def profile_arrays(prof, nz: int):
    """Radial columns of the driven initial state (``seed.init_driven``):
    ``psi(z) = Z1(z) e^{i theta(z)}``, ``A_t(z)``, ``A_y(z) = -Vy1(z)`` and the
    boundary charge, on ``nz`` points."""
    import importlib
    seed = importlib.import_module("ads4-holographic-quantum-turbulence_b200.seed")
    z, (Z1p, Z2p, Vy1p, rhop) = seed.regrid(prof, nz)
    theta = seed._theta_profile(z, Z2p)
    return dict(psi_z=Z1p * np.exp(1j * theta), at_z=Z2p, ay_z=-Vy1p,
                rho_b=np.float64(rhop[-1]))


def initial_state(fx, nx: int, ny: int, amp: float, seed: int):
    """``seed.init_driven`` with complex noise, rebuilt from stored columns."""
    psi_z, at_z, ay_z = fx["psi_z"], fx["at_z"], fx["ay_z"]
    nz = psi_z.size
    rng = np.random.default_rng(seed)
    pert = 1.0 + amp * (rng.standard_normal((nx, ny)) + 1j * rng.standard_normal((nx, ny)))
    Z1 = (pert[:, :, None] * psi_z[None, None, :]).astype(np.complex128)
    Z2 = np.broadcast_to(at_z[None, None, :], (nx, ny, nz)).copy()
    Z3 = np.zeros((nx, ny, nz))
    Z4 = np.broadcast_to(ay_z[None, None, :], (nx, ny, nz)).copy()
    rhoi = np.full((nx, ny, nz), float(fx["rho_b"]))
    return Z1, Z2, Z3, Z4, rhoi


def sketch(a: np.ndarray, rows: int = SKETCH_ROWS, seed: int = SKETCH_SEED) -> np.ndarray:
    """Rademacher projections of ``a`` over its column-major linear index
    (complex arrays: the same rows applied to the real and imaginary parts)."""
    v = np.asarray(a).ravel(order="F")
    rng = np.random.default_rng(seed)
    out = np.zeros(rows, dtype=np.complex128 if np.iscomplexobj(v) else np.float64)
    for k in range(rows):
        r = rng.integers(0, 2, size=v.size, dtype=np.int8).astype(np.float64) * 2.0 - 1.0
        out[k] = r @ v.real + (1j * (r @ v.imag) if np.iscomplexobj(v) else 0.0)
    return out


def sketch_rel(s_got: np.ndarray, s_want: np.ndarray) -> float:
    """Sketch estimate of ``||got - want|| / ||want||``."""
    return float(np.linalg.norm(s_got - s_want) / max(np.linalg.norm(s_want), 1e-300))


def state_sketches(Z1, Z2, Z3, Z4, rhoi) -> dict:
    """Sketches of the five fields; rhoi by its boundary plane."""
    return dict(Z1=sketch(Z1), Z2=sketch(Z2), Z3=sketch(Z3), Z4=sketch(Z4),
                rho=sketch(np.asarray(rhoi)[:, :, -1]))


LATTICE128 = dict(nx=128, nz=25, L=32.0, mu=6.0, dt=0.02, vortices=26, seed=1,
                  every=50, max_steps=3000)


def lattice_state(prof, w):
    """The vortex-lattice initial fields of ``seed.init_lattice`` for the
    configuration ``w`` (bare atan2 imprint, as tevol_lattice.m:109-135)."""
    import importlib
    seed = importlib.import_module("ads4-holographic-quantum-turbulence_b200.seed")
    rng = np.random.default_rng(w["seed"])
    nv, L = w["vortices"], w["L"]
    xs, ys = rng.uniform(0, L, nv), rng.uniform(0, L, nv)
    q = np.r_[np.ones(nv // 2), -np.ones(nv - nv // 2)]
    return seed.init_lattice(w["nx"], w["nx"], w["nz"], prof, L, L, xs, ys, q,
                             periodic_images=0)


def profile_from(d):
    """A ``seed.StationaryProfile`` from its stored arrays."""
    import importlib
    seed = importlib.import_module("ads4-holographic-quantum-turbulence_b200.seed")
    z = np.asarray(d["z"])
    return seed.StationaryProfile(6.0, 0.0, z, np.asarray(d["Z1"]), np.asarray(d["Z2"]),
                                  np.asarray(d["Vy1"]), np.asarray(d["rhoi"]), 0)
