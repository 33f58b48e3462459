"""Host-side FP64 seeding: stationary radial profiles and initial fields.

Everything here runs once per run on the host in FP64, exactly as in the
reference (the Newton solve is a 3*nz dense system).  The CUDA library only
evolves the fields these functions produce.

* ``chebdif``          -- ``third_party/dmsuite/chebdif.m:25-53`` (D1 only)
* ``NewtonRaphson_vy`` -- ``src/solvers/NewtonRaphson_vy.m:1-105``
* ``regrid``           -- the ``interp1(...,'spline')`` of
  ``scripts/simulation/tevol_driven_cluster.m:84`` (not-a-knot cubic spline)
* ``init_driven``      -- ``tevol_driven_cluster.m:85-102``
* ``init_lattice``     -- ``tevol_lattice.m:86-136`` (vortex imprint)
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

__all__ = ["chebdif", "radial_grid", "NewtonRaphson_vy", "StationaryProfile",
           "stationary_profile", "regrid", "init_driven", "init_lattice",
           "random_vortices"]


def chebdif(N: int):
    """Chebyshev points ``x`` (``x[0]=+1``) and first-derivative matrix.

    Same construction as ``third_party/dmsuite/chebdif.m:25-53`` with M=1:
    trigonometric differences with the flipping trick and the
    negative-row-sum diagonal.
    """
    k = np.arange(N)
    th = k * np.pi / (N - 1)
    x = np.sin(np.pi * np.arange(N - 1, -N, -2) / (2.0 * (N - 1)))
    half = th / 2
    DX = 2.0 * np.sin(half[None, :] + half[:, None]) * \
        np.sin(half[None, :] - half[:, None])
    n1, n2 = N // 2, int(math.ceil(N / 2))
    DX = np.concatenate([DX[:n1], -DX[:n2][::-1, ::-1]], axis=0)
    np.fill_diagonal(DX, 1.0)
    sgn = (-1.0) ** k
    C = sgn[:, None] * sgn[None, :]
    C[0, :] *= 2.0
    C[-1, :] *= 2.0
    C[:, 0] /= 2.0
    C[:, -1] /= 2.0
    Z = 1.0 / DX
    np.fill_diagonal(Z, 0.0)
    # first derivative: D = Z .* (C .* diag(I) - I), then the diagonal fix
    D = Z * (C - np.eye(N))
    np.fill_diagonal(D, 0.0)
    np.fill_diagonal(D, -D.sum(axis=1))
    return x, D


def radial_grid(nz: int):
    """Radial coordinate ``z`` (1 at the horizon, 0 at the AdS boundary) and
    ``Lz = 2*D1`` on ``nz`` Chebyshev points (``NewtonRaphson_vy.m:12-20``)."""
    x, D = chebdif(nz)
    return (x - 1.0) / 2.0 + 1.0, 2.0 * D


def NewtonRaphson_vy(nz: int, Z1, Z2, vy1, vy: float, zh: float = 1.0,
                     it_max: int = 1000, tol: float = 1e-6):
    """Stationary profiles ``(Psi, A_t, A_y)`` with the boundary flow ``vy``.

    Restates ``src/solvers/NewtonRaphson_vy.m``: the three coupled radial
    equations (:32-34), the analytic block Jacobian (:37-39), the four
    endpoint rows replaced by identity rows (:50-52,60-66), ``y=-J\\F``
    (:69) and the stop test ``max|F_next| < 1e-6`` (:92).  Returns
    ``(Z1, Z2, Vy1, iterations, update_norm)``.
    """
    z, Lz = radial_grid(nz)
    LLz = Lz @ Lz
    f = 1.0 - (z / zh) ** 3
    df = -3.0 * z ** 2 / zh ** 3
    Z1 = np.asarray(Z1, dtype=np.float64).reshape(nz).copy()
    Z2 = np.asarray(Z2, dtype=np.float64).reshape(nz).copy()
    vy1 = np.asarray(vy1, dtype=np.float64).reshape(nz).copy()

    def z2_over_f(Z2v):
        out = np.zeros(nz)
        out[1:] = Z2v[1:] / (1.0 - (z[1:] / zh) ** 3)
        out[0] = -(Lz @ Z2v)[0] / 3.0
        return out

    def fun(Z1v, Z2v, Vy1v, Z2f):
        return np.concatenate([
            f * (LLz @ Z1v) + df * (Lz @ Z1v) - Vy1v ** 2 * Z1v
            + Z2v * Z2f * Z1v - z * Z1v,
            f * (LLz @ Z2v) - 2.0 * Z1v ** 2 * Z2v,
            -f * (LLz @ Vy1v) - df * (Lz @ Vy1v) + 2.0 * Vy1v * Z1v ** 2])

    def dfun(Z1v, Z2v, Vy1v, Z2f):
        J = np.zeros((3 * nz, 3 * nz))
        A = f[:, None] * LLz + df[:, None] * Lz
        J[:nz, :nz] = A + np.diag(Z2v * Z2f - Vy1v ** 2 - z)
        J[:nz, nz:2 * nz] = np.diag(2.0 * Z2f * Z1v)
        J[:nz, 2 * nz:] = np.diag(-2.0 * Vy1v * Z1v)
        J[nz:2 * nz, :nz] = np.diag(-4.0 * Z1v * Z2v)
        J[nz:2 * nz, nz:2 * nz] = f[:, None] * LLz - np.diag(2.0 * Z1v ** 2)
        J[2 * nz:, :nz] = np.diag(4.0 * Vy1v * Z1v)
        J[2 * nz:, 2 * nz:] = -A + np.diag(2.0 * Z1v ** 2)
        return J

    Z2f = z2_over_f(Z2)
    vy1 = vy1 - vy1[nz - 1]
    Vy1 = vy + vy1
    # rows (1-based) nz, nz+1, 2nz, 3nz are replaced by endpoint conditions
    bc_rows = np.array([nz - 1, nz, 2 * nz - 1, 3 * nz - 1])
    BCz = np.zeros((4, 3 * nz))
    BCz[np.arange(4), bc_rows] = 1.0
    K = 0
    err = float("nan")
    Fun_next = None
    while K < it_max:
        if K == 0:
            Fun = fun(Z1, Z2, Vy1, Z2f)
            Fun[bc_rows] = 0.0
        else:
            Fun = Fun_next
        dFun = dfun(Z1, Z2, Vy1, Z2f)
        dFun[bc_rows, :] = BCz
        y = -np.linalg.solve(dFun, Fun)
        Z1t = Z1 + y[:nz]
        Z2t = Z2 + y[nz:2 * nz]
        Vy1t = Vy1 + y[2 * nz:]
        Z2ft = z2_over_f(Z2t)
        Fun_next = fun(Z1t, Z2t, Vy1t, Z2ft)
        Fun_next[bc_rows] = 0.0
        err2 = float(np.max(np.abs(Fun_next)))
        Z1, Z2, Vy1, Z2f = Z1t, Z2t, Vy1t, Z2ft
        err = float(np.max(np.abs(y)))
        if math.isnan(err):
            break
        if err2 < tol:
            break
        K += 1
    return Z1, Z2, Vy1, K, err


@dataclass
class StationaryProfile:
    """Radial profiles on ``nz`` Chebyshev points (index 0 = horizon)."""
    mu: float
    vy: float
    z: np.ndarray
    Z1: np.ndarray      # Psi(z)
    Z2: np.ndarray      # A_t(z)
    Vy1: np.ndarray     # A_y(z) of the stationary flowing state
    rhoi: np.ndarray    # -Lz*Z2
    iterations: int


def stationary_profile(mu: float = 6.0, vy: float = 0.0, nz0: int = 30,
                       step: float = 0.25) -> StationaryProfile:
    """Stationary state at chemical potential ``mu`` and boundary flow ``vy``.

    The reference seeds its runs from a stored profile that its seed
    notebook obtained by Newton continuation
    (``scripts/legacy/Statinary_state_with_v.m:15-56``).  Here the same
    solver (``NewtonRaphson_vy``) starts on the condensed branch at
    ``mu=6, vy=0`` from the analytic guess ``Psi=3z(1-z/2)``,
    ``A_t=6(1-z)``, ``A_y=0`` and is continued in ``mu`` (rescaling ``A_t`` by
    ``mu_new/mu_old`` as at ``Statinary_state_with_v.m:50``) and then in
    ``vy``, in steps of at most ``step``.  ``rhoi=-Lz*Z2``
    (``Statinary_state_with_v.m:53``).
    """
    z, Lz = radial_grid(nz0)
    Z1, Z2, Vy1, it, _ = NewtonRaphson_vy(nz0, 3.0 * z * (1.0 - 0.5 * z),
                                          6.0 * (1.0 - z), np.zeros(nz0), 0.0)
    if not Z1[0] > 0.1:
        raise RuntimeError("stationary solve did not reach the condensed branch")
    cur = 6.0
    nmu = max(1, int(math.ceil(abs(mu - cur) / step)))
    for m in np.linspace(cur, mu, nmu + 1)[1:]:
        Z2 = Z2 * (m / cur)
        Z1, Z2, Vy1, k, _ = NewtonRaphson_vy(nz0, Z1, Z2, Vy1, 0.0)
        it += k
        cur = m
    nvy = max(1, int(math.ceil(abs(vy) / step)))
    for v in np.linspace(0.0, vy, nvy + 1)[1:]:
        Z1, Z2, Vy1, k, _ = NewtonRaphson_vy(nz0, Z1, Z2, Vy1, v)
        it += k
    if not (np.all(np.isfinite(Z1)) and np.all(np.isfinite(Z2))
            and Z1[0] > 0.0):
        raise RuntimeError("stationary Newton solve did not converge")
    return StationaryProfile(float(mu), float(vy), z, Z1, Z2, Vy1,
                             -(Lz @ Z2), it)


def regrid(prof: StationaryProfile, nz: int):
    """Profiles on ``nz`` points by not-a-knot cubic spline
    (``interp1(Z,.,zz0,'spline')``, ``tevol_driven_cluster.m:84``)."""
    from scipy.interpolate import CubicSpline
    znew, _ = radial_grid(nz)
    order = np.argsort(prof.z)
    out = []
    for v in (prof.Z1, prof.Z2, prof.Vy1, prof.rhoi):
        cs = CubicSpline(prof.z[order], v[order], bc_type="not-a-knot")
        out.append(cs(znew))
    return znew, out


def _theta_profile(z: np.ndarray, Z2: np.ndarray) -> np.ndarray:
    """``theta = -Lzr(Z2_f)`` with ``Z2_f = Z2/f`` and its horizon limit
    ``-dZ2/3`` (``tevol_driven_cluster.m:90-93``)."""
    nz = z.size
    _, Lz = radial_grid(nz)
    Z2f = np.zeros(nz)
    Z2f[1:] = Z2[1:] / (1.0 - z[1:] ** 3)
    Z2f[0] = -(Lz @ Z2)[0] / 3.0
    Lz1 = np.linalg.solve(Lz[:nz - 1, :nz - 1], np.eye(nz - 1))
    theta = np.zeros(nz)
    theta[:nz - 1] = -(Lz1 @ Z2f[:nz - 1])
    return theta


def init_driven(nx: int, ny: int, nz: int, prof: StationaryProfile,
                noise: str = "complex", amplitude: float = 1e-3,
                seed: int = 0, zero_flow_profile: bool = False):
    """Initial fields ``(Z1, Z2, Z3, Z4, rhoi)`` as ``(nx, ny, nz)`` arrays.

    Restates ``tevol_driven_cluster.m:85-102``: the regridded profile is
    repeated over the plane, ``Psi = Z1*exp(i*theta)``, ``A_x = Lx*theta``
    (zero, since ``theta`` is uniform in x), ``A_y = -Vy1`` and ``rhoi`` is the
    boundary value of the charge profile repeated along z.

    ``noise`` selects the perturbation.  ``"reference"`` is the reference's
    ``Z1.*(1+a*randn(nx,ny))`` (real, repeated along z, default a=1e-2 there);
    ``"complex"`` multiplies by ``1+a*(xi_r+i*xi_i)`` with complex Gaussian
    ``xi`` per (x, y) point; ``"none"`` leaves the profile unperturbed.  The
    draw comes from ``numpy.random.default_rng(seed)``.
    """
    z, (Z1p, Z2p, Vy1p, rhop) = regrid(prof, nz)
    if zero_flow_profile:
        Vy1p = np.zeros_like(Vy1p)
    theta = _theta_profile(z, Z2p)
    psi = Z1p * np.exp(1j * theta)
    rng = np.random.default_rng(seed)
    if noise == "reference":
        pert = 1.0 + amplitude * rng.standard_normal((nx, ny))
    elif noise == "complex":
        pert = 1.0 + amplitude * (rng.standard_normal((nx, ny))
                                  + 1j * rng.standard_normal((nx, ny)))
    elif noise == "none":
        pert = np.ones((nx, ny))
    else:
        raise ValueError(f"unknown noise mode {noise!r}")
    Z1 = pert[:, :, None] * psi[None, None, :]
    Z2 = np.broadcast_to(Z2p[None, None, :], (nx, ny, nz)).copy()
    Z3 = np.zeros((nx, ny, nz))
    Z4 = np.broadcast_to(-Vy1p[None, None, :], (nx, ny, nz)).copy()
    rhoi = np.full((nx, ny, nz), float(rhop[-1]))
    return Z1.astype(np.complex128), Z2, Z3, Z4, rhoi


def random_vortices(count: int, Lx: float, Ly: float, seed: int):
    """``count`` positions uniform on the torus and charges, half +1 and
    half -1 (odd counts get the extra +1), shuffled by ``default_rng(seed)``.
    """
    rng = np.random.default_rng(seed)
    xs = rng.uniform(0.0, Lx, count)
    ys = rng.uniform(0.0, Ly, count)
    q = np.where(np.arange(count) < (count + 1) // 2, 1, -1)
    rng.shuffle(q)
    return xs, ys, q


def init_lattice(nx: int, ny: int, nz: int, prof: StationaryProfile,
                 Lx: float, Ly: float, xs, ys, charges, sigma: float = 3.0,
                 periodic_images: int = 4):
    """Vortex imprint of ``tevol_lattice.m:101-135``.

    ``Psi = z1 * (1 - sum_v exp(-|r-r_v|^2/sigma^2)) * prod_v e^{i q_v phi_v}``.
    The reference uses the bare ``atan2`` angle for ``phi_v``, which is not
    periodic on the torus.  Here ``phi_v`` is the angle of
    ``prod_m sin(pi*((x-x_v) + i*(y-y_v-m*Ly))/Lx)`` over ``|m| <= periodic_images``
    image rows: exactly periodic in x for an even number of unit charges, and
    periodic in y up to a uniform phase and exponentially small terms for a
    charge-neutral set.  ``periodic_images=0`` with a huge
    ``Lx`` recovers the bare ``atan2`` imprint.  Distances in the Gaussian dips
    use the minimum image.
    """
    z, (Z1p, Z2p, Vy1p, rhop) = regrid(prof, nz)
    theta = _theta_profile(z, Z2p)
    x = np.arange(nx) * Lx / nx
    y = np.arange(ny) * Ly / ny
    X, Y = np.meshgrid(x, y, indexing="ij")
    dip = np.zeros((nx, ny))
    plane = np.ones((nx, ny), dtype=np.complex128)
    for xv, yv, q in zip(xs, ys, charges):
        dx = (X - xv + Lx / 2) % Lx - Lx / 2
        dy = (Y - yv + Ly / 2) % Ly - Ly / 2
        dip += np.exp(-(dx ** 2 + dy ** 2) / sigma ** 2)
        ux, uy = X - xv, Y - yv
        for m in range(-periodic_images, periodic_images + 1):
            s = np.sin(np.pi * (ux + 1j * (uy - m * Ly)) / Lx)
            u = s / np.maximum(np.abs(s), 1e-300)
            plane *= u if q > 0 else np.conj(u)
            if abs(q) > 1:
                plane *= (u if q > 0 else np.conj(u)) ** (abs(q) - 1)
    plane *= (1.0 - dip)
    psi = Z1p * np.exp(1j * theta)
    Z1 = plane[:, :, None] * psi[None, None, :]
    Z2 = np.broadcast_to(Z2p[None, None, :], (nx, ny, nz)).copy()
    Z3 = np.zeros((nx, ny, nz))
    Z4 = np.broadcast_to(-Vy1p[None, None, :], (nx, ny, nz)).copy()
    rhoi = np.full((nx, ny, nz), float(rhop[-1]))
    return Z1.astype(np.complex128), Z2, Z3, Z4, rhoi
