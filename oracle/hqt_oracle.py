"""CPU oracle for the AdS4 holographic-superfluid RK4 step (TEST INFRASTRUCTURE).

This module is the parity checker, not the product.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may
import it.  The product path (the CUDA library behind ``include/hqt.h``)
never calls into this file.

It is a plain FP64 NumPy restatement of the reference's MATLAB time step,
kept deliberately close to the reference's operator nesting: dense
``fourdif`` / ``chebdif`` spectral matrices, ``Lz1 = inv(Lz(1:nz-1,1:nz-1))``,
the ``func_Lzr`` radial integration, the real/imaginary split Fourier filter
``ff`` and the literal ``countN`` plaquette winding.  Every function cites the
reference file and lines it restates (paths relative to the reference
project root).

Parity status
-------------
* Pinned by the reference's own known-answer tests
  (``tests/hqt_smoke_test.m``): ``fourdif`` (:129-130), ``chebdif`` (:131-133),
  ``ff`` with an empty mask (:141), ``countN`` n/np/nm = 4/2/2 (:148-151), and
  Newton convergence from the shipped seed (:180-183, checked against the
  product's host-side seed solver in the tests).
* The RK4 step, constraint, winding removal and filter are **parity
  unpinned**: the reference's evolution test only asserts finiteness
  (``tests/hqt_smoke_test.m:189-198,305-307``), ships no golden checkpoints,
  and its runtime (MATLAB R2025a + Parallel Computing Toolbox) is not present
  here.  The step below is a line-by-line restatement of
  ``scripts/simulation/tevol_driven_cluster.m:11-142``.

Array convention: NumPy arrays of shape ``(nx, ny, nz)`` indexed like the
MATLAB arrays ``[nx, ny, nz]`` (x first, z index ``nz-1`` = AdS boundary).
``np.asfortranarray`` of such an array has the reference's column-major
memory layout.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
from scipy.linalg import toeplitz

__all__ = [
    "fourdif", "chebdif", "matlab_round", "filter_mask", "ff", "countN",
    "Operators", "build_operators", "OracleState", "rhs", "rk4_step",
    "boundary_order_parameter", "winding_number",
]


# ---------------------------------------------------------------------------
# dmsuite operators
# ---------------------------------------------------------------------------
def fourdif(N: int, m: int):
    """Fourier spectral differentiation matrix on ``x_j = 2*pi*j/N``.

    Restates ``third_party/dmsuite/fourdif.m:30-71`` for ``m`` in {0, 1, 2}
    (the only orders the time-evolution scripts use): the first column is
    built with the cot/csc "flipping trick" formulas and the matrix is the
    Toeplitz matrix of (first column, first row).
    """
    x = 2.0 * np.pi * np.arange(N) / N                       # fourdif.m:30
    h = 2.0 * np.pi / N                                      # :31
    kk = np.arange(1, N)                                     # :33
    n1 = (N - 1) // 2                                        # :34
    n2 = int(math.ceil((N - 1) / 2))
    sgn = (-1.0) ** kk
    if m == 0:                                               # :35-37
        col1 = np.zeros(N)
        col1[0] = 1.0
        row1 = col1
    elif m == 1:                                             # :39-47
        if N % 2 == 0:
            topc = 1.0 / np.tan(np.arange(1, n2 + 1) * h / 2)
            col1 = np.r_[0.0, 0.5 * sgn * np.r_[topc, -topc[:n1][::-1]]]
        else:
            topc = 1.0 / np.sin(np.arange(1, n2 + 1) * h / 2)
            col1 = np.r_[0.0, 0.5 * sgn * np.r_[topc, topc[:n1][::-1]]]
        row1 = -col1
    elif m == 2:                                             # :49-57
        if N % 2 == 0:
            topc = 1.0 / np.sin(np.arange(1, n2 + 1) * h / 2) ** 2
            col1 = np.r_[-np.pi ** 2 / 3 / h ** 2 - 1.0 / 6,
                         -0.5 * sgn * np.r_[topc, topc[:n1][::-1]]]
        else:
            t = np.arange(1, n2 + 1) * h / 2
            topc = (1.0 / np.sin(t)) * (1.0 / np.tan(t))
            col1 = np.r_[-np.pi ** 2 / 3 / h ** 2 + 1.0 / 12,
                         -0.5 * sgn * np.r_[topc, -topc[:n1][::-1]]]
        row1 = col1
    else:
        raise ValueError("fourdif: only m in {0,1,2} is restated")
    return x, toeplitz(col1, row1)                           # :71


def chebdif(N: int, M: int):
    """Chebyshev differentiation matrices ``D1..DM`` on ``N`` points.

    Restates ``third_party/dmsuite/chebdif.m:25-53``: points
    ``x_k = sin(pi*(N-1-2k)/(2(N-1)))`` (so ``x[0] = +1`` and ``x[-1] = -1``),
    trigonometric differences with the flipping trick, and the negative-sum
    diagonal.  Returns ``x`` and an array ``DM`` of shape ``(M, N, N)``.
    """
    I = np.eye(N)                                            # chebdif.m:25
    n1 = N // 2                                              # :28
    n2 = int(math.ceil(N / 2))
    k = np.arange(N)                                         # :30
    th = k * np.pi / (N - 1)                                 # :31
    x = np.sin(np.pi * np.arange(N - 1, -N, -2) / (2.0 * (N - 1)))  # :33
    T = np.tile((th / 2)[:, None], (1, N))                   # :35
    DX = 2.0 * np.sin(T.T + T) * np.sin(T.T - T)             # :36
    DX = np.r_[DX[:n1, :], -np.flipud(np.fliplr(DX[:n2, :]))]  # :37
    DX[I.astype(bool)] = 1.0                                 # :38
    C = toeplitz((-1.0) ** k)                                # :40
    C[0, :] *= 2.0
    C[N - 1, :] *= 2.0                                       # :41
    C[:, 0] /= 2.0
    C[:, N - 1] /= 2.0                                       # :42
    Z = 1.0 / DX                                             # :44
    Z[I.astype(bool)] = 0.0                                  # :45
    D = np.eye(N)                                            # :47
    DM = np.zeros((M, N, N))
    for ell in range(1, M + 1):                              # :49-53
        D = ell * Z * (C * np.tile(np.diag(D)[:, None], (1, N)) - D)
        D[I.astype(bool)] = -np.sum(D, axis=1)
        DM[ell - 1] = D
    return x, DM


def matlab_round(v):
    """MATLAB ``round``: halves away from zero (NumPy rounds halves to even)."""
    v = np.asarray(v, dtype=np.float64)
    return np.sign(v) * np.floor(np.abs(v) + 0.5)


# ---------------------------------------------------------------------------
# Fourier filter
# ---------------------------------------------------------------------------
def filter_mask(nx: int, ny: int) -> np.ndarray:
    """Logical mask of zeroed Fourier modes, ``fx | fy`` (shape ``(nx, ny)``).

    Restates ``scripts/simulation/tevol_driven_cluster.m:27-31``:
    ``fx(round(round(nx/3)):round(nx/3*2)) = 1`` with 1-based MATLAB indices.
    """
    return filter_band(nx)[:, None] | filter_band(ny)[None, :]


def filter_band(n: int) -> np.ndarray:
    """``fx(round(round(n/3)):round(n/3*2)) = 1`` (1-based) of
    ``tevol_driven_cluster.m:27-29`` along one axis of ``n >= 2`` points."""
    f = np.zeros(n, dtype=bool)
    lo = int(matlab_round(matlab_round(n / 3)))
    hi = int(matlab_round(n / 3 * 2))
    f[lo - 1:hi] = True
    return f


def ff(x: np.ndarray, mask: np.ndarray) -> np.ndarray:
    """``real(ifft2(b))`` with ``b = fft2(x)`` and masked modes zeroed.

    Restates ``src/numerics/ff.m:7-11``; the 2-D transform acts on the first
    two axes of each z-slice.  ``mask`` has shape ``(nx, ny)`` (broadcast along
    z, as ``repmat(fx|fy,[1,1,nz])`` does at
    ``tevol_driven_cluster.m:31``).
    """
    b = np.fft.fft2(x, axes=(0, 1))
    if x.ndim == 3:
        b[mask, :] = 0
    else:
        b[mask] = 0
    return np.real(np.fft.ifft2(b, axes=(0, 1)))


# ---------------------------------------------------------------------------
# Vortex count
# ---------------------------------------------------------------------------
def countN(x1: np.ndarray):
    """Plaquette winding count on a periodic complex 2-D field.

    Restates ``src/diagnostics/countN.m:7-21`` literally: neighbours by
    ``circshift`` (x2=(i+1,j), x3=(i+1,j+1), x4=(i,j+1)), the winding
    ``w = (angle(x1/x2)+angle(x2/x3)+angle(x3/x4)+angle(x4/x1))/(2*pi)`` and
    the +-1 tolerance window of 1e-4.  Returns ``(n, np, nm)``.
    """
    x1 = np.asarray(x1, dtype=np.complex128)
    x2 = np.roll(x1, -1, axis=0)                      # circshift(x1,[-1,0])
    x3 = np.roll(np.roll(x1, -1, axis=0), -1, axis=1)  # circshift(x1,[-1,-1])
    x4 = np.roll(x1, -1, axis=1)                      # circshift(x1,[0,-1])
    w = 1.0 / (2.0 * np.pi) * (np.angle(x1 / x2) + np.angle(x2 / x3)
                               + np.angle(x3 / x4) + np.angle(x4 / x1))
    Lp = (w >= 1 - 1e-4) & (w <= 1 + 1e-4)
    Lm = (w <= -1 + 1e-4) & (w >= -1 - 1e-4)
    Lall = Lp.astype(np.int64) + Lm.astype(np.int64)
    return int(np.count_nonzero(Lall == 1)), int(np.count_nonzero(Lp)), \
        int(np.count_nonzero(Lm))


# ---------------------------------------------------------------------------
# Operators and the right-hand side
# ---------------------------------------------------------------------------
@dataclass
class Operators:
    nx: int
    ny: int
    nz: int
    Lx: np.ndarray      # (2*pi/Lx_len) * fourdif(nx,1)
    Ly: np.ndarray
    Lz: np.ndarray      # 2 * chebdif(nz,1)
    Lz1: np.ndarray     # inv(Lz(1:nz-1,1:nz-1))
    zz: np.ndarray      # radial coordinate, z[0]=1 (horizon) .. z[-1]=0
    mask: np.ndarray    # zeroed Fourier modes (nx, ny)
    Lx_len: float
    Ly_len: float


def build_operators(nx: int, ny: int, nz: int, Lx_len: float,
                    Ly_len: float | None = None) -> Operators:
    """Operators of ``scripts/simulation/tevol_driven_cluster.m:13-54``.

    ``Lx=px*Dx`` with ``px=2*pi/L0`` (:38,47), ``Lz=pz*Dz`` with ``pz=2``
    (``dlz=1``, :36-40,49), ``zz=(zcheb-1)*dlz/2+zf`` (:44) and
    ``Lz1=Lz(1:nz-1,1:nz-1)\\eye(nz-1)`` (:52).  ``nz`` is the number of
    Chebyshev points (``chebdif(nz,1)`` returns ``nz`` points).
    """
    if Ly_len is None:
        Ly_len = Lx_len
    _, Dx = fourdif(nx, 1)
    _, Dy = fourdif(ny, 1)
    z, DM = chebdif(nz, 1)
    Dz = DM[0]
    small, D = 0.0, 0.0
    zi, zf = D, 1.0 - small
    dlz = zf - zi
    px = 2.0 * np.pi / Lx_len
    py = 2.0 * np.pi / Ly_len
    pz = 2.0 / dlz
    zz = (z - 1.0) * dlz / 2.0 + zf
    Lz = pz * Dz
    Lz1 = np.linalg.solve(Lz[:nz - 1, :nz - 1], np.eye(nz - 1))
    return Operators(nx, ny, nz, px * Dx, py * Dy, Lz, Lz1, zz,
                     filter_mask(nx, ny), float(Lx_len), float(Ly_len))


def _along(M: np.ndarray, x: np.ndarray, axis: int) -> np.ndarray:
    """Apply the real matrix ``M`` along ``axis`` (real and imaginary parts
    separately, as a real matrix times a complex array does)."""
    if np.iscomplexobj(x):
        return _along(M, x.real, axis) + 1j * _along(M, x.imag, axis)
    y = np.tensordot(M, x, axes=([1], [axis]))
    return np.moveaxis(y, 0, axis)


class _Funcs:
    """The anonymous operators of ``tevol_driven_cluster.m:60-65``."""

    def __init__(self, op: Operators):
        self.op = op

    def Lx(self, x):            # func_Lx, :60
        return _along(self.op.Lx, x, 0)

    def Ly(self, x):            # func_Ly, :61
        return _along(self.op.Ly, x, 1)

    def Lz(self, x):            # func_Lz, :62
        return _along(self.op.Lz, x, 2)

    def Lzr(self, x):           # func_Lzr, :63-65: [[Lz1,0]*x; 0]
        nz = self.op.nz
        y = np.zeros_like(x)
        y[:, :, :nz - 1] = _along(self.op.Lz1, x[:, :, :nz - 1], 2)
        return y


def rhs(op: Operators, y1, y2, y3, y4):
    """``F1, F3, F4`` (full 3-D) and ``F2`` of ``tevol_driven_cluster.m:70-76``.

    ``y1`` is the complex scalar Psi, ``y2=A_t``, ``y3=A_x``, ``y4=A_y``.
    """
    fn = _Funcs(op)
    zz = op.zz[None, None, :]
    zh = 1.0
    fac = 1.0 - (zz / zh) ** 3
    Lzy1 = fn.Lz(y1)
    F1 = fn.Lzr(1j * y2 * Lzy1 + 0.5j * y1 * fn.Lz(y2)
                + 0.5 * fac * fn.Lz(Lzy1)
                - 0.5 * 3 * zz ** 2 / zh ** 3 * Lzy1
                - 0.5 * zz * y1 - 0.5 * y3 * y3 * y1 - 0.5 * y4 * y4 * y1
                + 1.0 * 0.5 * fn.Lx(fn.Lx(y1))
                + 1.0 * 0.5 * fn.Ly(fn.Ly(y1))
                - 1.0 * 0.5j * y1 * (fn.Lx(y3) + fn.Ly(y4))
                - 1j * (y3 * fn.Lx(y1) + y4 * fn.Ly(y1)))       # :72-73
    Lxy1 = fn.Lx(y1)
    Lyy1 = fn.Ly(y1)
    cy1 = np.conj(y1)
    F3 = np.real(fn.Lzr(0.5 * fn.Lz(fn.Lx(y2) + fac * fn.Lz(y3))
                        + 0.5 * fn.Ly(fn.Ly(y3) - fn.Lx(y4))
                        - 0.5j * (cy1 * Lxy1 - y1 * fn.Lx(cy1))
                        - y3 * y1 * cy1))                       # :74
    F4 = np.real(fn.Lzr(0.5 * fn.Lz(fn.Ly(y2) + fac * fn.Lz(y4))
                        + 0.5 * fn.Lx(-fn.Ly(y3) + fn.Lx(y4))
                        - 0.5j * (cy1 * Lyy1 - y1 * fn.Ly(cy1))
                        - y4 * y1 * cy1))                       # :75
    F2 = (1.0 - zz ** 3) * fn.Lz(fn.Lx(y3) + fn.Ly(y4))        # :76
    return F1, F2, F3, F4


def boundary_order_parameter(op: Operators, Z1) -> np.ndarray:
    """``O = func_Lz(Z1)(:,:,end)`` (``tevol_driven_cluster.m:136``)."""
    return _Funcs(op).Lz(Z1)[:, :, -1]


def winding_number(O: np.ndarray) -> int:
    """``round(mean(sum(angle(circshift(O,-1,2)./O),1))/(2*pi))``
    (``tevol_driven_cluster.m:137``)."""
    inc = np.angle(np.roll(O, -1, axis=1) / O)
    return int(matlab_round(np.mean(np.sum(inc, axis=0)) / (2.0 * np.pi)))


@dataclass
class OracleState:
    Z1: np.ndarray      # complex (nx, ny, nz)
    Z2: np.ndarray      # A_t
    Z3: np.ndarray      # A_x
    Z4: np.ndarray      # A_y
    rhoi: np.ndarray    # (nx, ny, nz), replicated along z

    def copy(self) -> "OracleState":
        return OracleState(self.Z1.copy(), self.Z2.copy(), self.Z3.copy(),
                           self.Z4.copy(), self.rhoi.copy())


def rk4_step(op: Operators, s: OracleState, h: float, mu: float, vy: float,
             remove_winding: bool = True, apply_filter: bool = True):
    """One pass of the loop body ``tevol_driven_cluster.m:120-142``.

    Four RK stages with ``A_t`` frozen (:120-123), the combine (:124,128),
    the constraint rebuild of ``A_t`` (:129-131), the AdS-boundary rows
    (:133), the global winding removal (:136-139; off for the lattice
    script, ``tevol_lattice.m:168-170``) and the real/imaginary split
    Fourier filter (:142).  Returns ``(new_state, winding)``.
    """
    nz = op.nz
    fn = _Funcs(op)
    Z1, Z2, Z3, Z4, rhoi = s.Z1, s.Z2, s.Z3, s.Z4, s.rhoi

    def stage(y1, y3, y4):
        F1, F2, F3, F4 = rhs(op, y1, Z2, y3, y4)
        k1, k3, k4 = h * F1, h * F3, h * F4
        k1[:, :, nz - 1] = 0
        k3[:, :, nz - 1] = 0
        k4[:, :, nz - 1] = 0
        return k1, h * F2, k3, k4

    k11, k21, k31, k41 = stage(Z1, Z3, Z4)                               # :120
    k12, k22, k32, k42 = stage(Z1 + k11 / 2, Z3 + k31 / 2, Z4 + k41 / 2)  # :121
    k13, k23, k33, k43 = stage(Z1 + k12 / 2, Z3 + k32 / 2, Z4 + k42 / 2)  # :122
    k14, k24, k34, k44 = stage(Z1 + k13, Z3 + k33, Z4 + k43)             # :123
    k1 = (1 / 6) * (k11 + 2 * k12 + 2 * k13 + k14)                       # :124
    k3 = (1 / 6) * (k31 + 2 * k32 + 2 * k33 + k34)
    k4 = (1 / 6) * (k41 + 2 * k42 + 2 * k43 + k44)
    k2 = (1 / 6) * (k21 + 2 * k22 + 2 * k23 + k24)
    Z1, Z3, Z4 = Z1 + k1, Z3 + k3, Z4 + k4                                # :128
    rhoi = rhoi - np.repeat(k2[:, :, nz - 1:nz], nz, axis=2)
    cons = np.real(fn.Lz(fn.Lx(Z3) + fn.Ly(Z4))
                   + 1j * (np.conj(Z1) * fn.Lz(Z1)
                           - Z1 * fn.Lz(np.conj(Z1))))                  # :129
    Z2 = fn.Lzr(fn.Lzr(cons) - rhoi) + mu                                # :131
    Z1 = Z1.copy()
    Z1[:, :, nz - 1] = 0                                                 # :133
    Z3[:, :, nz - 1] = 0
    Z2[:, :, nz - 1] = mu
    Z4[:, :, nz - 1] = -vy
    winding = 0
    if remove_winding:                                                   # :136-139
        O = boundary_order_parameter(op, Z1)
        winding = winding_number(O)
        yy = (2.0 * np.pi * np.arange(op.ny) / op.ny) * op.Ly_len / 2 / np.pi
        Z1 = Z1 * np.exp(-1j * 2 * np.pi * yy[None, :, None] / op.Ly_len
                         * (winding + 0))
    if apply_filter:                                                     # :142
        Z1 = ff(np.real(Z1), op.mask) + 1j * ff(np.imag(Z1), op.mask)
        Z2 = ff(Z2, op.mask)
        Z3 = ff(Z3, op.mask)
        Z4 = ff(Z4, op.mask)
    return OracleState(Z1, Z2, Z3, Z4, rhoi), winding


def run(op: Operators, s: OracleState, nsteps: int, h: float, mu: float,
        vy: float, remove_winding: bool = True):
    """Advance ``nsteps`` steps; stops at the first NaN like the guard at
    ``tevol_driven_cluster.m:182-185``.  Returns ``(state, windings)``."""
    windings = []
    for _ in range(nsteps):
        s, w = rk4_step(op, s, h, mu, vy, remove_winding)
        windings.append(w)
        if (np.isnan(s.Z1).any() or np.isnan(s.Z2).any()
                or np.isnan(s.Z3).any() or np.isnan(s.Z4).any()):
            break
    return s, windings


# ---------------------------------------------------------------------------
# Energy spectrum of the boundary superflow
# ---------------------------------------------------------------------------
def signed_wavenumbers(n: int) -> np.ndarray:
    """Integer wavenumbers of an n-point FFT: ``[0:n/2-1, -n/2:-1]`` for even
    n (as ``scripts/analysis/movie_show.m:148-149`` builds them) and
    ``[0:(n-1)/2, -(n-1)/2:-1]`` for odd n.  The reference's expression yields
    n-1 entries for odd n (300 for n=301) and mis-shapes its shell mask; this
    restatement uses the n-point grid for both parities."""
    if n % 2 == 0:
        return np.r_[np.arange(0, n // 2), np.arange(-n // 2, 0)].astype(np.float64)
    h = (n - 1) // 2
    return np.r_[np.arange(0, h + 1), np.arange(-h, 0)].astype(np.float64)


def boundary_velocity(O: np.ndarray, Lx: float, Ly: float):
    """``(vx, vy)``: ``VX_temp``, ``VY_temp`` of
    ``scripts/analysis/plots_cluster.m:92-93`` (= ``movie_show.m:93-94``),
    ``|O|./max(|O|) .* real(-1i*(func_Lx(O) - func_Lx(|O|).*O./|O|)./O)`` on
    the boundary slice, with spectral derivatives (``fourdif``: ``ik``,
    Nyquist 0).  ``max`` of the nx x ny slice is MATLAB's column max: one
    maximum over x per y index."""
    O = np.asarray(O, dtype=np.complex128)
    nx, ny = O.shape
    ikx = 1j * (2.0 * np.pi / Lx) * signed_wavenumbers(nx)
    iky = 1j * (2.0 * np.pi / Ly) * signed_wavenumbers(ny)
    if nx % 2 == 0:
        ikx[nx // 2] = 0
    if ny % 2 == 0:
        iky[ny // 2] = 0
    Ohat = np.fft.fft2(O)
    dOx = np.fft.ifft2(ikx[:, None] * Ohat)
    dOy = np.fft.ifft2(iky[None, :] * Ohat)
    a = np.abs(O)
    ahat = np.fft.fft2(a)
    dax = np.real(np.fft.ifft2(ikx[:, None] * ahat))
    day = np.real(np.fft.ifft2(iky[None, :] * ahat))
    w = a / np.max(a, axis=0, keepdims=True)
    vx = w * np.real(-1j * (dOx - dax * O / a) / O)
    vy = w * np.real(-1j * (dOy - day * O / a) / O)
    return vx, vy


def boundary_fields(op: Operators, Z1: np.ndarray):
    """One frame of ``scripts/analysis/plots_cluster.m:89-97``:
    ``(O, vx, vy, NofV)`` with ``O = func_Lz(Z1)(:,:,nz)`` and ``NofV`` the
    first output of ``countN``."""
    O = boundary_order_parameter(op, Z1)
    vx, vy = boundary_velocity(O, op.Lx_len, op.Ly_len)
    n, _, _ = countN(O)
    return O, vx, vy, n


def observables(op: Operators, Z1: np.ndarray, rhoi: np.ndarray):
    """Global observables of a state, build-defined (the reference computes no
    global charge or energy in its loop): ``Q = sum rhoi(:,:,nz) dx dy``, the
    boundary charge that the update ``rhoi = rhoi - k2(:,:,nz)``
    (``tevol_driven_cluster.m:128``) conserves in exact arithmetic (``k2`` is
    a spectral divergence, whose plane sum vanishes); ``E_kin = sum |u|^2/2
    dx dy`` of the velocity of :func:`boundary_velocity`; ``N_O = sum |O|^2
    dx dy``.  Sums are exact-rounded (``math.fsum``)."""
    import math
    O = boundary_order_parameter(op, Z1)
    vx, vy = boundary_velocity(O, op.Lx_len, op.Ly_len)
    area = (op.Lx_len / op.nx) * (op.Ly_len / op.ny)
    q = area * math.fsum(np.asarray(rhoi)[:, :, -1].ravel())
    e = area * math.fsum((0.5 * (vx * vx + vy * vy)).ravel())
    n = area * math.fsum((O.real ** 2 + O.imag ** 2).ravel())
    return q, e, n


def energy_spectrum(O: np.ndarray, Lx: float, Ly: float):
    """Incompressible/compressible kinetic-energy spectrum of the boundary flow.

    Restates ``scripts/analysis/movie_show.m``: the density-weighted velocity
    ``u = |O|/max|O| * Re(-i(dO - d|O| O/|O|)/O)`` (:93-94, with spectral
    derivatives; ``max`` of the slice is per y column, MATLAB's column max), the mean removed (:140-141), ``E2d = |u^|^2/2`` (:142-145),
    shell sums ``sum(E2d(K >= kbins(i) & K < kbins(i+1)))`` over
    ``kbins = 0:dk:kmax``, ``dk = 2*pi/L0``, ``kmax = floor(max K)`` (:146-160),
    and the Helmholtz split ``u_c = grad Phi``, ``lap Phi = div u`` (:217-233)
    done in Fourier space as ``u_c^ = k (k.u^)/|k|^2``.  Returns
    ``(kplot, E, E_c, E_i)``.
    """
    O = np.asarray(O, dtype=np.complex128)
    nx, ny = O.shape
    kx = (2.0 * np.pi / Lx) * signed_wavenumbers(nx)
    ky = (2.0 * np.pi / Ly) * signed_wavenumbers(ny)
    ux, uy = boundary_velocity(O, Lx, Ly)
    ux = ux - np.mean(ux)
    uy = uy - np.mean(uy)
    uxh = np.fft.fft2(ux)
    uyh = np.fft.fft2(uy)
    KX, KY = np.meshgrid(kx, ky, indexing="ij")
    K2 = KX * KX + KY * KY
    K = np.sqrt(K2)
    kdotu = KX * uxh + KY * uyh
    with np.errstate(invalid="ignore", divide="ignore"):
        s = np.where(K2 > 0, kdotu / np.where(K2 > 0, K2, 1.0), 0.0)
    ucx, ucy = KX * s, KY * s
    uix, uiy = uxh - ucx, uyh - ucy
    E2d = 0.5 * (np.abs(uxh) ** 2 + np.abs(uyh) ** 2)
    E2c = 0.5 * (np.abs(ucx) ** 2 + np.abs(ucy) ** 2)
    E2i = 0.5 * (np.abs(uix) ** 2 + np.abs(uiy) ** 2)
    dk = 2.0 * np.pi / Lx
    kmax = np.floor(np.max(K))
    nbins = int(np.floor(kmax / dk))       # len(0:dk:kmax) - 1
    idx = np.floor(K / dk).astype(np.int64)
    sel = idx < nbins
    E = np.bincount(idx[sel], weights=E2d[sel], minlength=nbins)[:nbins]
    Ec = np.bincount(idx[sel], weights=E2c[sel], minlength=nbins)[:nbins]
    Ei = np.bincount(idx[sel], weights=E2i[sel], minlength=nbins)[:nbins]
    kplot = (np.arange(nbins) + 0.5) * dk
    return kplot, E, Ec, Ei


# ---------------------------------------------------------------------------
# Vortex positions and structure factors
# ---------------------------------------------------------------------------
def _find_colmajor(mask: np.ndarray):
    """MATLAB ``[r, c] = find(mask)``: 1-based indices in column-major order."""
    r, c = np.nonzero(mask.T)          # rows of mask.T are the columns of mask
    return c + 1, r + 1


def find_vortices_coarse(O: np.ndarray):
    """``find_vortices_old`` (``src/diagnostics/find_vortices.m:80-118``):
    plaquette charges ``round((d1+d2+d3+d4)/(2*pi))`` with
    ``d = angle(p_next .* conj(p))`` around p1=(i,j), p2=(i+1,j),
    p3=(i+1,j+1), p4=(i,j+1) (periodic); returns 1-based ``[row, col]``
    arrays of the +1 and -1 plaquettes in ``find`` order and the charges."""
    O = np.asarray(O, dtype=np.complex128)
    p1 = O
    p2 = np.roll(O, -1, axis=0)
    p3 = np.roll(np.roll(O, -1, axis=0), -1, axis=1)
    p4 = np.roll(O, -1, axis=1)
    W = (np.angle(p2 * np.conj(p1)) + np.angle(p3 * np.conj(p2))
         + np.angle(p4 * np.conj(p3)) + np.angle(p1 * np.conj(p4)))
    charge = matlab_round(W / (2.0 * np.pi))
    vr, vc = _find_colmajor(charge == 1)
    ar, ac = _find_colmajor(charge == -1)
    return (np.stack([vr, vc], axis=1).astype(np.float64),
            np.stack([ar, ac], axis=1).astype(np.float64), charge)


def refine_vortex(pos, density: np.ndarray, threshold: float, radius: int):
    """``refine_positions`` (``find_vortices.m:30-78``): centroid of the
    periodic (2r+1)^2 window cells with density below the threshold, in
    1-based matrix-index units; ``pos + 0.5`` when no cell qualifies."""
    nx, ny = density.shape
    r_c, c_c = int(pos[0]), int(pos[1])
    off = np.arange(-radius, radius + 1)
    rows = np.mod(r_c + off - 1, nx)
    cols = np.mod(c_c + off - 1, ny)
    local = density[np.ix_(rows, cols)]
    mask = local < threshold
    s = int(mask.sum())
    if s == 0:
        return np.array([r_c + 0.5, c_c + 0.5])
    dR, dC = off[:, None] * np.ones((1, off.size)), np.ones((off.size, 1)) * off[None, :]
    orr = float(np.sum(dR * mask)) / s
    occ = float(np.sum(dC * mask)) / s
    return np.array([np.mod(r_c + orr - 1, nx) + 1, np.mod(c_c + occ - 1, ny) + 1])


def find_vortices(O: np.ndarray, threshold: float, radius: int):
    """``find_vortices`` (``src/diagnostics/find_vortices.m:1-28``): coarse
    plaquettes refined on ``density = |O|^2 / max(|O|^2,[],'all')``.  The k-th
    vortex and the k-th antivortex are refined for k = 1..#vortices (the
    routine assumes equal counts: extra antivortices are dropped, fewer
    raise, as MATLAB's indexing would)."""
    v, av, _ = find_vortices_coarse(O)
    if len(v) == 0:
        return np.zeros((0, 2)), np.zeros((0, 2))
    if len(av) < len(v):
        raise IndexError("fewer antivortices than vortices")
    a2 = np.abs(np.asarray(O)) ** 2
    density = a2 / np.max(a2)
    sv = np.array([refine_vortex(p, density, threshold, radius) for p in v])
    sa = np.array([refine_vortex(p, density, threshold, radius) for p in av[:len(v)]])
    return sv, sa


def shell_index(K: np.ndarray, dk: float) -> np.ndarray:
    """Bin b with ``b*dk <= K < (b+1)*dk`` (edges as products, so a value
    on an edge lands in the upper bin whatever the division rounds to)."""
    b = np.floor(K / dk)
    b = np.where(K < b * dk, b - 1, b)
    b = np.where(K >= (b + 1) * dk, b + 1, b)
    return b.astype(np.int64)


def vortex_structure_factor(Phi: np.ndarray, Lx: float, Ly: float):
    """``compute_vortex_structure_factor``
    (``src/diagnostics/compute_vortex_structure_factor.m:1-104``).

    ``Phi`` is ``[Ny, Nx]`` (rows = y).  Charges
    ``round(sum(mod(dtheta + pi, 2 pi) - pi)/(2 pi))`` around theta ->
    theta_x (next column) -> theta_xy -> theta_y (next row); positions
    ``((ix-0.5) dx, (iy-0.5) dy)`` in ``find`` order; spacing from the density
    and the mean minimum-image nearest-neighbour distance;
    ``S = |fft2(W)|^2 / Nv`` for W = charge and |charge|, averaged over shells
    ``k_edges = 0:dk:k_max`` (``dk = min(dkx, dky)``,
    ``k_max = min(max|kx|, max|ky|)``).  Returns
    ``(k_bin, Sc, Sn, vortices, spacing)``; ``spacing`` is a dict with
    rho, d_density, d_nnd, k_density, k_nnd.  No vortices: all empty/None.
    """
    Phi = np.asarray(Phi, dtype=np.complex128)
    Ny, Nx = Phi.shape
    dx, dy = Lx / Nx, Ly / Ny
    th = np.angle(Phi)
    tx = np.roll(th, -1, axis=1)
    ty = np.roll(th, -1, axis=0)
    txy = np.roll(np.roll(th, -1, axis=0), -1, axis=1)
    tp = 2.0 * np.pi
    d1 = np.mod(tx - th + np.pi, tp) - np.pi
    d2 = np.mod(txy - tx + np.pi, tp) - np.pi
    d3 = np.mod(ty - txy + np.pi, tp) - np.pi
    d4 = np.mod(th - ty + np.pi, tp) - np.pi
    charge = matlab_round((d1 + d2 + d3 + d4) / tp)
    iy, ix = _find_colmajor(np.abs(charge) > 0.5)
    q = charge[iy - 1, ix - 1]
    Nv = len(q)
    if Nv == 0:
        return np.zeros(0), np.zeros(0), np.zeros(0), np.zeros((0, 3)), None
    xv, yv = (ix - 0.5) * dx, (iy - 0.5) * dy
    vort = np.stack([xv, yv, q], axis=1)
    rho = Nv / (Lx * Ly)
    d_density = 1.0 / np.sqrt(rho)
    ddx = np.abs(xv[:, None] - xv[None, :])
    ddx = np.minimum(ddx, Lx - ddx)
    ddy = np.abs(yv[:, None] - yv[None, :])
    ddy = np.minimum(ddy, Ly - ddy)
    d2m = ddx ** 2 + ddy ** 2
    np.fill_diagonal(d2m, np.inf)
    nnd = np.sqrt(np.min(d2m, axis=1))
    d_nnd = float(np.mean(nnd))
    spacing = {"rho": rho, "d_density": d_density, "d_nnd": d_nnd,
               "k_density": 2 * np.pi / d_density, "k_nnd": 2 * np.pi / d_nnd}
    Sc2 = np.abs(np.fft.fft2(charge)) ** 2 / Nv
    Sn2 = np.abs(np.fft.fft2(np.abs(charge))) ** 2 / Nv
    dkx, dky = 2 * np.pi / Lx, 2 * np.pi / Ly
    # unshifted FFT index -> signed frequency of (-floor(N/2) : ceil(N/2)-1)
    kx = dkx * signed_wavenumbers(Nx)
    ky = dky * signed_wavenumbers(Ny)
    KX, KY = np.meshgrid(kx, ky)                     # [Ny, Nx], like Phi
    K = np.sqrt(KX * KX + KY * KY)                   # hypot(KX, KY)
    dk = min(dkx, dky)
    kmax = min(np.floor(Nx / 2) * dkx, np.floor(Ny / 2) * dky)
    nb = int(np.floor(kmax / dk + 1e-9))             # len(0:dk:k_max) - 1
    b = shell_index(K, dk)
    sel = (b >= 0) & (b < nb)
    cnt = np.bincount(b[sel], minlength=nb)[:nb]
    sc = np.bincount(b[sel], weights=Sc2[sel], minlength=nb)[:nb]
    sn = np.bincount(b[sel], weights=Sn2[sel], minlength=nb)[:nb]
    with np.errstate(invalid="ignore", divide="ignore"):
        Sc = np.where(cnt > 0, sc / np.maximum(cnt, 1), 0.0)
        Sn = np.where(cnt > 0, sn / np.maximum(cnt, 1), 0.0)
    k_bin = (np.arange(nb) + 0.5) * dk
    return k_bin, Sc, Sn, vort, spacing


# ---------------------------------------------------------------------------
# The same step in C + OpenMP (oracle/hqt_step_omp.c, built by oracle/Makefile)
# ---------------------------------------------------------------------------
_OMP_LIB = None


def omp_library():
    """ctypes handle of ``oracle/libhqt_oracle_omp.so`` (``make -C oracle``)."""
    global _OMP_LIB
    if _OMP_LIB is None:
        import ctypes
        from pathlib import Path
        path = Path(__file__).resolve().parent / "libhqt_oracle_omp.so"
        if not path.exists():
            raise RuntimeError(f"{path} is not built: run `make -C oracle`")
        lib = ctypes.CDLL(str(path))
        dp = ctypes.POINTER(ctypes.c_double)
        lib.hqt_omp_run.restype = ctypes.c_int
        lib.hqt_omp_run.argtypes = ([ctypes.c_int] * 3 + [ctypes.c_double] + [dp] * 9
                                    + [dp] * 5 + [ctypes.c_int, ctypes.c_double,
                                                  ctypes.c_double, ctypes.c_double,
                                                  ctypes.c_int, ctypes.c_int,
                                                  ctypes.POINTER(ctypes.c_int)])
        _OMP_LIB = lib
    return _OMP_LIB


def filter_matrices(n: int):
    """Real and imaginary parts of the circulant ``W = F^-1 diag(m) F`` with
    ``m`` the kept modes of ``tevol_driven_cluster.m:27-31`` along one axis
    (``ff`` keeps mode (kx, ky) iff both indices are outside the band)."""
    m = (~filter_band(n)).astype(np.float64)
    W = np.fft.ifft(m[:, None] * np.fft.fft(np.eye(n), axis=0), axis=0)
    return np.ascontiguousarray(W.real), np.ascontiguousarray(W.imag)


def omp_run(op: Operators, s: OracleState, nsteps: int, h: float, mu: float, vy: float,
            remove_winding: bool = True, apply_filter: bool = True):
    """``nsteps`` steps of :func:`rk4_step` in C + OpenMP on all host cores.

    Returns ``(state, windings, bad_step)``: ``bad_step`` is 0, or the 1-based
    step at which a NaN appeared (the run stops there, like :func:`run`)."""
    import ctypes
    lib = omp_library()
    dp = ctypes.POINTER(ctypes.c_double)
    Rx, Ix = filter_matrices(op.nx)
    Ry, Iy = filter_matrices(op.ny)
    mats = [np.ascontiguousarray(a, dtype=np.float64) for a in
            (op.Lx, op.Ly, op.Lz, op.Lz1, op.zz, Rx, Ix, Ry, Iy)]
    Z1 = np.asfortranarray(s.Z1, dtype=np.complex128).copy(order="F")
    Z2, Z3, Z4, rh = (np.asfortranarray(a, dtype=np.float64).copy(order="F")
                      for a in (s.Z2, s.Z3, s.Z4, s.rhoi))
    w = np.zeros(max(nsteps, 1), dtype=np.int32)
    ptr = lambda a: a.ctypes.data_as(dp)
    bad = lib.hqt_omp_run(op.nx, op.ny, op.nz, op.Ly_len, *[ptr(a) for a in mats],
                          ptr(Z1), ptr(Z2), ptr(Z3), ptr(Z4), ptr(rh), int(nsteps),
                          float(h), float(mu), float(vy), int(bool(remove_winding)),
                          int(bool(apply_filter)), w.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    nrun = bad if bad else nsteps
    return OracleState(Z1, Z2, Z3, Z4, rh), [int(v) for v in w[:nrun]], int(bad)
