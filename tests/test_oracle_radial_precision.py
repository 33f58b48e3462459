"""Why the mixed-precision step keeps its radial (Chebyshev) contractions FP64.

Measured on the oracle, not on the GPU: the oracle step is re-run with the
arithmetic of two mixed-precision designs and compared with the FP64 oracle
after 100 steps of a driven 32x32x21 run (L = 25, mu = 6, dt = 0.02, drive
2 pi 7/20, winding removal and filter on; the spacing of the benchmark grid).

* ``lines32``: the built mixed step.  Every x/y derivative is taken in FP32
  from the slice-mean-removed field (operands rounded to FP32, FP32 sums),
  the radial contractions, pointwise terms and state in FP64.
* ``radial32``: the same, and every D_z / Lzr contraction inside the
  right-hand side (``tevol_driven_cluster.m:62-65,72-75``) in FP32 as well
  (operands and matrices rounded to FP32, FP32 accumulation): the FP32
  D_z of the "split-BF16 or 3xTF32 accumulated in FP32" design at best.
  The boundary row F2 (:76) stays FP64 in both.

FP32 line derivatives cost ~5e-11 after 100 steps; FP32 radial contractions
cost ~1e-6, the whole 1e-6 error budget of 100 steps (D_z enters twice in
d_z^2 Psi and there is no radial filter to remove the rounding noise).
"""
import numpy as np
import pytest

F32 = np.float32
VY7 = 2 * np.pi * 7 / 20


def _along32(M, x, axis):
    if np.iscomplexobj(x):
        return _along32(M, x.real, axis) + 1j * _along32(M, x.imag, axis)
    y = np.tensordot(M.astype(F32), x.astype(F32), axes=([1], [axis]))
    return np.moveaxis(y.astype(np.float64), 0, axis)


def _line32(M, x, axis):
    # a derivative annihilates the slice mean, so it is removed before rounding
    if np.iscomplexobj(x):
        return _line32(M, x.real, axis) + 1j * _line32(M, x.imag, axis)
    return _along32(M, x - x.mean(axis=(0, 1), keepdims=True), axis)


def _funcs(oracle, op, radial32):
    class Funcs(oracle._Funcs):
        def Lx(self, x):
            return _line32(self.op.Lx, x, 0)

        def Ly(self, x):
            return _line32(self.op.Ly, x, 1)

        def Lz(self, x):
            return _along32(self.op.Lz, x, 2) if radial32 else super().Lz(x)

        def Lzr(self, x):
            if not radial32:
                return super().Lzr(x)
            nz = self.op.nz
            y = np.zeros_like(x)
            y[:, :, :nz - 1] = _along32(self.op.Lz1, x[:, :, :nz - 1], 2)
            return y
    return Funcs(op)


def _rhs(oracle, radial32):
    """``oracle.rhs`` (``tevol_driven_cluster.m:70-76``) with the emulated
    arithmetic; F2 keeps the FP64 radial row."""
    def rhs(op, y1, y2, y3, y4):
        fn = _funcs(oracle, op, radial32)
        zz = op.zz[None, None, :]
        fac = 1.0 - zz ** 3
        Lzy1 = fn.Lz(y1)
        F1 = fn.Lzr(1j * y2 * Lzy1 + 0.5j * y1 * fn.Lz(y2) + 0.5 * fac * fn.Lz(Lzy1)
                    - 1.5 * zz ** 2 * Lzy1 - 0.5 * zz * y1 - 0.5 * y3 * y3 * y1
                    - 0.5 * y4 * y4 * y1 + 0.5 * fn.Lx(fn.Lx(y1)) + 0.5 * fn.Ly(fn.Ly(y1))
                    - 0.5j * y1 * (fn.Lx(y3) + fn.Ly(y4))
                    - 1j * (y3 * fn.Lx(y1) + y4 * fn.Ly(y1)))
        cy1 = np.conj(y1)
        F3 = np.real(fn.Lzr(0.5 * fn.Lz(fn.Lx(y2) + fac * fn.Lz(y3))
                            + 0.5 * fn.Ly(fn.Ly(y3) - fn.Lx(y4))
                            - 0.5j * (cy1 * fn.Lx(y1) - y1 * fn.Lx(cy1)) - y3 * y1 * cy1))
        F4 = np.real(fn.Lzr(0.5 * fn.Lz(fn.Ly(y2) + fac * fn.Lz(y4))
                            + 0.5 * fn.Lx(-fn.Ly(y3) + fn.Lx(y4))
                            - 0.5j * (cy1 * fn.Ly(y1) - y1 * fn.Ly(cy1)) - y4 * y1 * cy1))
        F2 = (1.0 - zz ** 3) * oracle._Funcs(op).Lz(fn.Lx(y3) + fn.Ly(y4))
        return F1, F2, F3, F4
    return rhs


def _rel(a, b, scale=None):
    return float(np.linalg.norm(a - b) / (np.linalg.norm(b) if scale is None else scale))


def test_fp32_radial_contractions_use_the_error_budget(hqt, oracle, monkeypatch):
    nx, nz, L, mu, nsteps = 32, 21, 25.0, 6.0, 100
    prof = hqt.seed.stationary_profile(mu, VY7)
    st = hqt.seed.init_driven(nx, nx, nz, prof, noise="complex", amplitude=1e-3, seed=0)
    op = oracle.build_operators(nx, nx, nz, L, L)
    s0 = oracle.OracleState(np.asarray(st[0], complex), *[np.asarray(a, float) for a in st[1:]])

    def run(rhs):
        if rhs is not None:
            monkeypatch.setattr(oracle, "rhs", rhs)
        s = s0.copy()
        for _ in range(nsteps):
            s, _ = oracle.rk4_step(op, s, 0.02, mu, VY7, True)
        monkeypatch.undo()
        return s

    ref = run(None)
    errs = {}
    for name, radial32 in (("lines32", False), ("radial32", True)):
        s = run(_rhs(oracle, radial32))
        assert np.isfinite(s.Z1).all()
        errs[name] = {"Psi": _rel(s.Z1, ref.Z1), "A_t": _rel(s.Z2, ref.Z2),
                      "A_x": _rel(s.Z3, ref.Z3, np.linalg.norm(ref.Z2)),
                      "A_y": _rel(s.Z4, ref.Z4), "rho": _rel(s.rhoi, ref.rhoi)}
    print("relative L2 after 100 steps:", errs)
    lines, radial = max(errs["lines32"].values()), max(errs["radial32"].values())
    assert lines < 1e-9
    assert radial > 3e-7          # a third or more of the 1e-6 budget
    assert radial > 1e4 * lines
