"""Host-side interface of the B200 RK4 step, mirroring the reference workflow.

The reference drives its step from MATLAB scripts operating on the workspace
arrays ``Z1`` (complex Psi), ``Z2`` (A_t), ``Z3`` (A_x), ``Z4`` (A_y) and
``rhoi`` (``scripts/simulation/tevol_driven_cluster.m:117-187``).
:class:`Simulation` owns one C-ABI context (``include/hqt.h``) and exposes
the loop body, the right-hand side ``F1..F4``, the filter ``ff``, the
boundary order parameter, the winding and ``countN`` on the same arrays.

Host arrays are NumPy arrays indexed ``[x, y, z]`` like the MATLAB arrays
(any memory order; they are passed in column-major order).  Device arrays
are CUDA tensors in the same column-major layout, i.e. torch tensors of shape
``(nz, ny, nx)`` (``(ny, nx)`` for 2-D fields), contiguous.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import HQT_FP64, HQT_MIXED, HQTError, NonfiniteEvolution, check

__all__ = ["Simulation", "Ensemble", "StepInfo", "HQTError", "NonfiniteEvolution",
           "assign_runs"]


@dataclass
class StepInfo:
    steps_done: int
    nonfinite_step: int
    last_winding: int
    records: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), np.int32))
    # per record: (Q, E_kin, N_O) of hqt_observables_device
    observables: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Simulation:
    """A context for one grid and parameter set on one GPU.

    Parameters follow ``tevol_driven_cluster.m``: ``nx, ny`` periodic grid,
    ``nz`` Chebyshev points, box lengths ``Lx, Ly`` (``L0, L``), chemical
    potential ``mu``, drive ``vy`` (boundary value ``A_y = -vy``), time step
    ``dt`` (``h``), ``remove_winding`` (driven script) and ``apply_filter``.
    ``autotune`` times the line-pass geometries (transform engine per axis,
    lines per block) at creation and keeps the fastest
    (:meth:`config_report` shows the choice).
    """

    def __init__(self, nx: int, ny: int | None = None, nz: int = 21,
                 Lx: float | None = None, Ly: float | None = None,
                 mu: float = 6.0, vy: float = 0.0, dt: float = 0.02,
                 remove_winding: bool = True, precision: str = "fp64",
                 diag_every: int = 0, apply_filter: bool = True,
                 device: int = 0, autotune: bool = False):
        ny = nx if ny is None else ny
        Lx = (nx - 1) / 2 if Lx is None else Lx
        Ly = Lx if Ly is None else Ly
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.device = int(device)
        prec = {"fp64": HQT_FP64, "mixed": HQT_MIXED}[precision]
        self.params = _lib.hqt_params(self.nx, self.ny, self.nz, float(Lx),
                                      float(Ly), float(mu), float(vy),
                                      float(dt), int(bool(remove_winding)),
                                      prec, int(diag_every),
                                      int(bool(apply_filter)), int(bool(autotune)))
        self._lib = _lib.load()
        ctx = ctypes.c_void_p()
        code = self._lib.hqt_create(ctypes.byref(self.params), self.device,
                                    ctypes.byref(ctx))
        check(code, None)
        self._ctx = ctx
        self._stream = None

    # -- lifetime ---------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_ctx", None):
            self._lib.hqt_destroy(self._ctx)
            self._ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz)

    # -- helpers ----------------------------------------------------------
    def _check(self, code: int) -> None:
        check(code, self._ctx)

    def _sync_stream(self) -> None:
        """Order the library after torch's work.  On a torch side stream the
        library launches on that stream; on the legacy default stream (which
        cannot be graph-captured) it keeps its own stream and the device is
        synchronised first."""
        import torch
        s = torch.cuda.current_stream(self.device).cuda_stream
        if s != self._stream:
            self._check(self._lib.hqt_set_stream(self._ctx, ctypes.c_void_p(s or None)))
            self._stream = s
        if not s:
            torch.cuda.synchronize(self.device)

    def _host3(self, a, dtype) -> np.ndarray:
        a = np.asarray(a)
        if a.shape != self.shape:
            raise ValueError(f"expected shape {self.shape}, got {a.shape}")
        return np.asfortranarray(a, dtype=dtype)

    def _dev(self, t, shape, dtype):
        import torch
        if not (isinstance(t, torch.Tensor) and t.is_cuda):
            raise TypeError("expected a CUDA tensor")
        if tuple(t.shape) != shape or t.dtype != dtype or not t.is_contiguous():
            raise ValueError(f"expected contiguous {dtype} of shape {shape}")
        return ctypes.c_void_p(t.data_ptr())

    def _dev3(self, t, complex_=False):
        import torch
        return self._dev(t, (self.nz, self.ny, self.nx),
                         torch.complex128 if complex_ else torch.float64)

    def _dev2(self, t, complex_=False):
        import torch
        return self._dev(t, (self.ny, self.nx),
                         torch.complex128 if complex_ else torch.float64)

    def _diag(self, records: int):
        buf = np.zeros((max(records, 0), 4), dtype=np.int32)
        obs = np.zeros((max(records, 0), 3))
        d = _lib.hqt_diag()
        d.capacity = int(records)
        if records > 0:
            d.records = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
            d.obs = obs.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        return d, (buf, obs)

    @staticmethod
    def _info(d, bufs) -> StepInfo:
        buf, obs = bufs
        return StepInfo(int(d.steps_done), int(d.nonfinite_step),
                        int(d.last_winding), buf[:d.n_records].copy(),
                        obs[:d.n_records].copy())

    # -- the loop body ----------------------------------------------------
    def step(self, Z1, Z2, Z3, Z4, rhoi, nsteps: int = 1, records: int = 0,
             inplace: bool = False):
        """Advance host arrays ``nsteps`` RK4 steps (loop body
        ``tevol_driven_cluster.m:120-142``).  Returns the new
        ``(Z1, Z2, Z3, Z4, rhoi)`` as column-major arrays and a
        :class:`StepInfo`; raises :class:`NonfiniteEvolution` on NaN/Inf.
        With ``inplace=True`` column-major arrays of the right dtype (for
        example pinned buffers) are updated in place instead of copied."""
        z1 = self._host3(Z1, np.complex128)
        z2 = self._host3(Z2, np.float64)
        z3 = self._host3(Z3, np.float64)
        z4 = self._host3(Z4, np.float64)
        rh = self._host3(rhoi, np.float64)
        if not inplace and (z1 is Z1 or z2 is Z2 or z3 is Z3 or z4 is Z4 or rh is rhoi):
            z1, z2, z3, z4, rh = (z1.copy(order="F"), z2.copy(order="F"),
                                  z3.copy(order="F"), z4.copy(order="F"),
                                  rh.copy(order="F"))
        d, buf = self._diag(records)
        code = self._lib.hqt_step(
            self._ctx, z1.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            _dptr(z2), _dptr(z3), _dptr(z4), _dptr(rh), int(nsteps),
            ctypes.byref(d))
        info = self._info(d, buf)
        if code == _lib.HQT_ENONFINITE:
            err = NonfiniteEvolution(code, self._lib.hqt_last_error(self._ctx).decode())
            err.state = (z1, z2, z3, z4, rh)
            err.info = info
            raise err
        self._check(code)
        return (z1, z2, z3, z4, rh), info

    def step_device(self, Z1, Z2, Z3, Z4, rhoi, nsteps: int = 1,
                    records: int = 0) -> StepInfo:
        """Advance CUDA tensors in place (shape ``(nz, ny, nx)``)."""
        ptrs = [self._dev3(Z1, True), self._dev3(Z2), self._dev3(Z3),
                self._dev3(Z4), self._dev3(rhoi)]
        self._sync_stream()
        d, buf = self._diag(records)
        code = self._lib.hqt_step_device(self._ctx, *ptrs, int(nsteps),
                                         ctypes.byref(d))
        info = self._info(d, buf)
        if code == _lib.HQT_ENONFINITE:
            err = NonfiniteEvolution(code, self._lib.hqt_last_error(self._ctx).decode())
            err.info = info
            raise err
        self._check(code)
        return info

    # -- instrumentation --------------------------------------------------
    def profile(self, enable: bool) -> None:
        """Reset the launch counters; with ``enable`` every launch is timed
        with CUDA events (outside the step graph)."""
        self._check(self._lib.hqt_profile(self._ctx, int(bool(enable))))

    def config_report(self) -> dict:
        """The line-pass geometry in use (and the autotuner's timings)."""
        import json
        buf = ctypes.create_string_buffer(1 << 16)
        self._check(self._lib.hqt_config_report(self._ctx, buf, len(buf)))
        return json.loads(buf.value.decode())

    def profile_report(self) -> dict:
        import json
        buf = ctypes.create_string_buffer(1 << 16)
        self._check(self._lib.hqt_profile_report(self._ctx, buf, len(buf)))
        return json.loads(buf.value.decode())

    # -- individual operators ---------------------------------------------
    def rhs_device(self, Z1, Z2, Z3, Z4):
        """``F1, F3, F4`` and ``F2`` at the boundary slice
        (``tevol_driven_cluster.m:72-76``), without the factor ``h``."""
        import torch
        dev = Z1.device
        F1 = torch.empty_like(Z1)
        F3 = torch.empty((self.nz, self.ny, self.nx), dtype=torch.float64, device=dev)
        F4 = torch.empty_like(F3)
        F2b = torch.empty((self.ny, self.nx), dtype=torch.float64, device=dev)
        ptrs = [self._dev3(Z1, True), self._dev3(Z2), self._dev3(Z3),
                self._dev3(Z4), self._dev3(F1, True), self._dev3(F3),
                self._dev3(F4), self._dev2(F2b)]
        self._sync_stream()
        self._check(self._lib.hqt_rhs_device(self._ctx, *ptrs))
        return F1, F2b, F3, F4

    def filter_device(self, x, out=None):
        """``ff(x, fxyz)`` (``src/numerics/ff.m``) of real fields, a tensor of
        shape ``(nf, nz, ny, nx)`` or ``(nz, ny, nx)``."""
        import torch
        if x.dtype != torch.float64 or not x.is_cuda or not x.is_contiguous():
            raise ValueError("expected a contiguous float64 CUDA tensor")
        nf = 1 if x.dim() == 3 else x.shape[0]
        if tuple(x.shape[-3:]) != (self.nz, self.ny, self.nx):
            raise ValueError("bad field shape")
        out = torch.empty_like(x) if out is None else out
        self._sync_stream()
        self._check(self._lib.hqt_filter_device(
            self._ctx, ctypes.c_void_p(x.data_ptr()),
            ctypes.c_void_p(out.data_ptr()), nf))
        return out

    def order_parameter_device(self, Z1):
        """``O = func_Lz(Z1)(:,:,nz)`` as a ``(ny, nx)`` complex tensor."""
        import torch
        O = torch.empty((self.ny, self.nx), dtype=torch.complex128, device=Z1.device)
        p = [self._dev3(Z1, True), self._dev2(O, True)]
        self._sync_stream()
        self._check(self._lib.hqt_boundary_order_parameter_device(self._ctx, *p))
        return O

    def winding_device(self, O) -> int:
        w = ctypes.c_int32()
        p = self._dev2(O, True)
        self._sync_stream()
        self._check(self._lib.hqt_winding_device(self._ctx, p, ctypes.byref(w)))
        return int(w.value)

    def observables_device(self, Z1, rhoi) -> dict:
        """Global observables of a device state (``hqt_observables_device``):
        ``Q`` = sum of the boundary charge rhoi(:,:,nz) dx dy, ``E_kin`` =
        sum |u|^2/2 dx dy of the density-weighted boundary velocity of
        ``scripts/analysis/movie_show.m:93-94`` and ``N_O`` = sum |O|^2 dx dy,
        as compensated FP64 sums."""
        out = np.zeros(3)
        p = [self._dev3(Z1, True), self._dev3(rhoi)]
        self._sync_stream()
        self._check(self._lib.hqt_observables_device(self._ctx, *p, _dptr(out)))
        return {"Q": float(out[0]), "E_kin": float(out[1]), "N_O": float(out[2])}

    def energy_spectrum_device(self, O):
        """``(k, E, E_c, E_i)`` of the boundary superflow of a ``(ny, nx)``
        complex CUDA tensor ``O`` (``scripts/analysis/movie_show.m:140-276``)."""
        cap = self.nx + self.ny + 4
        k, E, Ec, Ei = (np.zeros(cap) for _ in range(4))
        nb = ctypes.c_int32()
        p = self._dev2(O, True)
        self._sync_stream()
        self._check(self._lib.hqt_energy_spectrum_device(
            self._ctx, p, cap, _dptr(k), _dptr(E), _dptr(Ec), _dptr(Ei), ctypes.byref(nb)))
        n = nb.value
        return k[:n].copy(), E[:n].copy(), Ec[:n].copy(), Ei[:n].copy()

    def boundary_velocity_device(self, O):
        """``(vx, vy)``, real ``(ny, nx)`` tensors, of a ``(ny, nx)`` complex
        CUDA tensor ``O``: ``VX_temp``, ``VY_temp`` of
        ``scripts/analysis/plots_cluster.m:92-93``."""
        import torch
        p = self._dev2(O, True)
        vx = torch.empty((self.ny, self.nx), dtype=torch.float64, device=O.device)
        vy = torch.empty_like(vx)
        self._sync_stream()
        self._check(self._lib.hqt_boundary_velocity_device(
            self._ctx, p, ctypes.c_void_p(vx.data_ptr()), ctypes.c_void_p(vy.data_ptr())))
        return vx, vy

    def boundary_fields_device(self, Z1):
        """One frame of the boundary-field extraction
        (``scripts/analysis/plots_cluster.m:89-97``): ``O = func_Lz(Z1)(:,:,nz)``,
        the velocity observables ``vx, vy`` and ``NofV`` (the total of
        ``countN``).  Returns ``(O, vx, vy, NofV)`` with device tensors."""
        O = self.order_parameter_device(Z1)
        vx, vy = self.boundary_velocity_device(O)
        n, _, _ = self.count_vortices_device(O)
        return O, vx, vy, n

    def find_vortices_device(self, O, threshold: float, window_radius: int):
        """``find_vortices(O, threshold, window_radius)``
        (``src/diagnostics/find_vortices.m:1-28``) of a ``(ny, nx)`` complex
        CUDA tensor: ``(vortices, antivortices)``, each ``(n, 2)`` host arrays
        of refined 1-based ``[row, col]`` positions."""
        cap = max(self.nx * self.ny // 2, 1)
        v, a = np.zeros((cap, 2)), np.zeros((cap, 2))
        n = ctypes.c_int32()
        p = self._dev2(O, True)
        self._sync_stream()
        self._check(self._lib.hqt_find_vortices_device(
            self._ctx, p, float(threshold), int(window_radius), cap, _dptr(v), _dptr(a),
            ctypes.byref(n)))
        k = n.value
        return v[:k].copy(), a[:k].copy()

    def vortex_structure_factor_device(self, Phi, Lx: float, Ly: float):
        """``compute_vortex_structure_factor(Phi, Lx, Ly)``
        (``src/diagnostics/compute_vortex_structure_factor.m:1-104``) of a
        ``(ny, nx)`` complex CUDA tensor read as the routine's ``[Ny, Nx]``
        matrix with ``Ny = nx``: ``(k_bin, Sc, Sn, vortices, spacing)``;
        ``vortices`` rows are ``[x, y, charge]``; ``spacing`` a dict (None
        without vortices)."""
        cap = self.nx * self.ny
        bcap = self.nx + self.ny + 4
        vort = np.zeros((cap, 3))
        kb, Sc, Sn, sp = np.zeros(bcap), np.zeros(bcap), np.zeros(bcap), np.zeros(5)
        nv, nb = ctypes.c_int32(), ctypes.c_int32()
        p = self._dev2(Phi, True)
        self._sync_stream()
        self._check(self._lib.hqt_vortex_structure_factor_device(
            self._ctx, p, float(Lx), float(Ly), cap, _dptr(vort), ctypes.byref(nv), bcap,
            _dptr(kb), _dptr(Sc), _dptr(Sn), ctypes.byref(nb), _dptr(sp)))
        k, b = nv.value, nb.value
        spacing = None if k == 0 else dict(zip(
            ("rho", "d_density", "d_nnd", "k_density", "k_nnd"), map(float, sp)))
        return kb[:b].copy(), Sc[:b].copy(), Sn[:b].copy(), vort[:k].copy(), spacing

    def count_vortices(self, O) -> tuple[int, int, int]:
        """``countN`` of a host ``(nx, ny)`` complex field."""
        O = np.asarray(O)
        if O.shape != (self.nx, self.ny):
            raise ValueError("expected shape (nx, ny)")
        o = np.asfortranarray(O, dtype=np.complex128)
        n, p, m = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        self._check(self._lib.hqt_count_vortices(
            self._ctx, o.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            ctypes.byref(n), ctypes.byref(p), ctypes.byref(m)))
        return int(n.value), int(p.value), int(m.value)

    def count_vortices_device(self, O) -> tuple[int, int, int]:
        n, p, m = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        ptr = self._dev2(O, True)
        self._sync_stream()
        self._check(self._lib.hqt_count_vortices_device(
            self._ctx, ptr, ctypes.byref(n), ctypes.byref(p), ctypes.byref(m)))
        return int(n.value), int(p.value), int(m.value)


class Ensemble:
    """Independent runs advanced together (``hqt_ensemble_*`` of the C ABI).

    The reference runs one simulation per MATLAB session; a parameter scan
    (grids, ``nz``, ``mu``, seeds) is many such runs.  ``Ensemble`` groups
    :class:`Simulation` objects of one GPU and advances all of them with one
    CUDA-graph launch per step: each member's captured step graph is a child
    node of the ensemble graph, with no dependencies between members.  The
    members stay owned by the caller and must outlive the ensemble.
    """

    def __init__(self, members):
        self.members = list(members)
        if not self.members:
            raise ValueError("an ensemble needs members")
        self._lib = _lib.load()
        arr = (ctypes.c_void_p * len(self.members))(*[m._ctx for m in self.members])
        h = ctypes.c_void_p()
        code = self._lib.hqt_ensemble_create(arr, len(self.members), ctypes.byref(h))
        if code:
            raise HQTError(code, self._lib.hqt_ensemble_last_error(None).decode())
        self._ens = h

    def close(self) -> None:
        if getattr(self, "_ens", None):
            self._lib.hqt_ensemble_destroy(self._ens)
            self._ens = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step_device(self, states, nsteps: int = 1) -> list[StepInfo]:
        """Advance every member ``nsteps`` RK4 steps in place.  ``states[i]``
        is member i's ``(Z1, Z2, Z3, Z4, rhoi)`` as CUDA tensors of shape
        ``(nz, ny, nx)``.  Raises :class:`NonfiniteEvolution` (with ``.info``,
        one :class:`StepInfo` per member) when a member's fields became
        non-finite."""
        import torch
        if len(states) != len(self.members):
            raise ValueError("one state per member")
        cols = [[], [], [], [], []]
        for m, st in zip(self.members, states):
            ptrs = [m._dev3(st[0], True), m._dev3(st[1]), m._dev3(st[2]),
                    m._dev3(st[3]), m._dev3(st[4])]
            for c, p in zip(cols, ptrs):
                c.append(p.value)
        arrs = [(ctypes.c_void_p * len(c))(*c) for c in cols]
        diags = (_lib.hqt_diag * len(self.members))()
        # the graph runs on torch's current stream when it is a side stream
        # (the legacy default stream cannot hold graph launches ordered with
        # torch's work, so the device is synchronised instead)
        s = torch.cuda.current_stream(self.members[0].device).cuda_stream
        self._lib.hqt_ensemble_set_stream(self._ens, ctypes.c_void_p(s or None))
        torch.cuda.synchronize(self.members[0].device)
        code = self._lib.hqt_ensemble_step_device(self._ens, *arrs, int(nsteps), diags)
        infos = [StepInfo(int(d.steps_done), int(d.nonfinite_step), int(d.last_winding))
                 for d in diags]
        if code:
            msg = self._lib.hqt_ensemble_last_error(self._ens).decode()
            err = (NonfiniteEvolution(code, msg) if code == _lib.HQT_ENONFINITE
                   else HQTError(code, msg))
            err.info = infos
            raise err
        return infos


def assign_runs(costs, world_size: int) -> list[list[int]]:
    """Bin-pack independent runs onto ``world_size`` GPUs: longest run
    first onto the least-loaded GPU (costs are site counts or any additive
    work measure).  Returns the run indices of each rank, each list in
    ascending order; every run appears exactly once."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world_size
    out: list[list[int]] = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(o) for o in out]


def to_device(a: np.ndarray, device: int = 0):
    """A host ``[x, y, z]`` array as a column-major CUDA tensor
    (shape ``(nz, ny, nx)``)."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(np.asarray(a).T))
    return t.to(f"cuda:{device}")


def from_device(t) -> np.ndarray:
    """Inverse of :func:`to_device`: a host ``[x, y, z]`` array."""
    return t.detach().cpu().numpy().T
