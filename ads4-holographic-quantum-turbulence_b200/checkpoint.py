"""Checkpoint files in the reference's format.

``check_point_t=<t>.mat`` holds ``Z1, Z2, Z3, Z4, rhoi`` as ``[nx, ny, nz]``
arrays (``scripts/simulation/tevol_driven_cluster.m:178-181``,
``docs/DATA_DICTIONARY.md:27-39``).  They are written as MAT v5 with
``scipy.io.savemat`` (the reference's default ``save`` may produce v7.3/HDF5,
which needs h5py, absent here); the grid and run parameters, which the
reference does not store, go to a JSON sidecar ``<file>.json``.

Processed boundary-field files ``driven_mu=<mu>,v=<v>_20.mat`` hold
``NofV`` (1 x nt), ``O``, ``vx``, ``vy`` (nx x ny x nt) of sampled frames
(``scripts/analysis/plots_cluster.m:77-99``, ``docs/DATA_DICTIONARY.md:41-51``);
``extract_boundary_fields`` computes them on the GPU from checkpoints or
in-memory states, also written as MAT v5.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

__all__ = ["checkpoint_name", "save_checkpoint", "load_checkpoint", "num2str",
           "driven_name", "extract_boundary_fields", "save_boundary_fields",
           "load_boundary_fields"]


def checkpoint_name(t: float) -> str:
    """``['check_point_t=',num2str(t),'.mat']``
    (``scripts/simulation/tevol_driven_cluster.m:179``)."""
    return f"check_point_t={num2str(t)}.mat"


def save_checkpoint(path, Z1, Z2, Z3, Z4, rhoi, params: dict | None = None):
    from scipy.io import savemat
    path = Path(path)
    savemat(path, {"Z1": np.asarray(Z1), "Z2": np.asarray(Z2),
                   "Z3": np.asarray(Z3), "Z4": np.asarray(Z4),
                   "rhoi": np.asarray(rhoi)}, do_compression=False)
    if params is not None:
        path.with_suffix(path.suffix + ".json").write_text(
            json.dumps(params, indent=1, sort_keys=True))
    return path


def load_checkpoint(path):
    """Returns ``(Z1, Z2, Z3, Z4, rhoi, params_or_None)``."""
    from scipy.io import loadmat
    path = Path(path)
    d = loadmat(path)
    side = path.with_suffix(path.suffix + ".json")
    params = json.loads(side.read_text()) if side.exists() else None
    return (d["Z1"].astype(np.complex128), d["Z2"], d["Z3"], d["Z4"],
            d["rhoi"], params)


def num2str(x: float) -> str:
    """MATLAB ``num2str`` of a real scalar: integers in full, otherwise
    ``%.<d>g`` with ``d = max(floor(log10|x|) + 5, 5)`` significant digits
    (at most 16): four digits after the leading one, and at least five."""
    x = float(x)
    if np.isfinite(x) and x == np.round(x):
        return str(int(np.round(x)))
    digits = min(max(int(np.floor(np.log10(abs(x)))) + 5, 5), 16)
    return f"{x:.{digits}g}"


def driven_name(mu: float, vy_load: float) -> str:
    """``['driven_mu=',num2str(mu),',v=',num2str(-vy_load*20/2/pi),'_20.mat']``
    (``scripts/analysis/plots_cluster.m:99``)."""
    return f"driven_mu={num2str(mu)},v={num2str(-vy_load * 20 / 2 / np.pi)}_20.mat"


def extract_boundary_fields(sim, frames, device: int = 0):
    """Boundary fields of sampled frames (``plots_cluster.m:83-98``).

    ``frames`` is an iterable of checkpoint paths or of ``Z1`` arrays
    (``[nx, ny, nz]`` complex, host or CUDA).  Each frame goes through
    ``sim.boundary_fields_device``: ``O = func_Lz(Z1)(:,:,nz)``, the velocity
    observables ``vx, vy`` and the vortex count.  Returns host arrays
    ``(NofV, O, vx, vy)`` shaped ``(1, nt)`` and ``(nx, ny, nt)``.
    """
    import torch
    from .api import from_device, to_device
    Os, vxs, vys, nv = [], [], [], []
    for fr in frames:
        if isinstance(fr, (str, Path)):
            fr = load_checkpoint(fr)[0]
        if not torch.is_tensor(fr):
            fr = to_device(np.asarray(fr, dtype=np.complex128), device)
        O, vx, vy, n = sim.boundary_fields_device(fr)
        Os.append(from_device(O))
        vxs.append(from_device(vx))
        vys.append(from_device(vy))
        nv.append(n)
    nt = len(nv)
    shape = (sim.nx, sim.ny, nt)
    stack = lambda xs, dt: (np.stack(xs, axis=-1) if xs else np.zeros(shape, dt))
    return (np.asarray(nv, dtype=np.float64).reshape(1, nt), stack(Os, np.complex128),
            stack(vxs, np.float64), stack(vys, np.float64))


def save_boundary_fields(path, NofV, O, vx, vy):
    """``save(..., 'NofV','O','vx','vy')`` of ``plots_cluster.m:99`` as MAT v5
    (the reference writes ``-v7.3``, which needs HDF5)."""
    from scipy.io import savemat
    path = Path(path)
    savemat(path, {"NofV": np.asarray(NofV, dtype=np.float64), "O": np.asarray(O),
                   "vx": np.asarray(vx), "vy": np.asarray(vy)}, do_compression=False)
    return path


def load_boundary_fields(path):
    """Returns ``(NofV, O, vx, vy)`` of a boundary-field file."""
    from scipy.io import loadmat
    d = loadmat(Path(path))
    return d["NofV"], d["O"].astype(np.complex128), d["vx"], d["vy"]
