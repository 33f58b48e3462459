"""Checkpoint files in the reference's format.

``check_point_t=<t>.mat`` holds ``Z1, Z2, Z3, Z4, rhoi`` as ``[nx, ny, nz]``
arrays (``scripts/simulation/tevol_driven_cluster.m:178-181``,
``docs/DATA_DICTIONARY.md:27-39``).  They are written as MAT v5 with
``scipy.io.savemat`` (the reference's default ``save`` may produce v7.3/HDF5,
which needs h5py, absent here); the grid and run parameters, which the
reference does not store, go to a JSON sidecar ``<file>.json``.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

__all__ = ["checkpoint_name", "save_checkpoint", "load_checkpoint"]


def checkpoint_name(t: float) -> str:
    """``['check_point_t=',num2str(t),'.mat']`` -- num2str keeps up to four
    decimals and drops trailing zeros."""
    s = f"{t:.4f}".rstrip("0").rstrip(".")
    return f"check_point_t={s}.mat"


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
