"""Regenerate the golden fixtures of this directory from the reference.

Reads the reference's shipped stationary seed
``data/reference/mu=6,nz=30,vy=7_20.mat`` (MAT v5; its SHA-256 is recorded
in the reference's ``data/metadata/manifest.csv:10``) and stores its arrays
as ``seed_mu6_nz30_vy7.npz``.  Run it where a reference checkout exists,
giving the checkout's root directory:

    python tests/golden/make_golden.py <reference-root>
"""
import hashlib
import json
import sys
from pathlib import Path

import numpy as np
from scipy.io import loadmat


def main(ref_root: str) -> None:
    src = Path(ref_root) / "data" / "reference" / "mu=6,nz=30,vy=7_20.mat"
    raw = src.read_bytes()
    d = loadmat(src)
    out = Path(__file__).resolve().parent
    np.savez(out / "seed_mu6_nz30_vy7.npz",
             Z1=d["Z1"].ravel(), Z2=d["Z2"].ravel(), Vy1=d["Vy1"].ravel(),
             rhoi=d["rhoi"].ravel(), mu=np.float64(d["mu"].ravel()[0]))
    (out / "seed_mu6_nz30_vy7.json").write_text(json.dumps({
        "source": "data/reference/mu=6,nz=30,vy=7_20.mat",
        "sha256": hashlib.sha256(raw).hexdigest(),
        "keys": ["Z1", "Z2", "Vy1", "rhoi", "mu"],
        "nz0": 30, "mu": 6, "vy": "-2*pi*7/20"}, indent=1))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference-root>")
    main(sys.argv[1])
