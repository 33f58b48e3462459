"""Regenerate the seed fixtures of this directory from the reference.

Reads the reference's three shipped stationary seeds
``data/reference/mu=6,nz=30,vy=7_20.mat`` (MAT v5),
``data/reference/mu=5,nz=30,vy=3.8_20.mat`` and
``data/reference/mu=8,nz=30,vy=13.5_20.mat`` (MAT v7.3, i.e. HDF5 behind a
512-byte MATLAB header; their SHA-256 are in the reference's
``data/metadata/manifest.csv:9-11``) and stores their arrays as
``seed_mu<mu>_nz30_vy<n>.npz`` with a JSON sidecar.  Run it where a
reference checkout exists, giving the checkout's root directory:

    python tests/golden/make_golden.py <reference-root>

h5py is not installed here, so ``read_mat73`` reads the little HDF5 these
files use: a version-0 superblock, one root group (a level-0 v1 B-tree of
symbol-table nodes and a local heap of names) and version-1 object headers
of contiguous or compact IEEE float64 datasets.  Anything else raises.
"""
import hashlib
import json
import struct
import sys
from pathlib import Path

import numpy as np
from scipy.io import loadmat

SEEDS = [  # (file, output stem, mu, n in vy = -2*pi*n/20)
    ("mu=6,nz=30,vy=7_20.mat", "seed_mu6_nz30_vy7", 6, "7"),
    ("mu=5,nz=30,vy=3.8_20.mat", "seed_mu5_nz30_vy3.8", 5, "3.8"),
    ("mu=8,nz=30,vy=13.5_20.mat", "seed_mu8_nz30_vy13.5", 8, "13.5"),
]


def read_mat73(raw: bytes) -> dict:
    """Top-level float64 arrays of a MAT v7.3 file, MATLAB (column-major) shape."""
    sb = raw.index(b"\x89HDF\r\n\x1a\n")
    if raw[sb + 8] != 0 or raw[sb + 13] != 8 or raw[sb + 14] != 8:
        raise ValueError("unsupported superblock")
    base = struct.unpack_from("<Q", raw, sb + 24)[0]
    root = sb + 24 + 32                      # root group symbol-table entry
    btree, heap = struct.unpack_from("<QQ", raw, root + 24)

    def at(addr):
        return base + addr

    h = at(heap)
    if raw[h:h + 4] != b"HEAP":
        raise ValueError("no local heap")
    names = at(struct.unpack_from("<Q", raw, h + 24)[0])

    def name(off):
        return raw[names + off:raw.index(b"\0", names + off)].decode()

    t = at(btree)
    if raw[t:t + 4] != b"TREE" or raw[t + 4] != 0 or raw[t + 5] != 0:
        raise ValueError("root group is not one level-0 B-tree node")
    nchild = struct.unpack_from("<H", raw, t + 6)[0]
    out = {}
    for i in range(nchild):
        s = at(struct.unpack_from("<Q", raw, t + 32 + 16 * i)[0])
        if raw[s:s + 4] != b"SNOD":
            raise ValueError("no symbol-table node")
        for j in range(struct.unpack_from("<H", raw, s + 6)[0]):
            lno, oha = struct.unpack_from("<QQ", raw, s + 8 + 40 * j)
            out[name(lno)] = _dataset(raw, at, at(oha))
    return out


def _dataset(raw, at, oh):
    if raw[oh] != 1:
        raise ValueError("object header version")
    nmsg, _, size = struct.unpack_from("<HII", raw, oh + 2)
    blocks, seen = [(oh + 16, size)], 0
    dims = dtype = data = None
    while blocks and seen < nmsg:
        p, size = blocks.pop(0)
        end = p + size
        while p + 8 <= end and seen < nmsg:
            mtype, msize = struct.unpack_from("<HH", raw, p)
            d, seen = p + 8, seen + 1
            if mtype == 0x0001:                  # dataspace
                nd = raw[d + 1]
                dims = struct.unpack_from("<%dQ" % nd, raw, d + (8 if raw[d] == 1 else 4))
            elif mtype == 0x0003:                # datatype: class, size
                dtype = (raw[d] & 0x0F, struct.unpack_from("<I", raw, d + 4)[0])
            elif mtype == 0x0008:                # data layout, version 3
                if raw[d] != 3 or raw[d + 1] not in (0, 1):
                    raise ValueError("unsupported layout")
                if raw[d + 1] == 0:
                    n = struct.unpack_from("<H", raw, d + 2)[0]
                    data = raw[d + 4:d + 4 + n]
                else:
                    addr, n = struct.unpack_from("<QQ", raw, d + 2)
                    data = raw[at(addr):at(addr) + n]
            elif mtype == 0x0010:                # continuation block
                blocks.append((at(struct.unpack_from("<Q", raw, d)[0]),
                               struct.unpack_from("<Q", raw, d + 8)[0]))
            p = d + msize
    if dtype != (1, 8) or dims is None or data is None:
        raise ValueError("not a float64 dataset")
    return np.frombuffer(data, "<f8").reshape(tuple(dims[::-1]), order="F")


def main(ref_root: str) -> None:
    out = Path(__file__).resolve().parent
    for fname, stem, mu, n in SEEDS:
        src = Path(ref_root) / "data" / "reference" / fname
        raw = src.read_bytes()
        d = loadmat(src) if raw.startswith(b"MATLAB 5.0") else read_mat73(raw)
        np.savez(out / f"{stem}.npz",
                 Z1=d["Z1"].ravel(), Z2=d["Z2"].ravel(), Vy1=d["Vy1"].ravel(),
                 rhoi=d["rhoi"].ravel(), mu=np.float64(d["mu"].ravel()[0]))
        (out / f"{stem}.json").write_text(json.dumps({
            "source": f"data/reference/{fname}",
            "sha256": hashlib.sha256(raw).hexdigest(),
            "keys": ["Z1", "Z2", "Vy1", "rhoi", "mu"],
            "nz0": 30, "mu": mu, "vy": f"-2*pi*{n}/20"}, indent=1))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference-root>")
    main(sys.argv[1])
