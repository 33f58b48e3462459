"""Build ``libhqt.so`` (the C ABI of ``include/hqt.h``) in-tree for sm_100a.

Every ``.cu``/``.cpp`` under ``csrc/`` is compiled by ``nvcc`` with
``-gencode arch=compute_100a,code=sm_100a`` in parallel (the column kernels
are one translation unit per compile-time column length), then linked into
``libhqt.so`` next to this file.  Objects are cached in ``_build/`` by
content hash, so an unchanged source is not recompiled.

Usage: ``python build.py [-v] [--ptxas]``
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
OUT = PKG / "libhqt.so"
OBJDIR = PKG / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
          "-I" + str(INCLUDE), "-I" + str(CSRC)]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"),
                 "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers_digest() -> str:
    h = hashlib.sha256()
    for p in sorted(list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h"))
                    + list(INCLUDE.glob("*.h"))):
        h.update(p.name.encode())
        h.update(p.read_bytes())
    return h.hexdigest()[:16]


def _compile(nvcc: str, src: Path, hdr: str, ptxas: bool, verbose: bool):
    h = hashlib.sha256(src.read_bytes() + hdr.encode()
                       + " ".join(ARCH + COMMON).encode()).hexdigest()[:16]
    obj = OBJDIR / f"{src.stem}.{h}.o"
    if obj.exists() and not ptxas:
        return obj, ""
    cmd = [nvcc, *ARCH, *COMMON, "-c", str(src), "-o", str(obj)]
    if ptxas:
        cmd.insert(1, "-Xptxas=-v")
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose: bool = False, ptxas: bool = False) -> Path:
    """Compile and link ``libhqt.so``; returns its path."""
    nvcc = _nvcc()
    OBJDIR.mkdir(exist_ok=True)
    hdr = _headers_digest()
    srcs = _sources()
    logs = []
    with cf.ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        futs = [ex.submit(_compile, nvcc, s, hdr, ptxas, verbose) for s in srcs]
        objs = []
        for f in futs:
            o, log = f.result()
            objs.append(o)
            logs.append(log)
    keep = {o.name for o in objs}
    for stale in OBJDIR.glob("*.o"):
        if stale.name not in keep:
            stale.unlink()
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs),
           "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, OUT)
    if ptxas:
        sys.stderr.write("".join(logs))
    return OUT


if __name__ == "__main__":
    path = build(verbose="-v" in sys.argv, ptxas="--ptxas" in sys.argv)
    print(path)
