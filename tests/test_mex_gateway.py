"""The MATLAB MEX gateway source (``mex/hqt_step_mex.c``).

MATLAB is not installed here, so the gateway is compiled against a minimal
declaration stub of the MEX API (``tests/mex_stub/mex.h``) and linked with a
small stand-in runtime (``tests/mex_stub/fake_mex.c``) that plays MATLAB's
part of ``[Z1,Z2,Z3,Z4,rhoi,info] = hqt_step_mex(Z1,Z2,Z3,Z4,rhoi,P,nsteps)``.
On a GPU the gateway's outputs must equal the Python binding's ``hqt_step``
bit for bit (both are the same library call).
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "ads4-holographic-quantum-turbulence_b200"
STUB = ROOT / "tests" / "mex_stub"
GATEWAY = PKG / "mex" / "hqt_step_mex.c"


def test_gateway_compiles_against_the_mex_api(hqt):
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-fsyntax-only",
                    "-I", str(STUB), "-I", str(ROOT / "include"), str(GATEWAY)], check=True)


def build_fake_mex(hqt, out: Path) -> Path:
    hqt._lib.load()  # builds libhqt.so if missing
    exe = out / "fake_mex"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", str(STUB),
                    "-I", str(ROOT / "include"), str(STUB / "fake_mex.c"), str(GATEWAY),
                    "-L", str(PKG), "-lhqt", f"-Wl,-rpath,{PKG}", "-o", str(exe)], check=True)
    return exe


def test_gateway_links_against_the_library(hqt, tmp_path):
    assert build_fake_mex(hqt, tmp_path).exists()


@pytest.mark.gpu
def test_gateway_step_matches_python_binding(hqt, cuda, tmp_path):
    nx, ny, nz, L, mu, vy, h, nsteps = 40, 36, 12, 20.0, 6.0, -2 * np.pi * 7 / 20, 0.02, 5
    prof = hqt.seed.stationary_profile(mu, vy)
    state = hqt.seed.init_driven(nx, ny, nz, prof, noise="complex", amplitude=1e-2, seed=3)
    exe = build_fake_mex(hqt, tmp_path)
    src, dst = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(src, "wb") as f:
        for a in state:
            f.write(np.asfortranarray(a).tobytes(order="F"))
    subprocess.run([str(exe), str(src), str(dst), str(nx), str(ny), str(nz), repr(L), repr(L),
                    repr(mu), repr(vy), repr(h), "1", str(nsteps)], check=True)
    raw = np.fromfile(dst, dtype=np.float64)
    n = nx * ny * nz
    got = [raw[:2 * n].view(np.complex128).reshape((nx, ny, nz), order="F")]
    off = 2 * n
    for _ in range(4):
        got.append(raw[off:off + n].reshape((nx, ny, nz), order="F"))
        off += n
    info = raw[off:off + 2]
    with hqt.Simulation(nx, ny, nz, Lx=L, Ly=L, mu=mu, vy=vy, dt=h, remove_winding=True) as sim:
        want, winfo = sim.step(*state, nsteps=nsteps)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    assert info[0] == nsteps and info[1] == winfo.last_winding
