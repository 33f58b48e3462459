"""The allocation-free vortex count against the context-based path.

``hqt_count_vortices_field_noalloc`` serves callers that cannot call
cudaMalloc (a MEX gateway whose device memory belongs to MATLAB's gpuArray
pool, a framework whose caching allocator owns a fixed budget, a real-time
host that must not allocate after start-up).  It keeps its scratch in
file-scope device arrays, so two calls in a row must both agree with the
context path (``hqt_boundary_order_parameter_device`` followed by
``hqt_count_vortices_device``), including a second call on a different field
(the counters are cleared per call).  Vortex counts are integers: exact.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def vortex_field(nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    x = np.arange(nx)[:, None] * 2 * np.pi / nx
    y = np.arange(ny)[None, :] * 2 * np.pi / ny
    psi = np.ones((nx, ny), dtype=complex)
    for _ in range(3):
        kx, ky = rng.integers(1, 4, size=2)
        psi *= (np.sin(kx * x + rng.uniform(0, 6)) + 1j * np.sin(ky * y + rng.uniform(0, 6))
                + 0.2)
    z = np.linspace(1, 0, nz)
    return psi[:, :, None] * (z * (1.5 - z))[None, None, :]


def noalloc_count(lib, t, nx, ny, nz):
    n, p, m = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    code = lib.hqt_count_vortices_field_noalloc(ctypes.c_void_p(t.data_ptr()), nx, ny, nz,
                                                ctypes.byref(n), ctypes.byref(p),
                                                ctypes.byref(m), None)
    assert code == 0, lib.hqt_noalloc_last_error()
    return n.value, p.value, m.value


@pytest.mark.parametrize("nx,ny,nz", [(64, 48, 12), (301, 301, 21)])
def test_noalloc_count_matches_context_path(hqt, cuda, nx, ny, nz):
    torch = cuda
    api = __import__(hqt.__name__ + ".api", fromlist=["to_device"])
    lib = hqt._lib.load()
    fields = [vortex_field(nx, ny, nz, s) for s in (0, 1)]
    with hqt.Simulation(nx, ny, nz, Lx=10.0) as sim:
        want = [sim.count_vortices_device(sim.order_parameter_device(api.to_device(f)))
                for f in fields]
    assert want[0] != (0, 0, 0)
    # two calls in a row on the first field, then one on the second field
    t0, t1 = api.to_device(fields[0]), api.to_device(fields[1])
    torch.cuda.synchronize()
    assert noalloc_count(lib, t0, nx, ny, nz) == want[0]
    assert noalloc_count(lib, t0, nx, ny, nz) == want[0]
    assert noalloc_count(lib, t1, nx, ny, nz) == want[1]


def test_noalloc_rejects_planes_beyond_the_scratch(hqt, cuda):
    torch = cuda
    lib = hqt._lib.load()
    t = torch.zeros(2, dtype=torch.complex128, device="cuda")
    n = ctypes.c_int32()
    code = lib.hqt_count_vortices_field_noalloc(ctypes.c_void_p(t.data_ptr()), 2048, 1024,
                                                8, ctypes.byref(n), ctypes.byref(n),
                                                ctypes.byref(n), None)
    assert code == 1
    assert b"scratch plane" in lib.hqt_noalloc_last_error()
