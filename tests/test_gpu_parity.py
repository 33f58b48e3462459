"""CUDA path (through the C ABI) against the FP64 oracle on identical inputs.

Tolerances: FP64 results of single operators agree to 1e-11 relative to the
field's maximum (FFT versus dense-matrix derivatives differ at roundoff);
evolved fields agree to 1e-10 relative L2 after 100 steps, the drop-in
requirement; vortex counts and windings are bit-exact integers.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VY7 = -2 * np.pi * 7 / 20


def relmax(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def random_fields(nx, ny, nz, seed, amp=1.0):
    """Smooth-ish random fields with content up to the Nyquist modes."""
    rng = np.random.default_rng(seed)

    def smooth(shape):
        a = rng.standard_normal(shape)
        f = np.fft.fftn(a, axes=(0, 1))
        kx = np.fft.fftfreq(shape[0])[:, None, None]
        ky = np.fft.fftfreq(shape[1])[None, :, None]
        f *= np.exp(-(kx ** 2 + ky ** 2) * 20.0) + 0.02
        return np.real(np.fft.ifftn(f, axes=(0, 1)))

    s = (nx, ny, nz)
    Z1 = amp * (smooth(s) + 1j * smooth(s))
    return Z1, 6.0 + smooth(s), 0.3 * smooth(s), 0.3 * smooth(s)


GRIDS = [(33, 33, 10), (64, 64, 21), (48, 40, 17), (30, 22, 12), (53, 59, 8),
         (128, 96, 25), (301, 40, 8), (1024, 24, 5), (20, 1024, 5), (512, 36, 6)]


@pytest.mark.parametrize("nx,ny,nz", GRIDS)
def test_rhs_parity(hqt, oracle, dev, nx, ny, nz):
    to_d, from_d = dev
    Lx, Ly = 0.5 * nx, 0.45 * ny
    Z1, Z2, Z3, Z4 = random_fields(nx, ny, nz, seed=nx * 7 + nz)
    op = oracle.build_operators(nx, ny, nz, Lx, Ly)
    F1, F2, F3, F4 = oracle.rhs(op, Z1, Z2, Z3, Z4)
    with hqt.Simulation(nx, ny, nz, Lx=Lx, Ly=Ly) as sim:
        g1, g2b, g3, g4 = sim.rhs_device(to_d(Z1), to_d(Z2), to_d(Z3), to_d(Z4))
    g1, g3, g4 = from_d(g1), from_d(g3), from_d(g4)
    g2b = g2b.cpu().numpy().T
    assert relmax(g1, F1) < 1e-11
    assert relmax(g3, F3) < 1e-11
    assert relmax(g4, F4) < 1e-11
    assert relmax(g2b, F2[:, :, -1]) < 1e-11
    assert np.all(g1[:, :, -1] == 0) and np.all(g3[:, :, -1] == 0)


@pytest.mark.parametrize("nx,ny,nz", [(33, 33, 10), (64, 64, 21), (301, 301, 5),
                                      (53, 59, 8), (30, 22, 12),
                                      # x and y on different line engines: the
                                      # x inverse must read the weight-zeroed
                                      # columns as zero whatever the y pass did
                                      (64, 301, 4), (40, 301, 3), (301, 64, 4),
                                      (512, 48, 3), (48, 512, 3)])
def test_filter_parity(hqt, oracle, cuda, nx, ny, nz):
    torch = cuda
    rng = np.random.default_rng(nx + ny)
    fields = rng.standard_normal((3, nx, ny, nz))
    mask = oracle.filter_mask(nx, ny)
    want = np.stack([oracle.ff(f, mask) for f in fields])
    x = torch.from_numpy(np.ascontiguousarray(fields.transpose(0, 3, 2, 1))).cuda()
    with hqt.Simulation(nx, ny, nz, Lx=10.0) as sim:
        y = sim.filter_device(x)
    got = y.cpu().numpy().transpose(0, 3, 2, 1)
    assert relmax(got, want) < 1e-12


def vortex_field(nx, ny, nz, nv, seed):
    rng = np.random.default_rng(seed)
    x = np.arange(nx)[:, None] * 2 * np.pi / nx
    y = np.arange(ny)[None, :] * 2 * np.pi / ny
    psi = np.ones((nx, ny), dtype=complex)
    for _ in range(nv):
        kx, ky = rng.integers(1, 4, size=2)
        psi *= (np.sin(kx * x + rng.uniform(0, 6)) + 1j * np.sin(ky * y + rng.uniform(0, 6)) + 0.2)
    z = np.linspace(1, 0, nz)
    return psi[:, :, None] * (z * (1.5 - z))[None, None, :]


@pytest.mark.parametrize("nx,ny,nz", [(33, 33, 10), (64, 64, 21), (301, 301, 21)])
def test_order_parameter_winding_countN(hqt, oracle, dev, nx, ny, nz):
    to_d, from_d = dev
    for seed in range(3):
        Z1 = vortex_field(nx, ny, nz, 3, seed)
        wind = (seed - 1) * 2
        Z1 = Z1 * np.exp(2j * np.pi * wind * np.arange(ny) / ny)[None, :, None]
        op = oracle.build_operators(nx, ny, nz, 10.0)
        O_ref = oracle.boundary_order_parameter(op, Z1)
        with hqt.Simulation(nx, ny, nz, Lx=10.0) as sim:
            O = sim.order_parameter_device(to_d(Z1))
            assert relmax(O.cpu().numpy().T, O_ref) < 1e-12
            # identical field for the integer diagnostics
            O_same = to_d(O_ref[:, :, None])[0]
            assert sim.winding_device(O_same) == oracle.winding_number(O_ref)
            assert sim.count_vortices_device(O_same) == oracle.countN(O_ref)
            assert sim.count_vortices(O_ref) == oracle.countN(O_ref)


def test_countN_reference_kat(hqt, cuda):
    g = np.arange(33) * 2 * np.pi / 33
    x, y = np.meshgrid(g, g, indexing="ij")
    phi = np.sin(x + 0.271) + 1j * np.sin(y + 0.613)
    with hqt.Simulation(33, 33, 5, Lx=10.0) as sim:
        assert sim.count_vortices(phi) == (4, 2, 2)
        assert sim.count_vortices(np.ones((33, 33), complex)) == (0, 0, 0)


def driven_state(hqt, nx, ny, nz, seed=0, noise="complex", amp=1e-3, vy=VY7, mu=6.0):
    prof = hqt.seed.stationary_profile(mu, vy)
    return hqt.seed.init_driven(nx, ny, nz, prof, noise=noise, amplitude=amp, seed=seed)


def run_oracle(oracle, nx, ny, nz, L, state, nsteps, dt, mu, vy, remove_winding=True):
    op = oracle.build_operators(nx, ny, nz, L)
    s = oracle.OracleState(*[a.copy() for a in state])
    ws = []
    for _ in range(nsteps):
        s, w = oracle.rk4_step(op, s, dt, mu, vy, remove_winding)
        ws.append(w)
    return s, ws


@pytest.mark.parametrize("nx,nz,L,vy,noise,rw", [
    (33, 10, 16.0, VY7, "reference", True),     # smoke-test grid, driven
    (64, 21, 50.0, 0.0, "complex", True),       # CPU-runnable config
    (48, 17, 30.0, VY7, "complex", False),      # lattice script: no winding removal
    (40, 25, 20.0, VY7, "complex", True),       # 25 levels: trimmed staged tiles
    (36, 23, 18.0, VY7, "complex", True),       # 23 levels in the 25-level kernel
    (32, 33, 16.0, 0.0, "complex", True),       # 33 levels (large single run)
])
def test_single_step_parity(hqt, oracle, nx, nz, L, vy, noise, rw, cuda):
    state = driven_state(hqt, nx, nx, nz, noise=noise, amp=1e-2, vy=vy)
    ref, _ = run_oracle(oracle, nx, nx, nz, L, state, 1, 0.02, 6.0, vy, rw)
    with hqt.Simulation(nx, nx, nz, Lx=L, mu=6.0, vy=vy, dt=0.02, remove_winding=rw) as sim:
        (g1, g2, g3, g4, gr), info = sim.step(*state, nsteps=1)
    assert info.steps_done == 1
    for got, want in ((g1, ref.Z1), (g2, ref.Z2), (g4, ref.Z4), (gr, ref.rhoi)):
        assert rel_l2(got, want) < 1e-12
    # A_x starts at zero: compare on the scale of the gauge fields
    assert np.max(np.abs(g3 - ref.Z3)) < 1e-12 * np.max(np.abs(ref.Z2))


def test_hundred_steps_fp64_parity(hqt, oracle, cuda):
    """64x64x21, L=50, mu=6, dt=0.02, 100 steps: the 1e-10 drop-in bar."""
    nx, nz, L = 64, 21, 50.0
    state = driven_state(hqt, nx, nx, nz, noise="complex", amp=1e-3, vy=0.0)
    ref, ws = run_oracle(oracle, nx, nx, nz, L, state, 100, 0.02, 6.0, 0.0)
    with hqt.Simulation(nx, nx, nz, Lx=L, mu=6.0, vy=0.0, dt=0.02) as sim:
        (g1, g2, g3, g4, gr), info = sim.step(*state, nsteps=100)
    assert info.steps_done == 100 and info.nonfinite_step == -1
    errs = [rel_l2(a, b) for a, b in ((g1, ref.Z1), (g2, ref.Z2), (g3, ref.Z3 + 1e-300),
                                      (g4, ref.Z4), (gr, ref.rhoi))]
    assert max(errs[0], errs[1], errs[3], errs[4]) < 1e-10, errs
    assert np.max(np.abs(g3 - ref.Z3)) < 1e-10 * max(1.0, np.max(np.abs(ref.Z3)))
    assert info.last_winding == ws[-1]


def test_driven_301_parity(hqt, oracle, cuda):
    """The 301x301x21 driven configuration for a few steps."""
    nx, nz, L = 301, 21, 100.0
    state = driven_state(hqt, nx, nx, nz, noise="complex", amp=1e-3)
    ref, ws = run_oracle(oracle, nx, nx, nz, L, state, 3, 0.02, 6.0, VY7)
    with hqt.Simulation(nx, nx, nz, Lx=L, mu=6.0, vy=VY7, dt=0.02) as sim:
        (g1, g2, g3, g4, gr), info = sim.step(*state, nsteps=3)
    for got, want in ((g1, ref.Z1), (g2, ref.Z2), (g4, ref.Z4), (gr, ref.rhoi)):
        assert rel_l2(got, want) < 1e-11
    assert np.max(np.abs(g3 - ref.Z3)) < 1e-11 * max(1.0, np.max(np.abs(ref.Z3)))


def test_winding_removal_matches(hqt, oracle, cuda):
    nx, nz, L = 40, 9, 20.0
    state = list(driven_state(hqt, nx, nx, nz, noise="complex", amp=1e-2))
    # imprint a net winding of 3 along y
    state[0] = state[0] * np.exp(2j * np.pi * 3 * np.arange(nx) / nx)[None, :, None]
    ref, ws = run_oracle(oracle, nx, nx, nz, L, state, 2, 0.02, 6.0, VY7)
    assert ws[0] == 3
    with hqt.Simulation(nx, nx, nz, Lx=L, mu=6.0, vy=VY7, dt=0.02) as sim:
        (g1, *_), info = sim.step(*state, nsteps=2)
    assert rel_l2(g1, ref.Z1) < 1e-12


def test_device_step_matches_host_step(hqt, dev):
    to_d, from_d = dev
    nx, nz = 32, 12
    state = driven_state(hqt, nx, nx, nz)
    with hqt.Simulation(nx, nx, nz, Lx=16.0, vy=VY7) as sim:
        (h1, h2, h3, h4, hr), _ = sim.step(*state, nsteps=5)
    with hqt.Simulation(nx, nx, nz, Lx=16.0, vy=VY7) as sim:
        t = [to_d(a) for a in state]
        sim.step_device(*t, nsteps=5)
    for a, b in zip((h1, h2, h3, h4, hr), t):
        assert np.array_equal(a, from_d(b))


def test_vortex_records_in_loop(hqt, oracle, cuda):
    nx, nz, L = 48, 9, 24.0
    state = driven_state(hqt, nx, nx, nz, noise="complex", amp=0.3)
    with hqt.Simulation(nx, nx, nz, Lx=L, vy=VY7, diag_every=2) as sim:
        (g1, *_), info = sim.step(*state, nsteps=4, records=8)
    assert info.records.shape == (2, 4)
    assert list(info.records[:, 0]) == [2, 4]
    op = oracle.build_operators(nx, nx, nz, L)
    O = oracle.boundary_order_parameter(op, g1)
    assert tuple(info.records[1, 1:]) == oracle.countN(O)


def test_nonfinite_guard(hqt, cuda):
    nx, nz = 24, 8
    state = list(driven_state(hqt, nx, nx, nz))
    state[2] = state[2].copy()
    state[2][3, 4, 2] = np.nan
    with hqt.Simulation(nx, nx, nz, Lx=12.0) as sim:
        with pytest.raises(hqt.NonfiniteEvolution) as e:
            sim.step(*state, nsteps=10)
        assert e.value.info.nonfinite_step == 1
        assert e.value.info.steps_done == 1
        # the context stays usable after the error
        (g1, *_), info = sim.step(*driven_state(hqt, nx, nx, nz), nsteps=1)
        assert np.all(np.isfinite(g1))


def test_nonfinite_run_stops_at_the_bad_step(hqt, dev):
    """Like the reference's guard (tevol_driven_cluster.m:182-185), a run stops
    at the first non-finite step: the device skips every later step, so the
    fields returned after asking for 100 steps equal those after 1 step."""
    to_d, from_d = dev
    nx, nz = 24, 8
    state = list(driven_state(hqt, nx, nx, nz))
    state[2] = state[2].copy()
    state[2][3, 4, 2] = np.nan
    out = []
    for nsteps in (1, 100):
        t = [to_d(a) for a in state]
        with hqt.Simulation(nx, nx, nz, Lx=12.0) as sim:
            with pytest.raises(hqt.NonfiniteEvolution) as e:
                sim.step_device(*t, nsteps=nsteps)
        assert e.value.info.nonfinite_step == 1 and e.value.info.steps_done == 1
        out.append([from_d(x) for x in t])
    for a, b in zip(*out):
        assert np.array_equal(a, b, equal_nan=True)


def test_device_diagnostics_reject_misaligned_arrays(hqt, cuda):
    """Interleaved-complex device arguments must be 16-byte aligned: a
    misaligned pointer is HQT_EINVAL, not a fault on the GPU."""
    torch = cuda
    lib = hqt._lib.load()
    nx, nz = 16, 8
    buf = torch.zeros(2 * nx * nx * nz + 2, dtype=torch.float64, device="cuda")
    bad = ctypes.c_void_p(buf.data_ptr() + 8)
    good = ctypes.c_void_p(buf.data_ptr())
    n = ctypes.c_int32()
    with hqt.Simulation(nx, nx, nz, Lx=8.0) as sim:
        ctx = sim._ctx
        assert lib.hqt_boundary_order_parameter_device(ctx, bad, good) == 1
        assert lib.hqt_count_vortices_device(ctx, bad, ctypes.byref(n), ctypes.byref(n),
                                             ctypes.byref(n)) == 1
        assert lib.hqt_winding_device(ctx, bad, ctypes.byref(n)) == 1
        assert b"aligned" in lib.hqt_last_error(ctx)


@pytest.mark.parametrize("engine", ["runtime", "stockham"])
@pytest.mark.parametrize("nx,ny,nz", [(64, 64, 21), (301, 301, 9), (53, 59, 8)])
def test_runtime_line_engine_parity(hqt, oracle, dev, monkeypatch, nx, ny, nz, engine):
    """The other line-transform engines on the same RHS and filter checks:
    the runtime-plan engine (line lengths without a compile-time transform)
    and the compile-time Stockham engine (which the prime-factor tensor-core
    engine replaces for its lengths)."""
    monkeypatch.setenv("HQT_LINE_ENGINE", engine)
    to_d, from_d = dev
    Lx, Ly = 0.5 * nx, 0.45 * ny
    Z1, Z2, Z3, Z4 = random_fields(nx, ny, nz, seed=nx + nz)
    op = oracle.build_operators(nx, ny, nz, Lx, Ly)
    F1, F2, F3, F4 = oracle.rhs(op, Z1, Z2, Z3, Z4)
    with hqt.Simulation(nx, ny, nz, Lx=Lx, Ly=Ly) as sim:
        g1, g2b, g3, g4 = sim.rhs_device(to_d(Z1), to_d(Z2), to_d(Z3), to_d(Z4))
        x = to_d(Z3)[None].contiguous()
        y = sim.filter_device(x)
    assert relmax(from_d(g1), F1) < 1e-11
    assert relmax(from_d(g3), F3) < 1e-11
    assert relmax(from_d(g4), F4) < 1e-11
    assert relmax(g2b.cpu().numpy().T, F2[:, :, -1]) < 1e-11
    assert relmax(from_d(y[0]), oracle.ff(Z3, op.mask)) < 1e-12


@pytest.mark.parametrize("nx,ny,nz", [(64, 64, 9), (301, 301, 9), (53, 48, 8)])
def test_energy_spectrum_parity(hqt, oracle, dev, nx, ny, nz):
    to_d, from_d = dev
    Lx, Ly = 0.4 * nx, 0.4 * ny
    Z1 = vortex_field(nx, ny, nz, 4, seed=nx)
    op = oracle.build_operators(nx, ny, nz, Lx, Ly)
    O = oracle.boundary_order_parameter(op, Z1)
    k, E, Ec, Ei = oracle.energy_spectrum(O, Lx, Ly)
    with hqt.Simulation(nx, ny, nz, Lx=Lx, Ly=Ly) as sim:
        gk, gE, gEc, gEi = sim.energy_spectrum_device(to_d(O[:, :, None])[0])
    assert len(gk) == len(k)
    assert np.allclose(gk, k, rtol=1e-14)
    scale = E.max()
    for got, want in ((gE, E), (gEc, Ec), (gEi, Ei)):
        assert np.max(np.abs(got - want)) < 1e-9 * scale


def test_mixed_precision_error_100_steps(hqt, oracle, cuda):
    """Mixed precision (FP32 line passes on slice-mean-removed copies, FP64
    columns and state) against the FP64 oracle after 100 steps at 64x64x21.
    Relative L2 per field; A_x and A_y start at zero without a drive, so they
    are measured against the gauge-field scale max|A_t|."""
    nx, nz, L = 64, 21, 50.0
    state = driven_state(hqt, nx, nx, nz, noise="complex", amp=1e-3, vy=0.0)
    ref, _ = run_oracle(oracle, nx, nx, nz, L, state, 100, 0.02, 6.0, 0.0)
    with hqt.Simulation(nx, nx, nz, Lx=L, mu=6.0, vy=0.0, dt=0.02, precision="mixed") as sim:
        (g1, g2, g3, g4, gr), info = sim.step(*state, nsteps=100)
    scale = np.max(np.abs(ref.Z2))
    errs = {"Z1": rel_l2(g1, ref.Z1), "Z2": rel_l2(g2, ref.Z2), "rhoi": rel_l2(gr, ref.rhoi),
            "Z3_abs": float(np.max(np.abs(g3 - ref.Z3)) / scale),
            "Z4_abs": float(np.max(np.abs(g4 - ref.Z4)) / scale)}
    print("mixed-precision errors after 100 steps:", errs)
    assert max(errs.values()) < 1e-8, errs


def test_mixed_precision_driven_301(hqt, cuda, dev):
    """301x301x21 driven: mixed against the FP64 GPU path (itself pinned to the
    oracle) after 100 steps.  A_x, which the drive keeps small, is measured
    against the gauge-field scale max|A_t|; the others by relative L2."""
    to_d, from_d = dev
    nx, nz, L = 301, 21, 100.0
    state = driven_state(hqt, nx, nx, nz, noise="complex", amp=1e-3)
    out = {}
    for prec in ("fp64", "mixed"):
        t = [to_d(a) for a in state]
        with hqt.Simulation(nx, nx, nz, Lx=L, mu=6.0, vy=VY7, dt=0.02, precision=prec) as sim:
            sim.step_device(*t, nsteps=100)
        out[prec] = [from_d(x) for x in t]
    m, f = out["mixed"], out["fp64"]
    errs = {"Z1": rel_l2(m[0], f[0]), "Z2": rel_l2(m[1], f[1]), "Z4": rel_l2(m[3], f[3]),
            "rhoi": rel_l2(m[4], f[4]),
            "Z3_abs": float(np.max(np.abs(m[2] - f[2])) / np.max(np.abs(f[1])))}
    print("mixed vs fp64 after 100 steps (301^2x21):", errs)
    assert max(errs.values()) < 1e-8, errs


@pytest.mark.parametrize("nx,ny,nz", [(64, 64, 21), (301, 301, 9), (53, 48, 8)])
def test_observables_parity(hqt, oracle, dev, nx, ny, nz):
    """Q, E_kin, N_O (compensated FP64 sums) against the oracle's exactly
    rounded sums on the same state."""
    to_d, from_d = dev
    L = 0.5 * nx
    state = driven_state(hqt, nx, ny, nz, noise="complex", amp=0.05)
    op = oracle.build_operators(nx, ny, nz, L)
    want = oracle.observables(op, state[0], state[4])
    with hqt.Simulation(nx, ny, nz, Lx=L) as sim:
        got = sim.observables_device(to_d(state[0]), to_d(state[4]))
    for k, w in zip(("Q", "E_kin", "N_O"), want):
        assert abs(got[k] - w) <= 1e-12 * abs(w), (k, got[k], w)


def test_observable_records_in_loop(hqt, dev):
    """With records, every diag_every steps the step records (Q, E_kin, N_O)
    of the state at that step; the charge stays conserved to roundoff."""
    to_d, from_d = dev
    nx, nz, L = 48, 12, 24.0
    state = driven_state(hqt, nx, nx, nz, noise="complex", amp=0.05)
    with hqt.Simulation(nx, nx, nz, Lx=L, vy=VY7, diag_every=3) as sim:
        t = [to_d(a) for a in state]
        q0 = sim.observables_device(t[0], t[4])
        info = sim.step_device(*t, nsteps=6, records=4)
        last = sim.observables_device(t[0], t[4])
    assert info.observables.shape == (2, 3)
    assert list(info.records[:, 0]) == [3, 6]
    assert tuple(info.observables[1]) == (last["Q"], last["E_kin"], last["N_O"])
    assert abs(info.observables[1, 0] - q0["Q"]) < 1e-12 * abs(q0["Q"])
