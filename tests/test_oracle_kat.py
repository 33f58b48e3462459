"""The oracle against the reference's own known-answer tests
(tests/hqt_smoke_test.m of the reference)."""
import numpy as np


def test_fourdif_kat(oracle):
    # hqt_smoke_test.m:129-130
    x, D = oracle.fourdif(33, 1)
    assert np.max(np.abs(D @ np.sin(3 * x) - 3 * np.cos(3 * x))) < 1e-10


def test_chebdif_kat(oracle):
    # hqt_smoke_test.m:131-133
    z, DM = oracle.chebdif(20, 2)
    assert np.max(np.abs(DM[0] @ z ** 4 - 4 * z ** 3)) < 1e-10
    assert np.max(np.abs(DM[1] @ z ** 4 - 12 * z ** 2)) < 1e-8


def test_chebdif_points_descend(oracle):
    z, _ = oracle.chebdif(21, 1)
    assert z[0] == 1.0 and z[-1] == -1.0 and np.all(np.diff(z) < 0)


def test_ff_empty_mask_kat(oracle):
    # hqt_smoke_test.m:139-141
    rng = np.random.default_rng(11)
    field = rng.standard_normal((17, 19)) + 1j * rng.standard_normal((17, 19))
    empty = np.zeros(field.shape, dtype=bool)
    assert np.max(np.abs(oracle.ff(field, empty) - field.real)) < 1e-12


def test_countN_kat(oracle):
    # hqt_smoke_test.m:148-151: phi = sin(x+0.271) + i sin(y+0.613), 33x33
    g = np.arange(33) * 2 * np.pi / 33
    x, y = np.meshgrid(g, g, indexing="ij")
    phi = np.sin(x + 0.271) + 1j * np.sin(y + 0.613)
    assert oracle.countN(phi) == (4, 2, 2)


def test_countN_empty_field(oracle):
    assert oracle.countN(np.ones((9, 9), dtype=complex)) == (0, 0, 0)


def test_fourdif_equals_spectral_multiplier(oracle):
    # the property the GPU path relies on: fourdif D1 == FFT i*k (Nyquist 0)
    rng = np.random.default_rng(0)
    for n in (33, 64, 301, 192):
        _, D = oracle.fourdif(n, 1)
        u = rng.standard_normal(n)
        k = np.fft.fftfreq(n, 1.0 / n)
        ik = 1j * k
        if n % 2 == 0:
            ik[n // 2] = 0
        du = np.real(np.fft.ifft(ik * np.fft.fft(u)))
        assert np.max(np.abs(D @ u - du)) <= 1e-12 * np.max(np.abs(du))


def test_filter_mask_band(oracle):
    # fx(round(round(n/3)):round(n/3*2)) = 1 (1-based), tevol_driven_cluster.m:28
    m = oracle.filter_mask(301, 301)
    zeroed = np.where(m[:, 0])[0]
    assert zeroed[0] == 99 and zeroed[-1] == 200
    m = oracle.filter_mask(64, 64)
    zeroed = np.where(m[:, 0])[0]
    assert zeroed[0] == 20 and zeroed[-1] == 42


def test_matlab_round(oracle):
    assert oracle.matlab_round(2.5) == 3 and oracle.matlab_round(-2.5) == -3
    assert oracle.matlab_round(0.49) == 0


def test_rk4_step_finite_smoke_size(oracle, hqt):
    # hqt_smoke_test.m:189-198: nx=33, nz=10, 4 steps of 0.02, finite fields
    prof = hqt.seed.stationary_profile(6.0, -2 * np.pi * 7 / 20)
    Z1, Z2, Z3, Z4, rhoi = hqt.seed.init_driven(33, 33, 10, prof,
                                                noise="reference",
                                                amplitude=1e-2, seed=0)
    op = oracle.build_operators(33, 33, 10, 16.0)
    s = oracle.OracleState(Z1, Z2, Z3, Z4, rhoi)
    s, w = oracle.run(op, s, 4, 0.02, 6.0, -2 * np.pi * 7 / 20)
    for f in (s.Z1, s.Z2, s.Z3, s.Z4):
        assert np.all(np.isfinite(f))
    assert np.all(s.Z1[:, :, -1] == 0)
    assert np.max(np.abs(s.Z2[:, :, -1] - 6.0)) < 1e-12


def test_energy_spectrum_helmholtz_split(oracle):
    # E = E_c + E_i (the split is orthogonal mode by mode); a single vortex
    # dipole carries mostly incompressible energy
    n = 48
    g = np.arange(n) * 2 * np.pi / n
    x, y = np.meshgrid(g, g, indexing="ij")
    O = np.tanh(np.hypot(np.sin((x - 2) / 2), np.sin((y - 3) / 2)) * 6) * 0 + 1.0
    O = O * (np.sin(x - 2.0) + 1j * np.sin(y - 3.0) + 0.3)
    k, E, Ec, Ei = oracle.energy_spectrum(O, 2 * np.pi, 2 * np.pi)
    assert len(k) > 10 and np.all(E >= 0) and np.all(Ec >= 0) and np.all(Ei >= 0)
    assert np.allclose(E, Ec + Ei, rtol=1e-12, atol=1e-12 * E.max())
    assert Ei.sum() > Ec.sum()


def test_signed_wavenumbers(oracle):
    assert list(oracle.signed_wavenumbers(4)) == [0, 1, -2, -1]
    assert list(oracle.signed_wavenumbers(5)) == [0, 1, 2, -2, -1]
