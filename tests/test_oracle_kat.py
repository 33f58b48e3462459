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


def _smoke_phi():
    # tests/hqt_smoke_test.m:148: [x, y] = ndgrid((0:32)*2*pi/33, ...)
    g = np.arange(33) * 2 * np.pi / 33
    x, y = np.meshgrid(g, g, indexing="ij")
    return np.sin(x + 0.271) + 1j * np.sin(y + 0.613)


def test_find_vortices_smoke_pins(oracle):
    # tests/hqt_smoke_test.m:154-157: two refined vortices and antivortices on
    # phi; none on a uniform field
    phi = _smoke_phi()
    pos, neg = oracle.find_vortices(phi, 0.4, 2)
    assert pos.shape == (2, 2) and neg.shape == (2, 2)
    n, npos, nneg = oracle.countN(phi)
    assert (npos, nneg) == (len(pos), len(neg))
    pos, neg = oracle.find_vortices(np.ones((9, 9)), 0.4, 2)
    assert pos.size == 0 and neg.size == 0
    # refined positions stay within the window of the coarse plaquette
    v, av, q = oracle.find_vortices_coarse(phi)
    pos, neg = oracle.find_vortices(phi, 0.4, 2)
    assert np.all(np.abs(pos - v) <= 2.5) and np.all(np.abs(neg - av[:2]) <= 2.5)
    assert int(np.sum(q == 1)) == npos and int(np.sum(q == -1)) == nneg


def test_structure_factor_smoke_pins(oracle):
    # tests/hqt_smoke_test.m:158-159: equal bin counts, one row per vortex of
    # countN, finite nearest-neighbour spacing
    phi = _smoke_phi()
    k, Sc, Sn, vort, spacing = oracle.vortex_structure_factor(phi.T, 2 * np.pi, 2 * np.pi)
    assert len(k) == len(Sc) == len(Sn) > 0
    n, _, _ = oracle.countN(phi)
    assert vort.shape == (n, 3) and np.isfinite(spacing["d_nnd"])
    assert sorted(vort[:, 2]) == [-1, -1, 1, 1]
    # the k = 0 cell of S_n is Nv^2/Nv = Nv and sits in the first shell
    assert np.all(Sc >= 0) and np.all(Sn >= 0)
    none = oracle.vortex_structure_factor(np.ones((8, 8), complex), 1.0, 1.0)
    assert none[0].size == 0 and none[3].shape == (0, 3) and none[4] is None


def test_shell_index_edges(oracle):
    dk = 0.1
    K = np.array([0.0, 0.1, 0.3, 0.29999999999999993, 0.7, 1.05])
    b = oracle.shell_index(K, dk)
    for Ki, bi in zip(K, b):
        assert bi * dk <= Ki < (bi + 1) * dk
