"""MAT-v5 checkpoints in the reference's variable layout."""
import numpy as np


def test_name_formatting(hqt):
    assert hqt.checkpoint.checkpoint_name(50.0) == "check_point_t=50.mat"
    assert hqt.checkpoint.checkpoint_name(0.08) == "check_point_t=0.08.mat"
    # t accumulated as t = t + h carries rounding noise that num2str hides
    t = 0.0
    for _ in range(4):
        t += 0.02
    assert hqt.checkpoint.checkpoint_name(t) == "check_point_t=0.08.mat"
    assert hqt.checkpoint.checkpoint_name(0.123456) == "check_point_t=0.12346.mat"


def test_num2str_known_answers(hqt):
    """MATLAB num2str of non-integers: max(floor(log10|x|)+5, 5) significant
    digits; integers in full."""
    n2s = hqt.checkpoint.num2str
    assert n2s(0.123456) == "0.12346"
    assert n2s(3.14159) == "3.1416"
    assert n2s(123.456789) == "123.4568"
    assert n2s(-0.5) == "-0.5"
    assert n2s(7.0) == "7"
    assert n2s(-2.0) == "-2"


def test_round_trip(hqt, tmp_path):
    rng = np.random.default_rng(0)
    shape = (5, 4, 3)
    Z1 = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    Z2, Z3, Z4, rho = (rng.standard_normal(shape) for _ in range(4))
    p = hqt.save_checkpoint(tmp_path / "check_point_t=1.mat", Z1, Z2, Z3, Z4,
                            rho, params={"nx": 5, "mu": 6.0})
    from scipy.io import loadmat
    raw = loadmat(p)
    assert set(k for k in raw if not k.startswith("__")) == {"Z1", "Z2", "Z3", "Z4", "rhoi"}
    out = hqt.load_checkpoint(p)
    for a, b in zip(out[:5], (Z1, Z2, Z3, Z4, rho)):
        assert np.array_equal(a, b)
    assert out[5] == {"nx": 5, "mu": 6.0}
