"""The bench's JSON contract on CPU: the reference arm's line and the
per-kernel roofline rows (no GPU needed for either)."""
import json
import subprocess
import sys

import pytest

from conftest import ROOT

sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def test_kernel_rows_roofline_fraction():
    ks = [{"kernel": "zstage", "launches": 80, "ms": 9.44},
          {"kernel": "winding", "launches": 20, "ms": 0.2}]
    rows = bench.kernel_rows(ks, 9.64, 301 * 301 * 21, 6545.9)
    z = rows["zstage"]
    gbs = bench.ALG_BYTES["zstage"] * 301 * 301 * 21 * 80 / 9.44e-3 / 1e9
    assert z["launches"] == 80 and z["share"] == round(9.44 / 9.64, 4)
    assert z["alg_gbs"] == round(gbs, 1) and z["hbm_frac"] == round(gbs / 6545.9, 4)
    # kernels without algorithmic bytes, and rows without a peak, carry no fraction
    assert "hbm_frac" not in rows["winding"]
    assert "hbm_frac" not in bench.kernel_rows(ks, 9.64)["zstage"]


def test_both_arms_share_the_config():
    w = bench.WORKLOADS["driven301"]
    c = bench.bench_config("driven301", w, 1)
    for key in ("workload", "nx", "ny", "nz", "L", "mu", "vy", "dt", "remove_winding",
                "filter", "precision"):
        assert key in c
    assert (c["nx"], c["ny"], c["nz"], c["L"], c["dt"]) == (301, 301, 21, 100.0, 0.02)


@pytest.mark.timeout(600)
def test_reference_arm_line():
    """``bench.py --impl reference`` times the C + OpenMP restatement on the
    host cores and prints one line with the contract's keys."""
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True,
                       cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d["impl"] == "reference" and d["metric"] == "RK4 site-updates/s"
    assert d["unit"] == "site-updates/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert d["config"] == bench.bench_config("driven301", bench.WORKLOADS["driven301"], 1)
