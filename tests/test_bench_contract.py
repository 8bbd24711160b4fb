"""The benchmark's output contract, checked on the CPU: the reference arm (the oracle port) on a
16³ grid prints one JSON line with the keys the driver reads, and the algorithmic byte counts
behind the roofline follow the pruned design."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--grid", "16",
                          "--tracers", "50", "--steps", "1", "--warmup", "0"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "steps/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["scaling"] == "weak"
    assert "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_algorithmic_bytes_follow_the_pruned_design():
    sys.path.insert(0, ROOT)
    import bench
    N, K, w = 512, 170, 16
    b = bench.algorithmic_bytes_per_step(N, K, w)
    KX1, NY2 = K + 1, 2 * K + 1
    assert b["x_products"] == 5 * N * N * KX1 * 13 * w                     # 7 spectra in, 6 out, 5 stages
    assert b["y_inverse"] == (4 * 7 + 4 + 3) * N * KX1 * (NY2 + N) * w     # first stage 4 slots, deposit 3
    assert b["y_forward"] == 5 * 6 * N * KX1 * (N + NY2) * w
    assert all(v > 0 for v in b.values())
    v = bench.algorithmic_bytes_per_step(N, K, w, has_scalar=False)
    assert v["x_products"] == 5 * N * N * KX1 * 9 * w
