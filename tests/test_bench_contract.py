"""The bench.py JSON line, on the CPU: the reference arm (the C/OpenMP oracle
timed on the host cores) on the small uniform channel, its silence on ranks
other than 0, and the algorithmic byte counts the roofline divides by."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BENCH = os.path.join(ROOT, "bench.py")


def _run(extra_env=None):
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        env.pop(k, None)
    env.update(extra_env or {})
    return subprocess.run([sys.executable, BENCH, "--impl", "reference", "--config", "c1", "--steps", "1",
                           "--warmup", "0"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)


def test_reference_arm_prints_one_contract_line():
    r = _run()
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference"
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["higher_is_better"] is True
    assert d["config"]["workload"] == "c1-128x128x64-uniform"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["unit"] == d["unit"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_is_silent_on_other_ranks():
    r = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""


def test_algorithmic_bytes_of_the_stages():
    sys.path.insert(0, ROOT)
    try:
        import bench
    finally:
        sys.path.remove(ROOT)
    nx, ny, nz = 512, 384, 256
    N, K = nx * ny * nz, (nx // 2 + 1) * ny * nz
    ab = bench.alg_bytes(nx, ny, nz)
    # recip reads rho, writes 1/rho; the correction reads u*, psi, psi^n,
    # psi^(n-1), 1/rho and writes u (10 doubles per cell)
    assert ab["recip"] == pytest.approx(16.0 * N)
    assert ab["correct"] == pytest.approx(80.0 * N)
    # each spectral pass reads and writes the half spectrum once
    for k in ("fftz_fwd", "tridiag", "fftz_inv"):
        assert ab[k] == pytest.approx(32.0 * K)
