"""
The benchmark's output contract, checked without a GPU: the reference arm
(`bench.py --impl reference`, the reference's own CPU kernels) prints one
JSON line with the keys the contract names, the same `config` block that the
GPU arm prints for the same grid, and a zero-copy `e2e`; the config's L2
note follows the state size.
"""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_config_l2_note_follows_the_state_size():
    big = bench.bench_config(4096, "exact")
    small = bench.bench_config(1024, "exact")
    assert big["zones"] == 4096 ** 2 and big["parallelism"] == "single"
    assert "exceed" in big["l2"] and "403 MB" in big["l2"]
    assert "fit in L2" in small["l2"]
    assert big["workload"].startswith("cbdiso_2d circumbinary disk 4096x4096 FP64 RK2")


@pytest.mark.skipif(not os.path.isdir(os.path.join(ROOT, "oracle")), reason="oracle sources absent")
def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--size", "256", "--steps", "2",
                          "--warmup", "1"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference"
    assert line["metric"] == "zone-updates/s" and line["unit"] == "zone-updates/s"
    assert line["higher_is_better"] is True and line["value"] > 0
    assert line["steps"] == 2 and line["n_gpus"] == 1
    assert line["config"] == bench.bench_config(256, "exact")
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["cores"] >= 1 and cb["kind"] in ("reference", "port") and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
