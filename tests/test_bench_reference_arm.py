"""The reference arm of bench.py on the CPU (`--impl reference`): one JSON
line with the GPU arm's metric, unit, direction and workload, the reference
decoder's own throughput as value, cpu_baseline describing the run and an
e2e block without host-device copies."""
import json
import os
import subprocess
import sys

import pytest

import bench
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not oracle.ref_available("avx2"), reason="reference build missing")
def test_reference_arm_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == "Gbit/s" and line["higher_is_better"] is True
    assert line["steps"] == 1 and line["warmup"] == 1 and line["n_gpus"] == 1
    assert line["value"] > 0
    assert line["config"]["workload"] == "dvbs2-normal-3_5-8psk-awgn-sweep"
    assert line["config"]["frames_per_step"] == 4096
    cpu = line["cpu_baseline"]
    assert cpu["kind"] in ("reference", "port") and cpu["cores"] >= 1 and cpu["value"] == line["value"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
