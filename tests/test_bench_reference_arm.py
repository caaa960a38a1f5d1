"""bench.py --impl reference without a GPU: the reference kernels compiled from their own
source, timed on the host cores, print one JSON line with the same metric as the GPU arm;
under torchrun only rank 0 works and prints."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT


def _run(env_extra, mode="disparity"):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config", "small",
                           "--mode", mode, "--steps", "1", "--warmup", "0"], capture_output=True, text=True, env=env,
                          cwd=ROOT, timeout=600)


@pytest.mark.parametrize("mode,metric", [("disparity", "Mpixel·iterations/s"), ("depth", "Mpixel·iterations/s"),
                                         ("vpm", "Mpixel·iterations/s"), ("svpm", "Mpixel·passes/s")])
def test_reference_arm_prints_one_contract_line(orc, mode, metric):
    p = _run({}, mode)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    if "unavailable" in d:   # the compiled reference is missing on this host
        assert d["impl"] == "reference"
        return
    assert d["impl"] == "reference"
    assert d["metric"] == metric and d["unit"] == d["metric"] and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 0 and d["n_gpus"] == 1
    assert d["config"]["workload"] == "small"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] >= 1 and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_exit_without_work(orc):
    p = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert p.returncode == 0, p.stderr[-2000:]
    assert not [l for l in p.stdout.splitlines() if l.startswith("{")]
