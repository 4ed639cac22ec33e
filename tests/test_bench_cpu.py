"""CPU: the benchmark's command-line contract.  The reference arm times the
reference's own CPU solver (compiled from its sources into the oracle's
build folder) and prints one JSON line; our arm needs a GPU and is covered
by the GPU runs."""
import json
import os
import subprocess
import sys

import pytest

from conftest import REPO

BENCH = os.path.join(REPO, "bench.py")


def _run(*args, timeout=600):
    p = subprocess.run([sys.executable, BENCH, *args], capture_output=True, text=True,
                       timeout=timeout, cwd=REPO)
    return p


def test_help_lists_the_contract_options():
    p = _run("--help", timeout=120)
    assert p.returncode == 0
    for opt in ("--gpus", "--steps", "--warmup", "--impl", "--cdist"):
        assert opt in p.stdout


@pytest.mark.skipif(not os.path.exists(os.path.join(REPO, "oracle", "_ref",
                                                    "libref_fused.so")),
                    reason="reference not compiled here")
def test_reference_arm_prints_one_json_line():
    p = _run("--impl", "reference", "--steps", "1", "--warmup", "3")
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    j = json.loads(lines[0])
    assert j["impl"] == "reference"
    assert j["value"] > 0 and j["unit"] == "pairs/s"
    assert j["higher_is_better"] is True and j["steps"] == 1 and j["warmup"] == 3
    assert j["cpu_baseline"]["kind"] in ("reference", "port")
    assert j["cpu_baseline"]["cores"] >= 1
    assert j["cpu_baseline"]["value"] == j["value"]
    assert j["e2e"]["h2d_bytes_per_step"] == 0 and j["e2e"]["d2h_bytes_per_step"] == 0
    assert j["config"]["workload"]
