"""bench.py's reference arm on the CPU: the upstream PLAPACK (oracle/_ref)
timed on the host cores, one JSON line with the contract's keys.

The arm runs PLA_General_solve of the compiled reference on a bounded sample
of the C3 matrix family and scales it to the stated n by n^3; under torchrun
only rank 0 works and prints.  A small n keeps the sample to a second or two.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libplapack_ref_openblas.so")


def run_bench(*args, env=None):
    e = dict(os.environ, OPENBLAS_NUM_THREADS="4")
    if env:
        e.update(env)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], env=e,
                       capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stdout + r.stderr
    return [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="oracle/_ref not built")
def test_reference_arm_prints_one_contract_line():
    lines = run_bench("--impl", "reference", "--n", "2048", "--steps", "1", "--warmup", "0",
                      "--cpu-seconds", "1")
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["unit"] == "s" and d["higher_is_better"] is False
    assert d["metric"].startswith("n=32768 solve time")
    assert d["value"] > 0 and d["ms_per_step"] == pytest.approx(d["value"] * 1e3)
    assert d["steps"] == 1 and d["n_gpus"] == 1 and d["config"]["n"] == 2048
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] == 4
    assert "upstream PLA_General_solve" in cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    assert run_bench("--impl", "reference", "--n", "2048", env={"RANK": "1"}) == []
