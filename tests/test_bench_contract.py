"""bench.py's reference arm on the CPU: the upstream PLAPACK (oracle/_ref)
timed on the host cores, one JSON line with the contract's keys.

The arm runs PLA_General_solve of the compiled reference on the n x n system
of the C3 matrix family itself (no sampling, no scaling); under torchrun only
rank 0 works and prints.  A small n keeps the solve to a second or two.
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
    lines = run_bench("--impl", "reference", "--n", "2048", "--steps", "5", "--warmup", "2")
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["unit"] == "s" and d["higher_is_better"] is False
    assert d["metric"].startswith("n=32768 solve time")
    assert d["value"] > 0 and d["ms_per_step"] == pytest.approx(d["value"] * 1e3)
    # one timed solve at the stated n whatever --steps asked, reported as such
    assert d["steps"] == 1 and d["steps_requested"] == 5 and d["warmup"] == 1
    assert d["n_gpus"] == 1 and d["config"]["n"] == 2048
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] == 4
    assert "upstream PLA_LU" in cb["sample"] and "n=2048" in cb["sample"]
    assert "scaled" not in cb["sample"]
    assert cb["backward_error"] < 2048 * 2.0 ** -53
    assert d["e2e"] == {"value": d["value"], "unit": "s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    assert run_bench("--impl", "reference", "--n", "2048", env={"RANK": "1"}) == []
