"""The parts of bench.py that run without a GPU: the byte model behind the
roofline, the ncu traffic it reads from the committed summaries, and the
reference arm's JSON line (the FP64 oracle on the host cores)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from dynaquant_b200 import systems  # noqa: E402


def test_spmm_bytes_counts_slabs_and_csr_once():
    s = systems.tube(6, 10, cutoff=25.0)
    B = 32
    nnz_off = s.nnz - s.n
    assert nnz_off > 0
    # q_j (8 B) + diagonal (4 B) read, w (8 B) written per site-trajectory; CSR values, columns, row pointers
    assert bench.spmm_bytes(s, B) == 20.0 * s.n * B + 8.0 * nnz_off + 4.0 * (s.n + 1)


def test_every_named_profile_carries_its_traffic():
    named = {k: v[1] for k, v in bench.SPMM_FORMS.items() if v[1]}
    assert 5 in named, "the autotuner's choice on the tube has a committed summary"
    for staged, name in named.items():
        assert os.path.exists(os.path.join(ROOT, "profiles", name)), name
        traffic, src = bench.measured_traffic(staged)
        assert traffic is not None and traffic > 0, name
        assert src == "profiles/" + name
    assert bench.measured_traffic(2) == (None, None)


def test_blk_profile_traffic_matches_its_byte_model():
    # the L1 form's captured launch (j = 4) reads q_{j-1} too: 28 B per site-trajectory plus the CSR
    s = bench.build_system()
    B = bench.WORKLOAD["B"]
    alg = bench.spmm_bytes(s, B) + 8.0 * s.n * B
    traffic, _ = bench.measured_traffic(5)
    assert abs(traffic / alg - 1.0) < 0.05


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["metric"] == bench.METRIC and d["unit"] == "traj-steps/s" and d["higher_is_better"] is True
    assert d["config"]["workload"] == bench.WORKLOAD["name"]
    assert np.isfinite(d["value"]) and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "traj-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_contexts_are_made_on_the_ranks_device(monkeypatch):
    # under torchrun every rank's contexts must land on its LOCAL_RANK device, not on device 0
    import dynaquant_b200 as dq

    made = []

    class FakePropagator:
        def __init__(self, *a, **kw):
            made.append(kw)

        def __getattr__(self, name):
            return lambda *a, **kw: None

    monkeypatch.setattr(dq, "Propagator", FakePropagator)
    monkeypatch.setattr(bench, "DEVICE", 3)
    s = systems.tube(6, 10, cutoff=25.0)
    bench.make_prop(s, 2, dq.PREC_MIXED, 1, max_steps=8)
    assert made and made[-1]["device"] == 3
