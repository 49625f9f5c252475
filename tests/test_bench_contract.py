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


class _FakeProp:
    """Stands in for dynaquant_b200.Propagator in the bench's control-flow tests (no GPU)."""

    def __init__(self, n, **kw):
        self.n, self.kw, self.stream = n, kw, 0

    def autotune(self):
        return {"traj_chunk": 64, "vec": 2, "ctas_per_sm": 1, "rows_per_block": 3, "staged": 5, "groups": 1,
                "ms_per_iter": 0.15, "cached": True}

    def profile_step(self, n_steps=1):
        from dynaquant_b200 import _lib
        return {k: (0.1, 2 * n_steps) for k in _lib.KIND_NAMES}

    def populations(self):
        return np.zeros((2, self.n))

    def correlation(self):
        return np.zeros(3, dtype=np.complex128)

    def __getattr__(self, name):
        return lambda *a, **kw: None


class _FakeEvent:
    def __init__(self, **kw):
        pass

    def record(self, stream=None):
        pass

    def elapsed_time(self, other):
        return 100.0


def _run_ours(monkeypatch, world, rank=0):
    import torch
    import dynaquant_b200 as dq

    class FakeClocks:
        def __init__(self, dev):
            pass

        def __enter__(self):
            return self

        def __exit__(self, *a):
            return False

        def summary(self):
            return {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 1}

    calls = []
    monkeypatch.setattr(bench, "DEVICE", 0)   # run_ours sets it; restored after the test
    monkeypatch.setattr(dq, "Propagator", _FakeProp)
    monkeypatch.setattr(bench, "Clocks", FakeClocks)
    monkeypatch.setattr(bench, "build_system", lambda: systems.tube(6, 10, cutoff=25.0))
    monkeypatch.setattr(torch.cuda, "set_device", lambda d: calls.append(("set_device", d)))
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a: None)
    monkeypatch.setattr(torch.cuda, "Event", _FakeEvent)
    monkeypatch.setattr(torch.cuda, "ExternalStream", lambda s: None)
    stub = {"stub": True}
    for leg in ("adjoint_leg", "aggregates_leg", "large_leg"):
        monkeypatch.setattr(bench, leg, lambda: stub)
    monkeypatch.setattr(bench, "zz_leg", lambda s, t: stub)
    monkeypatch.setattr(bench, "cpu_baseline_sample", lambda s, c: (800.0, "sample"))
    if world > 1:
        import torch.distributed as td
        monkeypatch.setattr(td, "barrier", lambda *a, **kw: calls.append(("barrier",)))
        monkeypatch.setattr(td, "all_reduce", lambda t, op=None, **kw: calls.append(("all_reduce",)))
        monkeypatch.setattr(torch, "tensor", lambda v, device=None: type("T", (), {"item": lambda self: v[0]})())
        import dynaquant_b200.ensemble as ens
        monkeypatch.setattr(ens, "allreduce_observables", lambda p, n, group=None: calls.append(("obs", n)))

    class Args:
        steps, warmup, gpus, impl = 10, 3, world, "ours"

    bench.run_ours(Args, rank, world, rank)
    return calls


def test_run_ours_line_at_one_gpu(monkeypatch, capsys):
    _run_ours(monkeypatch, 1)
    lines = [l for l in capsys.readouterr().out.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "e2e", "gpu_launches", "roofline", "cpu_baseline",
              "clocks", "plain_fp64", "adjoint", "zz_noise"):
        assert k in d, k
    assert d["n_gpus"] == 1 and d["steps"] == 10 and d["warmup"] == 3
    assert d["value"] == pytest.approx(bench.WORKLOAD["B"] * 10 / 0.1)   # 100 ms for 10 steps
    assert d["roofline"]["unit"] == "GB/s" and 0 < d["roofline"]["frac"]
    assert set(d["e2e"]) >= {"value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step"}
    assert d["cpu_baseline"]["kind"] == "port"


def test_run_ours_on_rank0_of_two_skips_the_n1_legs(monkeypatch, capsys):
    calls = _run_ours(monkeypatch, 2, rank=0)
    d = json.loads([l for l in capsys.readouterr().out.splitlines() if l.startswith("{")][0])
    assert d["n_gpus"] == 2 and "cpu_baseline" not in d and "adjoint" not in d
    assert d["value"] == pytest.approx(2 * bench.WORKLOAD["B"] * 10 / 0.1)
    assert ("obs", 2 * bench.WORKLOAD["B"]) in calls
    # every rank takes the same collective steps: barrier, max of the timed region, barrier, e2e max
    assert [c[0] for c in calls if c[0] in ("barrier", "all_reduce")] == ["barrier", "all_reduce", "barrier",
                                                                          "all_reduce"]


def test_run_ours_on_rank1_prints_nothing(monkeypatch, capsys):
    calls = _run_ours(monkeypatch, 2, rank=1)
    assert ("set_device", 1) in calls and bench.DEVICE == 1
    assert not [l for l in capsys.readouterr().out.splitlines() if l.startswith("{")]
