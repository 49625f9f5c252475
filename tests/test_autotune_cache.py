"""The autotuner's JSON cache: round trip, and stores from several processes
at once (one per rank on a node) leave a readable file."""
import json
import multiprocessing as mp
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from dynaquant_b200 import autotune  # noqa: E402


def _writer(path, tag, n):
    os.environ["DQ_TUNE_CACHE"] = path
    for i in range(n):
        autotune.store(f"{tag}|{i}", {"traj_chunk": 64, "vec": 2, "ctas_per_sm": 1, "rows_per_block": 3,
                                      "staged": 5, "groups": 1, "ms_per_iter": 0.1 + i})


def test_store_then_load(tmp_path, monkeypatch):
    path = str(tmp_path / "sub" / "tiling.json")
    monkeypatch.setenv("DQ_TUNE_CACHE", path)
    assert autotune.load_cache() == {}
    _writer(path, "a", 3)
    d = autotune.load_cache()
    assert sorted(d) == ["a|0", "a|1", "a|2"] and d["a|2"]["ms_per_iter"] == 2.1


def test_concurrent_stores_leave_valid_json(tmp_path):
    path = str(tmp_path / "tiling.json")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_writer, args=(path, f"r{r}", 40)) for r in range(4)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    with open(path) as f:
        d = json.load(f)
    assert len(d) >= 40   # the last writer's keys at least; racing read-modify-writes may drop others
    assert not [n for n in os.listdir(tmp_path) if n.endswith(".tmp")]
