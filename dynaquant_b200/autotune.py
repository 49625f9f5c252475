"""Tiling autotuner for the ensemble kernels, with a JSON cache.

dq_autotune (C ABI) times one Lanczos iteration (shared-CSR SpMM + axpy)
under every valid (trajectory chunk, vector width, CTAs per SM) and keeps the
fastest.  This module keys the winner by GPU model and problem shape (sites,
couplings, trajectories, precision) in a JSON file, so later contexts for
the same size class reuse it without re-timing.

Cache file: $DQ_TUNE_CACHE, else ~/.cache/dynaquant_b200/tiling.json.
"""
from __future__ import annotations

import json
import os


def cache_path() -> str:
    return os.environ.get("DQ_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "dynaquant_b200", "tiling.json"))


def _gpu_name(device: int) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:
        return "unknown-gpu"


def key(prop, nnz: int) -> str:
    c = prop.cfg
    # size class: sites and couplings rounded to 2 significant digits
    def sig2(x):
        if x <= 0:
            return 0
        e = len(str(int(x))) - 2
        return int(round(x / 10 ** max(e, 0))) * 10 ** max(e, 0)
    return (f"{_gpu_name(c.device)}|n~{sig2(c.n_sites)}|nnz~{sig2(nnz)}|B={c.n_traj}|"
            f"prec={c.precision}|dot={c.dot_mode}")


def load_cache() -> dict:
    p = cache_path()
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return {}


def store(k: str, entry: dict) -> None:
    p = cache_path()
    d = load_cache()
    d[k] = entry
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        tmp = f"{p}.{os.getpid()}.tmp"   # one per process: ranks of one node may store at once
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, p)
    except OSError:
        pass


def tune(prop, nnz: int, reps: int = 5, use_cache: bool = True) -> dict:
    """Chooses the tiling for `prop` (a dynaquant_b200.Propagator with its
    system set); returns {"traj_chunk", "vec", "ctas_per_sm", "rows_per_block",
    "ms_per_iter", "cached"}.  The ensemble is reset afterwards."""
    k = key(prop, nnz)
    if use_cache:
        e = load_cache().get(k)
        if e:
            try:
                prop.set_tiling(e["traj_chunk"], e["vec"], e["ctas_per_sm"], e["rows_per_block"], e["staged"],
                                e["groups"])
                prop.reset()
                return dict(e, cached=True)
            except Exception:
                pass
    ms = prop.autotune_raw(reps)
    tc, vec, cps, rpb, staged, groups = prop.get_tiling()
    entry = {"traj_chunk": tc, "vec": vec, "ctas_per_sm": cps, "rows_per_block": rpb, "staged": staged,
             "groups": groups, "ms_per_iter": ms}
    store(k, entry)
    return dict(entry, cached=False)
