"""Ensembles sharded over processes, one GPU per process.

The reference runs its numEnsembleRuns trajectories one after another on one
GPU and sums their observables (propagate.cu:167-298, popPrintClass.cu:160-522).
Trajectories are independent, so here rank r of a world of W runs trajectories
[r B, (r+1) B) of one ensemble of W B: dq_set_trajectory_offset keys every
random draw by the global trajectory index, so the union of the shards is
exactly the ensemble one context of W B trajectories would run.  Stepping
needs no exchange; at the end one all-reduce (torch.distributed: NCCL on GPUs,
gloo on CPU) sums the observable records (populations, correlation, IPR) and
installs them in every rank's context, whose getters and file writers then
report the whole ensemble.

The spectrum-loss gradient shards the same way (sharded_gradient): every rank
runs its trajectories forward, one all-reduce sums the correlation, each rank
computes the loss of the whole ensemble's mean and back-propagates through
its own trajectories, and a second all-reduce sums the gradients.

An engine is any object with set_trajectory_offset, run, observable_sums,
set_observable_sums and ipr_enabled (Propagator has them); sharded_gradient
also needs forward_shard, forward_reduced and backward.
"""
from __future__ import annotations

import numpy as np


def _dist():
    import torch.distributed as dist
    return dist


def shard_range(rank: int, n_traj_per_rank: int) -> tuple[int, int]:
    """Global trajectory indices [first, last) of a rank's shard."""
    return rank * n_traj_per_rank, (rank + 1) * n_traj_per_rank


def _allreduce(arr, group=None):
    """Sum of a float64 numpy array over the group's ranks (NCCL on the rank's GPU, or gloo)."""
    import torch
    dist = _dist()
    backend = dist.get_backend(group)
    device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float64)).to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def sharded_gradient(engine, n_traj_total: int, group=None):
    """Loss of the whole ensemble and this rank's share summed into the full gradient:
    (loss, grad_sites, grad_classes), identical on every rank."""
    corr = engine.forward_shard()
    corr_all = _allreduce(corr.view(np.float64), group).view(np.complex128)
    loss = engine.forward_reduced(corr_all, n_traj_total)
    gs, gc = engine.backward()
    flat = _allreduce(np.concatenate([gs, gc]), group)
    return loss, flat[:len(gs)], flat[len(gs):]


def allreduce_observables(engine, n_traj_total: int, group=None) -> None:
    """Sums the engine's observable records over the group's ranks (one all-reduce of one
    flat FP64 buffer) and installs the result as standing for n_traj_total trajectories."""
    import torch
    dist = _dist()
    pops, corr, ipr = engine.observable_sums(with_ipr=engine.ipr_enabled)
    parts = [pops.ravel(), corr.view(np.float64)] + ([ipr] if ipr is not None else [])
    flat = np.concatenate(parts)
    backend = dist.get_backend(group)
    device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.from_numpy(flat).to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    flat = t.cpu().numpy()
    k = pops.size
    pops = flat[:k].reshape(pops.shape)
    corr_r = flat[k:k + 2 * corr.size].copy().view(np.complex128)
    ipr_r = flat[k + 2 * corr.size:] if ipr is not None else None
    engine.set_observable_sums(pops, corr_r, ipr_r, n_traj_total)


class ShardedEnsemble:
    """One engine per rank over the rank's shard of the ensemble.

    make_engine(n_traj) builds the rank's engine (e.g. a configured Propagator on
    this rank's GPU); n_traj_per_rank must be even when the world has more than one
    rank (the random draws come in trajectory pairs)."""

    def __init__(self, make_engine, n_traj_per_rank: int, group=None):
        dist = _dist()
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        if self.world > 1 and n_traj_per_rank % 2:
            raise ValueError("n_traj_per_rank must be even on more than one rank")
        self.n_traj_per_rank = n_traj_per_rank
        self.n_traj_total = n_traj_per_rank * self.world
        self.engine = make_engine(n_traj_per_rank)
        self.engine.set_trajectory_offset(shard_range(self.rank, n_traj_per_rank)[0])

    def run(self, n_steps: int) -> None:
        """Advances the rank's shard; no collective."""
        self.engine.run(n_steps)

    def reduce(self) -> None:
        """Sums the observables over all ranks (every rank takes part)."""
        allreduce_observables(self.engine, self.n_traj_total, self.group)
