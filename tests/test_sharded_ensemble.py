"""An ensemble sharded over ranks (dynaquant_b200.ensemble): world-size-2 gloo ranks on the CPU,
each running its shard of trajectories through the oracle, all-reduce their observable sums; the
result equals one run of the whole ensemble (same Philox keys by global trajectory index)."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

B, T, PE = 4, 6, 2


def _system(oracle):
    from dynaquant_b200 import systems
    s = systems.chain(24, -200.0)
    rp, col, val, d = s.off_diagonal()
    S = oracle.System(rp, col, val, d, m=10, dt=2.0, dot_mode=1, noise=oracle.NOISE_OU, sigma=120.0, tau=50.0,
                      sigma_static=40.0, seed=11)
    psi0 = np.zeros(s.n, complex)
    psi0[s.n // 2] = 1.0
    return S, psi0


class OracleEngine:
    """The engine interface of ShardedEnsemble over the oracle's ensemble run."""
    ipr_enabled = True

    def __init__(self, S, psi0, n_traj):
        self.S, self.psi0, self.n_traj, self.t0 = S, psi0, n_traj, 0
        self.sums = None
        self.installed = None

    def set_trajectory_offset(self, t0):
        self.t0 = t0

    def run(self, n_steps):
        r = self.S.run(self.n_traj, n_steps, self.psi0, pop_every=PE, traj0=self.t0, threads=1)
        self.sums = (r["pops"] * self.n_traj, r["corr"] * self.n_traj, r["ipr"] * self.n_traj)

    def observable_sums(self, with_ipr=False):
        p, c, i = self.sums
        return p.copy(), c.copy(), (i.copy() if with_ipr else None)

    def set_observable_sums(self, pops, corr, ipr, n_traj_total):
        self.installed = (pops / n_traj_total, corr / n_traj_total, ipr / n_traj_total, n_traj_total)


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist

    from dynaquant_b200.ensemble import ShardedEnsemble
    from oracle import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        S, psi0 = _system(oracle)
        ens = ShardedEnsemble(lambda n: OracleEngine(S, psi0, n), B)
        assert ens.engine.t0 == rank * B and ens.n_traj_total == world * B
        ens.run(T)
        ens.reduce()
        p, c, i, tot = ens.engine.installed
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), pops=p, corr=c, ipr=i, total=tot)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_reproduce_one_ensemble(oracle, tmp_path):
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs)
    S, psi0 = _system(oracle)
    ref = S.run(world * B, T, psi0, pop_every=PE, threads=1)
    for r in range(world):
        got = np.load(tmp_path / f"rank{r}.npz")
        assert int(got["total"]) == world * B
        assert np.abs(got["pops"] - ref["pops"]).max() < 1e-14
        assert np.abs(got["corr"] - ref["corr"]).max() < 1e-14
        assert np.allclose(got["ipr"], ref["ipr"], rtol=1e-14)


def test_shard_ranges_cover_the_ensemble():
    from dynaquant_b200.ensemble import shard_range
    ranges = [shard_range(r, 6) for r in range(4)]
    assert ranges[0] == (0, 6) and ranges[-1] == (18, 24)
    assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))


class FakeGradEngine:
    """forward_shard / forward_reduced / backward of a made-up loss, to check the collective steps."""
    ipr_enabled = False

    def __init__(self, rank):
        self.rank = rank
        self.seen = None

    def set_trajectory_offset(self, t0):
        self.t0 = t0

    def forward_shard(self):
        return np.array([1.0 + self.rank, 2.0j * (self.rank + 1)])

    def forward_reduced(self, corr, n_total):
        self.seen = (corr.copy(), n_total)
        return float(abs(corr[0]) / n_total)

    def backward(self):
        return np.full(3, 10.0 ** self.rank), np.array([self.rank + 0.5])


def _grad_worker(rank, world, port, out_dir):
    import torch.distributed as dist

    from dynaquant_b200.ensemble import sharded_gradient
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        e = FakeGradEngine(rank)
        loss, gs, gc = sharded_gradient(e, 2 * world)
        np.savez(os.path.join(out_dir, f"g{rank}.npz"), loss=loss, gs=gs, gc=gc, corr=e.seen[0], n=e.seen[1])
    finally:
        dist.destroy_process_group()


def test_sharded_gradient_collectives(tmp_path):
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_grad_worker, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs)
    for r in range(world):
        g = np.load(tmp_path / f"g{r}.npz")
        assert np.allclose(g["corr"], [3.0, 6.0j])        # summed over both ranks
        assert int(g["n"]) == 4
        assert float(g["loss"]) == pytest.approx(0.75)
        assert np.allclose(g["gs"], 11.0) and np.allclose(g["gc"], [2.0])
