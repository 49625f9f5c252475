"""Sharded ensembles on the GPU: contexts over trajectory ranges [0, B) and [B, 2B)
(dq_set_trajectory_offset) sum to one context of 2B trajectories, on both paths; reduced sums
installed with dq_set_observable_sums drive the getters and writers; and the NCCL all-reduce of
ShardedEnsemble on a one-rank group."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

B, T, PE = 8, 10, 5


def _prop(n_traj, precision, offset=None, ipr=True):
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(20, 10)
    p = dq.Propagator(s.n, m=14, n_traj=n_traj, dt=2.0, noise=dq.NOISE_OU, sigma_static=60.0, seed=19,
                      dot=dq.DOT_HERMITIAN, pop_every=PE, max_steps=T, precision=precision)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, 150.0), np.full(s.n, 40.0))
    p.set_initial_state(s.bright_state())
    if ipr:
        p.set_ipr(True)
    if offset is not None:
        p.set_trajectory_offset(offset)
    return p


@pytest.mark.parametrize("precision", [0, 1])
def test_two_shards_equal_one_ensemble(precision, tmp_path):
    whole = _prop(2 * B, precision)
    whole.run(T)
    a, b = _prop(B, precision, 0), _prop(B, precision, B)
    a.run(T)
    b.run(T)
    sa, sb = a.observable_sums(with_ipr=True), b.observable_sums(with_ipr=True)
    pops, corr, ipr = (sa[0] + sb[0], sa[1] + sb[1], sa[2] + sb[2])
    tol = 1e-12
    assert np.abs(pops / (2 * B) - whole.populations()).max() < tol
    assert np.abs(corr / (2 * B) - whole.correlation()).max() < tol
    assert np.allclose(ipr / (2 * B), whole.ipr(), rtol=1e-12)
    # installing the reduced sums: getters and files report the whole ensemble
    a.set_observable_sums(pops, corr, ipr, 2 * B)
    assert np.abs(a.populations() - whole.populations()).max() < tol
    assert np.allclose(a.ipr(), whole.ipr(), rtol=1e-12)
    a.write_populations(tmp_path / "pops.dat")
    assert open(tmp_path / "pops.dat").readline().split() == ["numsims", str(2 * B)]
    import dynaquant_b200 as dq
    with pytest.raises(dq.DQError):
        a.run(1)                  # reduced sums: reset before stepping on
    # the per-trajectory path keys its draws the same way
    c = _prop(B, 0, B)
    c.run_plain(T)
    if precision == 0:
        assert np.abs(c.populations() - b.populations()).max() < 1e-10
    for p in (whole, a, b, c):
        p.close()


def test_sharded_ensemble_nccl_single_rank():
    import torch.distributed as dist

    from dynaquant_b200.ensemble import ShardedEnsemble
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        ens = ShardedEnsemble(lambda n: _prop(n, 1), B)
        ens.run(T)
        before = ens.engine.populations()
        ens.reduce()
        assert np.abs(ens.engine.populations() - before).max() == 0.0
        ens.engine.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("precision,tol", [(0, 1e-9), (1, 1e-5)])
def test_sharded_adjoint_equals_whole_ensemble(precision, tol):
    """Two shards of 8 trajectories (forward_shard, summed correlation, forward_reduced, summed
    gradients) give the loss and gradient of one context of 16 trajectories."""
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    N, T, LEN = 48, 10, 16
    s = systems.chain(N, -300.0)
    rng = np.random.default_rng(2)
    eps0 = rng.normal(0.0, 80.0, N)
    x = np.arange(N)
    psi0 = np.exp(-((x - N / 2) ** 2) / 30.0 + 0.4j * x)
    psi0 /= np.linalg.norm(psi0)
    target = rng.normal(0.0, 0.05, LEN)

    def make(B, offset=None):
        p = dq.Propagator(N, m=12, n_traj=B, dt=2.0, noise=dq.NOISE_OU, seed=23, dot=dq.DOT_HERMITIAN,
                          precision=precision, max_steps=T)
        p.set_system(s)
        p.set_noise_params(np.full(N, 60.0), np.full(N, 80.0))
        p.set_static_energies(eps0)
        p.set_initial_state(psi0)
        if offset is not None:
            p.set_trajectory_offset(offset)
        p.adjoint_setup(T, LEN, 1.0 / LEN, target, checkpoint_every=4)
        return p

    whole = make(16)
    loss_w = whole.forward()
    gs_w, gc_w = whole.backward()
    shards = [make(8, 0), make(8, 8)]
    corr = sum(p.forward_shard() for p in shards)
    losses = [p.forward_reduced(corr, 16) for p in shards]
    grads = [p.backward() for p in shards]
    gs = grads[0][0] + grads[1][0]
    gc = grads[0][1] + grads[1][1]
    assert losses[0] == losses[1]
    assert losses[0] == pytest.approx(loss_w, rel=tol)
    assert np.abs(gs - gs_w).max() <= tol * np.abs(gs_w).max()
    assert gc[0] == pytest.approx(gc_w[0], rel=tol)
    for p in [whole] + shards:
        p.close()
