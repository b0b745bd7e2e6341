"""The N>1 host path (one replica per GPU) on CPU: two gloo ranks exercise the
max-over-ranks timing reduction, the round-robin split of the differentiable
check's finite-difference directions and the gather that reassembles them."""
import os
import socket
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from simcraft_b200.replicas import Replicas, fd_check, fd_directions  # noqa: E402

SHAPE = (3, 4, 5, 6)
COUNT = 7
EPS = 1e-3


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _quadratic(scale_bug=1.0):
    """L(U) = 0.5 sum a U^2 + sum b U at a fixed U; its adjoint is a U + b.
    scale_bug != 1 plants a wrong adjoint (on the CPU) for the check to catch."""
    rng = np.random.default_rng(1)
    a, b, U = rng.uniform(0.5, 2.0, SHAPE), rng.standard_normal(SHAPE), rng.standard_normal(SHAPE)
    g = scale_bug * (a * U + b)

    def loss_at(d, sign):
        V = U + sign * EPS * d
        return float(0.5 * (a * V * V).sum() + (b * V).sum())

    def grad_dot(d):
        return float((g * d).sum())

    return loss_at, grad_dot


def _worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rep = Replicas(rank, world, dist, "cpu")
        res = {"max": rep.max(10.0 * rank + 1.0), "shard": rep.shard(COUNT),
               "gather": rep.gather({"rank": rank})}
        loss_at, grad_dot = _quadratic()
        res["errs"] = fd_check(loss_at, grad_dot, SHAPE, COUNT, 8, EPS, rep)
        loss_at, grad_dot = _quadratic(scale_bug=1.01)
        res["errs_bug"] = fd_check(loss_at, grad_dot, SHAPE, COUNT, 8, EPS, rep)
        rep.barrier()
        np.save(os.path.join(out_dir, f"r{rank}.npy"), np.array([res], dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


def test_replicas_two_gloo_ranks():
    world = 2
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(world, _free_port(), d), nprocs=world, join=True,
                           start_method="spawn")
        res = [np.load(os.path.join(d, f"r{r}.npy"), allow_pickle=True)[0] for r in range(world)]
    # the slowest replica's time on every rank
    assert all(r["max"] == 11.0 for r in res)
    # round robin: disjoint shares that cover every direction once
    assert res[0]["shard"] == [0, 2, 4, 6] and res[1]["shard"] == [1, 3, 5]
    assert all(r["gather"] == [{"rank": 0}, {"rank": 1}] for r in res)
    # the gathered check equals the single-process one, direction by direction
    loss_at, grad_dot = _quadratic()
    local = fd_check(loss_at, grad_dot, SHAPE, COUNT, 8, EPS)
    for r in res:
        assert r["errs"] == local
        assert max(r["errs"]) < 1e-8  # central differences are exact on a quadratic
        assert min(r["errs_bug"]) > 5e-3  # a 1% adjoint error is seen along every direction


def test_replicas_single_process():
    rep = Replicas()
    assert not rep.active and rep.max(3.5) == 3.5 and rep.shard(3) == [0, 1, 2]
    assert rep.gather("x") == ["x"] and rep.unshard(3, [[7, 8, 9]]) == [7, 8, 9]
    a = fd_directions((2, 3), 4, 8)
    b = fd_directions((2, 3), 4, 8)
    assert all((x == y).all() for x, y in zip(a, b))
