"""Multi-GPU layout on the CPU: the batch partition, the balanced assignment of uneven
batches, and the host-side reductions, run as world_size-2 ``gloo`` process groups.

Each rank integrates and differentiates its own shard with the oracle (the CUDA kernels
need a GPU); per-trajectory results must equal the full-batch results bit for bit, since
trajectories are independent and sharding only changes which process computes which row.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from gradsolve_b200.sharding import balanced_assignment, contiguous_slices


def test_contiguous_slices_partition():
    for n in (0, 1, 7, 64, 1000):
        for world in (1, 2, 3, 8):
            s = contiguous_slices(n, world)
            assert len(s) == world
            assert s[0][0] == 0 and s[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(s, s[1:]))
            sizes = [b - a for a, b in s]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        contiguous_slices(4, 0)


def test_balanced_assignment_partition_and_spread():
    rng = np.random.default_rng(5)
    # per-trajectory attempt counts of a mixed-horizon batch: heavy-tailed
    cost = np.exp(rng.uniform(np.log(4), np.log(8000), 10000)).round()
    for world in (1, 2, 4, 8):
        parts = balanced_assignment(cost, world)
        allidx = np.concatenate(parts)
        assert np.array_equal(np.sort(allidx), np.arange(cost.size))
        sums = np.array([cost[p].sum() for p in parts])
        assert sums.max() - sums.min() <= cost.max()
        for p in parts:
            assert np.all(np.diff(p) > 0)
    # contiguous slicing of the same costs is far less even
    sl = contiguous_slices(cost.size, 8)
    sorted_cost = np.sort(cost)
    sums = np.array([sorted_cost[a:b].sum() for a, b in sl])
    assert sums.max() - sums.min() > cost.max()
    with pytest.raises(ValueError):
        balanced_assignment([1.0, -1.0], 2)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _inputs(n):
    rng = np.random.default_rng(11)
    y0 = np.array([1.0, 0.0, 0.0]) + rng.normal(0.0, 0.1, (n, 3))
    rho = rng.uniform(20.0, 30.0, (n, 1))
    return y0, rho


def _rank_main(rank, world, port, n, mode, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    from oracle import oracle as O

    from gradsolve_b200.sharding import (balanced_assignment, contiguous_slices, global_sum,
                                         max_over_ranks)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        y0, rho = _inputs(n)
        if mode == "contiguous":
            a, b = contiguous_slices(n, world)[rank]
            idx = np.arange(a, b)
        else:
            # pilot: attempt counts of a loose-tolerance forward solve on every rank
            pilot = O.record("tsit5", "lorenz", y0, rho, 0.0, 1.0, 1e-5, 1e-5, cap=4096)
            cost = pilot["n_acc"] + pilot["n_rej"]
            idx = balanced_assignment(cost, world)[rank]
        r = O.record("tsit5", "lorenz", y0[idx], rho[idx], 0.0, 1.0, 1e-8, 1e-8, cap=4096)
        # loss = mean over the WHOLE ensemble of y_final^2: each rank's cotangent uses the
        # global count, and the loss value is a sum over ranks
        ybar = 2.0 * r["y_final"] / (n * 3)
        gy0, gp = O.replay_vjp("tsit5", "lorenz", y0[idx], rho[idx], r["dts"], ybar)
        loss = global_sum(float((r["y_final"] ** 2).sum()) / (n * 3))
        tmax = max_over_ranks(float(rank + 1))
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), idx=idx, gp=gp, gy0=gy0,
                 yf=r["y_final"], n_acc=r["n_acc"], loss=float(loss.item()), tmax=tmax)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("mode", ["contiguous", "balanced"])
def test_gloo_sharded_gradients_equal_full_batch(tmp_path, mode):
    from oracle import oracle as O
    O.build()
    n, world = 48, 2
    mp.start_processes(_rank_main, args=(world, _free_port(), n, mode, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    y0, rho = _inputs(n)
    r = O.record("tsit5", "lorenz", y0, rho, 0.0, 1.0, 1e-8, 1e-8, cap=4096)
    ybar = 2.0 * r["y_final"] / (n * 3)
    gy0, gp = O.replay_vjp("tsit5", "lorenz", y0, rho, r["dts"], ybar)
    seen = np.zeros(n, bool)
    for k in range(world):
        z = np.load(tmp_path / f"rank{k}.npz")
        idx = z["idx"]
        assert not seen[idx].any()
        seen[idx] = True
        np.testing.assert_array_equal(z["yf"], r["y_final"][idx])
        np.testing.assert_array_equal(z["n_acc"], r["n_acc"][idx])
        np.testing.assert_array_equal(z["gp"], gp[idx])
        np.testing.assert_array_equal(z["gy0"], gy0[idx])
        full = float((r["y_final"] ** 2).mean())
        assert abs(float(z["loss"]) - full) <= 1e-14 * full  # summation order differs
        assert float(z["tmax"]) == float(world)
    assert seen.all()
