"""Multi-rank decomposition on CPU: two gloo ranks each migrate their shot share with the CPU
oracle, sum the images with one all-reduce, and must reproduce the single-process image."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from imaging2d_wlsq_b200 import sharding, synthetic
from oracle import oracle


def test_assign_shots_balances_and_partitions():
    rng = np.random.default_rng(0)
    costs = rng.integers(256, 2049, 256)
    parts = sharding.assign_shots(costs, 4)
    allp = np.sort(np.concatenate(parts))
    np.testing.assert_array_equal(allp, np.arange(256))
    loads = [costs[p].sum() for p in parts]
    assert max(loads) / min(loads) < 1.02
    assert [len(p) for p in sharding.assign_shots([5, 5, 5], 5)].count(0) == 2


def test_sub_workload_repacks():
    w = synthetic.batched_uneven(scale=0.05)
    sub = sharding.sub_workload(w, [3, 1])
    np.testing.assert_array_equal(sub.block(sub.wave, 0), w.block(w.wave, 3))
    np.testing.assert_array_equal(sub.block(sub.shot, 1), w.block(w.shot, 1))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    w = synthetic.batched_uneven(scale=0.05)
    mine = sharding.assign_shots(w.shot_nx, world)[rank]
    sub = sharding.sub_workload(w, mine)
    stack, _, _, _ = oracle.migrate_workload_f64(sub)
    img = torch.from_numpy(stack.copy())
    sharding.sum_images(img)
    if rank == 0:
        q.put(img.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_reproduce_single_process_image():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    w = synthetic.batched_uneven(scale=0.05)
    ref, _, _, _ = oracle.migrate_workload_f64(w)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12


def _oracle_migrate(sub):
    """A rank's share migrated by the FP64 CPU oracle (stands in for the GPU plan on gloo ranks)."""
    stack, _, wo, so = oracle.migrate_workload_f64(sub)
    return (torch.from_numpy(stack.astype(np.float32)), torch.from_numpy(wo.astype(np.complex64)),
            torch.from_numpy(so.astype(np.complex64)))


def _sharded_rank(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    w = synthetic.batched_uneven(scale=0.05)
    img, mine, wave, shot = sharding.migrate_sharded(w, migrate_fn=_oracle_migrate)
    q.put((rank, img.numpy(), mine, wave.numpy(), shot.numpy()))
    dist.barrier()
    dist.destroy_process_group()


def test_migrate_sharded_two_gloo_ranks_strong_scaling():
    """One survey over two ranks through sharding.migrate_sharded: the shots are partitioned, every
    rank gets the same stacked image (float64 cross-rank sum), equal to the single-process image,
    and each rank's final wavefields are those of its own shots."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got.sort(key=lambda g: g[0])
    w = synthetic.batched_uneven(scale=0.05)
    ref, _, wo, so = oracle.migrate_workload_f64(w)
    np.testing.assert_array_equal(got[0][1], got[1][1])
    assert np.linalg.norm(got[0][1] - ref) / np.linalg.norm(ref) < 1e-6
    owned = np.sort(np.concatenate([g[2] for g in got]))
    np.testing.assert_array_equal(owned, np.arange(w.ns))
    off = w.offsets()
    for _, _, mine, wave, shot in got:
        exp_w = np.concatenate([wo[off[s]:off[s] + w.nf * w.shot_nx[s]] for s in mine])
        exp_s = np.concatenate([so[off[s]:off[s] + w.nf * w.shot_nx[s]] for s in mine])
        assert np.abs(wave - exp_w).max() <= 1e-6 * np.abs(exp_w).max()
        assert np.abs(shot - exp_s).max() <= 1e-6 * np.abs(exp_s).max()
