"""Multi-GPU decomposition: shots are independent through all depth steps and the stacked image
is a plain sum over shots, so ranks own disjoint shot sets and exchange only the image.

  assign_shots     longest-processing-time assignment of shots to ranks by cost (aperture width)
  sub_workload     the slice of a synthetic.Workload a rank migrates
  sum_images       one all-reduce of the stacked image partials (NCCL on GPUs, gloo on CPUs)
  migrate_sharded  one survey migrated over all ranks (strong scaling): each rank migrates its
                   LPT share of the shots and the partial images are summed in float64

One process per GPU (torch.distributed); no collective sits inside the depth loop.
"""
import numpy as np


def assign_shots(costs, world):
    """Greedy LPT: shots sorted by decreasing cost, each to the least loaded rank.
    Returns a list of index arrays (sorted) per rank; deterministic for equal costs."""
    costs = np.asarray(costs, dtype=np.int64)
    order = np.lexsort((np.arange(len(costs)), -costs))
    load = np.zeros(world, dtype=np.int64)
    owned = [[] for _ in range(world)]
    for s in order:
        r = int(np.argmin(load))
        owned[r].append(int(s))
        load[r] += costs[s]
    return [np.array(sorted(o), dtype=np.int64) for o in owned]


def sub_workload(w, shots):
    """Workload restricted to `shots` (packed spectra re-packed in that order)."""
    from .synthetic import Workload
    shots = np.asarray(shots, dtype=np.int64)
    sub = Workload(w.name, w.nz, w.nx, w.dx, w.dz, w.nf, w.M, w.nk, w.dk, w.omega, w.velocity, w.table,
                   w.shot_x0[shots], w.shot_nx[shots], w.shot_pos[shots], nextrap=w.nextrap, seed=w.seed)
    if len(shots):
        sub.wave = np.concatenate([w.block(w.wave, int(s)).reshape(-1) for s in shots])
        sub.shot = np.concatenate([w.block(w.shot, int(s)).reshape(-1) for s in shots])
    else:
        sub.wave = np.zeros(0, dtype=np.complex64)
        sub.shot = np.zeros(0, dtype=np.complex64)
    return sub


def sum_images(image, group=None):
    """In-place sum of the stacked image over all ranks (torch tensor)."""
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(image, group=group)
    return image


def sum_images_f64(image, group=None):
    """Sum of float32 image partials over all ranks, reduced in float64 (one all-reduce of
    nz * nx doubles) and rounded once to float32: the cross-rank sum adds no FP32 rounding of
    its own.  Returns a new float32 tensor on the image's device."""
    import torch
    import torch.distributed as dist
    acc = image.to(torch.float64)
    if dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(acc, group=group)
    return acc.to(torch.float32)


def _migrate_on_device(sub, device, plan_kw):
    """Migrate workload `sub` on `device` through a Plan; returns (image, wave, shot) tensors."""
    import torch
    from . import migration
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    plan = migration.Plan.for_workload(sub, **plan_kw)
    try:
        plan.set_model(torch.from_numpy(np.ascontiguousarray(sub.omega)).to(dev),
                       torch.from_numpy(np.ascontiguousarray(sub.velocity)).to(dev), sub.dk,
                       torch.from_numpy(np.ascontiguousarray(sub.table)).to(dev))
        wave = torch.from_numpy(sub.wave).to(dev)
        shot = torch.from_numpy(sub.shot).to(dev)
        image = torch.zeros((sub.nz, sub.nx), dtype=torch.float32, device=dev)
        plan.execute(wave, shot, image)
        torch.cuda.synchronize(dev)
    finally:
        plan.close()
    return image, wave, shot


def migrate_sharded(w, group=None, device=None, migrate_fn=None, **plan_kw):
    """Strong scaling of one survey: the shots of Workload-like `w` (fields of
    synthetic.Workload: geometry, omega, velocity, table, shot_x0/shot_nx, packed wave/shot) are
    split over the ranks of `group` by aperture width (assign_shots), each rank migrates its share
    on its GPU (one Plan, all its shots x frequencies in one persistent launch), and the partial
    images are summed in float64 (sum_images_f64).  The stacked image, as the reference forms it
    by summing shot images on the host (main.py:184-186), is returned on every rank.

    Returns (image (nz, nx) float32 tensor, identical on all ranks; this rank's shot indices;
    this rank's final source and receiver wavefields, packed in the order of those indices).
    migrate_fn(sub) -> (image, wave, shot) replaces the GPU migration of a rank's share (tests
    run the same decomposition with a CPU migration on gloo ranks).  A rank without shots
    contributes a zero image."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    mine = assign_shots(w.shot_nx, world)[rank]
    sub = sub_workload(w, mine)
    if len(mine):
        image, wave, shot = (migrate_fn or (lambda s: _migrate_on_device(s, device, plan_kw)))(sub)
    else:
        dev = device if device is not None else ("cuda" if migrate_fn is None else "cpu")
        image = torch.zeros((w.nz, w.nx), dtype=torch.float32, device=dev)
        wave = shot = torch.zeros(0, dtype=torch.complex64, device=dev)
    return sum_images_f64(image, group), mine, wave, shot
