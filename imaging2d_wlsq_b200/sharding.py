"""Multi-GPU decomposition: shots are independent through all depth steps and the stacked image
is a plain sum over shots, so ranks own disjoint shot sets and exchange only the image.

  assign_shots   longest-processing-time assignment of shots to ranks by cost (aperture width)
  sub_workload   the slice of a synthetic.Workload a rank migrates
  sum_images     one all-reduce of the stacked image partials (NCCL on GPUs, gloo on CPUs)

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
