"""Precision study of the operator-table storage modes.

The migration computes in FP32 with Kahan-compensated imaging.  The operator table may be stored as
complex64 (default) or as FP16 / BF16 (re, im) pairs.  This module runs each storage mode on the
GPU and compares the image with an FP64 CPU image of the same sub-volume.  A reduced-precision mode
is acceptable only if its relative-L2 image error stays within the tolerance the FP32 path meets
(1e-5).

The FP64 image is computed by a caller-supplied function (`reference(w)` returning the stacked
float64 image), so that this module does not depend on the checker.
"""
import numpy as np

from . import migration

TOLERANCE = 1e-5


def run_mode(w, table):
    import torch
    dev = torch.device("cuda")
    plan = migration.Plan.for_workload(w, table=table)
    plan.set_model(torch.from_numpy(w.omega).to(dev), torch.from_numpy(np.ascontiguousarray(w.velocity)).to(dev),
                   w.dk, torch.from_numpy(w.table).to(dev))
    wave = torch.from_numpy(w.wave.copy()).to(dev)
    shot = torch.from_numpy(w.shot.copy()).to(dev)
    img = torch.zeros((w.nz, w.nx), dtype=torch.float32, device=dev)
    plan.execute(wave, shot, img)
    torch.cuda.synchronize()
    d = plan.describe()
    plan.close()
    return img.cpu().numpy()[:w.nextrap].astype(np.float64), d


def study(w, reference, modes=("fp32", "fp16", "bf16")):
    """Image errors of each table storage mode against the FP64 image `reference(w)`."""
    ref = np.asarray(reference(w), dtype=np.float64)[:w.nextrap]
    scale = np.abs(ref).max()
    out = {}
    for m in modes:
        img, d = run_mode(w, m)
        rel = float(np.linalg.norm(img - ref) / np.linalg.norm(ref))
        out[m] = {"rel_l2": rel, "max_abs_rel": float(np.abs(img - ref).max() / scale),
                  "accepted": rel <= TOLERANCE, "kernel": d["kernel"], "table": d["table"]}
    return out
