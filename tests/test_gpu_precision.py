"""Precision study of the operator-table storage modes (FP32 arithmetic, Kahan imaging; table
stored as complex64, FP16 or BF16) against the FP64 CPU oracle.

The FP32 table must meet the 1e-5 relative-L2 bar.  The 16-bit tables are measured and reported;
whether they are accepted is decided by the same bar (precision.study marks `accepted`).
"""
import json
import os

import numpy as np
import pytest

from imaging2d_wlsq_b200 import precision, synthetic
from oracle import oracle

pytestmark = pytest.mark.gpu


def _fp64(w):
    stack, _, _, _ = oracle.migrate_workload_f64(w)
    return stack


def _report(name, res):
    print(f"\nprecision study {name}: " + json.dumps(res))
    out = os.environ.get("IMG2D_PRECISION_OUT")
    if out:
        with open(out, "a") as f:
            f.write(json.dumps({"case": name, "result": res}) + "\n")


def test_precision_modes_small():
    w = synthetic.precision(nx=1024, nextrap=60, nf=8, ns=16)
    res = precision.study(w, _fp64)
    _report("small", res)
    assert res["fp32"]["accepted"], res
    for m in ("fp16", "bf16"):
        assert np.isfinite(res[m]["rel_l2"]) and res[m]["table"] == m
        assert res[m]["rel_l2"] > res["fp32"]["rel_l2"]


def test_precision_study_subvolume():
    """The precision configuration's grid (nx=4096, dx=dz=5 m, 55 taps, nk=8000, thin layers)
    on a 200-depth-step sub-volume with all 64 full-aperture shots and 64 frequencies spread over
    2-60 Hz (3.4e9 points; the FP64 oracle takes a few minutes of host time)."""
    w = synthetic.precision(nextrap=200, nf=64, ns=64)
    res = precision.study(w, _fp64)
    _report("subvolume_200", res)
    assert res["fp32"]["accepted"], res
