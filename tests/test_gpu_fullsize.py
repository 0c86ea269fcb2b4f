"""Size-independent properties of the migration at the benchmark's full size (the 256-shot
uneven-aperture survey: nz=1000, nx=2048, 512 frequencies, 35 taps, 1.29e11 points), where the FP64
checker would take hours: the image is linear in the receiver spectra, and the image of all shots is
the sum of the images of any split of the shots (each half packed into its own lane slots).
Tolerance 1e-5 relative L2, the bar of the parity tests."""
import numpy as np
import pytest

from imaging2d_wlsq_b200 import migration, sharding, synthetic
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def _migrate(w, shot):
    img, _ = migration.migrate(w.ns, w.nextrap, w.nz, w.nx, w.nf, w.nt, w.M, w.nk, w.dk, w.omega, w.velocity,
                               w.table, w.wave.copy(), np.ascontiguousarray(shot, dtype=np.complex64).copy(),
                               shot_x0=w.shot_x0, shot_nx=w.shot_nx)
    return img


def test_full_size_linearity_and_shot_additivity():
    w = synthetic.batched_uneven()
    assert w.points() > 1e11
    rng = np.random.default_rng(21)
    d2 = (rng.standard_normal(w.shot.shape, dtype=np.float32)
          + 1j * rng.standard_normal(w.shot.shape, dtype=np.float32)).astype(np.complex64)
    img1 = _migrate(w, w.shot)
    img2 = _migrate(w, d2)
    img12 = _migrate(w, w.shot + np.float32(2.0) * d2)
    assert rel_l2(img12, img1.astype(np.float64) + 2.0 * img2) <= 1e-5
    halves = [np.arange(0, w.ns, 2), np.arange(1, w.ns, 2)]
    total = np.zeros_like(img1, dtype=np.float64)
    for idx in halves:
        sub = sharding.sub_workload(w, idx)
        total += _migrate(sub, sub.shot)
    assert rel_l2(total, img1) <= 1e-5
