"""The strong-scaling survey entry (sharding.migrate_sharded) on the GPU: with one rank it migrates
the whole survey through a Plan and must match the FP64 oracle within the compact-path bar
(relative L2 1e-5); the multi-rank decomposition itself is covered on gloo ranks in
tests/test_sharding.py."""
import numpy as np
import pytest

from imaging2d_wlsq_b200 import sharding, synthetic
from oracle import oracle
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def test_migrate_sharded_single_rank_matches_oracle():
    w = synthetic.batched_uneven(scale=0.08)
    img, mine, wave, shot = sharding.migrate_sharded(w)
    np.testing.assert_array_equal(mine, np.arange(w.ns))
    stack, _, wo, so = oracle.migrate_workload_f64(w)
    assert rel_l2(img.cpu().numpy(), stack) <= 1e-5
    assert rel_l2(wave.cpu().numpy(), wo) <= 1e-5 and rel_l2(shot.cpu().numpy(), so) <= 1e-5
