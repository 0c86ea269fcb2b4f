"""Error paths on the GPU, made on the host: an injected allocation failure (the library refuses an
allocation above a set limit before calling cudaMalloc) reported through the C ABI and through the
void drop-in shim, and the host entry point's per-device cache.  Nothing here faults the GPU."""
import os
import subprocess
import sys

import numpy as np
import pytest

from imaging2d_wlsq_b200 import _lib, migration, synthetic
from imaging2d_wlsq_b200._lib import LibraryError, lib
from oracle import oracle
from tests.conftest import ROOT, rel_l2

pytestmark = pytest.mark.gpu


def _small():
    return synthetic.plain_medium(nx=96, nz=6, nf=3, ns=2)


def test_injected_allocation_failure_is_reported_and_cleared():
    w = _small()
    lib().img2d_release_host_cache()  # buffers kept from earlier calls would need no allocation
    lib().img2d_set_alloc_limit(4096)
    try:
        with pytest.raises(LibraryError, match="allocation limit") as ei:
            migration.migrate_workload(w)
        assert ei.value.code == _lib.IMG2D_ENOMEM
    finally:
        lib().img2d_set_alloc_limit(0)
    # the failed call left nothing half-built behind: the next call runs and is correct
    img, _, _, _ = migration.migrate_workload(w)
    stack, _, _, _ = oracle.migrate_workload_f64(w)
    assert rel_l2(img, stack) <= 1e-5


def test_dropin_shim_aborts_with_the_error_text():
    """The reference ABI returns void: the shim prints the library's error and aborts instead of
    returning unfilled arrays (the allocation limit comes from the environment here)."""
    script = (
        "import ctypes, numpy as np\n"
        "lib = ctypes.CDLL(%r)\n"
        "ns, nz, nx, nf, M = 1, 3, 16, 2, 1\n"
        "op = np.zeros((nz, nf, nx, 2*M+1), np.complex64)\n"
        "wave = np.zeros((ns, nf, nx), np.complex64); shot = wave.copy()\n"
        "img = np.zeros((ns, nz, nx), np.float32)\n"
        "p = lambda a: a.ctypes.data_as(ctypes.c_void_p)\n"
        "lib.extrapolate(ns, nz, nz, nx, nf, nf, M, p(op), p(op), p(wave), p(shot), p(img))\n"
        "print('returned')\n" % os.path.join(_lib.DROPIN_DIR, "extrapolation_cpu.so"))
    env = dict(os.environ, IMG2D_ALLOC_LIMIT_BYTES="64")
    r = subprocess.run([sys.executable, "-c", script], capture_output=True, text=True, env=env, timeout=120,
                       cwd=ROOT)
    assert r.returncode != 0 and "returned" not in r.stdout
    assert "imaging2d_wlsq_b200: extrapolate failed (code 2)" in r.stderr, r.stderr
    assert "allocation limit" in r.stderr


def test_host_cache_is_kept_per_device():
    import torch
    w = _small()
    lib().img2d_release_host_cache()
    assert lib().img2d_host_cache_device_count() == 0
    migration.migrate_workload(w)
    assert lib().img2d_host_cache_device_count() == 1
    # the same device again reuses its entry
    migration.migrate_workload(w)
    assert lib().img2d_host_cache_device_count() == 1
    if torch.cuda.device_count() > 1:
        torch.cuda.set_device(1)
        try:
            img1, _, _, _ = migration.migrate_workload(w)
            assert lib().img2d_host_cache_device_count() == 2
        finally:
            torch.cuda.set_device(0)
        img0, _, _, _ = migration.migrate_workload(w)
        assert rel_l2(img0, img1) <= 1e-6
    lib().img2d_release_host_cache()
    assert lib().img2d_host_cache_device_count() == 0
    assert np.isfinite(migration.migrate_workload(w)[0]).all()
