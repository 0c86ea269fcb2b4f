"""The no-allocation entry point (img2d_migrate_compact_noalloc).

It exists for callers that cannot call cudaMalloc themselves or through the library: a plugin
inside a host application whose own pool owns all device memory, or a processing loop that must
not block on or fail in an allocation mid-run.  Its scratch is one fixed array inside the library.

Checked here through the C ABI: two calls in a row give the same image and wavefields as the
plan entry point (img2d_plan_execute) and as the FP64 CPU oracle, within the compact-path
tolerance (relative L2 1e-5); the second call is not disturbed by what the first left in the
shared scratch; and a problem whose scratch does not fit is refused with a message naming the
limit.  The file is collected last so
that a failure here does not hide the other tests; it also passes run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from imaging2d_wlsq_b200 import _lib, migration, synthetic
from oracle import oracle
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def _noalloc(w, dev, om, vel, tab, wave, shot, image):
    import torch
    x0 = np.ascontiguousarray(w.shot_x0, dtype=np.int32)
    wn = np.ascontiguousarray(w.shot_nx, dtype=np.int32)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    return _lib.lib().img2d_migrate_compact_noalloc(
        w.ns, w.nextrap, w.nz, w.nx, w.nf, w.nt, w.M, w.nk, float(w.dk), om.data_ptr(), vel.data_ptr(),
        tab.data_ptr(), x0.ctypes.data, wn.ctypes.data, wave.data_ptr(), shot.data_ptr(), image.data_ptr(), stream)


@pytest.mark.parametrize("maker,kw", [(synthetic.batched_uneven, dict(scale=0.08)),
                                      (synthetic.plain_small, dict(scale=1.0)),
                                      # 256 items, 0.5 MB image plane: fewer CTAs so their partials fit
                                      (synthetic.plain_medium, dict(nx=1024, nz=120, nf=64, ns=16))])
def test_noalloc_matches_plan_entry_two_calls(maker, kw):
    import torch
    dev = torch.device("cuda", 0)
    w = maker(**kw)
    om = torch.from_numpy(w.omega).to(dev)
    vel = torch.from_numpy(np.ascontiguousarray(w.velocity)).to(dev)
    tab = torch.from_numpy(w.table).to(dev)

    # existing entry point
    plan = migration.Plan.for_workload(w)
    plan.set_model(om, vel, w.dk, tab)
    wave_p = torch.from_numpy(w.wave.copy()).to(dev)
    shot_p = torch.from_numpy(w.shot.copy()).to(dev)
    img_p = torch.zeros((w.nz, w.nx), dtype=torch.float32, device=dev)
    plan.execute(wave_p, shot_p, img_p)
    torch.cuda.synchronize()
    plan.close()

    results = []
    for _ in range(2):
        wave = torch.from_numpy(w.wave.copy()).to(dev)
        shot = torch.from_numpy(w.shot.copy()).to(dev)
        img = torch.full((w.nz, w.nx), 7.0, dtype=torch.float32, device=dev)
        rc = _noalloc(w, dev, om, vel, tab, wave, shot, img)
        assert rc == _lib.IMG2D_OK, _lib.lib().img2d_last_error()
        torch.cuda.synchronize()
        results.append((img.cpu().numpy(), wave.cpu().numpy(), shot.cpu().numpy()))

    ref_img = img_p.cpu().numpy()
    stack64, _, wave64, shot64 = oracle.migrate_workload_f64(w)
    for img, wave, shot in results:
        assert rel_l2(img[:w.nextrap], ref_img[:w.nextrap]) <= 1e-5
        assert rel_l2(wave, wave_p.cpu().numpy()) <= 1e-5
        assert rel_l2(shot, shot_p.cpu().numpy()) <= 1e-5
        # and directly against the FP64 oracle
        assert rel_l2(img[:w.nextrap], stack64[:w.nextrap]) <= 1e-5
        assert rel_l2(wave, wave64) <= 1e-5
        assert rel_l2(shot, shot64) <= 1e-5
        assert np.all(img[w.nextrap:] == 7.0)  # rows below nextrap are not touched
    assert rel_l2(results[1][0], results[0][0]) <= 1e-5


def test_noalloc_rejects_problem_beyond_scratch():
    import torch
    dev = torch.device("cuda", 0)
    # index table alone: 512 frequencies x 1000 depths x 2048 positions x 2 B = 2 GB > 64 MiB
    ns, nextrap, nz, nx, nf, M, nk = 4, 1000, 1000, 2048, 512, 17, 400
    om = torch.ones(nf, dtype=torch.float64, device=dev)
    vel = torch.full((nz, nx), 2000.0, dtype=torch.float64, device=dev)
    tab = torch.zeros((nk, 2 * M + 1), dtype=torch.complex64, device=dev)
    wave = torch.zeros(ns * nf * nx, dtype=torch.complex64, device=dev)
    img = torch.zeros((nz, nx), dtype=torch.float32, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    rc = _lib.lib().img2d_migrate_compact_noalloc(ns, nextrap, nz, nx, nf, nf, M, nk, 1e-3, om.data_ptr(),
                                                   vel.data_ptr(), tab.data_ptr(), None, None, wave.data_ptr(),
                                                   wave.data_ptr(), img.data_ptr(), stream)
    assert rc == _lib.IMG2D_EINVAL
    assert b"MiB of fixed scratch" in _lib.lib().img2d_last_error()
