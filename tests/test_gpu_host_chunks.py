"""img2d_migrate_compact on large wavefields (64 MiB and more): the call splits the frequencies into
chunks whose host copies overlap the other chunks' kernels, on two alternating kernel streams with
two sets of image partials.  Checked against the device-resident plan (one launch over all items)
and the FP64 oracle, from pageable (numpy) and from pinned host memory."""
import numpy as np
import pytest

from imaging2d_wlsq_b200 import migration, synthetic
from oracle import oracle
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def _device_plan_result(w):
    import torch
    dev = torch.device("cuda")
    plan = migration.Plan.for_workload(w)
    plan.set_model(torch.from_numpy(w.omega).to(dev), torch.from_numpy(np.ascontiguousarray(w.velocity)).to(dev),
                   w.dk, torch.from_numpy(w.table).to(dev))
    wave = torch.from_numpy(w.wave.copy()).to(dev)
    shot = torch.from_numpy(w.shot.copy()).to(dev)
    img = torch.zeros((w.nz, w.nx), dtype=torch.float32, device=dev)
    plan.execute(wave, shot, img)
    plan.check_status()
    out = img.cpu().numpy(), wave.cpu().numpy(), shot.cpu().numpy()
    plan.close()
    return out


@pytest.mark.parametrize("pinned", [False, True], ids=["pageable", "pinned"])
def test_chunked_host_entry_matches_device_plan_and_oracle(pinned):
    import torch
    w = synthetic.batched_uneven(nz=6, nf=40)  # 2 x 81 MB of spectra: 8 chunks of 5 frequencies
    assert w.wave.nbytes >= 64 << 20
    img_d, wave_d, shot_d = _device_plan_result(w)
    if pinned:
        wave = torch.from_numpy(w.wave.copy()).pin_memory().numpy()
        shot = torch.from_numpy(w.shot.copy()).pin_memory().numpy()
    else:
        wave, shot = w.wave.copy(), w.shot.copy()
    img, _ = migration.migrate(w.ns, w.nextrap, w.nz, w.nx, w.nf, w.nt, w.M, w.nk, w.dk, w.omega, w.velocity,
                               w.table, wave, shot, shot_x0=w.shot_x0, shot_nx=w.shot_nx)
    # the per-position arithmetic does not depend on the launch split: identical wavefields
    np.testing.assert_array_equal(wave, wave_d)
    np.testing.assert_array_equal(shot, shot_d)
    assert rel_l2(img, img_d) <= 1e-6
    stack, _, wo, so = oracle.migrate_workload_f64(w)
    assert rel_l2(img, stack) <= 1e-5
    assert rel_l2(wave, wo) <= 1e-5 and rel_l2(shot, so) <= 1e-5
    # a second call on the cached plan and buffers gives the same result
    wave2, shot2 = w.wave.copy(), w.shot.copy()
    img2, _ = migration.migrate(w.ns, w.nextrap, w.nz, w.nx, w.nf, w.nt, w.M, w.nk, w.dk, w.omega, w.velocity,
                                w.table, wave2, shot2, shot_x0=w.shot_x0, shot_nx=w.shot_nx)
    np.testing.assert_array_equal(wave2, wave)
    assert rel_l2(img2, img) <= 1e-6


def test_chunked_host_entry_after_a_geometry_change():
    """A second geometry replaces the cached plan; the chunked call must rebuild its item lists for
    the new plan's groups, even where the new plan reuses the old one's memory."""
    from imaging2d_wlsq_b200 import sharding
    w = synthetic.batched_uneven(nz=6, nf=40)
    for idx in (np.arange(0, w.ns), np.arange(0, w.ns, 2), np.arange(1, w.ns, 2)):
        sub = sharding.sub_workload(w, idx)
        if sub.wave.nbytes < 64 << 20:
            sub = sharding.sub_workload(synthetic.batched_uneven(nz=6, nf=80), idx)
        assert sub.wave.nbytes >= 64 << 20
        img_d, wave_d, _ = _device_plan_result(sub)
        wave, shot = sub.wave.copy(), sub.shot.copy()
        img, _ = migration.migrate(sub.ns, sub.nextrap, sub.nz, sub.nx, sub.nf, sub.nt, sub.M, sub.nk, sub.dk,
                                   sub.omega, sub.velocity, sub.table, wave, shot, shot_x0=sub.shot_x0,
                                   shot_nx=sub.shot_nx)
        np.testing.assert_array_equal(wave, wave_d)
        assert rel_l2(img, img_d) <= 1e-6


def test_chunked_host_entry_with_more_rows_than_frequencies():
    """Packed spectra of nt > nf rows per shot (the reference's layout: only the first nf rows are
    extrapolated): the chunked call moves only those rows, leaves the others untouched, and gives
    the result of the tight layout."""
    w = synthetic.batched_uneven(nz=6, nf=40)
    nt = w.nf + 3
    img_ref, wave_ref, shot_ref = _device_plan_result(w)

    def pad(a, fill):
        out = []
        for s in range(w.ns):
            blk = w.block(a, s)
            extra = np.full((nt - w.nf, blk.shape[1]), fill, dtype=np.complex64)
            out.append(np.concatenate([blk, extra]).reshape(-1))
        return np.concatenate(out)

    wave = pad(w.wave, 7 + 7j)
    shot = pad(w.shot, -3 + 1j)
    assert wave.nbytes >= 64 << 20
    img, _ = migration.migrate(w.ns, w.nextrap, w.nz, w.nx, w.nf, nt, w.M, w.nk, w.dk, w.omega, w.velocity,
                               w.table, wave, shot, shot_x0=w.shot_x0, shot_nx=w.shot_nx)
    off = 0
    ref_off = 0
    for s in range(w.ns):
        n = int(w.shot_nx[s])
        blk_w = wave[off:off + nt * n].reshape(nt, n)
        blk_s = shot[off:off + nt * n].reshape(nt, n)
        np.testing.assert_array_equal(blk_w[:w.nf].reshape(-1), wave_ref[ref_off:ref_off + w.nf * n])
        np.testing.assert_array_equal(blk_s[:w.nf].reshape(-1), shot_ref[ref_off:ref_off + w.nf * n])
        assert np.all(blk_w[w.nf:] == np.complex64(7 + 7j)) and np.all(blk_s[w.nf:] == np.complex64(-3 + 1j))
        off += nt * n
        ref_off += w.nf * n
    assert rel_l2(img, img_ref) <= 1e-6
