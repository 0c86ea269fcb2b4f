"""The wide cluster kernel (8 lane slots x 1024 positions per CTA, clusters of half the size of the
cluster2 kernel's, each item's window split evenly over its CTAs) against the FP64 oracle
(relative L2 1e-5, the compact-path bar), in both its packed (FFMA2) and scalar FMA forms, with
and without the step-ahead stage, with its operator-pair ring filled by 16-byte cp.async or by 1-D
bulk copies, and bit for bit against the cluster2 kernel's final wavefields (the same FMA sequence
per element)."""
import numpy as np
import pytest

from imaging2d_wlsq_b200 import migration, operators, synthetic
from oracle import oracle
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

ARITH = [dict(wide=True), dict(wide_scalar=True), dict(wide_bulk=True)]
IDS = ["ffma2", "ffma", "bulk"]


def _with_M(w, M):
    w.M = M
    w.table = operators.design_compact_table(w.nx, w.dx, w.dz, M, w.nk, w.dk)
    return w


CASES = {
    "uneven_L35": lambda: synthetic.batched_uneven(scale=0.12),
    "medium_L31": lambda: synthetic.plain_medium(scale=0.125),
    "precision_L55": lambda: synthetic.precision(scale=0.05),
    "small_L25": lambda: synthetic.plain_small(scale=0.5),
    "uneven_L7": lambda: _with_M(synthetic.batched_uneven(nx=700, nz=10, nf=3, ns=40), 3),
    "uneven_L81": lambda: _with_M(synthetic.batched_uneven(nx=700, nz=10, nf=3, ns=40), 40),
    # windows wider than one cluster of 2: K = 3 (2600 positions) and K = 5 (4500 positions)
    "wide_K3": lambda: synthetic.batched_uneven(nx=2600, nz=6, nf=2, ns=24),
    "wide_K5": lambda: synthetic.plain_medium(nx=4500, nz=5, nf=2, ns=6),
}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("arith", ARITH, ids=IDS)
def test_wide_matches_fp64_oracle(case, arith):
    w = CASES[case]()
    d = migration.Plan.for_workload(w, **arith).describe()
    assert d["kernel"] == "migrate_wide" and d["G"] == 8, d
    img, _, wave, shot = migration.migrate_workload(w, **arith)
    stack, _, wo, so = oracle.migrate_workload_f64(w)
    assert rel_l2(img, stack) <= 1e-5
    assert rel_l2(wave, wo) <= 1e-5 and rel_l2(shot, so) <= 1e-5
    assert np.all(img[w.nextrap:] == 0)


@pytest.mark.parametrize("arith", ARITH, ids=IDS)
def test_wide_wavefields_bitwise_equal_cluster2(arith):
    w = synthetic.batched_uneven(scale=0.1)
    assert migration.Plan.for_workload(w, cluster2=True).describe()["kernel"] == "migrate_cluster2"
    _, _, wave_c, shot_c = migration.migrate_workload(w, cluster2=True)
    _, _, wave_w, shot_w = migration.migrate_workload(w, **arith)
    np.testing.assert_array_equal(wave_w, wave_c)
    np.testing.assert_array_equal(shot_w, shot_c)


def test_wide_per_shot_images():
    w = synthetic.batched_uneven(scale=0.08)
    img, imgs, wave, shot = migration.migrate_workload(w, image_shots=True, wide=True)
    _, shots_o, _, _ = oracle.migrate_workload_f64(w)
    assert rel_l2(imgs, shots_o) <= 1e-5
    for s in range(w.ns):
        x0, n = int(w.shot_x0[s]), int(w.shot_nx[s])
        assert np.all(imgs[s, :, :x0] == 0) and np.all(imgs[s, :, x0 + n:] == 0)
    assert rel_l2(imgs.sum(axis=0), img) <= 1e-6


def test_wide_device_plan_repeat_and_rows_beyond_nextrap():
    import torch
    w = synthetic.batched_uneven(scale=0.08)
    w.nextrap = w.nz - 3
    dev = torch.device("cuda")
    plan = migration.Plan.for_workload(w, wide=True)
    plan.set_model(torch.from_numpy(w.omega).to(dev), torch.from_numpy(np.ascontiguousarray(w.velocity)).to(dev),
                   w.dk, torch.from_numpy(w.table).to(dev))
    stack, _, wo, _ = oracle.migrate_workload_f64(w)
    for _ in range(2):
        wave = torch.from_numpy(w.wave.copy()).to(dev)
        shot = torch.from_numpy(w.shot.copy()).to(dev)
        img = torch.full((w.nz, w.nx), 5.0, dtype=torch.float32, device=dev)
        plan.execute(wave, shot, img)
        torch.cuda.synchronize()
        got = img.cpu().numpy()
        assert rel_l2(got[:w.nextrap], stack[:w.nextrap]) <= 1e-5
        assert np.all(got[w.nextrap:] == 5.0)
        assert rel_l2(wave.cpu().numpy(), wo) <= 1e-5
    plan.close()


def test_default_kernel_choice():
    """The wide kernel is the default where the 16-slot cluster kernel's clusters of 4 would leave
    SMs idle (2048-wide windows); the 16-slot kernel where its clusters fill the GPU."""
    w = synthetic.batched_uneven(nz=6, nf=2)
    assert migration.Plan.for_workload(w).describe()["kernel"] == "migrate_wide"
    w = synthetic.plain_medium(nz=6, nf=2)  # 32 full-aperture shots over 1024 positions: clusters of 2
    assert migration.Plan.for_workload(w).describe()["kernel"] == "migrate_cluster2"


def test_wide_bulk_plan_and_status():
    """The bulk-copy ring is a variant of the wide kernel (variant bit 4, with and without the
    stage), its launches report a clean status word, it gives the same wavefields as the cp.async
    ring, and it rejects the scalar-FMA flag."""
    import torch
    from imaging2d_wlsq_b200._lib import LibraryError
    w = synthetic.batched_uneven(scale=0.08)
    d = migration.Plan.for_workload(w, wide_bulk=True).describe()
    assert d["kernel"] == "migrate_wide" and d["variant"] == 7, d  # packed FMAs + stage + bulk
    w81 = CASES["uneven_L81"]()
    assert migration.Plan.for_workload(w81, wide_bulk=True).describe()["variant"] == 5  # no stage
    with pytest.raises(LibraryError):
        migration.Plan.for_workload(w, wide_bulk=True, wide_scalar=True)
    dev = torch.device("cuda")
    out = []
    for kw in (dict(wide=True), dict(wide_bulk=True)):
        plan = migration.Plan.for_workload(w, **kw)
        plan.set_model(torch.from_numpy(w.omega).to(dev),
                       torch.from_numpy(np.ascontiguousarray(w.velocity)).to(dev), w.dk,
                       torch.from_numpy(w.table).to(dev))
        wave = torch.from_numpy(w.wave.copy()).to(dev)
        shot = torch.from_numpy(w.shot.copy()).to(dev)
        img = torch.zeros((w.nz, w.nx), dtype=torch.float32, device=dev)
        plan.execute(wave, shot, img)
        plan.check_status()
        out.append((wave.cpu().numpy(), shot.cpu().numpy(), img.cpu().numpy()))
        plan.close()
    np.testing.assert_array_equal(out[1][0], out[0][0])
    np.testing.assert_array_equal(out[1][1], out[0][1])
    assert rel_l2(out[1][2], out[0][2]) <= 1e-6


def _narrow_shots(nx=2048, ns=48, nz=8, nf=3, seed=9):
    """Shots of 64-1024 traces on a 2048-wide model: the line packing chains them into 2048-wide
    items (clusters of 2), the window packing can use clusters of 1."""
    rng = np.random.default_rng(seed)
    v = synthetic.gaussian_random_field(nz, nx, 5.0, 1500.0, 4500.0, rng)
    width = rng.integers(64, 1025, ns).astype(np.int32)
    x0 = np.clip(rng.integers(0, nx, ns) - width // 2, 0, nx - width).astype(np.int32)
    pos = (x0 + width // 2).astype(np.int32)
    w = synthetic.Workload("narrow_shots", nz, nx, 10.0, 10.0, nf, 17, 256, 0.0, None, v, None, x0, width, pos,
                           nextrap=nz, seed=seed)
    return synthetic._finish(w, 2.0, 50.0, 20.0, rng, True)


@pytest.mark.parametrize("case", ["uneven", "narrow"])
def test_window_packing_matches_line_packing_and_oracle(case):
    """The window-first packing (the wide kernel's default where its modelled cost is lower) against
    the line packing: bit-identical wavefields (the per-point FMA sequence does not depend on the
    packing), images within 1e-6 of each other and 1e-5 of the FP64 oracle, and a lower modelled
    cost."""
    # modelled costs (window against line packing): 3.28 against 3.45, and 5.15 against 6.00
    w = synthetic.batched_uneven(seed=4, scale=0.25, nz=40, nf=16) if case == "uneven" else _narrow_shots()
    d_win = migration.Plan.for_workload(w, wide=True).describe()
    d_lin = migration.Plan.for_workload(w, wide=True, line_packing=True).describe()
    assert d_lin["packing"] == "lines"
    assert d_win["packing"] == "windows", d_win
    assert d_win["cost_units"] < d_lin["cost_units"]
    assert d_win["computed_per_useful"] < d_lin["computed_per_useful"]
    if case == "narrow":
        # windows of up to 2048 positions chain more of these shots per slot than clusters of 1
        assert d_win["cluster"] == 2 and d_lin["cluster"] == 2, (d_win, d_lin)
    img_w, _, wave_w, shot_w = migration.migrate_workload(w, wide=True)
    img_l, _, wave_l, shot_l = migration.migrate_workload(w, wide=True, line_packing=True)
    np.testing.assert_array_equal(wave_w, wave_l)
    np.testing.assert_array_equal(shot_w, shot_l)
    assert rel_l2(img_w, img_l) <= 1e-6
    stack, _, wo, so = oracle.migrate_workload_f64(w)
    assert rel_l2(img_w, stack) <= 1e-5
    assert rel_l2(wave_w, wo) <= 1e-5 and rel_l2(shot_w, so) <= 1e-5
