"""Demigration kernel (the adjoint of the migration), autograd bindings and least-squares migration
on the GPU, checked against the FP64 oracle (whose demigration is pinned to its migration by
test_oracle_adjoint.py).

Tolerances: demigrated data within 1e-5 relative L2 of the FP64 oracle (the FP32 bar of the
migration); dot-product test <F d, m> = Re sum d conj(F* m): the classic ratio
|<F d, m> - <d, F* m>| / |<F d, m>| within 1e-6 on five seeds per case for Gaussian m kept at least
3 norms of F d-projection away from orthogonality (for independent Gaussian vectors the ratio is
the FP32 error, a few 1e-7, divided by |z|, z ~ N(0, 1), and is only held to 2e-5), the same
difference within 1e-7 of ||F d|| ||m|| (the FP64 oracle pair passes at 1e-11); finite differences
of the quadratic misfit within 1e-3 relative.
"""
import numpy as np
import pytest

from imaging2d_wlsq_b200 import lsm, migration, operators, synthetic
from oracle import oracle
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def _with_M(w, M):
    """The same workload with another operator half-length (exercises the runtime-length kernel)."""
    w.M = M
    w.table = operators.design_compact_table(w.nx, w.dx, w.dz, M, w.nk, w.dk)
    return w


CASES = {
    "full_L31": lambda: synthetic.plain_medium(nx=200, nz=14, nf=5, ns=6),
    "uneven_L35": lambda: synthetic.batched_uneven(nx=300, nz=11, nf=4, ns=12),
    "small_L25": lambda: synthetic.plain_small(scale=0.1),
    "runtime_L11": lambda: _with_M(synthetic.plain_medium(nx=90, nz=9, nf=3, ns=3), 5),
    "one_shot_L31": lambda: synthetic.plain_medium(nx=64, nz=6, nf=2, ns=1),
}


def _op(w, slab=0):
    return lsm.MigrationOperator.for_workload(w, slab_depth=slab)


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("slab", [0, 1, 4, 1000])
def test_demigration_matches_oracle(case, slab):
    import torch
    w = CASES[case]()
    rng = np.random.default_rng(11)
    m = rng.standard_normal((w.nextrap, w.nx)).astype(np.float32)
    op = _op(w, slab)
    data = op.demigrate(torch.from_numpy(m).cuda()).cpu().numpy()
    ref = oracle.demigrate_workload_f64(w, m.astype(np.float64))
    assert rel_l2(data, ref) <= 1e-5
    # the source spectra are read only
    assert np.array_equal(op.wave.cpu().numpy(), w.wave)
    d = op.plan.describe_demigration()
    assert d["slabs"] == -(-w.nextrap // min(slab or 8, w.nextrap))
    op.plan.close()


def test_demigration_rows_beyond_nf_untouched():
    import torch
    w = synthetic.plain_medium(nx=64, nz=6, nf=3, ns=2)
    nt = 5
    plan = migration.Plan(w.ns, w.nextrap, w.nz, w.nx, w.nf, nt, w.M, w.nk)
    dev = torch.device("cuda")
    plan.set_model(torch.from_numpy(w.omega).to(dev), torch.from_numpy(np.ascontiguousarray(w.velocity)).to(dev),
                   w.dk, torch.from_numpy(w.table).to(dev))
    wave = np.zeros((w.ns, nt, w.nx), dtype=np.complex64)
    wave[:, :w.nf] = w.wave.reshape(w.ns, w.nf, w.nx)
    data = torch.full((w.ns, nt, w.nx), 3 + 4j, dtype=torch.complex64, device=dev)
    m = np.random.default_rng(2).standard_normal((w.nextrap, w.nx)).astype(np.float32)
    plan.demigrate(torch.from_numpy(m).to(dev), torch.from_numpy(wave).to(dev), data)
    out = data.cpu().numpy()
    assert np.all(out[:, w.nf:] == 3 + 4j)
    ref = oracle.demigrate_workload_f64(w, m.astype(np.float64)).reshape(w.ns, w.nf, w.nx)
    assert rel_l2(out[:, :w.nf], ref) <= 1e-5
    plan.close()


def test_demigration_rejects_bad_arguments():
    import torch
    from imaging2d_wlsq_b200._lib import LibraryError
    w = synthetic.plain_medium(nx=64, nz=6, nf=2, ns=1)
    op = _op(w)
    m = torch.zeros((w.nextrap, w.nx), device="cuda")
    with pytest.raises(LibraryError, match="alias"):
        op.plan.demigrate(m, op.wave, op.wave)
    two = migration.Plan.for_workload(w, two_tables=True)
    with pytest.raises(LibraryError, match="single-table"):
        two.demigrate(m, op.wave, op.zeros_data())
    two.close()
    op.plan.close()


@pytest.mark.parametrize("case", ["full_L31", "uneven_L35", "runtime_L11"])
def test_dot_product(case):
    w = CASES[case]()
    op = _op(w)
    sep, ind = [], []
    for seed in range(5):
        # m with |projection on F d| >= 3 (lsm.dot_product_test): the classic ratio measures the FP32 error
        lhs, rhs, rel, rel_norms = lsm.dot_product_test(op, seed=seed, separation=3.0)
        sep.append(rel)
        assert rel <= 1e-6 and rel_norms <= 1e-7, (seed, lhs, rhs, rel, rel_norms)
        # independent Gaussian m: the same FP32 error over |z|, z ~ N(0, 1)
        lhs, rhs, rel, rel_norms = lsm.dot_product_test(op, seed=seed)
        ind.append(rel)
        assert rel_norms <= 1e-7 and rel <= 2e-5, (seed, lhs, rhs, rel, rel_norms)
    print(f"\ndot product {case}: separated {[f'{r:.2e}' for r in sep]}, independent {[f'{r:.2e}' for r in ind]}")
    op.plan.close()


def test_dot_product_lsm_geometry():
    """The least-squares configuration's geometry (nx=1024, dx=dz=10 m, smooth random velocity, 31
    taps, nk=2000, 2-40 Hz, full-aperture shots) at a reduced size: 100 depth steps, 32 frequencies,
    16 shots.  The classic ratio |<F d, m> - <d, F* m>| / |<F d, m>| within 1e-6 on five seeds, for
    Gaussian d and Gaussian m separated from orthogonality to F d (lsm.dot_product_test,
    separation 3); independent Gaussian pairs within 2e-5 (FP32 error over |z|)."""
    w = synthetic.lsm(nz=100, nf=32, ns=16)
    op = _op(w)
    sep, ind = [], []
    for seed in range(5):
        lhs, rhs, rel, rel_norms = lsm.dot_product_test(op, seed=seed, separation=3.0)
        sep.append(rel)
        assert rel <= 1e-6 and rel_norms <= 1e-8, (seed, lhs, rhs, rel, rel_norms)
        lhs, rhs, rel, rel_norms = lsm.dot_product_test(op, seed=seed)
        ind.append(rel)
        assert rel <= 2e-5 and rel_norms <= 1e-8, (seed, lhs, rhs, rel, rel_norms)
    print(f"\ndot product lsm geometry (nz=100, nf=32, ns=16): separated {[f'{r:.2e}' for r in sep]}, "
          f"independent {[f'{r:.2e}' for r in ind]}")
    op.plan.close()


def test_dot_product_lsm_configuration():
    """The least-squares configuration in full (nz=500, nx=1024, nf=256, 31 taps, 64 shots):
    five seeds with separation 3.  At this size the FP32 difference |<F d, m> - <d, F* m>| reaches
    about 3e-6 of ||F d|| (rel_norms * sqrt(image size)), so the classic ratio of a separated pair
    is held to 2e-6."""
    w = synthetic.lsm()
    op = _op(w)
    rels = []
    for seed in range(5):
        lhs, rhs, rel, rel_norms = lsm.dot_product_test(op, seed=seed, separation=3.0)
        rels.append(rel)
        assert rel <= 2e-6 and rel_norms <= 1e-8, (seed, lhs, rhs, rel, rel_norms)
    print(f"\ndot product lsm configuration: separated {[f'{r:.2e}' for r in rels]}")
    op.plan.close()


def test_autograd_functions_are_the_operator_pair():
    import torch
    w = CASES["full_L31"]()
    op = _op(w)
    g = torch.Generator(device="cuda").manual_seed(3)
    m = torch.randn((w.nextrap, w.nx), device="cuda", generator=g).requires_grad_(True)
    d = lsm.demigrate(m, op)
    gd = torch.randn(d.shape, dtype=torch.complex64, device="cuda", generator=g)
    d.backward(gd)
    # the migration's image sum is split over per-CTA partials in queue order: equal to rounding
    assert rel_l2(m.grad.cpu().numpy(), op.migrate(gd).cpu().numpy()) <= 1e-6
    dd = torch.randn(d.shape, dtype=torch.complex64, device="cuda", generator=g).requires_grad_(True)
    img = lsm.migrate(dd, op)
    gi = torch.randn(img.shape, device="cuda", generator=g)
    img.backward(gi)
    # demigration writes every (shot, frequency) sample from one work item: deterministic
    assert torch.equal(dd.grad, op.demigrate(gi))
    op.plan.close()


def test_finite_differences():
    import torch
    w = synthetic.lsm(scale=0.08, nf=6)
    op = _op(w)
    m_true = torch.from_numpy(w.reflectivity[:w.nextrap]).cuda()
    d_obs = op.demigrate(m_true).clone()
    rng = np.random.default_rng(5)
    m0 = torch.from_numpy((0.5 * w.reflectivity[:w.nextrap]).astype(np.float32)).cuda()
    pts = [(int(rng.integers(0, w.nextrap)), int(rng.integers(0, w.nx))) for _ in range(16)]
    ga, fd = lsm.finite_difference_check(op, m0, d_obs, pts, h=1.0)
    scale = np.abs(ga).max()
    assert np.max(np.abs(ga - fd)) <= 1e-3 * scale, (ga, fd)
    op.plan.close()


def test_least_squares_migration_reduces_residual_and_solvers_agree():
    import torch
    w = synthetic.lsm(scale=0.08, nf=6)
    op = _op(w)
    m_true = torch.from_numpy(w.reflectivity[:w.nextrap]).cuda()
    d_obs = op.demigrate(m_true).clone()
    m_ag, hist_ag = lsm.lsm_cg(op, d_obs, niter=5)
    m_cg, hist_cg = lsm.cgls(op, d_obs, niter=5)
    r_ag = [h[1] for h in hist_ag]
    r_cg = [h[1] for h in hist_cg]
    assert r_ag[-1] < 0.5 * r_ag[0]
    assert all(b <= a * (1 + 1e-6) for a, b in zip(r_cg, r_cg[1:]))
    # CG with exact line search on a quadratic and CGLS produce the same iterates
    assert np.allclose(r_ag, r_cg, rtol=1e-3)
    assert rel_l2(m_ag.cpu().numpy(), m_cg.cpu().numpy()) <= 1e-3
    op.plan.close()


@pytest.mark.parametrize("case", ["uneven_L35", "runtime_L11", "full_L31"])
@pytest.mark.parametrize("slab", [0, 3])
def test_source_checkpoint_modes_agree(case, slab):
    """Recomputed, kept and reused source checkpoints give bit-identical demigrated data (the
    checkpoints are the same arithmetic), and match the FP64 oracle."""
    import torch
    from imaging2d_wlsq_b200._lib import LibraryError
    w = CASES[case]()
    op = _op(w, slab)
    plan = op.plan
    m = torch.from_numpy(np.random.default_rng(4).standard_normal((w.nextrap, w.nx)).astype(np.float32)).cuda()
    outs = {}
    with pytest.raises(LibraryError, match="kept source checkpoints"):
        plan.demigrate(m, op.wave, op.zeros_data(), slab_depth=slab, source="reuse")
    for mode in ("recompute", "keep", "reuse", "reuse"):
        d = op.zeros_data()
        plan.demigrate(m, op.wave, d, slab_depth=slab, source=mode)
        outs.setdefault(mode, []).append(d.cpu().numpy())
    ref = outs["recompute"][0]
    for mode, arrs in outs.items():
        for arr in arrs:
            assert np.array_equal(arr, ref), mode
    assert rel_l2(ref, oracle.demigrate_workload_f64(w, m.cpu().numpy().astype(np.float64))) <= 1e-5
    assert plan.describe_demigration()["source_cache_bytes"] > 0
    # a new model discards the kept checkpoints
    plan.set_model(torch.from_numpy(w.omega).cuda(), torch.from_numpy(np.ascontiguousarray(w.velocity)).cuda(),
                   w.dk, torch.from_numpy(w.table).cuda())
    with pytest.raises(LibraryError, match="kept source checkpoints"):
        plan.demigrate(m, op.wave, op.zeros_data(), slab_depth=slab, source="reuse")
    plan.close()


CLUSTER_CASES = {
    "cluster_full_L31": lambda: synthetic.plain_medium(nx=700, nz=12, nf=4, ns=16),
    "cluster_uneven_L35": lambda: synthetic.batched_uneven(nx=1300, nz=9, nf=3, ns=64),
    "cluster_runtime_L11": lambda: _with_M(synthetic.plain_medium(nx=600, nz=8, nf=3, ns=14), 5),
}


@pytest.mark.parametrize("case", list(CLUSTER_CASES))
@pytest.mark.parametrize("slab", [0, 3])
def test_cluster_demigration_matches_oracle_and_single_cta(case, slab):
    """The cluster demigration kernel (16 slots per item, window split over CTAs with halos in
    distributed shared memory) against the FP64 oracle, and bit for bit against the single-CTA
    kernel (same arithmetic per slot in the same order), in every source-checkpoint mode."""
    import torch
    w = CLUSTER_CASES[case]()
    m = torch.from_numpy(np.random.default_rng(8).standard_normal((w.nextrap, w.nx)).astype(np.float32)).cuda()
    op = _op(w, slab)
    data = {}
    for mode in ("recompute", "keep", "reuse"):
        d = op.zeros_data()
        op.plan.demigrate(m, op.wave, d, slab_depth=slab, source=mode)
        data[mode] = d.cpu().numpy()
    desc = op.plan.describe_demigration()
    assert desc["kernel"] == "demigrate_cluster" and desc["G"] == 16, desc
    assert desc["ring"] == (2 * w.M + 1 in (25, 31, 35, 55)), desc  # compile-time lengths
    if w.nx > 512:
        assert desc["cluster"] >= 2, desc
    single = lsm.MigrationOperator.for_workload(w, slab_depth=slab, no_cluster=True)
    d1 = single.zeros_data()
    single.plan.demigrate(m, single.wave, d1, slab_depth=slab, source="recompute")
    assert single.plan.describe_demigration()["kernel"] == "demigrate"
    ref = oracle.demigrate_workload_f64(w, m.cpu().numpy().astype(np.float64))
    assert rel_l2(data["recompute"], ref) <= 1e-5
    for mode in ("keep", "reuse"):
        assert np.array_equal(data[mode], data["recompute"]), mode
    assert np.array_equal(data["recompute"], d1.cpu().numpy())
    lhs, rhs, rel, rel_norms = lsm.dot_product_test(op, seed=2, separation=3.0)
    assert rel_norms <= 1e-7 and rel <= 1e-6, (lhs, rhs, rel, rel_norms)
    op.plan.close()
    single.plan.close()


def test_demigration_ring_matches_l1_path_bitwise():
    """The cluster demigration's forward steps read their operator pairs through a shared-memory ring
    (cp.async) by default; the same kernel reading them through L1 gives bit-identical data."""
    import torch
    w = synthetic.batched_uneven(nx=1300, nz=9, nf=3, ns=64)
    m = torch.from_numpy(np.random.default_rng(5).standard_normal((w.nextrap, w.nx)).astype(np.float32)).cuda()
    out = {}
    for ring in (True, False):
        op = lsm.MigrationOperator.for_workload(w, slab_depth=3, demig_ring=ring)
        out[ring] = op.demigrate(m).cpu().numpy()
        assert op.plan.describe_demigration()["ring"] == ring
        op.plan.close()
    assert np.array_equal(out[True], out[False])


def test_wide_window_non_portable_cluster_demigration():
    import torch
    w = synthetic.plain_medium(nx=6000, nz=4, nf=2, ns=12)
    op = _op(w)
    m = torch.from_numpy(np.random.default_rng(9).standard_normal((w.nextrap, w.nx)).astype(np.float32)).cuda()
    data = op.demigrate(m).cpu().numpy()
    desc = op.plan.describe_demigration()
    assert desc["kernel"] == "demigrate_cluster" and desc["cluster"] == 12, desc
    assert rel_l2(data, oracle.demigrate_workload_f64(w, m.cpu().numpy().astype(np.float64))) <= 1e-5
    op.plan.close()
