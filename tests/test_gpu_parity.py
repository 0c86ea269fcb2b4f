"""GPU parity: the CUDA library through its C ABI against the reference's known answers, the CPU
oracle (FP32 reference-order and FP64) and the reference demo.  Tolerances:
  known answers            1e-5 absolute, as the reference's own tests (test_cpp_src.py:13)
  dense ABI vs FP32 oracle  max |diff| <= 1e-5 * max|image| and wavefields likewise
  compact vs FP64 oracle    relative L2 of the image <= 1e-5 (single-table mode adds the
                            conj(T_forw) vs T_back rounding, still inside 1e-5)
"""
import ctypes
import os

import numpy as np
import pytest
from numpy.ctypeslib import ndpointer

from imaging2d_wlsq_b200 import DROPIN_DIR, interface, interface_cuda, migration, operators, synthetic
from oracle import oracle
from tests import kat_cases as K
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

HOST_CASES = K.cpu_cases() + [c[:7] for c in K.gpu_cases()] + K.py_float_cases()


def _host_call(fn, d, f, b, pf, pb):
    img = np.zeros((d["ns"], d["nz"], d["nx"]), dtype=np.float32)
    w, s = pf.copy(), pb.copy()
    fn(d["ns"], d["nextrap"], d["nz"], d["nx"], d["nf"], d["nt"], d["M"], f, b, w, s, img)
    return img, w, s


def _dev_call(fn, d, f, b, pf, pb):
    img = np.zeros((d["ns"], d["nz"], d["nx"]), dtype=np.float32)
    w, s = pf.copy(), pb.copy()
    fn(d["ns"], d["nextrap"], d["nz"], d["nt"], d["nf"], d["nx"], d["M"], f, w, b, s, img)
    return img, w, s


def _dropin(name, symbol="extrapolate"):
    # bound exactly as the reference's cpp_src/interface.py / interface_cuda.py bind it
    lib = ctypes.CDLL(os.path.join(DROPIN_DIR, name))
    f = getattr(lib, symbol)
    f.restype = ctypes.c_void_p
    f.argtypes = [ctypes.c_int] * 7 + [ndpointer(dtype=np.complex64, flags=("C", "A"))] * 4 + \
        [ndpointer(dtype=np.float32, flags=("C", "A"))]
    return f


@pytest.mark.parametrize("case", HOST_CASES, ids=[c[0] for c in HOST_CASES])
def test_known_answers_host_order(case):
    name, d, f, b, pf, pb, exp = case
    for fn in (interface.extrapolate, interface.extrapolate_v0, _dropin("extrapolation_cpu.so"),
               _dropin("extrapolation_cpu.so", "extrapolate_v0")):
        img, _, _ = _host_call(fn, d, f, b, pf, pb)
        ok, msg = K.check_image(img[0], exp, d["nz"], d["nx"])
        assert ok, f"{name}: {msg}"


@pytest.mark.parametrize("case", K.gpu_cases(), ids=[c[0] for c in K.gpu_cases()])
def test_known_answers_device_order(case):
    name, d, f, b, pf, pb, exp, waves = case
    (pi, pv), (ri, rv) = waves["pulse"], waves["pulse2"]
    for fn, wb in ((interface_cuda.extrapolate, False), (interface_cuda.extrapolate_revOp, True),
                   (interface_cuda.extrapolate_sh_revOp, True), (_dropin("extrapolation_gpu.so"), False),
                   (_dropin("extrapolation_revOp_gpu.so"), True), (_dropin("extrapolation_sh_revOp_gpu.so"), True)):
        img, w, s = _dev_call(fn, d, f, b, pf, pb)
        ok, msg = K.check_image(img[0], exp, d["nz"], d["nx"])
        assert ok, f"{name}: {msg}"
        if wb:
            assert abs(w[pi] - pv) <= K.SDELTA and abs(s[ri] - rv) <= K.SDELTA, name
        else:
            np.testing.assert_array_equal(w, pf)  # extrapolation_gpu.cu never writes wavefields back
            np.testing.assert_array_equal(s, pb)


def _rand_dense(ns, nextrap, nz, nx, nf, nt, M, seed):
    rng = np.random.default_rng(seed)
    L = 2 * M + 1

    def c(*shape):
        return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)

    scale = np.float32(0.6 / np.sqrt(L))
    return (c(nextrap, nf, nx, L) * scale).astype(np.complex64), (c(nextrap, nf, nx, L) * scale).astype(np.complex64), \
        c(ns, nt, nx), c(ns, nt, nx)


@pytest.mark.parametrize("ns,nextrap,nz,nx,nf,nt,M", [
    (1, 3, 5, 17, 5, 7, 2), (3, 6, 8, 40, 6, 6, 5), (5, 4, 4, 33, 9, 12, 12), (9, 7, 9, 150, 11, 11, 21),
    (2, 2, 3, 1, 2, 2, 1), (4, 5, 6, 64, 3, 3, 0), (16, 3, 3, 96, 4, 4, 7)])
def test_dense_abi_matches_oracle(ns, nextrap, nz, nx, nf, nt, M):
    f, b, pf, pb = _rand_dense(ns, nextrap, nz, nx, nf, nt, M, ns * 1000 + nx)
    d = dict(ns=ns, nextrap=nextrap, nz=nz, nx=nx, nf=nf, nt=nt, M=M)
    img_o = np.full((ns, nz, nx), 7.0, dtype=np.float32)
    wo, so = pf.copy(), pb.copy()
    oracle.extrapolate_f32(ns, nextrap, nz, nx, nf, nt, M, f, b, wo, so, img_o)
    img_g = np.full((ns, nz, nx), 7.0, dtype=np.float32)
    wg, sg = pf.copy(), pb.copy()
    interface.extrapolate(ns, nextrap, nz, nx, nf, nt, M, f, b, wg, sg, img_g)
    scale = np.abs(img_o[:, :nextrap]).max()
    assert np.abs(img_g - img_o).max() <= 1e-5 * scale + 1e-6
    assert np.all(img_g[:, nextrap:] == 7.0)  # rows >= nextrap untouched
    for g, o in ((wg, wo), (sg, so)):
        assert np.abs(g - o).max() <= 1e-5 * np.abs(o).max() + 1e-6
        np.testing.assert_array_equal(g[:, nf:], pf[:, nf:] if g is wg else pb[:, nf:])  # rows >= nf untouched


def _compact_check(w, img, wave, shot, two_tables=False, tol=1e-5):
    tab_b = None
    if two_tables:
        tab_b = w.table_back
    stack, _, wo, so = oracle.migrate_workload_f64(w, tab_back=tab_b)
    e_img = rel_l2(img, stack)
    e_w = rel_l2(wave, wo)
    e_s = rel_l2(shot, so)
    assert e_img <= tol, f"image rel-L2 {e_img:.2e}"
    assert e_w <= tol and e_s <= tol, f"wavefield rel-L2 {e_w:.2e} {e_s:.2e}"
    return e_img


@pytest.mark.parametrize("maker,scale", [(synthetic.plain_small, 0.5), (synthetic.plain_medium, 0.125),
                                         (synthetic.batched_uneven, 0.1), (synthetic.precision, 0.05)])
def test_compact_matches_fp64_oracle(maker, scale):
    w = maker(scale=scale)
    img, _, wave, shot = migration.migrate_workload(w)
    _compact_check(w, img, wave, shot)


def test_compact_generic_kernel_and_per_shot_images():
    w = synthetic.batched_uneven(scale=0.08)
    img, imgs, wave, shot = migration.migrate_workload(w, image_shots=True, generic=True)
    _compact_check(w, img, wave, shot)
    _, shots_o, _, _ = oracle.migrate_workload_f64(w)
    assert rel_l2(imgs, shots_o) <= 1e-5
    # per-shot images are zero outside each shot's aperture
    for s in range(w.ns):
        x0, n = int(w.shot_x0[s]), int(w.shot_nx[s])
        assert np.all(imgs[s, :, :x0] == 0) and np.all(imgs[s, :, x0 + n:] == 0)
    # stack == sum of per-shot images
    assert rel_l2(imgs.sum(axis=0), img) <= 1e-6


def test_compact_two_tables():
    from imaging2d_wlsq_b200 import operators as ops
    w = synthetic.plain_small(scale=0.4)
    w.table_back = ops.design_compact_table(w.nx, w.dx, w.dz, w.M, w.nk, w.dk, back=True)
    img, _, wave, shot = migration.migrate_workload(w, two_tables=True, table_back=w.table_back)
    _compact_check(w, img, wave, shot, two_tables=True)


def test_demo_matches_reference(golden_demo):
    g = golden_demo
    ns = g["src"].shape[0]
    nz, nx, nw, M, nk = (int(g[k]) for k in ("nz", "nx", "nw", "M", "nk"))
    for two in (True, False):
        wave, shot = g["src"].reshape(-1).copy(), g["rec"].reshape(-1).copy()
        img, _ = migration.migrate(ns, int(g["nextrap"]), nz, nx, nw, nw, M, nk, float(g["dk"]), g["omega"],
                                   g["velocity"], g["tab_f"], wave, shot, tab_back=g["tab_b"], two_tables=two)
        assert rel_l2(img, g["image_ref_cpu"]) <= 1e-5, two
        assert rel_l2(img, g["image_shipped"]) <= 3e-5, two
        assert np.all(img[int(g["nextrap"]):] == 0)


def test_plan_device_resident_matches_host_entry():
    import torch
    w = synthetic.batched_uneven(scale=0.08)
    img_h, _, wave_h, shot_h = migration.migrate_workload(w)
    plan = migration.Plan.for_workload(w)
    dev = torch.device("cuda")
    om = torch.from_numpy(w.omega).to(dev)
    vel = torch.from_numpy(np.ascontiguousarray(w.velocity)).to(dev)
    tab = torch.from_numpy(w.table).to(dev)
    wave = torch.from_numpy(w.wave.copy()).to(dev)
    shot = torch.from_numpy(w.shot.copy()).to(dev)
    img = torch.zeros((w.nz, w.nx), dtype=torch.float32, device=dev)
    plan.set_model(om, vel, w.dk, tab)
    plan.execute(wave, shot, img)
    torch.cuda.synchronize()
    assert rel_l2(img.cpu().numpy(), img_h) <= 1e-6
    assert rel_l2(wave.cpu().numpy(), wave_h) <= 1e-6
    d = plan.describe()
    assert d["G"] >= 1 and d["grid"] >= 1
    plan.close()


def test_naive_form_matches_batched():
    import torch
    w = synthetic.plain_medium(scale=0.06)
    dev = torch.device("cuda")
    plan = migration.Plan.for_workload(w)
    plan.set_model(torch.from_numpy(w.omega).to(dev), torch.from_numpy(np.ascontiguousarray(w.velocity)).to(dev),
                   w.dk, torch.from_numpy(w.table).to(dev))
    out = []
    for naive in (False, True):
        wave = torch.from_numpy(w.wave.copy()).to(dev)
        shot = torch.from_numpy(w.shot.copy()).to(dev)
        img = torch.zeros((w.nz, w.nx), dtype=torch.float32, device=dev)
        (plan.execute_naive if naive else plan.execute)(wave, shot, img)
        torch.cuda.synchronize()
        out.append((img.cpu().numpy(), wave.cpu().numpy()))
    assert rel_l2(out[1][0], out[0][0]) <= 1e-5
    assert rel_l2(out[1][1], out[0][1]) <= 1e-5
    plan.close()


def test_invalid_arguments_raise():
    from imaging2d_wlsq_b200 import LibraryError
    w = synthetic.plain_small(scale=0.2)
    with pytest.raises(LibraryError):
        migration.Plan(w.ns, w.nextrap, w.nz, w.nx, w.nf, w.nt, w.M, w.nk, shot_x0=[0, 0, 0, w.nx - 1],
                       shot_nx=[w.nx] * 4)
    with pytest.raises(LibraryError):
        migration.Plan(w.ns, w.nz + 1, w.nz, w.nx, w.nf, w.nt, w.M, w.nk)


@pytest.mark.parametrize("v1", [False, True], ids=["cluster2", "cluster1"])
@pytest.mark.parametrize("kind,nx,nz,nf,ns", [("medium", 256, 12, 6, 16), ("medium", 480, 10, 5, 24),
                                              ("uneven", 1000, 8, 5, 40), ("uneven", 2048, 6, 4, 64),
                                              ("medium", 2048, 5, 3, 32), ("medium", 3000, 4, 3, 20)])
def test_cluster_kernel_matches_oracle_and_single_cta(kind, nx, nz, nf, ns, v1):
    """Both cluster kernels (256 positions per CTA for the first, 512 for the second; clusters of
    1 to 8 CTAs) against the FP64 oracle and against the single-CTA kernel; few depth steps and
    frequencies keep the oracle fast."""
    if kind == "medium":
        w = synthetic.plain_medium(nx=nx, nz=nz, nf=nf, ns=ns, scale=1.0)
    else:
        w = synthetic.batched_uneven(nx=nx, nz=nz, nf=nf, ns=ns, scale=1.0)
    plan = migration.Plan.for_workload(w, cluster_v1=v1, cluster2=not v1)
    d = plan.describe()
    plan.close()
    if v1 and nx > 2048:
        assert d["kernel"] != "migrate_cluster", d  # 8 CTAs x 256 positions do not cover it
        return
    assert d["kernel"] == ("migrate_cluster" if v1 else "migrate_cluster2"), d
    pc = 256 if v1 else 512
    if kind == "medium":
        assert d["cluster"] >= -(-nx // pc), d
    img, imgs, wave, shot = migration.migrate_workload(w, image_shots=True, cluster_v1=v1, cluster2=not v1)
    e = _compact_check(w, img, wave, shot)
    img1, _, wave1, _ = migration.migrate_workload(w, no_cluster=True)
    assert rel_l2(img, img1) <= 2e-6 and rel_l2(wave, wave1) <= 2e-6
    _, shots_o, _, _ = oracle.migrate_workload_f64(w)
    assert rel_l2(imgs, shots_o) <= 1e-5
    assert e <= 1e-5


@pytest.mark.parametrize("variant", list(range(1, migration.N_CLUSTER2_VARIANTS + 1)))
def test_cluster2_variants_match_oracle(variant):
    """Every variant of the second-generation cluster kernel (warps per CTA, operator-pair
    prefetch, L1 row prefetch) on a window that needs a multi-CTA cluster."""
    w = synthetic.batched_uneven(nx=1500, nz=7, nf=4, ns=48, scale=1.0)
    plan = migration.Plan.for_workload(w, variant=variant)
    d = plan.describe()
    plan.close()
    assert d["kernel"] == "migrate_cluster2" and d["variant"] == variant - 1 and d["cluster"] >= 2, d
    wave, shot = w.wave.copy(), w.shot.copy()
    from imaging2d_wlsq_b200._lib import FLAG_VARIANT_SHIFT, check, lib, ptr
    img = np.zeros((w.nz, w.nx), dtype=np.float32)
    check(lib().img2d_migrate_compact(w.ns, w.nextrap, w.nz, w.nx, w.nf, w.nt, w.M, w.nk, float(w.dk), ptr(w.omega),
                                      ptr(np.ascontiguousarray(w.velocity)), ptr(w.table), None,
                                      ptr(np.ascontiguousarray(w.shot_x0)), ptr(np.ascontiguousarray(w.shot_nx)),
                                      ptr(wave), ptr(shot), ptr(img), None, variant << FLAG_VARIANT_SHIFT))
    _compact_check(w, img, wave, shot)


def test_staged_matches_unstaged_bitwise():
    """Variant 11 stages the next step's operator indices and Kahan partial rows in shared memory
    (cp.async); its per-point arithmetic is that of variant 1, so the final wavefields are
    bit-identical and the images agree to rounding of the partial split."""
    w = synthetic.batched_uneven(nx=1500, nz=9, nf=4, ns=48, scale=1.0)
    img0, _, wave0, shot0 = migration.migrate_workload(w, variant=11)
    img1, _, wave1, shot1 = migration.migrate_workload(w, variant=1)
    assert np.array_equal(wave0, wave1) and np.array_equal(shot0, shot1)
    assert rel_l2(img0, img1) <= 1e-6
    _compact_check(w, img0, wave0, shot0)


def _with_taps(w, taps):
    if taps != 2 * w.M + 1:
        w.M = (taps - 1) // 2
        w.table = operators.design_compact_table(w.nx, w.dx, w.dz, w.M, w.nk, w.dk)
    return w


def test_ring_default_matches_staged_bitwise():
    """The default (variant 12) reads the operator tap pairs from a per-lane-group shared-memory ring
    filled by 16-byte cp.async copies and keeps the next step's index and Kahan values in registers;
    the tap values and the FMA order are those of the staged variant 11, so final wavefields are
    bit-identical.  Runs an operator length with a middle loop (35 taps), the shortest one without
    (7 taps) and the longest whose ring still fits in shared memory (81 taps)."""
    for taps in (35, 7, 81):
        w = _with_taps(synthetic.batched_uneven(nx=1500, nz=9, nf=4, ns=48, scale=1.0), taps)
        d = migration.Plan.for_workload(w, cluster2=True).describe()
        assert d["kernel"] == "migrate_cluster2" and d["variant"] == 11, (taps, d)
        img0, _, wave0, shot0 = migration.migrate_workload(w, cluster2=True)
        img1, _, wave1, shot1 = migration.migrate_workload(w, variant=11)
        assert np.array_equal(wave0, wave1) and np.array_equal(shot0, shot1), taps
        assert rel_l2(img0, img1) <= 1e-6, taps
        _compact_check(w, img0, wave0, shot0)


def test_long_operator_falls_back_to_staged_variant():
    """91 taps leave no room for the 33 KB ring next to the wavefields and halos: the default plan
    takes the staged variant, still on the cluster kernel."""
    w = _with_taps(synthetic.batched_uneven(nx=1500, nz=5, nf=3, ns=48, scale=1.0), 91)
    d = migration.Plan.for_workload(w).describe()
    assert d["kernel"] == "migrate_cluster2" and d["variant"] == 10, d
    img, _, wave, shot = migration.migrate_workload(w)
    _compact_check(w, img, wave, shot)


def test_wide_window_non_portable_cluster():
    """A 6000-position full-aperture window needs 12 CTAs of 512 positions: a non-portable cluster
    size (up to 16 on B200 with the kernel's opt-in) for the 16-slot kernel; the default (wide)
    kernel covers it with 6 CTAs of 1024."""
    w = synthetic.plain_medium(nx=6000, nz=4, nf=2, ns=12)
    d = migration.Plan.for_workload(w, cluster2=True).describe()
    assert d["kernel"] == "migrate_cluster2" and d["cluster"] == 12, d
    img, _, wave, shot = migration.migrate_workload(w, cluster2=True)
    _compact_check(w, img, wave, shot)
    d = migration.Plan.for_workload(w).describe()
    assert d["kernel"] == "migrate_wide" and d["cluster"] == 6, d
    img, _, wave, shot = migration.migrate_workload(w)
    _compact_check(w, img, wave, shot)


@pytest.mark.skipif(not oracle.have_ref(), reason="oracle/_ref/extrapolation_cpu.so not built")
def test_plain_small_in_full_through_dense_dropin_matches_reference_library():
    """The plain small configuration in full (nz=200, nx=320, nf=64 over 2-30 Hz, 25 taps, 4
    full-aperture shots; dense tables 200 x 64 x 320 x 25) through the drop-in
    `extrapolation_cpu.so`, bound as cpp_src/interface.py binds it, against the reference's own
    extrapolation_cpu.so on the same dense tables and spectra, and against the FP64 oracle."""
    w = synthetic.plain_small()
    ns, nl, nz, nx, nf, M = w.ns, w.nextrap, w.nz, w.nx, w.nf, w.M
    tf = oracle.gather_dense_slab(0, nl, nx, 0, nx, nf, M, w.nk, w.dk, w.omega, w.velocity, w.table)
    tb = oracle.gather_dense_slab(0, nl, nx, 0, nx, nf, M, w.nk, w.dk, w.omega, w.velocity, w.table,
                                  conj_rows=True)
    wave0 = w.wave.reshape(ns, nf, nx)
    shot0 = w.shot.reshape(ns, nf, nx)
    img_r = np.zeros((ns, nz, nx), dtype=np.float32)
    wr, sr = wave0.copy(), shot0.copy()
    oracle.ref_extrapolate(ns, nl, nz, nx, nf, nf, M, tf, tb, wr, sr, img_r)
    img_g = np.zeros((ns, nz, nx), dtype=np.float32)
    wg, sg = wave0.copy(), shot0.copy()
    _dropin("extrapolation_cpu.so")(ns, nl, nz, nx, nf, nf, M, tf, tb, wg, sg, img_g)
    assert rel_l2(img_g, img_r) <= 1e-5
    assert rel_l2(wg, wr) <= 1e-5 and rel_l2(sg, sr) <= 1e-5
    _, shots64, w64, s64 = oracle.migrate_workload_f64(w)
    assert rel_l2(img_g, shots64) <= 1e-5
    assert rel_l2(wg.reshape(-1), w64) <= 1e-5 and rel_l2(sg.reshape(-1), s64) <= 1e-5
