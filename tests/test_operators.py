"""Host operator design (imaging2d_wlsq_b200.operators) against the reference's own Python outputs
(tests/golden/operators_small.npz, produced by py_src/operatorsPreparation with numba), and the
compact-table form against the reference demo (tests/golden/demo_case.npz)."""
import numpy as np

from imaging2d_wlsq_b200 import operators as ops
from oracle import oracle
from tests.conftest import rel_l2


def test_create_kappa(golden_ops):
    g = golden_ops
    k = ops.create_kappa(3000.0, 1500.0, float(g["dw"]), float(g["wmax"]), 0.25)
    np.testing.assert_array_equal(k, g["kappa"])


def test_find_nearest(golden_ops):
    g = golden_ops
    got = [ops.find_nearest(g["kappa"], v) for v in g["values"]]
    np.testing.assert_array_equal(got, g["nearest"])
    dk = g["kappa"][1] - g["kappa"][0]
    np.testing.assert_array_equal(ops.nearest_index(g["values"], 1.0, dk, len(g["kappa"])), g["nearest"])


def test_phase_shift_operators(golden_ops):
    g = golden_ops
    psf = ops.make_forw_ps_operators(g["kappa"], g["kx"], float(g["dz"]))
    psb = ops.make_back_ps_operators(g["kappa"], g["kx"], float(g["dz"]))
    np.testing.assert_allclose(psf, g["psf"], rtol=0, atol=2e-7)
    np.testing.assert_allclose(psb, g["psb"], rtol=0, atol=2e-7)
    # the receiver operators are the conjugates of the source operators (preparation.py:10-44)
    np.testing.assert_array_equal(psb, np.conjugate(psf))


def test_wlsq_operators(golden_ops):
    g = golden_ops
    M = int(g["M"])
    N = (int(g["nx"]) - 1) // 2
    op = ops.create_wlsq_operators(N, M, g["kx"], g["xilocal"])
    # every stencil bit-identical to the reference's createWLSQoperators (same cmath.exp per element)
    np.testing.assert_array_equal(op, g["op"])
    sym = ops.create_wlsq_operators(N, M, g["kx"], g["xilocal"], only_symmetric=True)
    np.testing.assert_array_equal(sym[M], op[M])


def test_dense_table_is_gather_of_compact(golden_ops):
    g = golden_ops
    M = int(g["M"])
    kappa = g["kappa"]
    dk = kappa[1] - kappa[0]
    comp_f = ops.compact_table(g["op"][M], g["psf"])
    comp_b = ops.compact_table(g["op"][M], g["psb"])
    nextrap, nx = g["vel"].shape
    dense_f = ops.dense_table(comp_f, g["w"], g["vel"], nextrap, dk=dk, nk=len(kappa))
    dense_b = ops.dense_table(comp_b, g["w"], g["vel"], nextrap, dk=dk, nk=len(kappa))
    # bitwise: the same numpy matmul per row as preparation.py:110
    np.testing.assert_array_equal(dense_f, g["table_f"])
    np.testing.assert_array_equal(dense_b, g["table_b"])
    # backward table == conj(forward) to rounding (exact in exact arithmetic for a symmetric kx grid)
    assert np.abs(comp_b - np.conjugate(comp_f)).max() <= 1e-6 * np.abs(comp_f).max()
    # the C gather used by tests and the CPU baseline agrees
    slab = oracle.gather_dense_slab(0, nextrap, nx, 0, nx, len(g["w"]), M, len(kappa), dk, g["w"], g["vel"], comp_f)
    np.testing.assert_array_equal(slab, g["table_f"])


def test_odd_grid_design_matches_reference_for_odd_nx(golden_ops):
    g = golden_ops
    N, kx = ops.odd_wavenumber_grid(int(g["nx"]), float(g["dx"]))
    np.testing.assert_allclose(kx, g["kx"], rtol=1e-14, atol=0)
    assert 2 * N + 1 == int(g["nx"])
    N2, kx2 = ops.odd_wavenumber_grid(320, 10.0)
    assert 2 * N2 + 1 == 321 and abs(np.abs(kx2).max() - np.pi / 10.0) < 1e-3


def test_demo_oracle_reproduces_reference_images(golden_demo):
    """FP64 compact oracle on the reference demo against the reference CPU library's image and the
    reference's shipped final_image.csv."""
    g = golden_demo
    ns = g["src"].shape[0]
    nz, nx, nw, M, nk = (int(g[k]) for k in ("nz", "nx", "nw", "M", "nk"))
    stack, _, _, _ = oracle.migrate_compact_f64(ns, int(g["nextrap"]), nz, nx, nw, nw, M, nk, float(g["dk"]),
                                                g["omega"], g["velocity"], g["tab_f"], g["src"].reshape(-1),
                                                g["rec"].reshape(-1), tab_back=g["tab_b"])
    assert rel_l2(stack, g["image_ref_cpu"]) < 2e-6
    assert rel_l2(stack, g["image_shipped"]) < 3e-5
    # single-table form (receiver uses conj of the forward table)
    stack1, _, _, _ = oracle.migrate_compact_f64(ns, int(g["nextrap"]), nz, nx, nw, nw, M, nk, float(g["dk"]),
                                                 g["omega"], g["velocity"], g["tab_f"], g["src"].reshape(-1),
                                                 g["rec"].reshape(-1))
    assert rel_l2(stack1, g["image_ref_cpu"]) < 1e-5
