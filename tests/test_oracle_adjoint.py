"""The FP64 oracle's demigration is the adjoint of its migration.

The oracle's migration (oracle_migrate_compact_f64) is pinned to the reference's known-answer tests
and to the reference library itself (test_oracle_kat.py).  Demigration has no reference
counterpart, so it is pinned here to that migration by the dot-product test
<F d, m> = Re sum d conj(F* m) in float64, for full and uneven apertures, and by an explicit
transpose on a tiny case.  The GPU kernels are then checked against this oracle.
"""
import numpy as np
import pytest

from imaging2d_wlsq_b200 import synthetic
from oracle import oracle


def _dot_test(w, seed, nextrap=None):
    n = nextrap or w.nextrap
    rng = np.random.default_rng(seed)
    d = (rng.standard_normal(w.shot.shape) + 1j * rng.standard_normal(w.shot.shape)).astype(np.complex128)
    m = rng.standard_normal((n, w.nx))
    stack, _, _, _ = oracle.migrate_compact_f64(w.ns, n, w.nz, w.nx, w.nf, w.nt, w.M, w.nk, w.dk, w.omega,
                                                w.velocity, w.table, w.wave, d, shot_x0=w.shot_x0,
                                                shot_nx=w.shot_nx, offsets=w.offsets())
    lhs = float(np.sum(stack[:n] * m))
    data = oracle.demigrate_workload_f64(w, m, nextrap=n)
    rhs = float(np.sum(d.real * data.real + d.imag * data.imag))
    return lhs, rhs


@pytest.mark.parametrize("maker,kw,seed", [
    (synthetic.plain_small, dict(scale=0.1), 0),
    (synthetic.plain_medium, dict(nx=96, nz=12, nf=5, ns=3), 1),
    (synthetic.batched_uneven, dict(scale=0.04, nz=10, nf=4), 2),
    (synthetic.lsm, dict(scale=0.06, nf=6), 3),
])
def test_oracle_dot_product(maker, kw, seed):
    w = maker(**kw)
    lhs, rhs = _dot_test(w, seed)
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), abs(rhs))


def test_oracle_adjoint_is_explicit_transpose():
    # tiny case: build F column by column (unit receiver samples) and compare F^T m with F* m
    w = synthetic.plain_medium(nx=32, nz=4, nf=2, ns=1)
    n = 3
    rng = np.random.default_rng(7)
    m = rng.standard_normal((n, w.nx))
    N = w.shot.size
    cols_re = np.zeros((n * w.nx, N))
    cols_im = np.zeros((n * w.nx, N))
    for e in range(N):
        for part, cols in ((1.0, cols_re), (1j, cols_im)):
            d = np.zeros(N, dtype=np.complex128)
            d[e] = part
            stack, _, _, _ = oracle.migrate_compact_f64(w.ns, n, w.nz, w.nx, w.nf, w.nt, w.M, w.nk, w.dk, w.omega,
                                                        w.velocity, w.table, w.wave, d)
            cols[:, e] = stack[:n].reshape(-1)
    # <F d, m> = Re sum d conj(F* m): Re(F* m) = F_re^T m, Im(F* m) = F_im^T m
    expect = cols_re.T @ m.reshape(-1) + 1j * (cols_im.T @ m.reshape(-1))
    got = oracle.demigrate_workload_f64(w, m, nextrap=n)
    np.testing.assert_allclose(got, expect, rtol=1e-12, atol=1e-12 * np.abs(expect).max())


def test_lsm_reflectivity_recipe():
    w = synthetic.lsm(scale=0.2, nf=4)
    r = w.reflectivity
    assert r.shape == (w.nz, w.nx) and r.dtype == np.float32
    # 0.5% spikes, each spread by the 3x3 kernel [1,2,1]/4 (x) [1,2,1]/4
    nonzero = np.count_nonzero(r)
    spikes = round(0.005 * w.nz * w.nx)
    assert spikes <= nonzero <= 9 * spikes
    again = synthetic.lsm(scale=0.2, nf=4)
    assert np.array_equal(again.reflectivity, r)
