"""The wide kernel's packing of shots into items (host logic, no GPU): every shot in exactly one lane
slot of one item, shots of a slot separated by at least M zero samples (the zero-halo semantics of
cpp_src/wfPad.h hold per shot), each item's window holding its shots and at most 8 slots, the
modelled cost recomputed from the windows, and the window-first packing cheaper than the line
packing on the benchmark survey."""
import math

import numpy as np
import pytest

from imaging2d_wlsq_b200 import migration, synthetic


def _item_cost(W, K):
    NC = min(1024, -(-W // (K * 256)) * 256)
    eff = 1.0 if NC >= 1024 else (0.92 if NC >= 768 else (0.87 if NC >= 512 else 0.62))
    return K * NC / 1024 / eff


def _check(x0, wn, nx, M, res):
    x1 = x0 + wn
    ng = len(res["width"])
    assert ng >= 1
    assert res["group"].min() >= 0 and res["group"].max() < ng
    assert res["slot"].min() >= 0 and res["slot"].max() < 8
    for g in range(ng):
        mine = np.flatnonzero(res["group"] == g)
        assert len(mine) > 0
        u0, W = int(res["u0"][g]), int(res["width"][g])
        assert u0 == x0[mine].min() and u0 + W == x1[mine].max()
        assert W <= res["K"] * 1024 if res["K"] > 0 else True
        for k in np.unique(res["slot"][mine]):
            line = mine[res["slot"][mine] == k]
            order = np.argsort(x0[line])
            a, b = x0[line][order], x1[line][order]
            assert np.all(a[1:] >= b[:-1] + M), (g, k)
    K = res["K"] if res["K"] > 0 else -(-int(res["width"].max()) // 1024)
    assert math.isclose(res["cost"], sum(_item_cost(int(W), K) for W in res["width"]), rel_tol=1e-9)


def _shots(seed, ns, nx, lo, hi):
    rng = np.random.default_rng(seed)
    wn = rng.integers(lo, hi + 1, ns).astype(np.int32)
    x0 = np.clip(rng.integers(0, nx, ns) - wn // 2, 0, nx - wn).astype(np.int32)
    return x0, wn


@pytest.mark.parametrize("seed,ns,nx,lo,hi", [(1, 40, 2048, 256, 2048), (2, 100, 2048, 64, 1024),
                                              (3, 7, 700, 50, 700), (4, 60, 5000, 100, 3000),
                                              (5, 1, 300, 300, 300)])
@pytest.mark.parametrize("windows", [False, True])
def test_packing_invariants(seed, ns, nx, lo, hi, windows):
    x0, wn = _shots(seed, ns, nx, lo, hi)
    M = 17
    res = migration.pack_shots(x0, wn, nx, M, windows=windows)
    _check(x0, wn, nx, M, res)


def test_window_packing_on_the_benchmark_survey():
    """256 shots of U[256, 2048] traces on 2048 positions (35 taps): the window-first packing models
    36.9 CTA units per frequency against 38.4 for the line packing (measured 4.1% faster)."""
    w = synthetic.batched_uneven(tables=False, nf=4)
    lines = migration.pack_shots(w.shot_x0, w.shot_nx, w.nx, w.M, windows=False)
    wins = migration.pack_shots(w.shot_x0, w.shot_nx, w.nx, w.M, windows=True)
    _check(w.shot_x0.astype(np.int64), w.shot_nx.astype(np.int64), w.nx, w.M, lines)
    _check(w.shot_x0.astype(np.int64), w.shot_nx.astype(np.int64), w.nx, w.M, wins)
    assert wins["cost"] < 0.97 * lines["cost"], (wins["cost"], lines["cost"])
    assert abs(wins["cost"] - 36.932) < 0.01 and abs(lines["cost"] - 38.410) < 0.01


def test_pack_shots_rejects_bad_input():
    from imaging2d_wlsq_b200._lib import LibraryError
    with pytest.raises(LibraryError):
        migration.pack_shots([10], [100], 64, 3)          # aperture outside [0, nx)
    with pytest.raises(LibraryError):
        migration.pack_shots([0], [2000], 2048, 3, K=1)   # a window of one CTA cannot hold the shot
