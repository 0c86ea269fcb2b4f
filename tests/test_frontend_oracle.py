"""The front-end checker (oracle/frontend_oracle.py) against the reference's own outputs: the
makeRickerWavelet known-answer test of unittests/test_py_src_util.py:17-50, the demo's wavelet and
record spectra (tests/golden/frontend_case.npz, demo_case.npz, generated by
tests/golden/make_golden.py from the reference code)."""
import math

import numpy as np

from oracle import frontend_oracle as fo
from tests.conftest import rel_l2


def test_ricker_matches_reference_unit_test():
    # unittests/test_py_src_util.py:19-50: isx=-600, nt=500, dt=1 ms, nx=151, dx=15, xmin=-800,
    # z1=0, z2=10, v=2600; expected (1 - 2 pi^2 30^2 tau^2) exp(-pi^2 30^2 tau^2) / sqrt(r) within 1e-5
    isx, nt, dt, nx, dx, xmin, z1, z2, v = -600, 500, 0.001, 151, 15, -800, 0, 10, 2600
    got = fo.ricker_sources(1, nt, nx, dt, xmin, dx, z2 - z1, v, [isx])[0]
    for i in range(0, nx, 7):
        r = math.sqrt((z2 - z1) ** 2 + (isx - (xmin + i * dx)) ** 2)
        for j in range(0, nt, 11):
            tau = j * dt - r / v
            term = math.pi ** 2 * 30.0 ** 2 * tau ** 2
            assert abs(got[j, i] - (1 - 2 * term) * math.exp(-term) / math.sqrt(r)) <= 1e-5


def test_ricker_and_record_spectra_match_reference_demo(golden_demo):
    g = dict(np.load("tests/golden/frontend_case.npz"))
    nt, nw, nx = int(g["nt"]), int(g["nw"]), int(g["nx"])
    dx, dz, dt, xmin, zinit, v = (float(g[k]) for k in ("dx", "dz", "dt", "xmin", "zinit", "v"))
    isx = g["shot_isx"]
    sx = xmin + isx * dx
    src_t = fo.ricker_sources(len(isx), nt, nx, dt, xmin + dx, dx, dz - zinit, v, sx)
    # the reference's makeRickerWavelet output for shot 0, to float32 rounding
    assert np.max(np.abs(src_t[0] - g["wavelet_t"])) <= 1e-6 * np.max(np.abs(g["wavelet_t"]))
    # source spectra of all shots (demo_case src = reference scipy.fftpack.fft, float32 FFT)
    src_f = fo.records_to_spectra(src_t, nw).reshape(len(isx), nw, nx)
    assert rel_l2(src_f, golden_demo["src"]) <= 1e-5
    rec_f = fo.records_to_spectra(g["rec_t"][None], nw).reshape(nw, nx)
    assert rel_l2(rec_f, g["rec_f"]) <= 1e-5
    assert rel_l2(rec_f, golden_demo["rec"][0]) <= 1e-5


def test_packed_apertures():
    rng = np.random.default_rng(3)
    rec = rng.standard_normal((3, 16, 20)).astype(np.float32)
    x0, wn = [0, 5, 12], [20, 7, 8]
    out = fo.records_to_spectra(rec, 5, nt_rows=6, shot_x0=x0, shot_nx=wn)
    off = 0
    for s in range(3):
        blk = out[off:off + 6 * wn[s]].reshape(6, wn[s])
        np.testing.assert_allclose(blk[:5], np.fft.fft(rec[s].astype(np.float64), axis=0)[:5, x0[s]:x0[s] + wn[s]])
        assert np.all(blk[5] == 0)
        off += 6 * wn[s]
