"""CPU restatement of the reference's per-shot data preparation (main.py:105-123).

TEST INFRASTRUCTURE ONLY: the checker for imaging2d_wlsq_b200.frontend.  The product never imports it.

  ricker_sources     util.makeRickerWavelet (py_src/operatorsPreparation/util.py:47-58) with the
                     wavelet of util.py:10-14, one source per shot: t - t0 is stored in float32 as the
                     reference's t_t0 array is, the wavelet is evaluated in float64 and stored in
                     float32
  records_to_spectra scipy.fftpack.fft(record, axis=0) of main.py:119/123 restricted to the first nf
                     rows (all the extrapolation reads), in float64, packed per shot aperture
Pinned by tests/test_frontend_oracle.py against tests/golden/frontend_case.npz and demo_case.npz (outputs
of the reference's own code) and against the reference's unit test of makeRickerWavelet
(unittests/test_py_src_util.py:17-50).
"""
import math

import numpy as np


def ricker_sources(ns, nt, nx, dt, x_first, dx, depth_offset, v, src_x, fpeak=30.0):
    out = np.zeros((ns, nt, nx), dtype=np.float32)
    xi = x_first + np.arange(nx, dtype=np.float64) * dx
    tj = np.arange(nt, dtype=np.float64) * dt
    for s in range(ns):
        r = np.sqrt(depth_offset ** 2 + (xi - src_x[s]) ** 2)
        tt = (tj[:, None] - (r / v)[None, :]).astype(np.float32).astype(np.float64)
        term = math.pi * math.pi * fpeak * fpeak * tt * tt
        out[s] = ((1.0 - 2.0 * term) * np.exp(-term) / np.sqrt(r)[None, :]).astype(np.float32)
    return out


def records_to_spectra(records, nf, nt_rows=None, shot_x0=None, shot_nx=None):
    records = np.asarray(records, dtype=np.float64)
    ns, nt, nx = records.shape
    nt_rows = nt_rows or nf
    x0 = np.zeros(ns, dtype=np.int64) if shot_x0 is None else np.asarray(shot_x0, dtype=np.int64)
    wn = np.full(ns, nx, dtype=np.int64) if shot_nx is None else np.asarray(shot_nx, dtype=np.int64)
    out = np.zeros(int(nt_rows * wn.sum()), dtype=np.complex128)
    off = 0
    for s in range(ns):
        spec = np.fft.fft(records[s][:, x0[s]:x0[s] + wn[s]], axis=0)[:nf]
        out[off:off + nf * wn[s]] = spec.reshape(-1)
        off += nt_rows * wn[s]
    return out
