"""Front end: source wavelets and receiver spectra on the device, in the migration's input layout.

Mirrors the per-shot preparation of the reference driver (main.py:105-123):

    pulse_forw_st[s] = util.makeRickerWavelet([xmin + shot_isx[s]*dx], zinit, nt, nx, tj, xi, dz, v)
    pulse_forw_fs[s] = scipy.fftpack.fft(pulse_forw_st[s], axis=0)
    pulse_back_st[s] = <the shot's CSV record>
    pulse_back_fs[s] = scipy.fftpack.fft(pulse_back_st[s], axis=0)

with tj = j*dt, xi = xmin + (i+1)*dx and v = velocity[0, 0] (main.py:111-113).  The wavelet and the
transform run as CUDA kernels (img2d_ricker_sources, img2d_records_to_spectra); only the first nf
frequency rows, the ones the extrapolation uses, are computed, straight into the packed per-shot
aperture layout of migration.Plan.
"""
import ctypes

import numpy as np

from ._lib import check, lib, ptr


def ricker_sources(ns, nt, nx, dt, x_first, dx, depth_offset, v, src_x, fpeak=30.0, device=None):
    """Time-domain source wavelets (ns, nt, nx) float32 on the device (util.py:47-58 semantics)."""
    import torch
    dev = device or torch.device("cuda")
    out = torch.empty((ns, nt, nx), dtype=torch.float32, device=dev)
    sx = np.ascontiguousarray(src_x, dtype=np.float64)
    if sx.shape != (ns,):
        raise ValueError("src_x must have one position per source")
    check(lib().img2d_ricker_sources(ns, nt, nx, float(dt), float(x_first), float(dx), float(depth_offset),
                                     float(v), float(fpeak), sx.ctypes.data, ptr(out),
                                     ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))
    return out


def records_to_spectra(records, nf, nt_rows=None, shot_x0=None, shot_nx=None, out=None):
    """First nf rows of the DFT along time of device records (ns, nt, nx) float32, packed per shot
    aperture with nt_rows rows per shot (default nf).  Returns the complex64 device vector."""
    import torch
    if records.dtype != torch.float32 or records.dim() != 3 or not records.is_cuda:
        raise TypeError("records must be a CUDA float32 tensor (ns, nt, nx)")
    records = records.contiguous()
    ns, nt, nx = records.shape
    nt_rows = nt_rows or nf
    x0 = None if shot_x0 is None else np.ascontiguousarray(shot_x0, dtype=np.int32)
    wn = None if shot_nx is None else np.ascontiguousarray(shot_nx, dtype=np.int32)
    widths = np.full(ns, nx, dtype=np.int64) if wn is None else wn.astype(np.int64)
    total = int(nt_rows * widths.sum())
    if out is None:
        out = torch.zeros(total, dtype=torch.complex64, device=records.device)
    elif out.numel() < total or out.dtype != torch.complex64:
        raise ValueError("out is too small or not complex64")
    check(lib().img2d_records_to_spectra(ns, nt, nx, int(nf), int(nt_rows), ptr(records),
                                         None if x0 is None else x0.ctypes.data,
                                         None if wn is None else wn.ctypes.data, ptr(out),
                                         ctypes.c_void_p(torch.cuda.current_stream(records.device).cuda_stream)))
    return out


def prepare_shots(records, shot_isx, nf, xmin, dx, dt, zinit, dz, v, fpeak=30.0, nt_rows=None):
    """Source and receiver spectra of main.py:105-123 for device records (ns, nt, nx) float32 and
    the shots' source indices.  Returns (wave, shot): packed complex64 device vectors with
    nt_rows (default nf) rows per shot, full aperture, ready for migration.Plan.execute."""
    ns, nt, nx = records.shape
    sx = xmin + np.asarray(shot_isx, dtype=np.float64) * dx
    src_t = ricker_sources(ns, nt, nx, dt, xmin + dx, dx, dz - zinit, v, sx, fpeak=fpeak, device=records.device)
    wave = records_to_spectra(src_t, nf, nt_rows=nt_rows)
    del src_t
    shot = records_to_spectra(records, nf, nt_rows=nt_rows)
    return wave, shot
