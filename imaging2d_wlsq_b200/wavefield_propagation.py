"""Mirror of the reference's Python extrapolation (py_src/wavefieldPropagation/extrapolation.py:38-66).

extrapolate(nextrap, nz, nx, nf, M, w_op_fs_forw, w_op_fs_back, wave_fs, shot_fs) -> image (nz, nx)
float32 for one shot, with the reference's arguments and result: dense operator tables
(nextrap, nf, nx, 2M+1), wavefields (nt, nx) of which the first nf rows are extrapolated, image rows
[0, nextrap) = Re sum_w S conj(R) after each depth step, the other rows zero; the caller's wavefields
are not modified.  It runs on the B200 through the dense-table entry point.  Differences: complex128
inputs are computed in FP32 (the reference's numba code keeps their dtype), and nz < nextrap raises
ValueError (the reference prints a message and fails later).
"""
import numpy as np

from ._lib import check, lib


def extrapolate(nextrap, nz, nx, nf, M, w_op_fs_forw, w_op_fs_back, wave_fs, shot_fs):
    if nz < nextrap:
        raise ValueError("nz must be equal or greater than nextrap")
    L = 2 * M + 1
    op_f = np.ascontiguousarray(w_op_fs_forw, dtype=np.complex64)
    op_b = np.ascontiguousarray(w_op_fs_back, dtype=np.complex64)
    if op_f.shape[:4] != (nextrap, nf, nx, L) or op_b.shape != op_f.shape:
        raise ValueError(f"operator tables must be ({nextrap}, {nf}, {nx}, {L})")
    wave = np.array(wave_fs, dtype=np.complex64, order="C", copy=True)
    shot = np.array(shot_fs, dtype=np.complex64, order="C", copy=True)
    if wave.ndim != 2 or wave.shape[1] != nx or wave.shape[0] < nf or shot.shape != wave.shape:
        raise ValueError(f"wavefields must be (nt >= {nf}, {nx}) and of equal shape")
    nt = wave.shape[0]
    image = np.zeros((1, nz, nx), dtype=np.float32)
    check(lib().img2d_extrapolate_host_order(1, nextrap, nz, nx, nf, nt, M, op_f, op_b, wave, shot, image))
    return image[0]
