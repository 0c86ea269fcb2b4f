"""Mirror of the reference's cpp_src/interface.py for the extrapolation entry points.

Same names, argument order and argument types as cpp_src/interface.py:49-70: `extrapolate` and
`extrapolate_v0` take (ns, nextrap, nz, nx, nf, nt, M, w_op_fs_forw, w_op_fs_back, wave_fs,
shot_fs, image) with complex64/float32 C-contiguous numpy arrays, fill rows [0, nextrap) of every
shot's image, and overwrite wave_fs/shot_fs with the final-depth wavefields
(cpp_src/extrapolation_cpu.cpp:91-99).  They run on the GPU through
libimaging2d_wlsq_b200.so.  Where the reference returns nothing and reports nothing, these raise
`LibraryError` on failure; ctypes still raises ArgumentError on a dtype or flag mismatch, as in
the reference.

The reference module also exposes MKL helpers (mkldot, mklmatvec, c64fft1dforw/back) from its own
mkl_linalg.so and mkl_fft.so; those are not part of the extrapolation path and are not provided.
"""
from ._lib import check, lib


def extrapolate(ns, nextrap, nz, nx, nf, nt, M, w_op_fs_forw, w_op_fs_back, wave_fs, shot_fs, image):
    """cpp_src/extrapolation_cpu.cpp:11-14 on the GPU."""
    check(lib().img2d_extrapolate_host_order(ns, nextrap, nz, nx, nf, nt, M, w_op_fs_forw, w_op_fs_back,
                                             wave_fs, shot_fs, image))


def extrapolate_v0(ns, nextrap, nz, nx, nf, nt, M, w_op_fs_forw, w_op_fs_back, wave_fs, shot_fs, image):
    """cpp_src/extrapolation_cpu.cpp:115-118 (same results as `extrapolate`; the reference keeps it
    only as a slower loop order)."""
    check(lib().img2d_extrapolate_host_order(ns, nextrap, nz, nx, nf, nt, M, w_op_fs_forw, w_op_fs_back,
                                             wave_fs, shot_fs, image))
