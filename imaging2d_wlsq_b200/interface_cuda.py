"""Mirror of the reference's cpp_src/interface_cuda.py.

Same names and device argument order as cpp_src/interface_cuda.py:17-52:
(ns, nextrap, nz, nt, nf, nx, M, w_op_forw, forw_pulse, w_op_back, back_pulse, image).

  extrapolate           cpp_src/extrapolation_gpu.cu:74-76; image only, the wavefields are left
                        untouched (that library never copies them back).
  extrapolate_revOp     cpp_src/extrapolation_revOp_gpu.cu:78-80; also writes the final-depth
                        wavefields back into forw_pulse/back_pulse.
  extrapolate_sh_revOp  cpp_src/extrapolation_sh_revOp_gpu.cu:87-89; as extrapolate_revOp.

The write-back uses the shot stride nt*nx of the input layout for every shot (the reference's
revOp/sh_revOp libraries use nf*(nx+2M), extrapolation_revOp_gpu.cu:189-190, which writes outside
the caller's array for ns > 1); for ns = 1 the results are identical.
"""
from ._lib import check, lib


def extrapolate(ns, nextrap, nz, nt, nf, nx, M, w_op_forw, forw_pulse, w_op_back, back_pulse, image):
    check(lib().img2d_extrapolate_device_order(ns, nextrap, nz, nt, nf, nx, M, w_op_forw, forw_pulse,
                                               w_op_back, back_pulse, image, 0))


def extrapolate_revOp(ns, nextrap, nz, nt, nf, nx, M, w_op_forw, forw_pulse, w_op_back, back_pulse, image):
    check(lib().img2d_extrapolate_device_order(ns, nextrap, nz, nt, nf, nx, M, w_op_forw, forw_pulse,
                                               w_op_back, back_pulse, image, 1))


def extrapolate_sh_revOp(ns, nextrap, nz, nt, nf, nx, M, w_op_forw, forw_pulse, w_op_back, back_pulse, image):
    check(lib().img2d_extrapolate_device_order(ns, nextrap, nz, nt, nf, nx, M, w_op_forw, forw_pulse,
                                               w_op_back, back_pulse, image, 1))
