/*
 * Drop-in shims: one small shared library per reference library, each exporting the reference's
 * void `extrapolate` symbol (and `extrapolate_v0` for the host library) with the reference's
 * argument order, forwarding to libimaging2d_wlsq_b200.so.  Built four times by
 * imaging2d_wlsq_b200/build.py:
 *   extrapolation_cpu.so           IMG2D_DROPIN_HOST      cpp_src/extrapolation_cpu.cpp:11-14, :115-118
 *   extrapolation_gpu.so           IMG2D_DROPIN_DEVICE=0  cpp_src/extrapolation_gpu.cu:74-76 (no write-back)
 *   extrapolation_revOp_gpu.so     IMG2D_DROPIN_DEVICE=1  cpp_src/extrapolation_revOp_gpu.cu:78-80
 *   extrapolation_sh_revOp_gpu.so  IMG2D_DROPIN_DEVICE=1  cpp_src/extrapolation_sh_revOp_gpu.cu:87-89
 * The reference ABI returns void and has no error channel; a failure prints the library's error
 * text to stderr and aborts rather than returning unfilled outputs.
 */
#include <stdio.h>
#include <stdlib.h>
#include "../../include/imaging2d_wlsq_b200.h"

static void img2d_dropin_check(int rc)
{
    if (rc != IMG2D_OK) {
        fprintf(stderr, "imaging2d_wlsq_b200: extrapolate failed (code %d): %s\n", rc, img2d_last_error());
        abort();
    }
}

#ifdef IMG2D_DROPIN_HOST
void extrapolate(int ns, int nextrap, int nz, int nx, int nf, int nt, int M, img2d_c64 *w_op_fs_forw,
                 img2d_c64 *w_op_fs_back, img2d_c64 *wave_fs, img2d_c64 *shot_fs, float *image)
{
    img2d_dropin_check(img2d_extrapolate_host_order(ns, nextrap, nz, nx, nf, nt, M, w_op_fs_forw, w_op_fs_back,
                                                    wave_fs, shot_fs, image));
}

void extrapolate_v0(int ns, int nextrap, int nz, int nx, int nf, int nt, int M, img2d_c64 *w_op_fs_forw,
                    img2d_c64 *w_op_fs_back, img2d_c64 *wave_fs, img2d_c64 *shot_fs, float *image)
{
    img2d_dropin_check(img2d_extrapolate_host_order(ns, nextrap, nz, nx, nf, nt, M, w_op_fs_forw, w_op_fs_back,
                                                    wave_fs, shot_fs, image));
}
#endif

#ifdef IMG2D_DROPIN_DEVICE
void extrapolate(int ns, int nextrap, int nz, int nt, int nf, int nx, int M, img2d_c64 *w_op_forw,
                 img2d_c64 *forw_pulse, img2d_c64 *w_op_back, img2d_c64 *back_pulse, float *image)
{
    img2d_dropin_check(img2d_extrapolate_device_order(ns, nextrap, nz, nt, nf, nx, M, w_op_forw, forw_pulse,
                                                      w_op_back, back_pulse, image, IMG2D_DROPIN_DEVICE));
}
#endif
