// Front end of the migration: source wavelets and frequency-domain records on the device.
//
// Reference (file:line within the reference project ahadji05/Imaging2D_WLSQ):
//   main.py:111-123           per shot: Ricker source wavelet sampled on (nt, nx), receiver record read
//                             from CSV, both transformed along time with scipy.fftpack.fft (axis 0);
//                             the extrapolation then uses the first nw frequency rows
//   py_src/operatorsPreparation/util.py:10-14   ricker_wv_map(t) = (1 - 2 pi^2 f^2 t^2) exp(-pi^2 f^2 t^2),
//                             f = 30 Hz
//   py_src/operatorsPreparation/util.py:47-58   makeRickerWavelet: r = sqrt((init_depth - isz)^2 +
//                             (xi - sx)^2), t0 = r / v, t_t0 = tj - t0 stored as float32, wavelet[j, i] =
//                             ricker(t_t0[j]) / sqrt(r), accumulated into a float32 array
//
// The transform along time is a batched single-precision real-to-complex cuFFT per group of shots
// (the reference's scipy.fftpack.fft of float32 records is a single-precision transform too); a
// kernel then packs the first nf rows of every shot's aperture into the layout the migration plan
// consumes.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "wlsq_kernels.cuh"

namespace img2d {

// out[s][j][i] (float32, time domain) for ns sources at sx[s] (model x in metres).
__global__ void ricker_sources_kernel(int ns, int nt, int nx, double dt, double x_first, double dx, double dzr,
                                      double v, double fpeak, const double *__restrict__ sx,
                                      float *__restrict__ out)
{
    const long long total = (long long)ns * nt * nx;
    const double pf2 = 9.869604401089358 * fpeak * fpeak;  // pi^2 f^2
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % nx);
        const long long r0 = e / nx;
        const int j = (int)(r0 % nt);
        const int s = (int)(r0 / nt);
        const double xi = x_first + i * dx;
        const double ddx = xi - sx[s];
        const double r = sqrt(dzr * dzr + ddx * ddx);
        const float tt = (float)((double)j * dt - r / v);  // the reference keeps t - t0 in float32
        const double term = pf2 * (double)tt * (double)tt;
        out[e] = (float)((1.0 - 2.0 * term) * exp(-term) / sqrt(r));
    }
}

// Packs the first nf rows of real-to-complex spectra into the migration's per-shot aperture layout.
// spec: (nsc, nt/2+1, nx) complex, the transforms along time of shots s0 .. s0+nsc-1; row j of the
// full spectrum is spec row j for j <= nt/2 and conj(spec row nt-j) above (real input).
// out: shot s's block at off[s], row j, column x - x0[s] for x in [x0[s], x0[s] + w[s]).
__global__ void pack_spectra_kernel(int s0, int nsc, int nt, int nx, int nf, const cpx *__restrict__ spec,
                                    const int *__restrict__ x0, const int *__restrict__ w,
                                    const long long *__restrict__ off, cpx *__restrict__ out)
{
    const int nh = nt / 2 + 1;
    const long long total = (long long)nsc * nf * nx;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(e % nx);
        const long long r = e / nx;
        const int j = (int)(r % nf);
        const int sl = (int)(r / nf);
        const int s = s0 + sl;
        const int xs = x0[s], ws = w[s];
        if (x < xs || x >= xs + ws) continue;
        cpx v;
        if (j < nh) {
            v = spec[((long long)sl * nh + j) * nx + x];
        } else {
            const cpx c = spec[((long long)sl * nh + (nt - j)) * nx + x];
            v = cpx{c.re, -c.im};
        }
        out[off[s] + (long long)j * ws + (x - xs)] = v;
    }
}

}  // namespace img2d
