/*
 * Support code linked into oracle/_ref/extrapolation_cpu.so (test infrastructure only).
 *
 * 1. cblas_cdotu_sub / cblas_cgemv: straightforward loops standing in for Intel MKL.
 * 2. Zero-filling operator new[]: the reference's padded-wavefield class allocates with
 *    `new fcomp[n]` and relies on the elements being zero in the halo (cpp_src/wfPad.h:76-84,
 *    100-108, where the explicit zeroing loop runs over `iy < My` with My = 0).  With CUDA 12.9
 *    thrust::complex<float> has a defaulted constructor, so those elements are uninitialised
 *    and the reference produces NaN images.  Returning zeroed storage from operator new[]
 *    gives the value-initialised behaviour the reference was written for, without editing
 *    its sources.  The library is linked with -Bsymbolic so its own calls bind here.
 */
#include <complex>
#include <cstdlib>
#include <new>
#include "mkl.h"

extern "C" void cblas_cdotu_sub(const MKL_INT n, const void *x, const MKL_INT incx,
                                const void *y, const MKL_INT incy, void *dotu)
{
    const std::complex<float> *a = static_cast<const std::complex<float> *>(x);
    const std::complex<float> *b = static_cast<const std::complex<float> *>(y);
    float re = 0.f, im = 0.f;
    for (MKL_INT i = 0; i < n; ++i) {
        std::complex<float> u = a[i * incx], v = b[i * incy];
        re += u.real() * v.real() - u.imag() * v.imag();
        im += u.real() * v.imag() + u.imag() * v.real();
    }
    *static_cast<std::complex<float> *>(dotu) = std::complex<float>(re, im);
}

extern "C" void cblas_cgemv(const CBLAS_LAYOUT layout, const CBLAS_TRANSPOSE trans,
                            const MKL_INT m, const MKL_INT n, const void *alpha, const void *a,
                            const MKL_INT lda, const void *x, const MKL_INT incx,
                            const void *beta, void *y, const MKL_INT incy)
{
    const std::complex<float> al = *static_cast<const std::complex<float> *>(alpha);
    const std::complex<float> be = *static_cast<const std::complex<float> *>(beta);
    const std::complex<float> *A = static_cast<const std::complex<float> *>(a);
    const std::complex<float> *X = static_cast<const std::complex<float> *>(x);
    std::complex<float> *Y = static_cast<std::complex<float> *>(y);
    for (MKL_INT r = 0; r < m; ++r) {
        std::complex<float> acc(0.f, 0.f);
        for (MKL_INT c = 0; c < n; ++c) {
            std::complex<float> av = (layout == CblasRowMajor) ? A[r * lda + c] : A[c * lda + r];
            acc += av * X[c * incx];
        }
        Y[r * incy] = al * acc + be * Y[r * incy];
    }
    (void)trans;
}

void *operator new[](std::size_t n)
{
    void *p = std::calloc(n ? n : 1, 1);
    if (!p) throw std::bad_alloc();
    return p;
}
void operator delete[](void *p) noexcept { std::free(p); }
void operator delete[](void *p, std::size_t) noexcept { std::free(p); }
