/*
 * wlsq_oracle.c -- CPU restatement of the Imaging2D_WLSQ extrapolation + imaging path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library in
 * imaging2d_wlsq_b200/ and the "port" CPU-baseline arm of bench.py.  Nothing in the
 * product path links, loads or calls it; the product fails loudly when its CUDA
 * library is missing instead of falling back here.
 *
 * Parity pins: the functions below are checked (tests/test_oracle_*.py) against
 *   - every known-answer test of the reference for this path
 *     (unittests/test_cpp_src.py:113-295, unittests/test_cpp_src_cuda.py:23-384,
 *      unittests/test_py_src_extrapolation.py:150-314),
 *   - the reference CPU library itself, compiled from cpp_src/extrapolation_cpu.cpp into
 *     oracle/_ref by oracle/build_ref.sh, on seeded random inputs,
 *   - the reference's shipped end-to-end result demo-result/final_image.csv (through the
 *     committed fixture tests/golden/demo_case.npz).
 *
 * Reference semantics restated (file:line within the reference project):
 *   cpp_src/extrapolation_cpu.cpp:11-107   extrapolate(): depth loop, per-point complex dot of
 *                                           2M+1 taps for source and receiver, ping-pong swap,
 *                                           imaging Re(sum_w F*conj(B)), in-place final write-back
 *   cpp_src/wfPad.h:89-115                  zero halo of width M on both sides of x
 *   cpp_src/mkl_linalg.cpp:7-11             c64dot = unconjugated complex dot (cblas_cdotu_sub)
 *   py_src/operatorsPreparation/util.py:5-8 find_nearest = argmin |kappa - k|, first index on ties
 *   py_src/operatorsPreparation/util.py:39-45 kappa[i] = i*deltak
 *   py_src/operatorsPreparation/preparation.py:101-115 dense table T[l,j,i,:] = table row of
 *                                           find_nearest(kappa, w[j]/v[l,i])
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { float re, im; } cf32;
typedef struct { double re, im; } cf64;

/* find_nearest(kappa, value) with kappa[i] = i*dk (float64), ties -> lowest index.
 * Restates util.py:5-8 (np.argmin of np.abs(kappa - value)) and util.py:43. */
int oracle_nearest_kappa(double value, double dk, int nk)
{
    double q = value / dk;
    long i0;
    if (!(q > 0.0)) i0 = 0;
    else if (q >= (double)(nk - 1)) i0 = nk - 1;
    else i0 = (long)floor(q);
    long lo = i0 - 1, hi = i0 + 2;
    if (lo < 0) lo = 0;
    if (hi > nk - 1) hi = nk - 1;
    long best = lo;
    double bestd = INFINITY;
    for (long i = lo; i <= hi; ++i) {
        double d = fabs((double)i * dk - value);
        if (d < bestd) { bestd = d; best = i; }
    }
    return (int)best;
}

/* ------------------------------------------------------------------------------------
 * Dense-table form, reference argument order of extrapolation_cpu.cpp:11-14.
 *   opF, opB : (nextrap, nf, nx, L) complex64, L = 2M+1
 *   wave, shot: (ns, nt, nx) complex64, first nf rows used; overwritten with final wavefields
 *   image     : (ns, nz, nx) float32, rows [0, nextrap) of each shot overwritten
 * FP32 arithmetic in the reference's loop order (k ascending per dot, w ascending per image
 * point).  One extra leading dimension of work is spread over threads (OpenMP over w),
 * exactly as extrapolation_cpu.cpp:43 does.
 * ----------------------------------------------------------------------------------*/
void oracle_extrapolate_dense_f32(int ns, int nextrap, int nz, int nx, int nf, int nt, int M,
                                  const cf32 *opF, const cf32 *opB, cf32 *wave, cf32 *shot,
                                  float *image)
{
    const int L = 2 * M + 1;
    const long dimx = nx + 2 * M;
    const long pulse = (long)nf * dimx;
    cf32 *of = (cf32 *)calloc((size_t)ns * pulse, sizeof(cf32));
    cf32 *nf_ = (cf32 *)calloc((size_t)ns * pulse, sizeof(cf32));
    cf32 *ob = (cf32 *)calloc((size_t)ns * pulse, sizeof(cf32));
    cf32 *nb = (cf32 *)calloc((size_t)ns * pulse, sizeof(cf32));
    for (int s = 0; s < ns; ++s)
        for (int j = 0; j < nf; ++j)
            for (int i = 0; i < nx; ++i) {
                of[s * pulse + j * dimx + i + M] = wave[(long)s * nt * nx + (long)j * nx + i];
                ob[s * pulse + j * dimx + i + M] = shot[(long)s * nt * nx + (long)j * nx + i];
            }
    for (int l = 0; l < nextrap; ++l) {
        const long depth = (long)l * nf * nx * L;
#pragma omp parallel for schedule(dynamic, 1)
        for (int j = 0; j < nf; ++j) {
            for (int s = 0; s < ns; ++s) {
                for (int i = 0; i < nx; ++i) {
                    const cf32 *tf = opF + depth + ((long)j * nx + i) * L;
                    const cf32 *tb = opB + depth + ((long)j * nx + i) * L;
                    const cf32 *xf = of + s * pulse + j * dimx + i;
                    const cf32 *xb = ob + s * pulse + j * dimx + i;
                    float fr = 0.f, fi = 0.f, br = 0.f, bi = 0.f;
                    for (int k = 0; k < L; ++k) {
                        fr += tf[k].re * xf[k].re - tf[k].im * xf[k].im;
                        fi += tf[k].re * xf[k].im + tf[k].im * xf[k].re;
                        br += tb[k].re * xb[k].re - tb[k].im * xb[k].im;
                        bi += tb[k].re * xb[k].im + tb[k].im * xb[k].re;
                    }
                    nf_[s * pulse + j * dimx + i + M] = (cf32){fr, fi};
                    nb[s * pulse + j * dimx + i + M] = (cf32){br, bi};
                }
            }
        }
        cf32 *t = of; of = nf_; nf_ = t;
        t = ob; ob = nb; nb = t;
        for (int s = 0; s < ns; ++s)
            for (int i = 0; i < nx; ++i) {
                float cr = 0.f, ci = 0.f;
                for (int j = 0; j < nf; ++j) {
                    cf32 a = of[s * pulse + j * dimx + i + M];
                    cf32 b = ob[s * pulse + j * dimx + i + M];
                    cr += a.re * b.re + a.im * b.im;  /* Re(a*conj(b)) */
                    ci += a.im * b.re - a.re * b.im;
                }
                (void)ci;
                image[(long)s * nz * nx + (long)l * nx + i] = cr;
            }
    }
    for (int s = 0; s < ns; ++s)
        for (int j = 0; j < nf; ++j)
            for (int i = 0; i < nx; ++i) {
                wave[(long)s * nt * nx + (long)j * nx + i] = of[s * pulse + j * dimx + i + M];
                shot[(long)s * nt * nx + (long)j * nx + i] = ob[s * pulse + j * dimx + i + M];
            }
    free(of); free(nf_); free(ob); free(nb);
}

/* Same as above in float64 (inputs promoted), image returned as float64. */
void oracle_extrapolate_dense_f64(int ns, int nextrap, int nz, int nx, int nf, int nt, int M,
                                  const cf32 *opF, const cf32 *opB, cf64 *wave, cf64 *shot,
                                  double *image)
{
    const int L = 2 * M + 1;
    const long dimx = nx + 2 * M;
    const long pulse = (long)nf * dimx;
    cf64 *of = (cf64 *)calloc((size_t)ns * pulse, sizeof(cf64));
    cf64 *nf_ = (cf64 *)calloc((size_t)ns * pulse, sizeof(cf64));
    cf64 *ob = (cf64 *)calloc((size_t)ns * pulse, sizeof(cf64));
    cf64 *nb = (cf64 *)calloc((size_t)ns * pulse, sizeof(cf64));
    for (int s = 0; s < ns; ++s)
        for (int j = 0; j < nf; ++j)
            for (int i = 0; i < nx; ++i) {
                of[s * pulse + j * dimx + i + M] = wave[(long)s * nt * nx + (long)j * nx + i];
                ob[s * pulse + j * dimx + i + M] = shot[(long)s * nt * nx + (long)j * nx + i];
            }
    for (int l = 0; l < nextrap; ++l) {
        const long depth = (long)l * nf * nx * L;
#pragma omp parallel for schedule(dynamic, 1)
        for (int j = 0; j < nf; ++j)
            for (int s = 0; s < ns; ++s)
                for (int i = 0; i < nx; ++i) {
                    const cf32 *tf = opF + depth + ((long)j * nx + i) * L;
                    const cf32 *tb = opB + depth + ((long)j * nx + i) * L;
                    const cf64 *xf = of + s * pulse + j * dimx + i;
                    const cf64 *xb = ob + s * pulse + j * dimx + i;
                    double fr = 0, fi = 0, br = 0, bi = 0;
                    for (int k = 0; k < L; ++k) {
                        fr += (double)tf[k].re * xf[k].re - (double)tf[k].im * xf[k].im;
                        fi += (double)tf[k].re * xf[k].im + (double)tf[k].im * xf[k].re;
                        br += (double)tb[k].re * xb[k].re - (double)tb[k].im * xb[k].im;
                        bi += (double)tb[k].re * xb[k].im + (double)tb[k].im * xb[k].re;
                    }
                    nf_[s * pulse + j * dimx + i + M] = (cf64){fr, fi};
                    nb[s * pulse + j * dimx + i + M] = (cf64){br, bi};
                }
        cf64 *t = of; of = nf_; nf_ = t;
        t = ob; ob = nb; nb = t;
        for (int s = 0; s < ns; ++s)
            for (int i = 0; i < nx; ++i) {
                double cr = 0;
                for (int j = 0; j < nf; ++j) {
                    cf64 a = of[s * pulse + j * dimx + i + M];
                    cf64 b = ob[s * pulse + j * dimx + i + M];
                    cr += a.re * b.re + a.im * b.im;
                }
                image[(long)s * nz * nx + (long)l * nx + i] = cr;
            }
    }
    for (int s = 0; s < ns; ++s)
        for (int j = 0; j < nf; ++j)
            for (int i = 0; i < nx; ++i) {
                wave[(long)s * nt * nx + (long)j * nx + i] = of[s * pulse + j * dimx + i + M];
                shot[(long)s * nt * nx + (long)j * nx + i] = ob[s * pulse + j * dimx + i + M];
            }
    free(of); free(nf_); free(ob); free(nb);
}

/* ------------------------------------------------------------------------------------
 * Compact-table form (what the dense tables of preparation.py:101-115 are a gather of).
 *   tabF      : (nk, L) forward rows; the dense table is T[l,j,i,:] = tabF[idx(l,j,i)]
 *   tabB      : (nk, L) receiver rows, or NULL to use conj(tabF) (exact in exact arithmetic
 *               for a symmetric kx grid, preparation.py:10-44)
 *   idx(l,j,i) = find_nearest(kappa, omega[j] / vel[l, i])        (util.py:5-8)
 *   shot s lives on the window [x0[s], x0[s] + wnx[s]) of the model grid, zero outside
 *   (x0 == NULL: full aperture).  wave/shot are packed: block s has nt rows of wnx[s]
 *   samples, block offsets given by woff[s] (elements).
 *   image_shots (optional, (ns, nz, nx) float64) and image_stack ((nz, nx) float64, summed
 *   over shots) receive rows [0, nextrap); other rows untouched.
 * Arithmetic is float64 throughout (the FP64 oracle of the precision study).
 * Work over (shot, w) pairs is spread over threads; each pair is independent.
 * ----------------------------------------------------------------------------------*/
void oracle_migrate_compact_f64(int ns, int nextrap, int nz, int nx, int nf, int nt, int M,
                                int nk, double dk, const double *omega, const double *vel,
                                const cf32 *tabF, const cf32 *tabB,
                                const int *x0, const int *wnx, const long *woff,
                                cf64 *wave, cf64 *shot, double *image_shots, double *image_stack)
{
    const int L = 2 * M + 1;
    const long npair = (long)ns * nf;
    /* per-pair image rows are accumulated in a private buffer then reduced, so the result
     * does not depend on the thread count */
    double *img = (double *)calloc((size_t)ns * nextrap * nx, sizeof(double));
    int *idx = (int *)malloc((size_t)nf * nextrap * nx * sizeof(int));
    for (int j = 0; j < nf; ++j)
        for (int l = 0; l < nextrap; ++l)
            for (int i = 0; i < nx; ++i)
                idx[((long)j * nextrap + l) * nx + i] =
                    oracle_nearest_kappa(omega[j] / vel[(long)l * nx + i], dk, nk);
    int nthreads = 1;
#ifdef _OPENMP
    nthreads = omp_get_max_threads();
#endif
    double *priv = (double *)calloc((size_t)nthreads * ns * nextrap * nx, sizeof(double));
#pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *mine = priv + (size_t)tid * ns * nextrap * nx;
        int maxw = nx + 2 * M;
        cf64 *f0 = (cf64 *)calloc(maxw, sizeof(cf64)), *f1 = (cf64 *)calloc(maxw, sizeof(cf64));
        cf64 *b0 = (cf64 *)calloc(maxw, sizeof(cf64)), *b1 = (cf64 *)calloc(maxw, sizeof(cf64));
#pragma omp for schedule(dynamic, 1)
        for (long p = 0; p < npair; ++p) {
            int s = (int)(p / nf), j = (int)(p % nf);
            int xs = x0 ? x0[s] : 0;
            int w = wnx ? wnx[s] : nx;
            long base = woff ? woff[s] : (long)s * nt * nx;
            memset(f0, 0, maxw * sizeof(cf64)); memset(f1, 0, maxw * sizeof(cf64));
            memset(b0, 0, maxw * sizeof(cf64)); memset(b1, 0, maxw * sizeof(cf64));
            for (int i = 0; i < w; ++i) {
                f0[i + M] = wave[base + (long)j * w + i];
                b0[i + M] = shot[base + (long)j * w + i];
            }
            for (int l = 0; l < nextrap; ++l) {
                const int *ix = idx + ((long)j * nextrap + l) * nx + xs;
                for (int i = 0; i < w; ++i) {
                    const cf32 *tf = tabF + (long)ix[i] * L;
                    const cf32 *tb = tabB ? tabB + (long)ix[i] * L : NULL;
                    double fr = 0, fi = 0, br = 0, bi = 0;
                    for (int k = 0; k < L; ++k) {
                        double tr = tf[k].re, ti = tf[k].im;
                        double ur = tb ? (double)tb[k].re : tr, ui = tb ? (double)tb[k].im : -ti;
                        fr += tr * f0[i + k].re - ti * f0[i + k].im;
                        fi += tr * f0[i + k].im + ti * f0[i + k].re;
                        br += ur * b0[i + k].re - ui * b0[i + k].im;
                        bi += ur * b0[i + k].im + ui * b0[i + k].re;
                    }
                    f1[i + M] = (cf64){fr, fi};
                    b1[i + M] = (cf64){br, bi};
                }
                cf64 *t = f0; f0 = f1; f1 = t;
                t = b0; b0 = b1; b1 = t;
                double *row = mine + ((long)s * nextrap + l) * nx + xs;
                for (int i = 0; i < w; ++i)
                    row[i] += f0[i + M].re * b0[i + M].re + f0[i + M].im * b0[i + M].im;
            }
            for (int i = 0; i < w; ++i) {
                wave[base + (long)j * w + i] = f0[i + M];
                shot[base + (long)j * w + i] = b0[i + M];
            }
        }
        free(f0); free(f1); free(b0); free(b1);
    }
    for (int t = 0; t < nthreads; ++t)
        for (long e = 0; e < (long)ns * nextrap * nx; ++e)
            img[e] += priv[(size_t)t * ns * nextrap * nx + e];
    for (int s = 0; s < ns; ++s)
        for (int l = 0; l < nextrap; ++l)
            for (int i = 0; i < nx; ++i) {
                double v = img[((long)s * nextrap + l) * nx + i];
                if (image_shots) image_shots[(long)s * nz * nx + (long)l * nx + i] = v;
            }
    if (image_stack)
        for (int l = 0; l < nextrap; ++l)
            for (int i = 0; i < nx; ++i) {
                double acc = 0;
                for (int s = 0; s < ns; ++s) acc += img[((long)s * nextrap + l) * nx + i];
                image_stack[(long)l * nx + i] = acc;
            }
    free(priv); free(img); free(idx);
}

/* Gather one depth slab of the dense table from the compact table:
 * out[(l-l0), j, i, :] = tab[find_nearest(omega[j]/vel[l, x0+i])] for l in [l0, l0+nl),
 * i in [0, w).  This is the dense table preparation.py:101-115 builds, restricted to a slab
 * and an x-window; used to drive the reference's own dense-table library in tests and in
 * the CPU baseline. */
void oracle_gather_dense_slab(int l0, int nl, int nx, int x0, int w, int nf, int M,
                              int nk, double dk, const double *omega, const double *vel,
                              const cf32 *tab, int conj_rows, cf32 *out)
{
    const int L = 2 * M + 1;
#pragma omp parallel for schedule(static)
    for (int l = 0; l < nl; ++l)
        for (int j = 0; j < nf; ++j)
            for (int i = 0; i < w; ++i) {
                int r = oracle_nearest_kappa(omega[j] / vel[(long)(l0 + l) * nx + x0 + i], dk, nk);
                cf32 *dst = out + (((long)l * nf + j) * w + i) * L;
                const cf32 *src = tab + (long)r * L;
                for (int k = 0; k < L; ++k) {
                    dst[k] = src[k];
                    if (conj_rows) dst[k].im = -dst[k].im;
                }
            }
}

/* Index table idx[j][l][i] = find_nearest(kappa, omega[j]/vel[l, i]) (int32), for tests of
 * the device index computation. */
void oracle_index_table(int nextrap, int nx, int nf, int nk, double dk, const double *omega,
                        const double *vel, int *out)
{
#pragma omp parallel for schedule(static)
    for (int j = 0; j < nf; ++j)
        for (int l = 0; l < nextrap; ++l)
            for (int i = 0; i < nx; ++i)
                out[((long)j * nextrap + l) * nx + i] =
                    oracle_nearest_kappa(omega[j] / vel[(long)l * nx + i], dk, nk);
}

/* ------------------------------------------------------------------------------------
 * Demigration (the adjoint of oracle_migrate_compact_f64 with respect to the receiver
 * spectra, single-table mode: receiver rows conj(tabF)).  No reference counterpart: the
 * reference only migrates.  For the real inner products <I, m> = sum I*m and
 * <u, v> = Re sum u*conj(v) this returns data = F* m such that
 *     <F d, m> = Re sum d * conj(F* m)
 * for the migration F of extrapolation_cpu.cpp:39-89 (source S fixed, receiver d):
 *     V_{n-1} = m_{n-1} S_n;   U_l = A_l^T V_l;   V_{l-1} = U_l + m_{l-1} S_l;   F* m = U_0,
 * where (A_l^T V)[i] = sum_k T(l, i')[k] V[i'], i' = i + M - k, inside the shot window (the
 * transpose of the zero-halo gather).  The source wavefield of every depth is kept in memory
 * (small test cases only).  refl: (nextrap, nx) float64; data: packed like wave, rows [0, nf)
 * of every shot block written.  Float64 throughout.
 * ----------------------------------------------------------------------------------*/
void oracle_demigrate_compact_f64(int ns, int nextrap, int nx, int nf, int nt, int M, int nk, double dk,
                                  const double *omega, const double *vel, const cf32 *tabF,
                                  const int *x0, const int *wnx, const long *woff,
                                  const cf64 *wave, const double *refl, cf64 *data)
{
    const int L = 2 * M + 1;
    const long npair = (long)ns * nf;
    int *idx = (int *)malloc((size_t)nf * nextrap * nx * sizeof(int));
    for (int j = 0; j < nf; ++j)
        for (int l = 0; l < nextrap; ++l)
            for (int i = 0; i < nx; ++i)
                idx[((long)j * nextrap + l) * nx + i] =
                    oracle_nearest_kappa(omega[j] / vel[(long)l * nx + i], dk, nk);
#pragma omp parallel
    {
        cf64 *S = (cf64 *)malloc((size_t)(nextrap + 1) * nx * sizeof(cf64));
        cf64 *V = (cf64 *)malloc((size_t)nx * sizeof(cf64));
        cf64 *U = (cf64 *)malloc((size_t)nx * sizeof(cf64));
#pragma omp for schedule(dynamic, 1)
        for (long p = 0; p < npair; ++p) {
            int s = (int)(p / nf), j = (int)(p % nf);
            int xs = x0 ? x0[s] : 0;
            int w = wnx ? wnx[s] : nx;
            long base = woff ? woff[s] : (long)s * nt * nx;
            for (int i = 0; i < w; ++i) S[i] = wave[base + (long)j * w + i];
            for (int l = 0; l < nextrap; ++l) {
                const int *ix = idx + ((long)j * nextrap + l) * nx + xs;
                const cf64 *cur = S + (long)l * w;
                cf64 *nxt = S + (long)(l + 1) * w;
                for (int i = 0; i < w; ++i) {
                    const cf32 *t = tabF + (long)ix[i] * L;
                    double re = 0, im = 0;
                    for (int k = 0; k < L; ++k) {
                        int ii = i + k - M;
                        if (ii < 0 || ii >= w) continue;
                        re += (double)t[k].re * cur[ii].re - (double)t[k].im * cur[ii].im;
                        im += (double)t[k].re * cur[ii].im + (double)t[k].im * cur[ii].re;
                    }
                    nxt[i] = (cf64){re, im};
                }
            }
            {
                const double *m = refl + (long)(nextrap - 1) * nx + xs;
                const cf64 *Sn = S + (long)nextrap * w;
                for (int i = 0; i < w; ++i) V[i] = (cf64){m[i] * Sn[i].re, m[i] * Sn[i].im};
            }
            for (int l = nextrap - 1; l >= 0; --l) {
                const int *ix = idx + ((long)j * nextrap + l) * nx + xs;
                for (int i = 0; i < w; ++i) {
                    double re = 0, im = 0;
                    for (int k = 0; k < L; ++k) {
                        int ii = i + M - k;
                        if (ii < 0 || ii >= w) continue;
                        const cf32 *t = tabF + (long)ix[ii] * L + k;
                        re += (double)t->re * V[ii].re - (double)t->im * V[ii].im;
                        im += (double)t->re * V[ii].im + (double)t->im * V[ii].re;
                    }
                    U[i] = (cf64){re, im};
                }
                if (l > 0) {
                    const double *m = refl + (long)(l - 1) * nx + xs;
                    const cf64 *Sl = S + (long)l * w;
                    for (int i = 0; i < w; ++i) V[i] = (cf64){U[i].re + m[i] * Sl[i].re, U[i].im + m[i] * Sl[i].im};
                } else {
                    for (int i = 0; i < w; ++i) data[base + (long)j * w + i] = U[i];
                }
            }
        }
        free(S); free(V); free(U);
    }
    free(idx);
}
