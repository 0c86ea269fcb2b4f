/*
 * imaging2d_wlsq_b200.h -- C ABI of the B200 extrapolation + imaging library.
 *
 * Library: imaging2d_wlsq_b200/libimaging2d_wlsq_b200.so (CUDA, sm_100a).
 * Drop-in shims with the reference's library names and its void `extrapolate` symbols are
 * built into imaging2d_wlsq_b200/dropin/ (csrc/dropin.c).
 *
 * Data conventions shared by every entry point:
 *   img2d_c64   interleaved (re, im) float32 pair, the layout of numpy.complex64 and of the
 *               reference's `fcomp` = thrust::complex<float> (cpp_src/types.h:9).
 *   All arrays are C-contiguous.  Host-pointer entry points copy to and from the current CUDA
 *   device inside the call and return when the results are back in host memory.
 *   Every int-returning function returns IMG2D_OK (0) or an IMG2D_E* code; the text of the last
 *   failure on the calling thread is available from img2d_last_error().
 */
#ifndef IMAGING2D_WLSQ_B200_H
#define IMAGING2D_WLSQ_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    float re, im;
} img2d_c64;

#define IMG2D_OK 0
#define IMG2D_EINVAL 1   /* invalid dimensions or pointers */
#define IMG2D_ENOMEM 2   /* device allocation failed */
#define IMG2D_ECUDA 3    /* a CUDA runtime call or kernel launch failed */
#define IMG2D_ENODEV 4   /* no CUDA device visible */

/* flags for the compact-table entry points */
#define IMG2D_FLAG_TWO_TABLES 1   /* use tab_back for the receiver instead of conj(tab_forw) */
#define IMG2D_FLAG_GENERIC 2      /* force the runtime-length kernel (testing) */
#define IMG2D_FLAG_NO_CLUSTER 4   /* use the single-CTA kernels even where the cluster kernel applies */
#define IMG2D_FLAG_CLUSTER_V1 8   /* first-generation cluster kernel (256 threads, fixed L) instead */
#define IMG2D_FLAG_TABLE_FP16 16  /* operator table stored as FP16 (re, im) pairs, arithmetic FP32 */
#define IMG2D_FLAG_TABLE_BF16 32  /* operator table stored as BF16 (re, im) pairs, arithmetic FP32 */
#define IMG2D_FLAG_DEMIG_NO_RING 64 /* demigration: forward steps read operator pairs through L1, not the ring */
#define IMG2D_FLAG_WIDE 128        /* wide cluster kernel: 8 slots x 1024 positions per CTA (packed FMAs) */
#define IMG2D_FLAG_WIDE_SCALAR (1 << 16) /* the wide cluster kernel with scalar instead of packed FMAs */
#define IMG2D_FLAG_CLUSTER2 (1 << 17)    /* 16-slot cluster kernel (512 positions per CTA) instead */
/* the wide cluster kernel (packed FMAs) with its operator-pair ring filled by 1-D bulk copies
 * (cp.async.bulk, completing on per-warp transaction barriers) instead of 16-byte cp.async */
#define IMG2D_FLAG_WIDE_BULK (1 << 18)
/* wide cluster kernel: keep the line packing of the other kernels (shots chained into lane-slot
 * lines across the model, lines grouped by extent) instead of the window-first packing, which the
 * plan otherwise uses where its modelled cost is lower */
#define IMG2D_FLAG_LINE_PACKING (1 << 19)
/* Default kernel choice: the wide cluster kernel where the 16-slot kernel's clusters would leave
 * SMs idle (or fewer than 12 lane slots), else the 16-slot cluster kernel; the single-CTA kernels
 * for fewer than 6 lane slots, operators shorter than 7 taps or windows beyond 16 CTAs. */
/* select variant v (1-based; 0 = default) of the second-generation cluster kernel: bits 8-15 */
#define IMG2D_FLAG_VARIANT_SHIFT 8
#define IMG2D_FLAG_VARIANT(v) ((v) << IMG2D_FLAG_VARIANT_SHIFT)

const char *img2d_last_error(void);
int img2d_version(void);

/* Failure injection for tests of the error path (no counterpart in the reference, which checks no
 * allocation).  Every device allocation of the library larger than max_bytes then fails with
 * IMG2D_ENOMEM on the host, before cudaMalloc is called; 0 removes the limit.  Until this is
 * called the limit comes from the environment variable IMG2D_ALLOC_LIMIT_BYTES (unset: none), so
 * it also reaches callers of the void drop-in shims, which then print the error and abort. */
void img2d_set_alloc_limit(size_t max_bytes);

/* ------------------------------------------------------------------------------------------
 * Drop-in entry points: the reference's dense-table ABI.
 * opF/opB are dense operator tables (nextrap, nf, nx, 2M+1); wavefields are (ns, nt, nx) with the
 * first nf rows used; image is (ns, nz, nx) float32 and rows [0, nextrap) of every shot are
 * overwritten with Re(sum_w S conj R).
 * ---------------------------------------------------------------------------------------- */

/* Replaces `extrapolate` and `extrapolate_v0` of cpp_src/extrapolation_cpu.cpp:11-14 and :115-118
 * (bound in cpp_src/interface.py:50-70).  Host argument order.  wave_fs and shot_fs are
 * overwritten with the final-depth wavefields (extrapolation_cpu.cpp:91-99). */
int img2d_extrapolate_host_order(int ns, int nextrap, int nz, int nx, int nf, int nt, int M,
                                 const img2d_c64 *op_forw, const img2d_c64 *op_back,
                                 img2d_c64 *wave_fs, img2d_c64 *shot_fs, float *image);

/* Replaces `extrapolate` of cpp_src/extrapolation_gpu.cu:74-76 (write_back = 0, that library does
 * not write the wavefields back), cpp_src/extrapolation_revOp_gpu.cu:78-80 and
 * cpp_src/extrapolation_sh_revOp_gpu.cu:87-89 (write_back = 1), bound in
 * cpp_src/interface_cuda.py:17-52.  Device argument order.  With write_back the final-depth
 * wavefields go to forw_pulse/back_pulse with shot stride nt*nx. */
int img2d_extrapolate_device_order(int ns, int nextrap, int nz, int nt, int nf, int nx, int M,
                                   const img2d_c64 *op_forw, img2d_c64 *forw_pulse,
                                   const img2d_c64 *op_back, img2d_c64 *back_pulse, float *image,
                                   int write_back);

/* ------------------------------------------------------------------------------------------
 * Compact-table entry point (replaces the dense-table gather of
 * py_src/operatorsPreparation/preparation.py:101-115 followed by the call of main.py:153-160).
 *   omega[nf]            angular frequencies w[j] (float64)
 *   velocity[nz*nx]      velocity model (float64), rows [0, nextrap) used
 *   tab_forw[nk*(2M+1)]  row i = forward WLSQ operator for kappa[i] = i*dk
 *   tab_back             row i = receiver operator, read only with IMG2D_FLAG_TWO_TABLES
 *   shot_x0, shot_nx     per-shot aperture [x0, x0+nx_s) inside [0, nx); NULL = full aperture
 *   wave_fs, shot_fs     packed per-shot blocks of nt rows x nx_s samples (first nf rows used),
 *                        blocks in shot order; overwritten with the final-depth wavefields
 *   image[nz*nx]         stacked image (sum over shots), rows [0, nextrap) overwritten; may be NULL
 *   image_shots          per-shot images (ns, nz, nx), rows [0, nextrap) overwritten; may be NULL
 * The operator for (depth l, frequency j, position x) is row find_nearest(kappa, w[j]/v[l,x])
 * (py_src/operatorsPreparation/util.py:5-8), evaluated in float64 on the device.
 * ---------------------------------------------------------------------------------------- */
int img2d_migrate_compact(int ns, int nextrap, int nz, int nx, int nf, int nt, int M, int nk,
                          double dk, const double *omega, const double *velocity,
                          const img2d_c64 *tab_forw, const img2d_c64 *tab_back,
                          const int *shot_x0, const int *shot_nx, img2d_c64 *wave_fs,
                          img2d_c64 *shot_fs, float *image, float *image_shots, int flags);
/* img2d_migrate_compact keeps, per device, its plan (for the last geometry on that device) and its
 * device buffers (grown to the largest sizes seen) between calls, so repeated calls allocate
 * nothing.  img2d_release_host_cache frees them on every device; img2d_host_cache_device_count
 * is the number of devices that hold such a cache.
 * With 64 MiB of wavefields or more (and no per-shot images) a call runs in 8 frequency chunks: the
 * host copies of each chunk overlap the kernels of the others (pinned host memory overlaps fully),
 * on streams of its own, with a second set of per-CTA image partials.  It returns when everything
 * is back in host memory, like a call in one piece. */
void img2d_release_host_cache(void);
int img2d_host_cache_device_count(void);

/* ------------------------------------------------------------------------------------------
 * Plan interface for device-resident data (the building block under the host entry points).
 * A plan fixes the geometry (dimensions, apertures) and owns its device workspace.
 * ---------------------------------------------------------------------------------------- */
typedef struct img2d_plan img2d_plan;

int img2d_plan_create(img2d_plan **plan, int ns, int nextrap, int nz, int nx, int nf, int nt,
                      int M, int nk, const int *shot_x0, const int *shot_nx, int flags);
/* Device pointers.  Copies the tables into the plan (rows padded for 16-byte loads) and builds
 * the operator index table for (omega, velocity, dk).  stream: cudaStream_t or NULL. */
int img2d_plan_set_model(img2d_plan *plan, const double *d_omega, const double *d_velocity,
                         double dk, const img2d_c64 *d_tab_forw, const img2d_c64 *d_tab_back,
                         void *stream);
/* Device pointers, packed layout of img2d_migrate_compact.  Asynchronous on `stream`. */
int img2d_plan_execute(img2d_plan *plan, img2d_c64 *d_wave, img2d_c64 *d_shot, float *d_image,
                       float *d_image_shots, void *stream);
/* Element offset of shot s's block inside the packed wavefield arrays, and their total size. */
long long img2d_plan_shot_offset(const img2d_plan *plan, int s);
/* Dense operator table of the reference's legacy ABI, (nextrap, nf, nx, 2M+1) complex64 written to
 * d_dense on the device from the plan's compact table and operator index (after set_model):
 * entry [l][j][x] is the table row of find_nearest(kappa, w[j]/v[l,x]).  which = 0: forward rows;
 * 1: receiver rows (tab_back in two-table plans, else the conjugated forward rows).  Replaces the
 * host-side gather of py_src/operatorsPreparation/preparation.py:101-115 (makeTableOfOperators)
 * for callers that keep passing dense tables to `extrapolate`.  Asynchronous on `stream`. */
int img2d_plan_dense_table(const img2d_plan *plan, int which, img2d_c64 *d_dense, void *stream);
long long img2d_plan_wavefield_elems(const img2d_plan *plan);
/* Device bytes held by the plan, and the kernel configuration it chose. */
size_t img2d_plan_workspace_bytes(const img2d_plan *plan);
int img2d_plan_describe(const img2d_plan *plan, char *buf, int buflen);
void img2d_plan_destroy(img2d_plan *plan);

/* Device time (ms) of the persistent migration kernel alone in the last img2d_plan_execute on this
 * plan, from CUDA events recorded around that launch on its stream (waits for it to finish). */
int img2d_plan_kernel_ms(img2d_plan *plan, float *ms);

/* Status of the last migration launch on this plan, read on `stream` after it (waits for it):
 * IMG2D_ECUDA if a bounded wait inside the kernel gave up (the bulk-copy ring of
 * IMG2D_FLAG_WIDE_BULK; the results of that launch are then invalid), else IMG2D_OK.
 * img2d_migrate_compact checks it by itself. */
int img2d_plan_status(img2d_plan *plan, void *stream);

/* Host only (no GPU needed): the wide kernel's packing of shots into items of up to 8 lane slots.
 * windows = 0: the line packing (K <= 0: clusters just wide enough for its widest group);
 * windows = 1: the window-first packing on clusters of K CTAs of 1024 positions.  Writes, per shot,
 * its group and lane slot; per group (arrays of at least ns entries, may be NULL) its window start
 * and width; the number of groups, and the modelled cost of one frequency's items in CTA units. */
int img2d_pack_shots(int ns, int nx, int M, const int *shot_x0, const int *shot_nx, int windows, int K,
                     int *group_of_shot, int *slot_of_shot, int *group_u0, int *group_w, int *n_groups,
                     double *cost_units);

/* FP32 FMA throughput of the current device in TFLOP/s, measured by a short kernel of independent
 * FMA chains (the denominator of the FP32 roofline; not part of the migration path). */
int img2d_measure_fp32_peak(double *tflops);

/* L2 read bandwidth of the current device in GB/s: all SMs stream a 32 MB L2-resident buffer with
 * L2-only loads (the denominator of the L2 roofline of the operator gathers). */
int img2d_measure_l2_bandwidth(double *gbs);

/* ------------------------------------------------------------------------------------------
 * Front end: the per-shot data preparation of main.py:111-123 on the device.
 *
 * img2d_ricker_sources replaces util.makeRickerWavelet (py_src/operatorsPreparation/util.py:47-58,
 * wavelet util.py:10-14) for ns single sources: d_out (ns, nt, nx) float32 gets
 *   (1 - 2 pi^2 f^2 tau^2) exp(-pi^2 f^2 tau^2) / sqrt(r),  r = sqrt(depth_offset^2 + (x_i - src_x[s])^2),
 *   tau = float32(j dt - r / v),  x_i = x_first + i dx,
 * with f = fpeak (the reference uses 30 Hz).  main.py:114-122 calls it with x_first = xmin + dx,
 * src_x[s] = xmin + shot_isx[s] dx, depth_offset = dz - zinit and v = velocity[0][0].  src_x is a
 * host array; the call returns when d_out is written.
 *
 * img2d_records_to_spectra replaces scipy.fftpack.fft(record, axis=0) of main.py:118-123 followed
 * by the use of its first nf rows: d_records (ns, nt, nx) float32 time-domain traces (receiver
 * records or the wavelets above) -> d_out packed like the migration's wave/shot buffers (per shot
 * nt_rows rows of that shot's aperture [shot_x0[s], shot_x0[s] + shot_nx[s]), NULL = full
 * aperture), rows j < nf set to sum_t rec[t][x] exp(-2 pi i j t / nt), other rows untouched.  The
 * transform is a single-precision real-to-complex cuFFT along time (as the reference's transform of
 * float32 records is single precision), rows above nt/2 by conjugate symmetry.  shot_x0 / shot_nx
 * are host arrays; the call returns when d_out is written.
 * ---------------------------------------------------------------------------------------- */
int img2d_ricker_sources(int ns, int nt, int nx, double dt, double x_first, double dx,
                         double depth_offset, double v, double fpeak, const double *src_x,
                         float *d_out, void *stream);
int img2d_records_to_spectra(int ns, int nt, int nx, int nf, int nt_rows, const float *d_records,
                             const int *shot_x0, const int *shot_nx, img2d_c64 *d_out, void *stream);

/* ------------------------------------------------------------------------------------------
 * No-allocation entry point.  No counterpart in the reference: the reference libraries allocate
 * their device memory inside every call.
 *
 * For callers that cannot call cudaMalloc: a plugin inside a host application that owns all
 * device memory through its own pool and forbids direct allocation, or a processing loop that
 * must not block on (cudaMalloc can synchronise the device) or fail in an allocation mid-run.
 * Same migration as img2d_plan_execute (single-table mode), with device pointers for every input
 * and output; shot_x0/shot_nx are host arrays (or NULL for full aperture).  Its scratch (operator
 * index table, padded table, work descriptors, per-CTA image partials) lives in one fixed device
 * array of IMG2D_NOALLOC_SCRATCH_BYTES inside the library, which every GPU that loads the library
 * holds until the process exits.  Problems whose scratch does not fit are rejected with
 * IMG2D_EINVAL and a message naming the limit; nothing is allocated.
 *  - The first call on a device looks up the array's device address (cudaGetSymbolAddress);
 *    make that first call before any stream capture.
 *  - All calls share the one array and it keeps the last call's contents (the entry point
 *    clears what must start at zero).  Calls that overlap on the GPU race: issue them on one
 *    stream, or wait for the previous call before the next.
 *  - Every call copies its work descriptors from pageable host memory to the array with
 *    cudaMemcpyAsync on `stream` and then calls cudaStreamSynchronize(stream), so it returns only
 *    after the work queued on `stream` before it has finished; the index-table build, the
 *    migration and the image reduction that follow are queued on `stream` without waiting.
 * ---------------------------------------------------------------------------------------- */
#define IMG2D_NOALLOC_SCRATCH_BYTES (64ull << 20)
int img2d_migrate_compact_noalloc(int ns, int nextrap, int nz, int nx, int nf, int nt, int M, int nk,
                                  double dk, const double *d_omega, const double *d_velocity,
                                  const img2d_c64 *d_tab_forw, const int *shot_x0, const int *shot_nx,
                                  img2d_c64 *d_wave, img2d_c64 *d_shot, float *d_image, void *stream);

/* ------------------------------------------------------------------------------------------
 * Demigration: the adjoint of img2d_plan_execute's stacked image with respect to the receiver
 * spectra.  No counterpart in the reference, which only migrates (cpp_src/extrapolation_cpu.cpp:
 * 11-107 is the forward map F that this is the adjoint of).
 *
 * For a fixed source (d_wave, packed like img2d_plan_execute's wave buffer, read only) the
 * migration is the real-linear map F: receiver spectra d -> image I[l][x], l < nextrap.  This
 * computes d_data = F* m for the reflectivity m = d_refl (rows [0, nextrap) of an nx-wide float
 * image), with <F d, m> = Re sum d conj(F* m).  It sweeps the depth steps in reverse order with
 * the transposed operators and recomputes the source wavefield per slab of slab_depth steps from
 * checkpoints (slab_depth <= 0: 8).  Writes rows [0, nf) of every shot block of d_data (packed like
 * d_wave, must not alias it).  Single-table mode only (T_back = conj(T_forw)); uses the FP32 table.
 * Asynchronous on `stream`; img2d_plan_kernel_ms then times this kernel.
 *
 * source_mode: the source wavefield does not depend on the reflectivity, so repeated
 * demigrations with the same source (a least-squares migration loop) can keep its checkpoints.
 *   IMG2D_SOURCE_RECOMPUTE  checkpoints in per-CTA scratch, recomputed by this call, not kept;
 *   IMG2D_SOURCE_KEEP       checkpoints computed by this call and kept on the plan
 *                           (items x slabs x window x slots x 8 bytes of device memory);
 *   IMG2D_SOURCE_REUSE      the kept checkpoints are read instead of computed (the checkpoint pass,
 *                           a third of the work, is skipped).  The caller guarantees the same
 *                           d_wave contents as the keeping call; img2d_plan_set_model and a
 *                           different slab_depth discard the kept checkpoints (IMG2D_EINVAL).
 * ---------------------------------------------------------------------------------------- */
#define IMG2D_SOURCE_RECOMPUTE 0
#define IMG2D_SOURCE_KEEP 1
#define IMG2D_SOURCE_REUSE 2
int img2d_plan_demigrate(img2d_plan *plan, const float *d_refl, const img2d_c64 *d_wave,
                         img2d_c64 *d_data, int slab_depth, int source_mode, void *stream);
/* Kernel configuration of the last demigration on this plan (JSON). */
int img2d_plan_describe_demigration(const img2d_plan *plan, char *buf, int buflen);

/* Naive comparison form: one kernel launch per (shot, frequency, depth), operators from the
 * compact table, wavefields in global memory.  Same arguments and results as
 * img2d_plan_execute (device pointers).  Used only to measure the batched kernel against. */
int img2d_plan_execute_naive(img2d_plan *plan, img2d_c64 *d_wave, img2d_c64 *d_shot,
                             float *d_image, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* IMAGING2D_WLSQ_B200_H */
