// Device kernels of the ω-x WLSQ extrapolation + cross-correlation imaging path.
//
// Reference semantics (file:line within the reference project ahadji05/Imaging2D_WLSQ):
//   cpp_src/extrapolation_cpu.cpp:39-89  depth loop: new[x] = sum_k T[z,w,x,k] * old[x+k-M] for the
//                                        source wavefield (forward table) and the receiver
//                                        wavefield (backward table), zero outside [0,nx),
//                                        then image[s,z,x] = Re(sum_w S * conj(R)).
//   cpp_src/extrapolation_revOp_gpu.cu:51-72 the same step as one CUDA thread per (x, w).
//   py_src/operatorsPreparation/preparation.py:101-115 the dense table is a gather of a compact
//                                        (nk, 2M+1) table by idx = find_nearest(kappa, w/v(z,x)).
//
// Work decomposition (B200): one CTA owns one work item = (group of G lane slots, one frequency)
// for the whole depth loop; both wavefields of every shot of the group stay resident in shared
// memory (ping-pong buffers) across all depth steps.  A slot holds one shot, or several shots
// whose apertures are disjoint (uneven-aperture surveys pack into fewer slots).  Lane q of a warp
// owns slot q (its source value S and receiver value R packed as one float4), lanes are split
// into 32/G position groups, and each position group sweeps blocks of X consecutive positions.  The
// operator row of a position is loaded once per lane group and broadcast to the G shots.
// The receiver is stored conjugated in the single-table mode: conj(R_new) = sum_k T_f conj(R_old)
// when T_b = conj(T_f), so source and receiver share every operator load.
//
// Imaging is fused: after each block the lanes form Re(S conj R) per shot, reduce over the G
// shots with warp shuffles and add the row into the CTA's private partial image with Kahan
// compensation (no global atomics on the stacked image).  A persistent grid pulls work items
// from an atomic counter; a final kernel sums the per-CTA partials.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace img2d {

struct cpx {
    float re, im;
};

enum OpMode : int {
    OP_CONJ = 0,   // compact table, receiver uses conj(tabF)
    OP_TWO = 1,    // compact tables tabF (source) and tabB (receiver)
    OP_DENSE = 2,  // dense tables (nextrap, nf, nx, L), reference layout
};

// A work group: up to G lane slots over a union window [u0, u0+W) of the model.  Each slot holds
// one or more shots whose apertures are disjoint and separated by at least M zero samples, so the
// FIR of one never reads another (the zero-halo semantics of cpp_src/wfPad.h hold per shot).
struct GroupDesc {
    int seg_begin, nseg;  // segments [seg_begin, seg_begin+nseg) of MigrateArgs::segs
    int u0, W;            // union window
    int nslots, owner_stride;
    long long owner_off;  // start of this group's owner table
};

// Everything a migration kernel launch needs (device pointers).
struct MigrateArgs {
    int nextrap;     // depth steps
    int nx;          // model width
    int nf;          // frequencies
    int M;           // half operator length, L = 2M+1
    int tab_stride;  // complex elements per compact-table row (even, >= L)
    int n_items;
    const int2 *items;       // x = group, y = frequency index, decreasing cost
    const GroupDesc *groups;
    const int4 *segs;        // x = shot, y = slot in its group, z = x0, w = nx_s
    const int16_t *owner;    // per group [slot][owner_stride]: shot id at each position, -1 outside
    const long long *shot_off;  // element offset of each shot's block in wave/shot
    const cpx *tabF;
    const cpx *tabB;
    const void *tab16;       // 16-bit copy of tabF (FP16 or BF16 (re, im) pairs), same row stride
    const uint16_t *idx;     // [nf][nextrap][idx_lstride] compact row index
    long long idx_jstride;
    int idx_lstride;
    const cpx *denseF;       // dense tables (OP_DENSE)
    const cpx *denseB;
    cpx *wave;               // source wavefields, overwritten with the final depth
    cpx *shot;               // receiver wavefields, overwritten with the final depth
    int write_back;
    float *partial;          // [gridDim.x][nextrap][nx] stacked partial image (or null)
    float *comp;             // Kahan compensation, same shape
    float *image_shots;      // per-shot images (or null), row l of shot s at s*img_sstride + l*nx
    long long img_sstride;
    int *counter;            // work-queue counter, zeroed before launch
    int *status;             // zeroed before launch; set non-zero by a kernel whose bounded wait gave up
};

__device__ __forceinline__ int pad_slot(int xl, int X) { return xl + xl / X; }

__device__ __forceinline__ void kahan_add(float *s, float *c, float v)
{
    float y = v - *c;
    float t = *s + y;
    *c = (t - *s) - y;
    *s = t;
}

// One work item: stage the wavefields of the group for frequency j into shared memory.
template <int G>
__device__ __forceinline__ void stage_in(const MigrateArgs &a, float4 *buf, const GroupDesc &grp, int j,
                                         int Mp, int X, bool conj_rec)
{
    for (int k = grp.seg_begin; k < grp.seg_begin + grp.nseg; ++k) {
        const int4 sg = a.segs[k];
        const cpx *ws = a.wave + a.shot_off[sg.x] + (long long)j * sg.w;
        const cpx *rs = a.shot + a.shot_off[sg.x] + (long long)j * sg.w;
        for (int i = threadIdx.x; i < sg.w; i += blockDim.x) {
            const int xl = sg.z - grp.u0 + i + Mp;
            const cpx S = ws[i], R = rs[i];
            buf[pad_slot(xl, X) * G + sg.y] = make_float4(S.re, S.im, R.re, conj_rec ? -R.im : R.im);
        }
    }
}

template <int G>
__device__ __forceinline__ void stage_out(const MigrateArgs &a, const float4 *buf, const GroupDesc &grp,
                                          int j, int Mp, int X, bool conj_rec)
{
    for (int k = grp.seg_begin; k < grp.seg_begin + grp.nseg; ++k) {
        const int4 sg = a.segs[k];
        cpx *ws = a.wave + a.shot_off[sg.x] + (long long)j * sg.w;
        cpx *rs = a.shot + a.shot_off[sg.x] + (long long)j * sg.w;
        for (int i = threadIdx.x; i < sg.w; i += blockDim.x) {
            const int xl = sg.z - grp.u0 + i + Mp;
            const float4 v = buf[pad_slot(xl, X) * G + sg.y];
            ws[i] = cpx{v.x, v.y};
            rs[i] = cpx{v.z, conj_rec ? -v.w : v.w};
        }
    }
}

// Shot ids of X consecutive positions of one slot (X = 4 or 8; 8- or 16-byte aligned rows).
template <int X>
__device__ __forceinline__ void load_owner(const int16_t *row, int16_t (&own)[X])
{
    if (row == nullptr) {
#pragma unroll
        for (int i = 0; i < X; ++i) own[i] = -1;
        return;
    }
    if (X == 8) {
        const int4 v = *reinterpret_cast<const int4 *>(row);
        const int w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int i = 0; i < X; ++i) own[i] = (int16_t)(w[i / 2] >> (16 * (i & 1)));
    } else {
        const int2 v = *reinterpret_cast<const int2 *>(row);
        const int w[2] = {v.x, v.y};
#pragma unroll
        for (int i = 0; i < X; ++i) own[i] = (int16_t)(w[i / 2] >> (16 * (i & 1)));
    }
}

// Imaging + masking epilogue for one position of a block.
// The G lanes of one position group always run the same block loop, but different position
// groups of a warp may not (their block counts can differ by one), so the reduction over shots
// synchronises only the group's own lanes.
template <int G>
__device__ __forceinline__ unsigned group_mask(int lane)
{
    return G == 32 ? 0xffffffffu : (((1u << G) - 1u) << ((lane / G) * G));
}

template <int G>
__device__ __forceinline__ void emit_position(const MigrateArgs &a, float4 *dst, int slot, int q,
                                              bool in_win, bool in_group, int xm, int l, int shot_id,
                                              float sr, float si, float rr, float ri, bool conj_rec,
                                              float *part_row, float *comp_row)
{
    if (!in_win) sr = si = rr = ri = 0.f;
    dst[slot * G + q] = make_float4(sr, si, rr, ri);
    // Re(S * conj(R)); the stored receiver is conj(R) in the single-table mode
    float img = conj_rec ? (sr * rr - si * ri) : (sr * rr + si * ri);
    if (a.image_shots && in_win)
        atomicAdd(a.image_shots + (long long)shot_id * a.img_sstride + (long long)l * a.nx + xm, img);
#pragma unroll
    for (int off = 1; off < G; off <<= 1) img += __shfl_xor_sync(group_mask<G>(threadIdx.x & 31), img, off);
    if (part_row && q == 0 && in_group) kahan_add(part_row + xm, comp_row + xm, img);
}

// Fast path: compile-time operator length L, X positions per lane block, G shots per CTA.
// Operator rows come from the compact table (row stride a.tab_stride, even, zero padded),
// loaded as tap pairs (16 B) through the read-only path and broadcast to the G lanes.
template <int G, int X, int L, int MODE>
__global__ void __launch_bounds__(256, 1) migrate_fixed_kernel(MigrateArgs a)
{
    static_assert(32 % G == 0, "G must divide 32");
    constexpr int P = 32 / G;
    constexpr int M = (L - 1) / 2;
    constexpr int Mp = ((M + X - 1) / X) * X;
    constexpr bool CONJ = (MODE == OP_CONJ);
    extern __shared__ float4 smem[];
    __shared__ int s_item;

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q = lane % G, p = lane / G;
    const int ngroups = (blockDim.x >> 5) * P;
    const int gid = warp * P + p;
    float *part = a.partial ? a.partial + (long long)blockIdx.x * a.nextrap * a.nx : nullptr;
    float *cmp = a.comp ? a.comp + (long long)blockIdx.x * a.nextrap * a.nx : nullptr;

    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(a.counter, 1);
        __syncthreads();
        const int it = s_item;
        __syncthreads();
        if (it >= a.n_items) break;
        const int2 item = a.items[it];
        const GroupDesc grp = a.groups[item.x];
        const int j = item.y, u0 = grp.u0, W = grp.W;
        const int Wp = ((W + X - 1) / X) * X;
        const int npos = Mp + Wp + Mp;
        const int nslot = npos / X * (X + 1);
        float4 *bufA = smem, *bufB = smem + nslot * G;
        for (int i = threadIdx.x; i < 2 * nslot * G; i += blockDim.x) smem[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        __syncthreads();
        stage_in<G>(a, bufA, grp, j, Mp, X, CONJ);
        __syncthreads();

        const int16_t *own_base =
            q < grp.nslots ? a.owner + grp.owner_off + (long long)q * grp.owner_stride : nullptr;
        const int nblocks = Wp / X;
        const uint16_t *idx_j = a.idx + (long long)j * a.idx_jstride;

        for (int l = 0; l < a.nextrap; ++l) {
            const uint16_t *idx_l = idx_j + (long long)l * a.idx_lstride;
            float *prow = part ? part + (long long)l * a.nx : nullptr;
            float *crow = cmp ? cmp + (long long)l * a.nx : nullptr;
            for (int b = gid; b < nblocks; b += ngroups) {
                const int xb = Mp + b * X;  // index-space position of the block's first output
                const float4 *rowF[X];
                const float4 *rowB[X];
#pragma unroll
                for (int jj = 0; jj < X; ++jj) {
                    int xm = u0 + b * X + jj;
                    xm = xm < a.nx ? xm : a.nx - 1;
                    const int r = idx_l[xm];
                    rowF[jj] = reinterpret_cast<const float4 *>(a.tabF + (long long)r * a.tab_stride);
                    if (!CONJ) rowB[jj] = reinterpret_cast<const float4 *>(a.tabB + (long long)r * a.tab_stride);
                }
                float sr[X], si[X], rr[X], ri[X];
#pragma unroll
                for (int jj = 0; jj < X; ++jj) sr[jj] = si[jj] = rr[jj] = ri[jj] = 0.f;
                float4 tf[X], tb[X];
#pragma unroll
                for (int t = 0; t < X + L - 1; ++t) {
                    const float4 v = bufA[pad_slot(xb - M + t, X) * G + q];
#pragma unroll
                    for (int jj = 0; jj < X; ++jj) {
                        const int k = t - jj;
                        if (k >= 0 && k < L) {
                            if ((k & 1) == 0) {
                                tf[jj] = __ldg(rowF[jj] + (k >> 1));
                                if (!CONJ) tb[jj] = __ldg(rowB[jj] + (k >> 1));
                            }
                            const float fr = (k & 1) ? tf[jj].z : tf[jj].x;
                            const float fi = (k & 1) ? tf[jj].w : tf[jj].y;
                            float br = fr, bi = fi;
                            if (!CONJ) {
                                br = (k & 1) ? tb[jj].z : tb[jj].x;
                                bi = (k & 1) ? tb[jj].w : tb[jj].y;
                            }
                            sr[jj] = fmaf(fr, v.x, sr[jj]);
                            sr[jj] = fmaf(-fi, v.y, sr[jj]);
                            si[jj] = fmaf(fr, v.y, si[jj]);
                            si[jj] = fmaf(fi, v.x, si[jj]);
                            rr[jj] = fmaf(br, v.z, rr[jj]);
                            rr[jj] = fmaf(-bi, v.w, rr[jj]);
                            ri[jj] = fmaf(br, v.w, ri[jj]);
                            ri[jj] = fmaf(bi, v.z, ri[jj]);
                        }
                    }
                }
                int16_t own[X];
                load_owner<X>(own_base ? own_base + b * X : nullptr, own);
#pragma unroll
                for (int jj = 0; jj < X; ++jj) {
                    const int xl = xb + jj;
                    const int xr = b * X + jj;  // position relative to u0
                    emit_position<G>(a, bufB, pad_slot(xl, X), q, own[jj] >= 0, xr < W,
                                     u0 + (xr < W ? xr : 0), l, own[jj], sr[jj], si[jj], rr[jj], ri[jj],
                                     CONJ, prow, crow);
                }
            }
            __syncthreads();
            float4 *t = bufA; bufA = bufB; bufB = t;
        }
        if (a.write_back) stage_out<G>(a, bufA, grp, j, Mp, X, CONJ);
        __syncthreads();
    }
}

// General path: runtime operator length, any of the three operator sources.  Same work
// decomposition as the fast path; the tap loop reads the wavefield window from shared memory
// directly, X = 4 outputs per lane block.
template <int G, int MODE>
__global__ void __launch_bounds__(256, 1) migrate_generic_kernel(MigrateArgs a)
{
    constexpr int P = 32 / G;
    constexpr int X = 4;
    constexpr bool CONJ = (MODE == OP_CONJ);
    extern __shared__ float4 smem[];
    __shared__ int s_item;
    const int M = a.M, L = 2 * a.M + 1;
    const int Mp = ((M + X - 1) / X) * X;

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q = lane % G, p = lane / G;
    const int ngroups = (blockDim.x >> 5) * P;
    const int gid = warp * P + p;
    float *part = a.partial ? a.partial + (long long)blockIdx.x * a.nextrap * a.nx : nullptr;
    float *cmp = a.comp ? a.comp + (long long)blockIdx.x * a.nextrap * a.nx : nullptr;

    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(a.counter, 1);
        __syncthreads();
        const int it = s_item;
        __syncthreads();
        if (it >= a.n_items) break;
        const int2 item = a.items[it];
        const GroupDesc grp = a.groups[item.x];
        const int j = item.y, u0 = grp.u0, W = grp.W;
        const int Wp = ((W + X - 1) / X) * X;
        const int npos = Mp + Wp + Mp;
        const int nslot = npos / X * (X + 1);
        float4 *bufA = smem, *bufB = smem + nslot * G;
        for (int i = threadIdx.x; i < 2 * nslot * G; i += blockDim.x) smem[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        __syncthreads();
        stage_in<G>(a, bufA, grp, j, Mp, X, CONJ);
        __syncthreads();

        const int16_t *own_base =
            q < grp.nslots ? a.owner + grp.owner_off + (long long)q * grp.owner_stride : nullptr;
        const int nblocks = Wp / X;

        for (int l = 0; l < a.nextrap; ++l) {
            float *prow = part ? part + (long long)l * a.nx : nullptr;
            float *crow = cmp ? cmp + (long long)l * a.nx : nullptr;
            for (int b = gid; b < nblocks; b += ngroups) {
                const int xb = Mp + b * X;
                const cpx *rowF[X];
                const cpx *rowB[X];
#pragma unroll
                for (int jj = 0; jj < X; ++jj) {
                    int xm = u0 + b * X + jj;
                    xm = xm < a.nx ? xm : a.nx - 1;
                    if (MODE == OP_DENSE) {
                        const long long off = (((long long)l * a.nf + j) * a.nx + xm) * L;
                        rowF[jj] = a.denseF + off;
                        rowB[jj] = a.denseB + off;
                    } else {
                        const int r = a.idx[(long long)j * a.idx_jstride + (long long)l * a.idx_lstride + xm];
                        rowF[jj] = a.tabF + (long long)r * a.tab_stride;
                        rowB[jj] = CONJ ? rowF[jj] : a.tabB + (long long)r * a.tab_stride;
                    }
                }
                float sr[X], si[X], rr[X], ri[X];
#pragma unroll
                for (int jj = 0; jj < X; ++jj) {
                    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
                    for (int k = 0; k < L; ++k) {
                        const float4 v = bufA[pad_slot(xb + jj - M + k, X) * G + q];
                        const cpx f = rowF[jj][k];
                        const cpx g = rowB[jj][k];
                        const float br = g.re, bi = g.im;
                        a0 = fmaf(f.re, v.x, a0); a0 = fmaf(-f.im, v.y, a0);
                        a1 = fmaf(f.re, v.y, a1); a1 = fmaf(f.im, v.x, a1);
                        a2 = fmaf(br, v.z, a2); a2 = fmaf(-bi, v.w, a2);
                        a3 = fmaf(br, v.w, a3); a3 = fmaf(bi, v.z, a3);
                    }
                    sr[jj] = a0; si[jj] = a1; rr[jj] = a2; ri[jj] = a3;
                }
                int16_t own[X];
                load_owner<X>(own_base ? own_base + b * X : nullptr, own);
#pragma unroll
                for (int jj = 0; jj < X; ++jj) {
                    const int xl = xb + jj;
                    const int xr = b * X + jj;
                    emit_position<G>(a, bufB, pad_slot(xl, X), q, own[jj] >= 0, xr < W,
                                     u0 + (xr < W ? xr : 0), l, own[jj], sr[jj], si[jj], rr[jj], ri[jj],
                                     CONJ, prow, crow);
                }
            }
            __syncthreads();
            float4 *t = bufA; bufA = bufB; bufB = t;
        }
        if (a.write_back) stage_out<G>(a, bufA, grp, j, Mp, X, CONJ);
        __syncthreads();
    }
}

// idx[j][l][x] = find_nearest(kappa, omega[j] / vel[l][x]) with kappa[i] = i*dk, ties to the
// lowest index (py_src/operatorsPreparation/util.py:5-8, 39-45), computed in float64 exactly as
// numpy does: |fl(i*dk) - fl(w/v)| compared over the candidates around floor(w/v/dk).
__global__ void index_table_kernel(const double *__restrict__ omega, const double *__restrict__ vel,
                                   int nf, int nextrap, int nx, int lstride, int nk, double dk,
                                   uint16_t *__restrict__ idx)
{
    const long long total = (long long)nf * nextrap * nx;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(e % nx);
        const long long r = e / nx;
        const int l = (int)(r % nextrap);
        const int j = (int)(r / nextrap);
        const double value = __ddiv_rn(omega[j], vel[(long long)l * nx + x]);
        const double qv = __ddiv_rn(value, dk);
        long long i0;
        if (!(qv > 0.0)) i0 = 0;
        else if (qv >= (double)(nk - 1)) i0 = nk - 1;
        else i0 = (long long)floor(qv);
        long long lo = i0 - 1, hi = i0 + 2;
        if (lo < 0) lo = 0;
        if (hi > nk - 1) hi = nk - 1;
        long long best = lo;
        double bestd = __longlong_as_double(0x7ff0000000000000ll);
        for (long long i = lo; i <= hi; ++i) {
            const double d = fabs(__dadd_rn(__dmul_rn((double)i, dk), -value));
            if (d < bestd) { bestd = d; best = i; }
        }
        idx[((long long)j * nextrap + l) * lstride + x] = (uint16_t)best;
    }
}

// image[l][x] = sum over CTAs of the Kahan pair (s - c), reduced with Kahan in a fixed order.
__global__ void reduce_partials_kernel(const float *__restrict__ partial, const float *__restrict__ comp,
                                       int nslots, long long plane, float *__restrict__ image)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < plane;
         e += (long long)gridDim.x * blockDim.x) {
        float s = 0.f, c = 0.f;
        for (int k = 0; k < nslots; ++k) {
            const float v = partial[(long long)k * plane + e] - comp[(long long)k * plane + e];
            kahan_add(&s, &c, v);
        }
        image[e] = s - c;
    }
}

// 16-bit copy of the padded operator table: (re, im) of each tap as half2 / bfloat162, rounded to
// nearest.  Used by the reduced-precision table storage modes of the cluster kernel.
__global__ void table_to_16bit_kernel(const cpx *__restrict__ src, long long n, int bf16, unsigned *__restrict__ dst)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const cpx v = src[e];
        if (bf16) {
            const __nv_bfloat162 h = __floats2bfloat162_rn(v.re, v.im);
            dst[e] = *reinterpret_cast<const unsigned *>(&h);
        } else {
            const __half2 h = __floats2half2_rn(v.re, v.im);
            dst[e] = *reinterpret_cast<const unsigned *>(&h);
        }
    }
}

}  // namespace img2d
