// Demigration: the adjoint of the migration with respect to the recorded receiver data.
//
// The migration of the reference (cpp_src/extrapolation_cpu.cpp:39-89) is, for a fixed source
// wavefield, a real-linear map F from receiver spectra d (per shot, frequency, position) to the
// stacked image:
//     S_{l+1} = A_l S_l                  A_l[x, x+k-M] = T(z_l, w, x)[k]   (source, forward table)
//     R_{l+1} = B_l R_l                  B_l = conj(A_l) elementwise        (receiver, T_b = conj(T_f))
//     I[l, x] = Re sum_{shots, w} S_{l+1}[x] conj(R_{l+1}[x]),  R_0 = d.
// With the real inner products <I, m> = sum I m and <u, v> = Re sum u conj(v) its adjoint is
//     F* m = sum_l B_0^H ... B_l^H (m_l S_{l+1}),   B_l^H = A_l^T,
// evaluated here by the reverse-depth recursion
//     V_{nextrap-1} = m_{nextrap-1} S_{nextrap};   U_l = A_l^T V_l;   V_{l-1} = U_l + m_{l-1} S_l;
//     F* m = U_0.
// A_l^T applies, at output y, tap y+M-i of the operator row of INPUT position i (the transpose of
// the gather of cpp_src/extrapolation_cpu.cpp:50-53), with the same zero halos.
//
// The source wavefield is needed in reverse depth order.  Instead of storing it for every depth,
// each CTA keeps checkpoints S_{cD} every D depth steps, and per slab recomputes S_{cD+1..cD+D}
// into a small per-CTA slab buffer (L2-resident) before sweeping the slab backwards.
//
// Work decomposition: as in the migration kernels, one persistent CTA takes a work item (group of
// G lane slots, one frequency) from an atomic counter.  Lane q of a warp owns slot q; 32/G position
// groups sweep blocks of X = 8 positions.  One complex wavefield per slot is resident in shared
// memory as float2, ping-pong, with one pad slot every X positions against bank conflicts.
#pragma once
#include "wlsq_kernels.cuh"

namespace img2d {

struct DemigrateArgs {
    int nextrap;     // depth steps
    int nx;          // model width
    int M;           // half operator length
    int tab_stride;  // complex elements per compact-table row (even)
    int n_items;
    int slab;        // D, depth steps per slab
    int nslab;       // ceil(nextrap / D)
    const int2 *items;
    const GroupDesc *groups;
    const int4 *segs;
    const int16_t *owner;
    const long long *shot_off;
    const cpx *tab;          // compact forward table
    const uint16_t *idx;     // [nf][nextrap][idx_lstride]
    long long idx_jstride;
    int idx_lstride;
    const cpx *wave;         // source spectra, packed like the migration's wave buffer; read only
    const float *refl;       // reflectivity rows [0, nextrap), row stride nx
    cpx *data;               // receiver spectra out, same packing as wave; rows [0, nf) written
    float2 *work;            // per CTA: ckpt[nslab][wmax*G], slab[D][wmax*G], save[wmax*G]
    long long work_cta;      // float2 elements per CTA
    int wmax;
    int *counter;
    // source checkpoints: 0 = per CTA, recomputed in every call; 1 = computed into the per-item
    // cache ckpt_items[item][nslab][wmax*G]; 2 = read from that cache (no checkpoint pass)
    int ckpt_mode;
    float2 *ckpt_items;
};

// Shared-memory words of one staged operator-index row: the positions [u0-Mp, u0+Wp+Mp) of a window,
// clipped to [0, nx), copied as aligned 32-bit words of the index table row.
__host__ __device__ inline int demig_idx_words(int Wp, int Mp) { return (Wp + 2 * Mp) / 2 + 2; }

// Copy the index row of depth step l covering the window into `dst` (cp.async, 4-byte words);
// returns nothing, the caller commits and waits.  Word k of dst holds table entries 2*(w0+k) and
// 2*(w0+k)+1 of the row, w0 = max(0, u0-Mp) / 2.
__device__ __forceinline__ void demig_stage_idx(const DemigrateArgs &a, const uint16_t *idx_j, int l, int u0,
                                                int Wp, int Mp, unsigned *dst)
{
    const int lo = max(0, u0 - Mp) >> 1;
    const int hi = (min(a.nx, u0 + Wp + Mp) + 1) >> 1;  // words [lo, hi) lie inside the padded row
    const unsigned *row = reinterpret_cast<const unsigned *>(idx_j + (long long)l * a.idx_lstride);
    for (int k = lo + (int)threadIdx.x; k < hi; k += blockDim.x) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(dst + (k - lo));
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(row + k) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// Wavefield slots (positions with pad slots) of one buffer for the widest window.
__host__ __device__ inline int nslot_max(int wmax, int Mp)
{
    const int X = 8;
    const int Wp = ((wmax + X - 1) / X) * X;
    return (Mp + Wp + Mp) / X * (X + 1);
}

// Dense [W][G] layout of one depth plane in the per-CTA work area.
__device__ __forceinline__ long long plane_elems(const DemigrateArgs &a, int G) { return (long long)a.wmax * G; }

template <int G, int X>
__device__ __forceinline__ void smem_to_plane(const float2 *buf, float2 *plane, int W, int Mp)
{
    for (int e = threadIdx.x; e < W * G; e += blockDim.x) {
        const int xr = e / G, q = e - xr * G;
        plane[e] = buf[pad_slot(Mp + xr, X) * G + q];
    }
}

template <int G, int X>
__device__ __forceinline__ void plane_to_smem(float2 *buf, const float2 *plane, int W, int Mp)
{
    for (int e = threadIdx.x; e < W * G; e += blockDim.x) {
        const int xr = e / G, q = e - xr * G;
        buf[pad_slot(Mp + xr, X) * G + q] = plane[e];
    }
}

// Forward step of the source wavefield for one block of X outputs (gather with output rows).
template <int X, int L, int G>
__device__ __forceinline__ void fir_forward(const DemigrateArgs &a, const float2 *src, const uint16_t *idx_l,
                                           int u0, int b, int xb, int q, float (&re)[X], float (&im)[X])
{
    constexpr int M = (L - 1) / 2;
    const float4 *row[X];
    const int hstride = a.tab_stride >> 1;
#pragma unroll
    for (int jj = 0; jj < X; ++jj) {
        int xm = u0 + b * X + jj;
        xm = xm < a.nx ? xm : a.nx - 1;
        row[jj] = reinterpret_cast<const float4 *>(a.tab) + (long long)idx_l[xm] * hstride;
        re[jj] = im[jj] = 0.f;
    }
    float4 tf[X];
#pragma unroll
    for (int t = 0; t < X + L - 1; ++t) {
        const float2 v = src[pad_slot(xb - M + t, X) * G + q];
#pragma unroll
        for (int jj = 0; jj < X; ++jj) {
            const int k = t - jj;
            if (k >= 0 && k < L) {
                if ((k & 1) == 0) tf[jj] = __ldg(row[jj] + (k >> 1));
                const float fr = (k & 1) ? tf[jj].z : tf[jj].x;
                const float fi = (k & 1) ? tf[jj].w : tf[jj].y;
                re[jj] = fmaf(fr, v.x, re[jj]);
                re[jj] = fmaf(-fi, v.y, re[jj]);
                im[jj] = fmaf(fr, v.y, im[jj]);
                im[jj] = fmaf(fi, v.x, im[jj]);
            }
        }
    }
}

// Transposed step for one block of X outputs: output y takes tap y+M-i of the row of input i.
template <int X, int L, int G>
__device__ __forceinline__ void fir_transposed(const DemigrateArgs &a, const float2 *src, const uint16_t *idx_l,
                                               int u0, int xb, int Mp, int q, float (&re)[X], float (&im)[X])
{
    constexpr int M = (L - 1) / 2;
    const int hstride = a.tab_stride >> 1;
#pragma unroll
    for (int jj = 0; jj < X; ++jj) re[jj] = im[jj] = 0.f;
#pragma unroll
    for (int t = 0; t < X + L - 1; ++t) {
        const int xi = xb - M + t;  // input position (index space)
        const float2 v = src[pad_slot(xi, X) * G + q];
        int xm = u0 + xi - Mp;
        xm = xm < 0 ? 0 : (xm < a.nx ? xm : a.nx - 1);
        const float4 *rp = reinterpret_cast<const float4 *>(a.tab) + (long long)idx_l[xm] * hstride;
        float4 cur = make_float4(0.f, 0.f, 0.f, 0.f);
        const int jj0 = t - 2 * M > 0 ? t - 2 * M : 0;
#pragma unroll
        for (int jj = 0; jj < X; ++jj) {
            const int k = jj + 2 * M - t;
            if (k >= 0 && k < L) {
                if ((k & 1) == 0 || jj == jj0) cur = __ldg(rp + (k >> 1));
                const float fr = (k & 1) ? cur.z : cur.x;
                const float fi = (k & 1) ? cur.w : cur.y;
                re[jj] = fmaf(fr, v.x, re[jj]);
                re[jj] = fmaf(-fi, v.y, re[jj]);
                im[jj] = fmaf(fr, v.y, im[jj]);
                im[jj] = fmaf(fi, v.x, im[jj]);
            }
        }
    }
}

// Runtime-length forms (any M), X = 8 outputs per block.
template <int X, int G>
__device__ __forceinline__ void fir_forward_rt(const DemigrateArgs &a, const float2 *src, const uint16_t *idx_l,
                                               int u0, int b, int xb, int q, float (&re)[X], float (&im)[X])
{
    const int M = a.M, L = 2 * a.M + 1;
#pragma unroll
    for (int jj = 0; jj < X; ++jj) {
        int xm = u0 + b * X + jj;
        xm = xm < a.nx ? xm : a.nx - 1;
        const cpx *row = a.tab + (long long)idx_l[xm] * a.tab_stride;
        float r0 = 0.f, i0 = 0.f;
        for (int k = 0; k < L; ++k) {
            const float2 v = src[pad_slot(xb + jj - M + k, X) * G + q];
            const cpx f = row[k];
            r0 = fmaf(f.re, v.x, r0); r0 = fmaf(-f.im, v.y, r0);
            i0 = fmaf(f.re, v.y, i0); i0 = fmaf(f.im, v.x, i0);
        }
        re[jj] = r0;
        im[jj] = i0;
    }
}

template <int X, int G>
__device__ __forceinline__ void fir_transposed_rt(const DemigrateArgs &a, const float2 *src, const uint16_t *idx_l,
                                                  int u0, int xb, int Mp, int q, float (&re)[X], float (&im)[X])
{
    const int M = a.M, L = 2 * a.M + 1;
#pragma unroll
    for (int jj = 0; jj < X; ++jj) {
        float r0 = 0.f, i0 = 0.f;
        for (int k = 0; k < L; ++k) {
            const int xi = xb + jj + M - k;
            const float2 v = src[pad_slot(xi, X) * G + q];
            int xm = u0 + xi - Mp;
            xm = xm < 0 ? 0 : (xm < a.nx ? xm : a.nx - 1);
            const cpx f = a.tab[(long long)idx_l[xm] * a.tab_stride + k];
            r0 = fmaf(f.re, v.x, r0); r0 = fmaf(-f.im, v.y, r0);
            i0 = fmaf(f.re, v.y, i0); i0 = fmaf(f.im, v.x, i0);
        }
        re[jj] = r0;
        im[jj] = i0;
    }
}

// L > 0: compile-time operator length; L == 0: runtime length a.M.
template <int G, int L, int NW>
__global__ void __launch_bounds__(NW * 32, 1) demigrate_kernel(DemigrateArgs a)
{
    static_assert(32 % G == 0, "G must divide 32");
    constexpr int X = 8;
    constexpr int P = 32 / G;
    extern __shared__ float2 smem2[];
    __shared__ int s_item;

    const int M = L > 0 ? (L - 1) / 2 : a.M;
    const int Mp = ((M + X - 1) / X) * X;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q = lane % G, p = lane / G;
    const int ngroups = NW * P;
    const int gid = warp * P + p;
    const long long pe = plane_elems(a, G);
    float2 *ckpt = a.work + (long long)blockIdx.x * a.work_cta;
    float2 *slabbuf = ckpt + (long long)a.nslab * pe;
    float2 *save = slabbuf + (long long)a.slab * pe;

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
        const int nslot = (Mp + Wp + Mp) / X * (X + 1);
        float2 *bufA = smem2, *bufB = smem2 + nslot * G;
        // staged operator-index rows (double buffer) after the two wavefield buffers
        const int iwords = demig_idx_words(((a.wmax + X - 1) / X) * X, Mp);
        unsigned *sidx0 = reinterpret_cast<unsigned *>(smem2 + 2 * (long long)nslot_max(a.wmax, Mp) * G);
        unsigned *sidx1 = sidx0 + iwords;
        const int ibase = 2 * (max(0, u0 - Mp) >> 1);  // table position of staged entry 0
        const uint16_t *idx_j = a.idx + (long long)j * a.idx_jstride;
        if (a.ckpt_mode != 0) ckpt = a.ckpt_items + (long long)it * a.nslab * pe;
        const int D = a.slab;
        const int first_l = a.ckpt_mode == 2 ? (a.nslab - 1) * D : 0;
        demig_stage_idx(a, idx_j, first_l, u0, Wp, Mp, sidx0);
        for (int i = threadIdx.x; i < 2 * nslot * G; i += blockDim.x) smem2[i] = make_float2(0.f, 0.f);
        __syncthreads();
        if (a.ckpt_mode != 2) {
            // source spectra of the group at frequency j
            for (int k = grp.seg_begin; k < grp.seg_begin + grp.nseg; ++k) {
                const int4 sg = a.segs[k];
                const cpx *ws = a.wave + a.shot_off[sg.x] + (long long)j * sg.w;
                for (int i = threadIdx.x; i < sg.w; i += blockDim.x) {
                    const cpx S = ws[i];
                    bufA[pad_slot(sg.z - u0 + i + Mp, X) * G + sg.y] = make_float2(S.re, S.im);
                }
            }
        }
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncthreads();

        const int16_t *own_base =
            q < grp.nslots ? a.owner + grp.owner_off + (long long)q * grp.owner_stride : nullptr;
        const int nblocks = Wp / X;
        // cur: staged index row of the current step; the next step's row is copied into nxt while
        // the current step computes, waited for before the step's closing barrier
        unsigned *cur = sidx0, *nxt = sidx1;
        auto step_idx = [&]() { return reinterpret_cast<const uint16_t *>(cur) - ibase; };
        auto stage_next = [&](int nl) {
            if (nl >= 0) demig_stage_idx(a, idx_j, nl, u0, Wp, Mp, nxt);
        };
        auto end_step = [&]() {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
            __syncthreads();
            unsigned *t = cur; cur = nxt; nxt = t;
        };

        // One forward step of the source, l -> l+1; optionally keeps S_{l+1} in a dense plane;
        // nl: depth step that comes next (its index row is staged meanwhile), -1 for none.
        auto forward_step = [&](int l, float2 *keep, int nl) {
            stage_next(nl);
            const uint16_t *idx_l = step_idx();
            for (int b = gid; b < nblocks; b += ngroups) {
                const int xb = Mp + b * X;
                float re[X], im[X];
                if (L > 0) fir_forward<X, (L > 0 ? L : 1), G>(a, bufA, idx_l, u0, b, xb, q, re, im);
                else fir_forward_rt<X, G>(a, bufA, idx_l, u0, b, xb, q, re, im);
                int16_t own[X];
                load_owner<X>(own_base ? own_base + b * X : nullptr, own);
#pragma unroll
                for (int jj = 0; jj < X; ++jj) {
                    const int xr = b * X + jj;
                    const bool in = own[jj] >= 0 && xr < W;
                    const float2 v = in ? make_float2(re[jj], im[jj]) : make_float2(0.f, 0.f);
                    bufB[pad_slot(xb + jj, X) * G + q] = v;
                    if (keep && xr < W) keep[(long long)xr * G + q] = v;
                }
            }
            end_step();
            float2 *t = bufA; bufA = bufB; bufB = t;
        };

        // Phase 1: checkpoints S_{cD}, c = 0 .. nslab-1 (skipped when they come from the cache).
        if (a.ckpt_mode != 2) {
            for (int c = 0; c < a.nslab; ++c) {
                smem_to_plane<G, X>(bufA, ckpt + (long long)c * pe, W, Mp);
                if (c == a.nslab - 1) break;
                for (int l = c * D; l < (c + 1) * D; ++l) forward_step(l, nullptr, l + 1);
            }
            __syncthreads();
        }

        // Phase 2: slabs in reverse depth order.
        for (int c = a.nslab - 1; c >= 0; --c) {
            const int lb = c * D;
            const int le = lb + D < a.nextrap ? lb + D : a.nextrap;
            if (c != a.nslab - 1 || a.ckpt_mode == 2) {
                plane_to_smem<G, X>(bufA, ckpt + (long long)c * pe, W, Mp);
                __syncthreads();
            }
            // the last forward step is followed by the backward step at the same depth
            for (int l = lb; l < le; ++l) forward_step(l, slabbuf + (long long)(l - lb) * pe, l + 1 < le ? l + 1 : l);
            // V_{le-1}: m_{le-1} S_{le} on the deepest slab, else the state saved by the slab below
            {
                const float *mrow = a.refl + (long long)(le - 1) * a.nx + u0;
                const float2 *Sle = slabbuf + (long long)(le - 1 - lb) * pe;
                for (int e = threadIdx.x; e < W * G; e += blockDim.x) {
                    const int xr = e / G, qq = e - xr * G;
                    float2 v;
                    if (c == a.nslab - 1) {
                        const float m = mrow[xr];
                        const float2 s = Sle[e];
                        v = make_float2(m * s.x, m * s.y);
                    } else {
                        v = save[e];
                    }
                    bufA[pad_slot(Mp + xr, X) * G + qq] = v;
                }
            }
            __syncthreads();
            for (int l = le - 1; l >= lb; --l) {
                // next: the step above, or the next slab's first forward step
                stage_next(l > lb ? l - 1 : (c > 0 ? (c - 1) * D : -1));
                const uint16_t *idx_l = step_idx();
                // where U_l goes and which source term joins it
                const bool to_save = (l == lb) && (l > 0);
                const float2 *Sl = (l > lb) ? slabbuf + (long long)(l - 1 - lb) * pe
                                            : ckpt + (long long)c * pe;  // S_l
                const float *mrow = l > 0 ? a.refl + (long long)(l - 1) * a.nx + u0 : nullptr;
                for (int b = gid; b < nblocks; b += ngroups) {
                    const int xb = Mp + b * X;
                    float re[X], im[X];
                    if (L > 0) fir_transposed<X, (L > 0 ? L : 1), G>(a, bufA, idx_l, u0, xb, Mp, q, re, im);
                    else fir_transposed_rt<X, G>(a, bufA, idx_l, u0, xb, Mp, q, re, im);
                    int16_t own[X];
                    load_owner<X>(own_base ? own_base + b * X : nullptr, own);
#pragma unroll
                    for (int jj = 0; jj < X; ++jj) {
                        const int xr = b * X + jj;
                        const bool in = own[jj] >= 0 && xr < W;
                        float2 v = make_float2(0.f, 0.f);
                        if (in) {
                            v = make_float2(re[jj], im[jj]);
                            if (mrow) {
                                const float m = mrow[xr];
                                const float2 s = Sl[(long long)xr * G + q];
                                v.x = fmaf(m, s.x, v.x);
                                v.y = fmaf(m, s.y, v.y);
                            }
                        }
                        if (to_save) {
                            if (xr < W) save[(long long)xr * G + q] = v;
                        } else {
                            bufB[pad_slot(xb + jj, X) * G + q] = v;
                        }
                    }
                }
                end_step();
                if (!to_save) {
                    float2 *t = bufA; bufA = bufB; bufB = t;
                }
            }
        }
        // bufA holds U_0 = F* m for this group and frequency
        for (int k = grp.seg_begin; k < grp.seg_begin + grp.nseg; ++k) {
            const int4 sg = a.segs[k];
            cpx *ds = a.data + a.shot_off[sg.x] + (long long)j * sg.w;
            for (int i = threadIdx.x; i < sg.w; i += blockDim.x) {
                const float2 v = bufA[pad_slot(sg.z - u0 + i + Mp, X) * G + sg.y];
                ds[i] = cpx{v.x, v.y};
            }
        }
        __syncthreads();
    }
}

}  // namespace img2d
