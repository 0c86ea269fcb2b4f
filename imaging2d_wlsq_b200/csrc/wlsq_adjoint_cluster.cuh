// Demigration over a thread-block cluster: the adjoint of wlsq_adjoint.cuh (same recursion, same
// checkpoints and slabs, same results) with the migration cluster kernel's work shape.
//
// One item = 16 lane slots x one frequency.  Its window is split over a cluster of K CTAs of 512
// positions each.  Lane q of an 8-lane group owns slots q and q+8 as one float4 (two complex
// values), so every 16-byte operator pair load feeds 16 FMAs per lane (the single-CTA kernel, one
// slot per lane, feeds 8).  Each CTA keeps two buffers (ping-pong) of its 512 positions plus halos
// of MP = ceil8(M) positions on each side.  The outputs of a depth step go to the CTA's next buffer
// and, for the MP positions at each edge, also into the neighbouring CTA's next buffer halo through
// distributed shared memory; one cluster barrier closes the step.  The neighbours only read their
// current buffers during the step, so no staging is needed.
#pragma once
#include "wlsq_adjoint.cuh"
#include "wlsq_cluster.cuh"
#include "wlsq_cluster2.cuh"

namespace img2d {

constexpr int kDcQ = 8, kDcP = 4, kDcX = 8, kDcNW = 16;
constexpr int kDcPC = kDcNW * kDcP * kDcX;  // 512 positions per CTA

__host__ __device__ inline int demigc_mp(int M) { return ((M + 7) / 8) * 8; }

// Dynamic shared memory: two float4 buffers of (PC + 2 MP) positions x 8 lanes, two staged
// operator-index rows.
__host__ __device__ inline size_t demigc_smem_bytes(int M)
{
    const int mp = demigc_mp(M);
    return 2 * (size_t)(kDcPC + 2 * mp) * kDcQ * 16 + 2 * (size_t)demig_idx_words(kDcPC, mp) * 4;
}

__device__ __forceinline__ void mac2(float (&c)[4], float fr, float fi, const float4 v)
{
    c[0] = fmaf(fr, v.x, c[0]); c[0] = fmaf(-fi, v.y, c[0]);
    c[1] = fmaf(fr, v.y, c[1]); c[1] = fmaf(fi, v.x, c[1]);
    c[2] = fmaf(fr, v.z, c[2]); c[2] = fmaf(-fi, v.w, c[2]);
    c[3] = fmaf(fr, v.w, c[3]); c[3] = fmaf(fi, v.z, c[3]);
}

// Forward step of a block of X outputs (rows of the outputs).  src points at buffer entry 0 of this
// lane (buf + q); output jj of the block sits at buffer position pb + jj, model position xm0 + jj.
template <int X, int L>
__device__ __forceinline__ void fir2_forward(const DemigrateArgs &a, const float4 *src, const uint16_t *sidx,
                                            int xm0, int pb, int M_rt, float (&acc)[X][4])
{
    const int hstride = a.tab_stride >> 1;
    const float4 *tab4 = reinterpret_cast<const float4 *>(a.tab);
    const float4 *row[X];
#pragma unroll
    for (int jj = 0; jj < X; ++jj) {
        const int xm = min(xm0 + jj, a.nx - 1);
        row[jj] = tab4 + (long long)sidx[xm] * hstride;
        acc[jj][0] = acc[jj][1] = acc[jj][2] = acc[jj][3] = 0.f;
    }
    if (L > 0) {
        constexpr int M = (L > 0 ? L - 1 : 0) / 2;
        float4 tf[X];
#pragma unroll
        for (int t = 0; t < X + L - 1; ++t) {
            const float4 v = src[(pb - M + t) * kDcQ];
#pragma unroll
            for (int jj = 0; jj < X; ++jj) {
                const int k = t - jj;
                if (k >= 0 && k < L) {
                    if ((k & 1) == 0) tf[jj] = __ldg(row[jj] + (k >> 1));
                    mac2(acc[jj], (k & 1) ? tf[jj].z : tf[jj].x, (k & 1) ? tf[jj].w : tf[jj].y, v);
                }
            }
        }
    } else {
        const int Lr = 2 * M_rt + 1;
#pragma unroll
        for (int jj = 0; jj < X; ++jj) {
            const cpx *r = reinterpret_cast<const cpx *>(row[jj]);
            for (int k = 0; k < Lr; ++k) {
                const float4 v = src[(pb + jj - M_rt + k) * kDcQ];
                const cpx f = r[k];
                mac2(acc[jj], f.re, f.im, v);
            }
        }
    }
}

// The forward step with the operator pairs read from the lane group's shared-memory ring (the
// migration kernel's scheme): lane q copies the pairs of output q's row with 16-byte cp.async through
// L2, three tap-loop iterations before they are read.  Output jj reads pair p at iteration
// u = p - (X - jj) / 2 from slot u mod 4; iteration u's reads happen at steps t = 2u+7 (odd jj) and
// 2u+8 (even jj).  The pairs with u < 0 are copied on entry, u = 0, 1, 2 after steps 0, 2, 4, and
// u + 3 at the start of iteration u, one commit group each.  Same taps, same FMA order as
// fir2_forward.
template <int X, int L>
__device__ __forceinline__ void fir2_forward_ring(const DemigrateArgs &a, const float4 *src, const uint16_t *sidx,
                                                 int xm0, int pb, int q, float4 *ring, float (&acc)[X][4])
{
    static_assert(L > 0 && X == 8 && kDcQ == X, "lane q owns output q of the block");
    constexpr int M = (L - 1) / 2, NP = (L + 1) / 2;
    const int hstride = a.tab_stride >> 1;
    const float4 *rowq = reinterpret_cast<const float4 *>(a.tab) + (long long)sidx[min(xm0 + q, a.nx - 1)] * hstride;
    const int cq = (X - q) >> 1;
    auto copy = [&](int u) {
        const int pr = u + cq;
        const bool ok = (unsigned)pr < (unsigned)NP;
        cp_async16_zfill(ring + q * kRingSlots + (u & (kRingSlots - 1)), rowq + (ok ? pr : 0), ok ? 16u : 0u);
    };
#pragma unroll
    for (int u = -(X / 2); u < 0; ++u) copy(u);
    cp_async_commit();
    cp_async_wait<0>();
    __syncwarp();
#pragma unroll
    for (int jj = 0; jj < X; ++jj) acc[jj][0] = acc[jj][1] = acc[jj][2] = acc[jj][3] = 0.f;
    float4 tf[X];
#pragma unroll
    for (int t = 0; t < X + L - 1; ++t) {
        if (t >= X - 1 && ((t - (X - 1)) & 1) == 0) {
            // start of iteration u: copy iteration u + 3, wait for iteration u
            const int u = (t - (X - 1)) >> 1;
            if (u + 3 <= NP - 1) {
                copy(u + 3);
                cp_async_commit();
            }
            const int newer = (u + 3 < NP - 1 ? u + 3 : NP - 1) - u;
            if (newer >= 3) cp_async_wait<3>();
            else if (newer == 2) cp_async_wait<2>();
            else if (newer == 1) cp_async_wait<1>();
            else cp_async_wait<0>();
            __syncwarp();
        }
        const float4 v = src[(pb - M + t) * kDcQ];
#pragma unroll
        for (int jj = 0; jj < X; ++jj) {
            const int k = t - jj;
            if (k >= 0 && k < L) {
                if ((k & 1) == 0) tf[jj] = ring[jj * kRingSlots + (((k >> 1) - ((X - jj) >> 1)) & (kRingSlots - 1))];
                mac2(acc[jj], (k & 1) ? tf[jj].z : tf[jj].x, (k & 1) ? tf[jj].w : tf[jj].y, v);
            }
        }
        if (t < 6 && (t & 1) == 0 && (t >> 1) <= NP - 1) {
            copy(t >> 1);
            cp_async_commit();
        }
    }
}

// Transposed step of a block of X outputs: output y takes tap y+M-i of the row of input i.
template <int X, int L>
__device__ __forceinline__ void fir2_transposed(const DemigrateArgs &a, const float4 *src, const uint16_t *sidx,
                                               int xm0, int pb, int M_rt, float (&acc)[X][4])
{
    const int hstride = a.tab_stride >> 1;
    const float4 *tab4 = reinterpret_cast<const float4 *>(a.tab);
#pragma unroll
    for (int jj = 0; jj < X; ++jj) acc[jj][0] = acc[jj][1] = acc[jj][2] = acc[jj][3] = 0.f;
    if (L > 0) {
        constexpr int M = (L > 0 ? L - 1 : 0) / 2;
#pragma unroll
        for (int t = 0; t < X + L - 1; ++t) {
            const float4 v = src[(pb - M + t) * kDcQ];
            int xm = xm0 - M + t;
            xm = xm < 0 ? 0 : (xm < a.nx ? xm : a.nx - 1);
            const float4 *rp = tab4 + (long long)sidx[xm] * hstride;
            float4 cur = make_float4(0.f, 0.f, 0.f, 0.f);
            const int jj0 = t - 2 * M > 0 ? t - 2 * M : 0;
#pragma unroll
            for (int jj = 0; jj < X; ++jj) {
                const int k = jj + 2 * M - t;
                if (k >= 0 && k < L) {
                    if ((k & 1) == 0 || jj == jj0) cur = __ldg(rp + (k >> 1));
                    mac2(acc[jj], (k & 1) ? cur.z : cur.x, (k & 1) ? cur.w : cur.y, v);
                }
            }
        }
    } else {
        const int Lr = 2 * M_rt + 1;
#pragma unroll
        for (int jj = 0; jj < X; ++jj) {
            for (int k = 0; k < Lr; ++k) {
                const int d = jj + M_rt - k;  // input offset from the block start
                const float4 v = src[(pb + d) * kDcQ];
                int xm = xm0 + d;
                xm = xm < 0 ? 0 : (xm < a.nx ? xm : a.nx - 1);
                const cpx f = a.tab[(long long)sidx[xm] * a.tab_stride + k];
                mac2(acc[jj], f.re, f.im, v);
            }
        }
    }
}

// Shared memory of the forward step's tap-pair ring (RING): per lane group X rows x kRingSlots
// pairs plus one 16-byte pad, after the index rows rounded up to 16 bytes.
__host__ __device__ inline size_t demigc_ring_offset(int M) { return (demigc_smem_bytes(M) + 15) / 16 * 16; }
__host__ __device__ inline size_t demigc_ring_smem_bytes(int M)
{
    return demigc_ring_offset(M) + (size_t)(kDcPC / kDcX) * (kDcX * kRingSlots + 1) * 16;
}

// L > 0: compile-time operator length; L == 0: runtime length a.M.  work / ckpt_items hold float4
// planes of PC x 8 lanes per CTA: per CTA ckpt[nslab], slab[D], save; the cache [item][rank][nslab].
// RING (L > 0): the forward steps read their operator pairs through the lane group's shared-memory
// ring (fir2_forward_ring), and the next step's index row is loaded into registers at the start of
// a step and stored to shared memory at its end, so the ring's cp.async groups are the only ones.
template <int L, bool RING = false>
__global__ void __launch_bounds__(kDcNW * 32, 1) demigrate_cluster_kernel(DemigrateArgs a)
{
    static_assert(!RING || L > 0, "the ring needs a compile-time operator length");
    constexpr int Q = kDcQ, P = kDcP, X = kDcX, PC = kDcPC;
    const int M = L > 0 ? (L - 1) / 2 : a.M;
    const int MP = demigc_mp(M);
    const int NPOS = PC + 2 * MP;
    extern __shared__ float4 sm4[];
    __shared__ int s_item;
    float4 *buf0 = sm4, *buf1 = sm4 + (size_t)NPOS * Q;
    unsigned *sidx0 = reinterpret_cast<unsigned *>(sm4 + (size_t)2 * NPOS * Q);
    unsigned *sidx1 = sidx0 + demig_idx_words(PC, MP);

    const unsigned crank = cluster_rank(), csize = cluster_size();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int p = lane / Q, q = lane % Q;
    const int b = warp * P + p;  // this lane group's block: local positions [b*X, b*X+X)
    const int c0 = (int)crank * PC;
    const bool has_left = crank > 0, has_right = crank + 1 < csize;
    float4 *const ring = reinterpret_cast<float4 *>(reinterpret_cast<char *>(sm4) + demigc_ring_offset(M)) +
                         (size_t)b * (X * kRingSlots + 1);
    const unsigned rank0_item = map_rank(&s_item, 0);
    const long long pe = (long long)PC * Q;  // float4 per plane
    float4 *work = reinterpret_cast<float4 *>(a.work) + (long long)blockIdx.x * (a.work_cta / 2);
    float4 *slabbuf = work + (long long)a.nslab * pe;
    float4 *save = slabbuf + (long long)a.slab * pe;
    const int D = a.slab;

    for (;;) {
        if (crank == 0 && threadIdx.x == 0) s_item = atomicAdd(a.counter, 1);
        cluster_arrive();
        cluster_wait();
        const int it = ld_cluster_s32(rank0_item);
        cluster_arrive();
        cluster_wait();
        if (it >= a.n_items) break;
        const int2 item = a.items[it];
        const GroupDesc grp = a.groups[item.x];
        const int j = item.y, u0 = grp.u0, W = grp.W;
        const int base = u0 + c0;  // model position of local position 0
        const uint16_t *idx_j = a.idx + (long long)j * a.idx_jstride;
        float4 *ckpt = a.ckpt_mode != 0
                           ? reinterpret_cast<float4 *>(a.ckpt_items) + ((long long)it * csize + crank) * a.nslab * pe
                           : work;
        const int first_l = a.ckpt_mode == 2 ? (a.nslab - 1) * D : 0;
        const int ibase = 2 * (max(0, base - MP) >> 1);
        demig_stage_idx(a, idx_j, first_l, base, PC, MP, sidx0);
        for (int i = threadIdx.x; i < 2 * NPOS * Q; i += blockDim.x) sm4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        __syncthreads();
        float4 *bufA = buf0, *bufB = buf1;
        if (a.ckpt_mode != 2) {
            // source spectra of the group at frequency j: interior and halos straight from global
            for (int k = grp.seg_begin; k < grp.seg_begin + grp.nseg; ++k) {
                const int4 sg = a.segs[k];
                const int r0 = sg.z - u0;
                const int lo = max(r0, c0 - MP), hi = min(r0 + sg.w, c0 + PC + MP);
                const cpx *ws = a.wave + a.shot_off[sg.x] + (long long)j * sg.w;
                float *dst = reinterpret_cast<float *>(bufA) + (sg.y / Q) * 2;
                for (int x = lo + (int)threadIdx.x; x < hi; x += blockDim.x) {
                    const cpx Sv = ws[x - r0];
                    float *e = dst + ((long long)(x - c0 + MP) * Q + (sg.y % Q)) * 4;
                    e[0] = Sv.re;
                    e[1] = Sv.im;
                }
            }
        }
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        // every CTA of the cluster has zeroed its buffers before any neighbour writes a halo
        cluster_arrive();
        cluster_wait();

        const bool blk_active = c0 + b * X < W;
        unsigned in_a = 0, in_b = 0;  // bit jj: output jj of slot q (q+8) lies in a shot's aperture
        {
            const int16_t *oa = (blk_active && q < grp.nslots)
                                    ? a.owner + grp.owner_off + (long long)q * grp.owner_stride + c0 + b * X
                                    : nullptr;
            const int16_t *ob = (blk_active && q + Q < grp.nslots)
                                    ? a.owner + grp.owner_off + (long long)(q + Q) * grp.owner_stride + c0 + b * X
                                    : nullptr;
            int16_t va[X], vb[X];
            load_owner<X>(oa, va);
            load_owner<X>(ob, vb);
#pragma unroll
            for (int jj = 0; jj < X; ++jj) {
                in_a |= (va[jj] >= 0 ? 1u : 0u) << jj;
                in_b |= (vb[jj] >= 0 ? 1u : 0u) << jj;
            }
        }
        const int xm0 = base + b * X;   // model position of this block's output 0
        const int pb = MP + b * X;      // its buffer position
        unsigned *cur = sidx0, *nxt = sidx1;
        auto step_idx = [&]() { return reinterpret_cast<const uint16_t *>(cur) - ibase; };
        // RING: this thread's word of the next step's index row (at most one: the row has fewer
        // words than the CTA has threads), loaded at the start of a step, stored at its end
        unsigned iw = 0;
        int iw_k = -1;
        auto stage_next = [&](int nl) {
            if (RING) {
                iw_k = -1;
                if (nl >= 0) {
                    const int lo = max(0, base - MP) >> 1, hi = (min(a.nx, base + PC + MP) + 1) >> 1;
                    const int k = lo + (int)threadIdx.x;
                    if (k < hi) {
                        iw = reinterpret_cast<const unsigned *>(idx_j + (long long)nl * a.idx_lstride)[k];
                        iw_k = k - lo;
                    }
                }
            } else if (nl >= 0) {
                demig_stage_idx(a, idx_j, nl, base, PC, MP, nxt);
            }
        };
        auto end_step = [&]() {
            if (RING) {
                if (iw_k >= 0) nxt[iw_k] = iw;
            } else {
                asm volatile("cp.async.wait_group 0;" ::: "memory");
            }
            cluster_arrive();
            cluster_wait();
            unsigned *t = cur; cur = nxt; nxt = t;
        };
        // value of local position x (0 <= x < PC) into buffer `dst` here and, at the edges, into the
        // neighbour's halo of the same buffer
        auto put = [&](float4 *dst, int x, float4 v, int lq) {
            dst[(x + MP) * Q + lq] = v;
            if (has_left && x < MP) st_cluster(map_rank(dst + (x + PC + MP) * Q + lq, crank - 1), v);
            if (has_right && x >= PC - MP) st_cluster(map_rank(dst + (x - PC + MP) * Q + lq, crank + 1), v);
        };
        // after the interior of `buf` was loaded: edges to the neighbours' halos, then the barrier
        auto exchange = [&](float4 *buf) {
            for (int e = threadIdx.x; e < 2 * MP * Q; e += blockDim.x) {
                const int side = e / (MP * Q), r = e - side * MP * Q;
                const int x = side ? PC - MP + r / Q : r / Q, lq = r % Q;
                const float4 v = buf[(x + MP) * Q + lq];
                if (side == 0 && has_left) st_cluster(map_rank(buf + (x + PC + MP) * Q + lq, crank - 1), v);
                if (side == 1 && has_right) st_cluster(map_rank(buf + (x - PC + MP) * Q + lq, crank + 1), v);
            }
            cluster_arrive();
            cluster_wait();
        };
        auto mask = [&](float (&c)[4], int jj) {
            const bool live = c0 + b * X + jj < W;
            if (!live || !((in_a >> jj) & 1u)) c[0] = c[1] = 0.f;
            if (!live || !((in_b >> jj) & 1u)) c[2] = c[3] = 0.f;
        };

        // forward step l -> l+1 of the source; keep: plane for S_{l+1} or null; nl: next depth step
        auto forward_step = [&](int l, float4 *keep, int nl) {
            stage_next(nl);
            float acc[X][4];
            if constexpr (RING) fir2_forward_ring<X, L>(a, bufA + q, step_idx(), xm0, pb, q, ring, acc);
            else fir2_forward<X, L>(a, bufA + q, step_idx(), xm0, pb, M, acc);
#pragma unroll
            for (int jj = 0; jj < X; ++jj) {
                mask(acc[jj], jj);
                const float4 v = make_float4(acc[jj][0], acc[jj][1], acc[jj][2], acc[jj][3]);
                put(bufB, b * X + jj, v, q);
                if (keep) keep[(b * X + jj) * Q + q] = v;
            }
            end_step();
            float4 *t = bufA; bufA = bufB; bufB = t;
        };

        // Phase 1: checkpoints S_{cD} (skipped when they come from the cache)
        if (a.ckpt_mode != 2) {
            for (int c = 0; c < a.nslab; ++c) {
                // checkpoints are read once, a slab sweep later: evict-first in L2, so that the slab
                // planes (re-read within D steps) keep their L2 lines
                for (int e = threadIdx.x; e < PC * Q; e += blockDim.x) __stcs(ckpt + (long long)c * pe + e, bufA[MP * Q + e]);
                if (c == a.nslab - 1) break;
                for (int l = c * D; l < (c + 1) * D; ++l) forward_step(l, nullptr, l + 1);
            }
            __syncthreads();
        }

        // Phase 2: slabs in reverse depth order
        for (int c = a.nslab - 1; c >= 0; --c) {
            const int lb = c * D;
            const int le = lb + D < a.nextrap ? lb + D : a.nextrap;
            if (c != a.nslab - 1 || a.ckpt_mode == 2) {
                for (int e = threadIdx.x; e < PC * Q; e += blockDim.x) bufA[MP * Q + e] = __ldcs(ckpt + (long long)c * pe + e);
                __syncthreads();
                exchange(bufA);
            }
            for (int l = lb; l < le; ++l)
                forward_step(l, slabbuf + (long long)(l - lb) * pe, l + 1 < le ? l + 1 : l);
            // V_{le-1}: m_{le-1} S_{le} on the deepest slab, else the state the slab below saved
            {
                const float *mrow = a.refl + (long long)(le - 1) * a.nx + base;
                const float4 *Sle = slabbuf + (long long)(le - 1 - lb) * pe;
                for (int e = threadIdx.x; e < PC * Q; e += blockDim.x) {
                    const int x = e / Q;
                    float4 v;
                    if (c == a.nslab - 1) {
                        const float m = c0 + x < W ? mrow[x] : 0.f;
                        const float4 s = Sle[e];
                        v = make_float4(m * s.x, m * s.y, m * s.z, m * s.w);
                    } else {
                        v = save[e];
                    }
                    bufA[MP * Q + e] = v;
                }
                __syncthreads();
                exchange(bufA);
            }
            for (int l = le - 1; l >= lb; --l) {
                stage_next(l > lb ? l - 1 : (c > 0 ? (c - 1) * D : -1));
                const bool to_save = (l == lb) && (l > 0);
                const float4 *Sl = (l > lb) ? slabbuf + (long long)(l - 1 - lb) * pe : ckpt + (long long)c * pe;
                const float *mrow = l > 0 ? a.refl + (long long)(l - 1) * a.nx + base : nullptr;
                if (mrow) {
                    // the source plane and reflectivity row the emission after the FIR reads, into L1
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(Sl + (long long)(b * X + q) * Q));
                    if (q == 0) asm volatile("prefetch.global.L1 [%0];" ::"l"(mrow + b * X));
                }
                float acc[X][4];
                fir2_transposed<X, L>(a, bufA + q, step_idx(), xm0, pb, M, acc);
#pragma unroll
                for (int jj = 0; jj < X; ++jj) {
                    mask(acc[jj], jj);
                    const int x = b * X + jj;
                    float4 v = make_float4(acc[jj][0], acc[jj][1], acc[jj][2], acc[jj][3]);
                    if (mrow && c0 + x < W) {
                        const float m = mrow[x];
                        const float4 s = Sl[x * Q + q];  // zero outside the apertures
                        v.x = fmaf(m, s.x, v.x);
                        v.y = fmaf(m, s.y, v.y);
                        v.z = fmaf(m, s.z, v.z);
                        v.w = fmaf(m, s.w, v.w);
                    }
                    if (to_save) save[x * Q + q] = v;
                    else put(bufB, x, v, q);
                }
                end_step();
                if (!to_save) {
                    float4 *t = bufA; bufA = bufB; bufB = t;
                }
            }
        }
        // bufA holds U_0 = F* m for this CTA's positions
        for (int k = grp.seg_begin; k < grp.seg_begin + grp.nseg; ++k) {
            const int4 sg = a.segs[k];
            const int r0 = sg.z - u0;
            const int lo = max(r0, c0), hi = min(r0 + sg.w, c0 + PC);
            cpx *ds = a.data + a.shot_off[sg.x] + (long long)j * sg.w;
            const float *srcf = reinterpret_cast<const float *>(bufA) + (sg.y / Q) * 2;
            for (int x = lo + (int)threadIdx.x; x < hi; x += blockDim.x) {
                const float *e = srcf + ((long long)(x - c0 + MP) * Q + (sg.y % Q)) * 4;
                ds[x - r0] = cpx{e[0], e[1]};
            }
        }
        __syncthreads();
    }
    cluster_arrive();
    cluster_wait();
}

}  // namespace img2d
