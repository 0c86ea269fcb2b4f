// Second-generation cluster kernel: same decomposition and results as migrate_cluster_kernel
// (wlsq_cluster.cuh), reshaped for latency hiding on B200:
//   * 512 threads (16 warps, 4 per scheduler) at <= 128 registers, one CTA per SM, each CTA owning
//     512 consecutive positions of the item's window (one X=8 block per lane group), so a
//     2048-wide window needs a cluster of 4 CTAs (clusters of 4 pack the GPCs better than 8);
//   * the tap loop is a compact runtime loop over tap pairs with a short static prologue and
//     epilogue, which keeps the loop body in the instruction cache and serves every odd operator
//     length L >= 7 with one instance;
//   * in the default form (OPT bit 3) the operator tap pairs reach the tap loop through a small
//     per-lane-group shared-memory ring filled by cp.async a few tap pairs ahead, and the next
//     depth step's operator index and Kahan partial-image values are loaded into registers one step
//     ahead, so neither the tap loop nor the imaging read-modify-write waits on L2 or DRAM.
//
// Tap loop (input-stationary): input position t (0 <= t < X+L-1, relative to block start - M)
// contributes to output jj with tap k = t - jj when 0 <= k < L.  Taps are loaded in pairs (k, k+1)
// as one float4 when k is even; output jj keeps its current pair in tp[jj].  For t in
// [X-1, L-1] every jj is active; that middle range has an even number of steps (L odd, X even) and
// runs as a loop of two steps: at the odd step the odd jj load a new pair, at the even step the
// even jj do, and every jj uses the other half of the pair it holds.
#pragma once
#include "wlsq_cluster.cuh"

namespace img2d {

template <int NWARPS>
struct Cluster2Shape {
    static constexpr int Q = 8;            // lanes per position group
    static constexpr int G = 2 * Q;        // lane slots per item (two per lane)
    static constexpr int P = 32 / Q;       // position groups per warp
    static constexpr int NW = NWARPS;      // warps per CTA
    static constexpr int X = 8;            // positions per block
    static constexpr int PC = NW * P * X;  // positions per CTA
};

__host__ __device__ inline int cluster2_mp(int M) { return ((M + 7) / 8) * 8; }

__host__ __device__ inline size_t cluster2_smem_bytes(int M, int pc)
{
    const int mp = cluster2_mp(M);
    return (size_t)((pc + 2 * mp) + 4 * mp) * 16 * 16;
}

// One step t of the tap loop for the outputs selected by ACTIVE(jj) (compile-time in the
// prologue/epilogue).  LOAD(jj) says whether output jj starts a new tap pair at this step.
// Packed form of IMG2D_MAC8 (sm_100 FFMA2): acc (re, im) += (fr, fr) (v.re, v.im) + (-fi, fi) (v.im, v.re).
// va/vb hold (S.re, S.im, conj R.re, conj R.im) of slots q and q+8; sw* are the same pairs swapped.
#define IMG2D_MAC8P(c, fr, fi, va, vb, swa0, swa1, swb0, swb1)                                      \
    do {                                                                                            \
        const float2 t1_ = make_float2(fr, fr), t2_ = make_float2(-(fi), fi);                       \
        float2 *c2_ = reinterpret_cast<float2 *>(c);                                                \
        c2_[0] = __ffma2_rn(t1_, make_float2(va.x, va.y), c2_[0]); c2_[0] = __ffma2_rn(t2_, swa0, c2_[0]); \
        c2_[1] = __ffma2_rn(t1_, make_float2(va.z, va.w), c2_[1]); c2_[1] = __ffma2_rn(t2_, swa1, c2_[1]); \
        c2_[2] = __ffma2_rn(t1_, make_float2(vb.x, vb.y), c2_[2]); c2_[2] = __ffma2_rn(t2_, swb0, c2_[2]); \
        c2_[3] = __ffma2_rn(t1_, make_float2(vb.z, vb.w), c2_[3]); c2_[3] = __ffma2_rn(t2_, swb1, c2_[3]); \
    } while (0)

// The same sixteen FMAs grouped by tap component: each accumulator's two FMAs are eight
// instructions apart and fr / fi stay in one operand slot for eight consecutive FMAs.  Per
// accumulator the operations and their order are those of IMG2D_MAC8 (bit-identical results).
#define IMG2D_MAC8G(c, fr, fi, va, vb)                                                  \
    do {                                                                                \
        c[0] = fmaf(fr, va.x, c[0]); c[1] = fmaf(fr, va.y, c[1]);                       \
        c[2] = fmaf(fr, va.z, c[2]); c[3] = fmaf(fr, va.w, c[3]);                       \
        c[4] = fmaf(fr, vb.x, c[4]); c[5] = fmaf(fr, vb.y, c[5]);                       \
        c[6] = fmaf(fr, vb.z, c[6]); c[7] = fmaf(fr, vb.w, c[7]);                       \
        c[0] = fmaf(-fi, va.y, c[0]); c[1] = fmaf(fi, va.x, c[1]);                      \
        c[2] = fmaf(-fi, va.w, c[2]); c[3] = fmaf(fi, va.z, c[3]);                      \
        c[4] = fmaf(-fi, vb.y, c[4]); c[5] = fmaf(fi, vb.x, c[5]);                      \
        c[6] = fmaf(-fi, vb.w, c[6]); c[7] = fmaf(fi, vb.z, c[7]);                      \
    } while (0)

#define IMG2D_MAC8(c, fr, fi, va, vb)                                                   \
    do {                                                                                \
        c[0] = fmaf(fr, va.x, c[0]); c[0] = fmaf(-fi, va.y, c[0]);                      \
        c[1] = fmaf(fr, va.y, c[1]); c[1] = fmaf(fi, va.x, c[1]);                       \
        c[2] = fmaf(fr, va.z, c[2]); c[2] = fmaf(-fi, va.w, c[2]);                      \
        c[3] = fmaf(fr, va.w, c[3]); c[3] = fmaf(fi, va.z, c[3]);                       \
        c[4] = fmaf(fr, vb.x, c[4]); c[4] = fmaf(-fi, vb.y, c[4]);                      \
        c[5] = fmaf(fr, vb.y, c[5]); c[5] = fmaf(fi, vb.x, c[5]);                       \
        c[6] = fmaf(fr, vb.z, c[6]); c[6] = fmaf(-fi, vb.w, c[6]);                      \
        c[7] = fmaf(fr, vb.w, c[7]); c[7] = fmaf(fi, vb.z, c[7]);                       \
    } while (0)

// Operator-table storage of the cluster kernel: complex64 taps, or (re, im) pairs in FP16 / BF16
// (4 bytes per tap, widened to FP32 in registers; the arithmetic stays FP32).
enum TableType : int { TAB_F32 = 0, TAB_F16 = 1, TAB_BF16 = 2 };

// Taps (2i, 2i+1) of a row as one float4 (re0, im0, re1, im1).
template <int TT>
__device__ __forceinline__ float4 load_tap_pair(const void *row, int i)
{
    if (TT == TAB_F32) return __ldg(reinterpret_cast<const float4 *>(row) + i);
    const uint2 u = __ldg(reinterpret_cast<const uint2 *>(row) + i);
    float2 a, b;
    if (TT == TAB_F16) {
        a = __half22float2(*reinterpret_cast<const __half2 *>(&u.x));
        b = __half22float2(*reinterpret_cast<const __half2 *>(&u.y));
    } else {
        a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.x));
        b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.y));
    }
    return make_float4(a.x, a.y, b.x, b.y);
}

// Asynchronous 4-byte global -> shared copies (cp.async), one commit group per depth step.
__device__ __forceinline__ void cp_async4(void *smem_dst, const void *gsrc)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
// 16-byte global -> shared copy through L2 only (no L1 allocation); `bytes` (0 or 16) are read
// from global memory and the rest of the 16 are zero-filled
__device__ __forceinline__ void cp_async16_zfill(void *smem_dst, const void *gsrc, unsigned bytes)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(gsrc), "r"(bytes) : "memory");
}
// wait until at most N of this thread's most recent commit groups are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Shared memory of the step-ahead stage (OPT bit 2): per parity, one 32-bit index word and the
// Kahan partial and compensation values of every position of the CTA.
__host__ __device__ inline size_t cluster2_stage_bytes(int pc) { return (size_t)pc * (2 * 4 + 2 * 2 * 4); }

// Operator-pair ring (OPT bit 3): per lane group, kRingSlots 16-byte tap pairs of each of its X
// output rows, plus one 16-byte pad per group so that the four groups of a warp read disjoint banks.
constexpr int kRingSlots = 4;
__host__ __device__ inline size_t cluster2_ring_bytes(int pc) { return (size_t)(pc / 8) * (8 * kRingSlots + 1) * 16; }

// NWARPS: warps per CTA (positions per CTA = 32 * NWARPS).  TAP_PF: operator tap pairs are loaded one
// step ahead into a second register set.  ROW_PF: the next depth step's operator rows are prefetched
// into L1 during the current step.  OPT bit 0: FMAs grouped by tap component (IMG2D_MAC8G);
// bit 1: the next depth step's operator indices are prefetched into L1 one step ahead; bit 2: the
// next step's operator indices and Kahan partial-image rows are copied into shared memory
// (cp.async) one step ahead, so neither the index loads at the start of a step nor the imaging
// read-modify-write at its end waits on DRAM; bit 3 (instead of bit 2): the operator tap pairs reach
// the tap loop through a per-lane-group shared-memory ring instead of L1, and the next step's
// operator index and Kahan values come one step ahead in registers (see RING below).
template <int NWARPS, bool TAP_PF, bool ROW_PF, bool PACKED = false, int TT = TAB_F32, int OPT = 0>
__global__ void __launch_bounds__(NWARPS * 32, 1) migrate_cluster2_kernel(MigrateArgs a)
{
    using S = Cluster2Shape<NWARPS>;
    constexpr int Q = S::Q, G = S::G, P = S::P, X = S::X, PC = S::PC;
    constexpr bool STAGE = (OPT & 4) != 0;
    static_assert(!STAGE || Q == X, "the stage gives lane q of a group position q of its block");
    // RING: lane q of a lane group owns output q of the group's block.  It copies the tap pairs of
    // that output's operator row into the group's shared-memory ring with 16-byte cp.async through
    // L2, three tap-loop iterations before they are read, so the tap loop reads its operator taps
    // from shared memory instead of waiting on L1 sector misses.  Output jj reads its pair p at
    // iteration u = p - (X - jj) / 2 of the tap loop (the prologue has u < 0, the middle loop
    // u = 0 .. nmid-1, the epilogue u = nmid .. nmid+3) from ring slot u mod 4, so all outputs of the
    // group read slot u mod 4 at iteration u, and one commit group per iteration lets the loop wait
    // for exactly the pairs it is about to read.  The pairs with u < 0 are copied at the end of the
    // previous depth step.  The next step's operator index and Kahan partial-image values of the
    // lane's own position are loaded into registers one step ahead; lane q also does the Kahan
    // update of its position, so no other staging is needed.
    constexpr bool RING = (OPT & 8) != 0;
    static_assert(!RING || (!STAGE && TT == TAB_F32 && !TAP_PF && !ROW_PF && !PACKED && Q == X && X == 8),
                  "the ring variant is built on the 16-byte FP32 tap loop with lane q owning output q");
    const int M = a.M, L = 2 * a.M + 1;
    const int MP = cluster2_mp(M);
    const int NEXT = PC + 2 * MP;
    extern __shared__ float4 smem[];
    float4 *ext = smem;                     // [NEXT][G]; local position x at index x + MP
    float4 *stg = smem + (size_t)NEXT * G;  // [parity][side][MP][G]; side 0 = left halo, 1 = right
    // step-ahead stage (STAGE): sidx[parity][PC] index words, spart[parity][partial|comp][PC]
    unsigned *sidx = reinterpret_cast<unsigned *>(stg + (size_t)4 * MP * G);
    float *spart = reinterpret_cast<float *>(sidx + 2 * PC);
    __shared__ int s_item;

    const unsigned crank = cluster_rank(), csize = cluster_size();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int p = lane / Q, q = lane % Q;
    const int b = warp * P + p;  // this lane group's block: local positions [b*X, b*X+X)
    const int c0 = (int)crank * PC;
    const unsigned gmask = 0xffu << (p * Q);
    float *part = a.partial ? a.partial + (long long)blockIdx.x * a.nextrap * a.nx : nullptr;
    float *cmp = a.comp ? a.comp + (long long)blockIdx.x * a.nextrap * a.nx : nullptr;
    const bool push_left = crank > 0 && b * X < MP;
    const bool push_right = crank + 1 < csize && b * X + X > PC - MP;
    // RING: this lane group's ring, [output][slot] float4 plus one pad, after the halo staging
    float4 *const ringb = smem + (size_t)(NEXT + 4 * MP) * G + (size_t)b * (X * kRingSlots + 1);
    const int npairs = (L + 1) >> 1, cq = (X - q) >> 1;
    const unsigned rank0_item = map_rank(&s_item, 0);
    // row r starts at byte r * row_bytes; taps are addressed in pairs through load_tap_pair
    const char *tabb = reinterpret_cast<const char *>(TT == TAB_F32 ? (const void *)a.tabF : a.tab16);
    const int row_bytes = a.tab_stride * (TT == TAB_F32 ? 8 : 4);

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

        for (int i = threadIdx.x; i < (NEXT + 4 * MP) * G; i += blockDim.x) smem[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        __syncthreads();
        for (int k = grp.seg_begin; k < grp.seg_begin + grp.nseg; ++k) {
            const int4 sg = a.segs[k];
            const int r0 = sg.z - u0;
            const int lo = max(r0, c0 - MP), hi = min(r0 + sg.w, c0 + PC + MP);
            const cpx *ws = a.wave + a.shot_off[sg.x] + (long long)j * sg.w;
            const cpx *rs = a.shot + a.shot_off[sg.x] + (long long)j * sg.w;
            for (int x = lo + (int)threadIdx.x; x < hi; x += blockDim.x) {
                const cpx Sv = ws[x - r0], Rv = rs[x - r0];
                ext[(x - c0 + MP) * G + sg.y] = make_float4(Sv.re, Sv.im, Rv.re, -Rv.im);
            }
        }
        // cluster-wide: no CTA may push step-0 halos into a peer that is still zeroing them
        cluster_arrive();
        cluster_wait();

        const bool blk_active = c0 + b * X < W;
        const int16_t *own_a = (blk_active && q < grp.nslots)
                                   ? a.owner + grp.owner_off + (long long)q * grp.owner_stride + c0 + b * X
                                   : nullptr;
        const int16_t *own_b = (blk_active && q + Q < grp.nslots)
                                   ? a.owner + grp.owner_off + (long long)(q + Q) * grp.owner_stride + c0 + b * X
                                   : nullptr;
        unsigned in_a = 0, in_b = 0;  // bit jj: output jj of slot q (q+8) is inside a shot's aperture
        {
            int16_t oa[X], ob[X];
            load_owner<X>(own_a, oa);
            load_owner<X>(own_b, ob);
#pragma unroll
            for (int jj = 0; jj < X; ++jj) {
                in_a |= (oa[jj] >= 0 ? 1u : 0u) << jj;
                in_b |= (ob[jj] >= 0 ? 1u : 0u) << jj;
            }
        }
        const uint16_t *idx_j = a.idx + (long long)j * a.idx_jstride;
        const int xg = u0 + c0 + b * X;  // model position of the block's first output
        const bool img_lane = part && q == 0 && blk_active;
        if (img_lane && !STAGE && !RING) {
            asm volatile("prefetch.global.L1 [%0];" ::"l"(part + xg));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(cmp + xg));
        }
        // STAGE: lane q copies, for depth step ls, the aligned index word holding position xg+q and
        // that position's partial and compensation values; one commit group per step
        const int spos = b * X + q;
        const int xq = min(xg + q, a.nx - 1);
        const bool stage_img = part && c0 + spos < W;
        auto stage_step = [&](int ls) {
            if (ls < a.nextrap) {
                const uint16_t *ip = idx_j + (long long)ls * a.idx_lstride + xq;
                cp_async4(sidx + (ls & 1) * PC + spos, reinterpret_cast<const void *>(
                                                              reinterpret_cast<uintptr_t>(ip) & ~(uintptr_t)3));
                if (stage_img) {
                    cp_async4(spart + ((ls & 1) * 2 + 0) * PC + spos, part + (long long)ls * a.nx + xg + q);
                    cp_async4(spart + ((ls & 1) * 2 + 1) * PC + spos, cmp + (long long)ls * a.nx + xg + q);
                }
            }
            cp_async_commit();
        };
        if (STAGE) stage_step(0);
        // RING state of the lane's own position xg + q: its operator row at the current step, its
        // row index at the next step, and the Kahan partial/compensation values of both steps
        const uint16_t *idx_q = idx_j + xq;
        const char *row_q = tabb;
        unsigned nidx = 0;
        float cur_s = 0.f, cur_c = 0.f, nxt_s = 0.f, nxt_c = 0.f;
        // branch-free: a pair outside the row becomes a zero-filled copy of nothing (never read)
        auto ring_copy = [&](int u) {
            const int pr = u + cq;
            const bool ok = (unsigned)pr < (unsigned)npairs;
            cp_async16_zfill(ringb + q * kRingSlots + (u & (kRingSlots - 1)), row_q + (ok ? pr : 0) * 16,
                             ok ? 16u : 0u);
        };
        if (RING) {
            row_q = tabb + (size_t)idx_q[0] * row_bytes;
            for (int u = -(X / 2); u < 0; ++u) ring_copy(u);
            cp_async_commit();
            if (stage_img) {
                nxt_s = part[xg + q];
                nxt_c = cmp[xg + q];
            }
        }

        for (int l = 0; l < a.nextrap; ++l) {
            const int par = l & 1;
            const uint16_t *idx_l = idx_j + (long long)l * a.idx_lstride;
            int roff[X];  // byte offset of each output's operator row
            if (STAGE) {
                // this step's words arrived during the previous step; the group's lanes wrote them
                cp_async_wait_all();
                __syncwarp(gmask);
#pragma unroll
                for (int jj = 0; jj < X; ++jj) {
                    const unsigned wv = sidx[par * PC + b * X + jj];
                    const int xj = min(xg + jj, a.nx - 1);
                    roff[jj] = (int)((wv >> (16 * (xj & 1))) & 0xffffu) * row_bytes;
                }
                stage_step(l + 1);
            } else if (RING) {
                // this step's prologue pairs (copied at the end of the previous step) for the group
                cp_async_wait_all();
                __syncwarp();  // control flow is warp-uniform here
                cur_s = nxt_s;
                cur_c = nxt_c;
                if (l + 1 < a.nextrap) {
                    nidx = idx_q[(long long)(l + 1) * a.idx_lstride];
                    if (stage_img) {
                        nxt_s = part[(long long)(l + 1) * a.nx + xg + q];
                        nxt_c = cmp[(long long)(l + 1) * a.nx + xg + q];
                    }
                }
            } else {
#pragma unroll
                for (int jj = 0; jj < X; ++jj) roff[jj] = (int)idx_l[min(xg + jj, a.nx - 1)] * row_bytes;
            }
            if (ROW_PF && l + 1 < a.nextrap) {
                // lane q of the group fetches the 16-byte pairs of output q's next-step row into L1
                const uint16_t *idx_n = idx_l + a.idx_lstride;
                const char *rn = tabb + (long long)idx_n[min(xg + q, a.nx - 1)] * row_bytes;
                for (int c = 0; c < row_bytes; c += 128) asm volatile("prefetch.global.L1 [%0];" ::"l"(rn + c));
            }
            if ((OPT & 2) && q == 0 && l + 1 < a.nextrap)
                asm volatile("prefetch.global.L1 [%0];" ::"l"(idx_l + a.idx_lstride + min(xg, a.nx - 1)));
            if (img_lane && !STAGE && !RING && l + 1 < a.nextrap) {
                asm volatile("prefetch.global.L1 [%0];" ::"l"(part + (long long)(l + 1) * a.nx + xg));
                asm volatile("prefetch.global.L1 [%0];" ::"l"(cmp + (long long)(l + 1) * a.nx + xg));
            }
#define IMG2D_MAC(c, fr, fi, va, vb)                 \
    do {                                             \
        if (OPT & 1) IMG2D_MAC8G(c, fr, fi, va, vb); \
        else IMG2D_MAC8(c, fr, fi, va, vb);          \
    } while (0)
            float acc[X][8];
#pragma unroll
            for (int jj = 0; jj < X; ++jj)
#pragma unroll
                for (int e = 0; e < 8; ++e) acc[jj][e] = 0.f;
            float4 tp[X];
            const float4 *src = ext + (size_t)(b * X + MP - M) * G + q;

            // prologue: t = 0 .. X-2, outputs jj <= t are active
#pragma unroll
            for (int t = 0; t < X - 1; ++t) {
                const float4 va = src[(size_t)t * G];
                const float4 vb = src[(size_t)t * G + Q];
#pragma unroll
                for (int jj = 0; jj < X; ++jj) {
                    const int k = t - jj;
                    if (k >= 0) {
                        if ((k & 1) == 0)
                            tp[jj] = RING ? ringb[jj * kRingSlots + (((k >> 1) - ((X - jj) >> 1)) & (kRingSlots - 1))]
                                          : load_tap_pair<TT>(tabb + roff[jj], (k >> 1));
                        const float fr = (k & 1) ? tp[jj].z : tp[jj].x;
                        const float fi = (k & 1) ? tp[jj].w : tp[jj].y;
                        IMG2D_MAC(acc[jj], fr, fi, va, vb);
                    }
                }
                // RING: after t = 2u the slot of iteration u - 4 has been read; copy iteration u
                if (RING && (t & 1) == 0 && (t >> 1) < 3) {
                    ring_copy(t >> 1);
                    cp_async_commit();
                }
            }
            // middle: t = X-1 .. L-1 in steps of two (odd t, then even t+1)
            const float4 *sp = src + (size_t)(X - 1) * G;
            const int nmid = (L - X + 1) / 2;
            if (!TAP_PF) {
                int kbase = X - 1;  // k of output 0 at the odd step
                for (int u = 0; u < nmid; ++u, sp += 2 * G, kbase += 2) {
                    const float4 *rs = ringb + (u & (kRingSlots - 1));
                    if (RING) {
                        // iteration u - 1 has read the slot of iteration u + 3; wait for iteration u
                        ring_copy(u + 3);
                        cp_async_commit();
                        cp_async_wait<3>();
                        __syncwarp();  // control flow is warp-uniform here
                    }
                    {
                        const float4 va = sp[0];
                        const float4 vb = sp[Q];
                        const float2 swa0 = make_float2(va.y, va.x), swa1 = make_float2(va.w, va.z);
                        const float2 swb0 = make_float2(vb.y, vb.x), swb1 = make_float2(vb.w, vb.z);
#pragma unroll
                        for (int jj = 0; jj < X; ++jj) {
                            // k = kbase - jj: even for odd jj (new pair), odd for even jj (held pair)
                            if (jj & 1)
                                tp[jj] = RING ? rs[jj * kRingSlots] : load_tap_pair<TT>(tabb + roff[jj], ((kbase - jj) >> 1));
                            const float fr = (jj & 1) ? tp[jj].x : tp[jj].z;
                            const float fi = (jj & 1) ? tp[jj].y : tp[jj].w;
                            if (PACKED) IMG2D_MAC8P(acc[jj], fr, fi, va, vb, swa0, swa1, swb0, swb1);
                            else IMG2D_MAC(acc[jj], fr, fi, va, vb);
                        }
                    }
                    {
                        const float4 va = sp[G];
                        const float4 vb = sp[G + Q];
                        const float2 swa0 = make_float2(va.y, va.x), swa1 = make_float2(va.w, va.z);
                        const float2 swb0 = make_float2(vb.y, vb.x), swb1 = make_float2(vb.w, vb.z);
#pragma unroll
                        for (int jj = 0; jj < X; ++jj) {
                            if (!(jj & 1))
                                tp[jj] = RING ? rs[jj * kRingSlots]
                                              : load_tap_pair<TT>(tabb + roff[jj], ((kbase + 1 - jj) >> 1));
                            const float fr = (jj & 1) ? tp[jj].z : tp[jj].x;
                            const float fi = (jj & 1) ? tp[jj].w : tp[jj].y;
                            if (PACKED) IMG2D_MAC8P(acc[jj], fr, fi, va, vb, swa0, swa1, swb0, swb1);
                            else IMG2D_MAC(acc[jj], fr, fi, va, vb);
                        }
                    }
                }
            } else {
                // Each output's new pairs come one iteration early: iteration u uses nx_[jj] loaded
                // during iteration u-1 (odd jj at the odd step, even jj at the even step) and loads
                // the pair of iteration u+1 into the other register set.
                float4 nx_[X];
#pragma unroll
                for (int jj = 0; jj < X; ++jj) {
                    const int k0 = (X - 1) - jj + ((jj & 1) ? 0 : 1);  // first new pair's even k
                    nx_[jj] = nmid > 0 ? load_tap_pair<TT>(tabb + roff[jj], (k0 >> 1)) : make_float4(0.f, 0.f, 0.f, 0.f);
                }
                int kbase = X - 1;
                for (int u = 0; u < nmid; ++u, sp += 2 * G, kbase += 2) {
                    const bool more = u + 1 < nmid;
                    {
                        const float4 va = sp[0];
                        const float4 vb = sp[Q];
#pragma unroll
                        for (int jj = 0; jj < X; ++jj) {
                            if (jj & 1) {
                                tp[jj] = nx_[jj];
                                if (more) nx_[jj] = load_tap_pair<TT>(tabb + roff[jj], ((kbase + 2 - jj) >> 1));
                            }
                            const float fr = (jj & 1) ? tp[jj].x : tp[jj].z;
                            const float fi = (jj & 1) ? tp[jj].y : tp[jj].w;
                            IMG2D_MAC(acc[jj], fr, fi, va, vb);
                        }
                    }
                    {
                        const float4 va = sp[G];
                        const float4 vb = sp[G + Q];
#pragma unroll
                        for (int jj = 0; jj < X; ++jj) {
                            if (!(jj & 1)) {
                                tp[jj] = nx_[jj];
                                if (more) nx_[jj] = load_tap_pair<TT>(tabb + roff[jj], ((kbase + 3 - jj) >> 1));
                            }
                            const float fr = (jj & 1) ? tp[jj].z : tp[jj].x;
                            const float fi = (jj & 1) ? tp[jj].w : tp[jj].y;
                            IMG2D_MAC(acc[jj], fr, fi, va, vb);
                        }
                    }
                }
            }
            // epilogue: t = L .. L+X-2, outputs jj > t-L are active (k = t - jj <= L-1)
            const float4 *ep = src + (size_t)L * G;
            if (RING) {
                ring_copy(nmid + 3);
                cp_async_commit();
            }
#pragma unroll
            for (int e = 0; e < X - 1; ++e) {
                const float4 va = ep[(size_t)e * G];
                const float4 vb = ep[(size_t)e * G + Q];
                if (RING && (e & 1) == 0) {
                    // steps e and e + 1 read iteration nmid + e / 2; later iterations may be in flight
                    switch (e >> 1) {
                        case 0: cp_async_wait<3>(); break;
                        case 1: cp_async_wait<2>(); break;
                        case 2: cp_async_wait<1>(); break;
                        default: cp_async_wait<0>(); break;
                    }
                    __syncwarp();  // control flow is warp-uniform here
                }
#pragma unroll
                for (int jj = 0; jj < X; ++jj) {
                    if (jj > e) {
                        // k = L + e - jj, parity of (1 + e - jj) since L is odd
                        const bool even = ((1 + e - jj) & 1) == 0;
                        if (even)
                            tp[jj] = RING ? ringb[jj * kRingSlots + ((nmid + (e >> 1)) & (kRingSlots - 1))]
                                          : load_tap_pair<TT>(tabb + roff[jj], ((L + e - jj) >> 1));
                        const float fr = even ? tp[jj].x : tp[jj].z;
                        const float fi = even ? tp[jj].y : tp[jj].w;
                        IMG2D_MAC(acc[jj], fr, fi, va, vb);
                    }
                }
            }
            // outputs outside every shot aperture of their slot stay zero; most lanes have none
            if ((in_a & in_b) != (1u << X) - 1u) {
#pragma unroll
                for (int jj = 0; jj < X; ++jj) {
                    if (!((in_a >> jj) & 1u)) acc[jj][0] = acc[jj][1] = acc[jj][2] = acc[jj][3] = 0.f;
                    if (!((in_b >> jj) & 1u)) acc[jj][4] = acc[jj][5] = acc[jj][6] = acc[jj][7] = 0.f;
                }
            }
            if (RING) {
                // every ring slot has been read: copy the next step's prologue pairs (u < 0) now, so
                // that they arrive during the halo exchange and the imaging
                if (l + 1 < a.nextrap) {
                    row_q = tabb + (size_t)nidx * row_bytes;
                    for (int u = -(X / 2); u < 0; ++u) ring_copy(u);
                }
                cp_async_commit();
            }
            // halos of step l+1 into the neighbours' staging (parity par^1); see wlsq_cluster.cuh
            if (push_left) {
                float4 *dst = stg + ((size_t)((par ^ 1) * 2 + 1) * MP) * G;
#pragma unroll
                for (int jj = 0; jj < X; ++jj) {
                    const int x = b * X + jj;
                    if (x < MP) {
                        const unsigned ra = map_rank(dst + (size_t)x * G + q, crank - 1);
                        st_cluster(ra, make_float4(acc[jj][0], acc[jj][1], acc[jj][2], acc[jj][3]));
                        st_cluster(ra + Q * 16, make_float4(acc[jj][4], acc[jj][5], acc[jj][6], acc[jj][7]));
                    }
                }
            }
            if (push_right) {
                float4 *dst = stg + ((size_t)((par ^ 1) * 2 + 0) * MP) * G;
#pragma unroll
                for (int jj = 0; jj < X; ++jj) {
                    const int x = b * X + jj - (PC - MP);
                    if (x >= 0) {
                        const unsigned ra = map_rank(dst + (size_t)x * G + q, crank + 1);
                        st_cluster(ra, make_float4(acc[jj][0], acc[jj][1], acc[jj][2], acc[jj][3]));
                        st_cluster(ra + Q * 16, make_float4(acc[jj][4], acc[jj][5], acc[jj][6], acc[jj][7]));
                    }
                }
            }
            __syncthreads();  // every read of step l's values in ext[] is done
            float4 *dst = ext + (size_t)(b * X + MP) * G + q;
#pragma unroll
            for (int jj = 0; jj < X; ++jj) {
                dst[(size_t)jj * G] = make_float4(acc[jj][0], acc[jj][1], acc[jj][2], acc[jj][3]);
                dst[(size_t)jj * G + Q] = make_float4(acc[jj][4], acc[jj][5], acc[jj][6], acc[jj][7]);
            }
            cluster_arrive();
            float *prow = part ? part + (long long)l * a.nx : nullptr;
            float *crow = cmp ? cmp + (long long)l * a.nx : nullptr;
            float img_q = 0.f;  // RING: the stacked image value of the lane's own position
#pragma unroll
            for (int jj = 0; jj < X; ++jj) {
                const float ia = acc[jj][0] * acc[jj][2] - acc[jj][1] * acc[jj][3];
                const float ib = acc[jj][4] * acc[jj][6] - acc[jj][5] * acc[jj][7];
                if (a.image_shots) {
                    // per-shot images (optional output): shot ids re-read from the owner table
                    if ((in_a >> jj) & 1u)
                        atomicAdd(a.image_shots + (long long)own_a[jj] * a.img_sstride + (long long)l * a.nx + xg + jj, ia);
                    if ((in_b >> jj) & 1u)
                        atomicAdd(a.image_shots + (long long)own_b[jj] * a.img_sstride + (long long)l * a.nx + xg + jj, ib);
                }
                float img = ia + ib;
#pragma unroll
                for (int off = 1; off < Q; off <<= 1) img += __shfl_xor_sync(RING ? 0xffffffffu : gmask, img, off);
                if (RING) {
                    if (jj == q) img_q = img;
                } else if (prow && q == 0 && c0 + b * X + jj < W) {
                    if (STAGE) {
                        // kahan_add on the staged values; the stores need not be waited for
                        float sum = spart[(par * 2 + 0) * PC + b * X + jj];
                        float c = spart[(par * 2 + 1) * PC + b * X + jj];
                        const float y = img - c;
                        const float t = sum + y;
                        c = (t - sum) - y;
                        prow[xg + jj] = t;
                        crow[xg + jj] = c;
                    } else {
                        kahan_add(prow + xg + jj, crow + xg + jj, img);
                    }
                }
            }
            if (RING && stage_img) {
                // kahan_add on the values loaded a step ahead (same operations as the other forms)
                const float y = img_q - cur_c;
                const float t = cur_s + y;
                prow[xg + q] = t;
                crow[xg + q] = (t - cur_s) - y;
            }
            cluster_wait();
            const float4 *hs = stg + (size_t)((par ^ 1) * 2) * MP * G;
            for (int i = threadIdx.x; i < 2 * MP * G; i += blockDim.x) {
                const int side = i / (MP * G), r = i % (MP * G);
                ext[(side ? (PC + MP) * G : 0) + r] = hs[i];
            }
            __syncthreads();
        }
        if (a.write_back) {
            for (int k = grp.seg_begin; k < grp.seg_begin + grp.nseg; ++k) {
                const int4 sg = a.segs[k];
                const int r0 = sg.z - u0;
                const int lo = max(r0, c0), hi = min(r0 + sg.w, c0 + PC);
                cpx *ws = a.wave + a.shot_off[sg.x] + (long long)j * sg.w;
                cpx *rs = a.shot + a.shot_off[sg.x] + (long long)j * sg.w;
                for (int x = lo + (int)threadIdx.x; x < hi; x += blockDim.x) {
                    const float4 v = ext[(x - c0 + MP) * G + sg.y];
                    ws[x - r0] = cpx{v.x, v.y};
                    rs[x - r0] = cpx{v.z, -v.w};
                }
            }
        }
        __syncthreads();
    }
    cluster_arrive();
    cluster_wait();
}

#undef IMG2D_MAC
#undef IMG2D_MAC8
#undef IMG2D_MAC8G
#undef IMG2D_MAC8P

}  // namespace img2d
