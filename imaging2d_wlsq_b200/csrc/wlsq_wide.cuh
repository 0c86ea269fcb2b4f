// Wide cluster kernel: the decomposition of migrate_cluster2_kernel (wlsq_cluster2.cuh) reshaped so
// that a 2048-wide window needs a cluster of 2 CTAs instead of 4.
//
// Why: one CTA per SM holds one share of an item for the whole depth loop.  Clusters of 4 fit 33
// times on the 148 SMs of a B200 (132 SMs busy, because clusters cannot span GPCs), clusters of 2
// fit 74 times (all 148).  Each CTA here owns 1024 consecutive positions of 8 lane slots instead of
// 512 positions of 16 slots: the same 8192 (slot, position) pairs, the same shared memory for the
// wavefields, the same per-lane work (2 slots x 8 outputs) and the same operator reuse per load
// (each 16-byte tap pair feeds 2 taps x 2 slots x (S, conj R) = 32 FMAs of one lane).  An item
// carries 8 slots (one frequency), so there are twice as many items, each half as tall.
//
// Layout.  Lane group = 4 lanes; lane q holds slots q and q+4 of the item; 8 groups per warp, each
// over a block of X = 8 consecutive positions; 16 warps.  The wavefields of a position are 128
// bytes: for each lane q two float4, A = (S_a.re, S_b.re, S_a.im, S_b.im) and B = the same of
// conj(R) (a = slot q, b = slot q+4), so the two slots of a lane form the (x, y) halves of packed
// pairs.  The 8 groups of a warp read rows 8 positions apart, which without care would all hit
// banks 0-15; the A and B columns of a row are therefore swapped in every other 8-row block
// (column 2q + (h ^ ((pos >> 3) & 1)) for half h), so each bank serves 4 of the 32 lanes and a
// warp's 512-byte read takes the minimum 4 wavefronts.
//
// Arithmetic (per input t, output jj, tap (fr, fi)), for each of A and B:
//   re.ab += fr * v.re.ab ; re.ab += -fi * v.im.ab ; im.ab += fr * v.im.ab ; im.ab += fi * v.re.ab
// in that order per element, which is the FMA sequence of every other kernel of this library
// (IMG2D_MAC8), so final wavefields are bit-identical to migrate_cluster2_kernel.  ARITH = 1 issues
// it as packed f32x2 FMAs (FFMA2: two lanes of work per instruction), ARITH = 0 as scalar FMAs.
//
// Operator taps reach the tap loop through the per-lane-group shared-memory ring of the cluster2
// ring variant: lane q owns outputs q and q+4 of its group's block and copies their tap pairs with
// 16-byte cp.async three tap-loop iterations before they are read.  The next depth step's operator
// indices and this step's Kahan partial-image values of those two positions reach the thread
// through a per-thread shared-memory stage filled by cp.async a step ahead (STAGE, where the
// shared memory allows), or are loaded into registers at the start of the step.  The BULK variant
// fills the same ring with 1-D bulk copies completing on per-warp transaction-count barriers.
//
// Per depth step: tap loop into registers; aperture mask; edge outputs pushed into the neighbour's
// halo staging (distributed shared memory, double-buffered by step parity); cluster barrier arrive
// (release of the pushes); the next step's first tap pairs copied; __syncthreads;
// in-place write; imaging (Re(S conj R), shuffle over the group's 4 lanes, Kahan update of the
// CTA's private partial row); cluster barrier wait; halo copy; __syncthreads.
#pragma once
#include "wlsq_cluster2.cuh"

namespace img2d {

struct WideShape {
    static constexpr int Q = 4;            // lanes per position group
    static constexpr int G = 2 * Q;        // lane slots per item (two per lane)
    static constexpr int P = 32 / Q;       // position groups per warp
    static constexpr int NW = 16;          // warps per CTA
    static constexpr int X = 8;            // positions per block
    static constexpr int PC = NW * P * X;  // positions per CTA (1024)
    static constexpr int NG = NW * P;      // lane groups per CTA (128)
    static constexpr int RING = 8 * kRingSlots + 1;  // float4 per lane group's ring (+1 pad)
};

// Shared memory: ext[PC + 2 MP] rows + staging[2 parity][2 side][MP] rows (8 float4 per row) +
// the operator-pair rings.
__host__ __device__ inline size_t wide_smem_bytes(int M)
{
    const int mp = cluster2_mp(M);
    return (size_t)((WideShape::PC + 2 * mp) + 4 * mp) * WideShape::G * 16 +
           (size_t)WideShape::NG * WideShape::RING * 16;
}

// Step-ahead stage (STAGE): per thread 6 words after the rings, the aligned index words holding the
// next depth step's operator indices of its two outputs and this step's Kahan partial and
// compensation values of its two positions.  Each thread reads only its own words, then refills
// them with cp.async for a later step.
constexpr int kWideStageWords = 6;
__host__ __device__ inline size_t wide_stage_smem_bytes(int M)
{
    return wide_smem_bytes(M) + (size_t)WideShape::NW * 32 * kWideStageWords * 4;
}

// BULK: two transaction-count barriers per warp after the stage words (or the rings), one per
// alternate ring chunk.
__host__ __device__ inline size_t wide_bulk_bar_offset(int M, bool stage)
{
    return stage ? wide_stage_smem_bytes(M) : wide_smem_bytes(M);
}
__host__ __device__ inline size_t wide_bulk_smem_bytes(int M, bool stage)
{
    return wide_bulk_bar_offset(M, stage) + (size_t)WideShape::NW * 2 * sizeof(unsigned long long);
}

// SM clock cycles (about a second) after which a ring-chunk wait gives up: the thread then records
// the failure in the launch's status word and neither waits for nor issues ring chunks again, so a
// phase that can never complete ends the launch instead of hanging it.
constexpr long long kBulkWaitCycles = 1ll << 31;

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// the initialisations above become visible to the asynchronous (bulk-copy) proxy
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// arrive on the barrier's current phase, first raising its expected transaction bytes
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
                     smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity)
{
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// 1-D bulk copy global -> this CTA's shared memory, completing bytes on the barrier (no multicast)
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// float4 column of half h (0 = S, 1 = conj R) of lane q in row pos
__device__ __forceinline__ int wide_col(int pos, int q, int h) { return 2 * q + (h ^ ((pos >> 3) & 1)); }

template <int ARITH>
__device__ __forceinline__ void wide_mac(float (&c)[8], float fr, float fi, const float4 &va, const float4 &vb)
{
    if (ARITH == 1) {
        const float2 frr = make_float2(fr, fr), nfi = make_float2(-fi, -fi), fii = make_float2(fi, fi);
        float2 *c2 = reinterpret_cast<float2 *>(c);
        c2[0] = __ffma2_rn(frr, make_float2(va.x, va.y), c2[0]);
        c2[0] = __ffma2_rn(nfi, make_float2(va.z, va.w), c2[0]);
        c2[1] = __ffma2_rn(frr, make_float2(va.z, va.w), c2[1]);
        c2[1] = __ffma2_rn(fii, make_float2(va.x, va.y), c2[1]);
        c2[2] = __ffma2_rn(frr, make_float2(vb.x, vb.y), c2[2]);
        c2[2] = __ffma2_rn(nfi, make_float2(vb.z, vb.w), c2[2]);
        c2[3] = __ffma2_rn(frr, make_float2(vb.z, vb.w), c2[3]);
        c2[3] = __ffma2_rn(fii, make_float2(vb.x, vb.y), c2[3]);
    } else {
        c[0] = fmaf(fr, va.x, c[0]); c[0] = fmaf(-fi, va.z, c[0]);
        c[1] = fmaf(fr, va.y, c[1]); c[1] = fmaf(-fi, va.w, c[1]);
        c[2] = fmaf(fr, va.z, c[2]); c[2] = fmaf(fi, va.x, c[2]);
        c[3] = fmaf(fr, va.w, c[3]); c[3] = fmaf(fi, va.y, c[3]);
        c[4] = fmaf(fr, vb.x, c[4]); c[4] = fmaf(-fi, vb.z, c[4]);
        c[5] = fmaf(fr, vb.y, c[5]); c[5] = fmaf(-fi, vb.w, c[5]);
        c[6] = fmaf(fr, vb.z, c[6]); c[6] = fmaf(fi, vb.x, c[6]);
        c[7] = fmaf(fr, vb.w, c[7]); c[7] = fmaf(fi, vb.y, c[7]);
    }
}

// STAGE: the next step's operator indices and this step's Kahan values reach the thread through its
// shared-memory stage words, copied by cp.async one step ahead (no register holds a pending load
// across the tap loop); otherwise they are loaded into registers at the start of the step.
//
// BULK: the operator-pair ring is filled by 1-D bulk copies (cp.async.bulk, the copy engine of
// the SM) instead of per-lane 16-byte cp.async.  Ring iterations are copied in chunks of two (v
// even: the slots of v and v + 1 are adjacent), one bulk copy of up to 32 bytes per output, each
// chunk completing on one of two transaction-count barriers of the warp (alternating), where the
// cp.async ring would wait for a commit group.  A chunk is issued where the cp.async ring copies
// its later iteration and waited for where the ring waits for its first one.
template <int ARITH, bool STAGE, bool BULK = false>
__global__ void __launch_bounds__(WideShape::NW * 32, 1) migrate_wide_kernel(MigrateArgs a)
{
    using S = WideShape;
    constexpr int Q = S::Q, G = S::G, P = S::P, X = S::X, PC = S::PC;
    const int M = a.M, L = 2 * a.M + 1;
    const int MP = cluster2_mp(M);
    const int NEXT = PC + 2 * MP;
    extern __shared__ float4 smem[];
    float4 *ext = smem;                     // [NEXT][G]; local position x at row x + MP
    float4 *stg = smem + (size_t)NEXT * G;  // [parity][side][MP][G]; side 0 = left halo, 1 = right
    float *extf = reinterpret_cast<float *>(ext);
    __shared__ int s_item;

    const unsigned crank = cluster_rank(), csize = cluster_size();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int p = lane / Q, q = lane % Q;
    const int b = warp * P + p;  // this lane group's block: local positions [b*X, b*X+X)
    // this lane group's ring, [output][slot] float4 plus one pad, after the halo staging
    float4 *const ringb = smem + (size_t)(NEXT + 4 * MP) * G + (size_t)b * S::RING;
    // STAGE: this thread's words [idx word of output q, of q+4, s0, c0, s1, c1]
    unsigned *const sst = reinterpret_cast<unsigned *>(smem + (size_t)(NEXT + 4 * MP) * G + (size_t)S::NG * S::RING) +
                          (size_t)threadIdx.x * kWideStageWords;
    const int npairs = (L + 1) >> 1;
    static_assert(X == 8 && kRingSlots == 4, "the ring schedule assumes 8 outputs per block and 4 slots");
    // BULK: this warp's two chunk barriers, the chunks it has issued and waited for (warp-uniform)
    unsigned long long *const wbar =
        reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(smem) + wide_bulk_bar_offset(M, STAGE)) +
        warp * 2;
    unsigned n_issued = 0, n_waited = 0;
    bool bulk_failed = false;
    if (BULK) {
        if (lane == 0) {
            mbar_init(wbar, 32);  // one arrival per lane and chunk
            mbar_init(wbar + 1, 32);
            mbar_init_fence();
        }
        __syncwarp();
    }
    const unsigned rank0_item = map_rank(&s_item, 0);
    const int row_bytes = a.tab_stride * 8;
    // register budget (512 threads at <= 128 registers): the partial-image, table and owner
    // pointers are formed from the kernel parameters where they are used

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
        // The item's window is split evenly over the cluster in units of 4 warps (256 positions, one
        // warp per SM sub-partition): each CTA owns NC <= PC consecutive positions starting at c0,
        // and warps past NC skip the step's work.  A narrow window then leaves every sub-partition
        // one warp less to run instead of computing positions past the window (finer units would
        // leave the busiest sub-partition as loaded as before).
        const int NC = min(PC, (W + (int)csize * 256 - 1) / ((int)csize * 256) * 256);
        const int c0 = (int)crank * NC;
        const int own = max(0, min(NC, W - c0));  // window positions this CTA owns (the rest are past W)
        const bool warp_active = warp * (P * X) < NC;
        const bool push_left = crank > 0 && b * X < MP;
        const bool push_right = crank + 1 < csize && b * X + X > NC - MP && b * X < NC;

        for (int i = threadIdx.x; i < (NEXT + 4 * MP) * G; i += blockDim.x) smem[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        __syncthreads();
        for (int k = grp.seg_begin; k < grp.seg_begin + grp.nseg; ++k) {
            const int4 sg = a.segs[k];
            const int r0 = sg.z - u0;
            const int lo = max(r0, c0 - MP), hi = min(r0 + sg.w, c0 + NC + MP);
            const cpx *ws = a.wave + a.shot_off[sg.x] + (long long)j * sg.w;
            const cpx *rs = a.shot + a.shot_off[sg.x] + (long long)j * sg.w;
            const int sq = sg.y & (Q - 1), sh = sg.y / Q;  // lane and half (x/z or y/w) of the slot
            for (int x = lo + (int)threadIdx.x; x < hi; x += blockDim.x) {
                const cpx Sv = ws[x - r0], Rv = rs[x - r0];
                const int pos = x - c0 + MP;
                float *fa = extf + ((size_t)pos * G + wide_col(pos, sq, 0)) * 4;
                float *fb = extf + ((size_t)pos * G + wide_col(pos, sq, 1)) * 4;
                fa[sh] = Sv.re;
                fa[2 + sh] = Sv.im;
                fb[sh] = Rv.re;
                fb[2 + sh] = -Rv.im;
            }
        }
        // cluster-wide: no CTA may push step-0 halos into a peer that is still zeroing them
        cluster_arrive();
        cluster_wait();

        const bool blk_active = b * X < own;
        unsigned in_a = 0, in_b = 0;  // bit jj: output jj of slot q (q+4) is inside a shot's aperture
        {
            const int16_t *own_a = (blk_active && q < grp.nslots)
                                       ? a.owner + grp.owner_off + (long long)q * grp.owner_stride + c0 + b * X
                                       : nullptr;
            const int16_t *own_b = (blk_active && q + Q < grp.nslots)
                                       ? a.owner + grp.owner_off + (long long)(q + Q) * grp.owner_stride + c0 + b * X
                                       : nullptr;
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
        // lane q owns outputs q and q+4 of the block: their operator rows (byte offsets into the
        // table), next-step indices and Kahan partial-image values
        const int xq0 = min(xg + q, a.nx - 1), xq1 = min(xg + q + Q, a.nx - 1);
        const bool img0 = a.partial && b * X + q < own, img1 = a.partial && b * X + q + Q < own;
        unsigned roff0 = (unsigned)idx_j[xq0] * (unsigned)row_bytes;
        unsigned roff1 = (unsigned)idx_j[xq1] * (unsigned)row_bytes;
        unsigned nidx01 = 0;  // next step's row indices of outputs q (low half) and q+4 (high half)
        // STAGE: copies of the aligned index words of step ls (outputs q and q+4) and of the Kahan
        // values of step lk (positions q and q+4) into this thread's stage words
        auto stage_idx = [&](int ls) {
            const uint16_t *ip = idx_j + (long long)ls * a.idx_lstride;
            cp_async4(sst + 0, ip + (xq0 & ~1));
            cp_async4(sst + 1, ip + (xq1 & ~1));
        };
        const long long prow0 = (long long)blockIdx.x * a.nextrap * a.nx + xg + q;  // partial element of step 0
        auto stage_kahan = [&](int lk) {
            const long long e = prow0 + (long long)lk * a.nx;
            if (img0) {
                cp_async4(sst + 2, a.partial + e);
                cp_async4(sst + 3, a.comp + e);
            }
            if (img1) {
                cp_async4(sst + 4, a.partial + e + Q);
                cp_async4(sst + 5, a.comp + e + Q);
            }
        };
        // branch-free: a pair outside the row becomes a zero-filled copy of nothing (never read)
        auto ring_copy = [&](int u) {
            const char *tabb = reinterpret_cast<const char *>(a.tabF);
            const int pr0 = u + ((X - q) >> 1), pr1 = u + ((X - q - Q) >> 1);
            const bool ok0 = (unsigned)pr0 < (unsigned)npairs, ok1 = (unsigned)pr1 < (unsigned)npairs;
            const int sl = u & (kRingSlots - 1);
            cp_async16_zfill(ringb + q * kRingSlots + sl, tabb + roff0 + (ok0 ? pr0 : 0) * 16, ok0 ? 16u : 0u);
            cp_async16_zfill(ringb + (q + Q) * kRingSlots + sl, tabb + roff1 + (ok1 ? pr1 : 0) * 16, ok1 ? 16u : 0u);
        };
        // BULK: the pairs of ring iterations v and v + 1 (v even; v + 1 only while <= vlast) of outputs
        // q and q + 4, one bulk copy per output into the two adjacent slots.  Pairs outside the row
        // are not copied (their slots are never read).  Every lane arrives on the chunk's barrier
        // with its own byte count before issuing its copies, so the phase completes only after all
        // 32 lanes' copies have landed.
        auto ring_chunk = [&](int v, int vlast) {
            const char *tabb = reinterpret_cast<const char *>(a.tabF);
            unsigned long long *bar = wbar + (n_issued & 1);
            ++n_issued;
            if (bulk_failed) return;  // never arrive on a phase that may still be open
            unsigned nb[2];
            const char *src[2];
            float4 *dst[2];
#pragma unroll
            for (int o = 0; o < 2; ++o) {
                const int p0 = v + ((X - q - o * Q) >> 1);
                const bool ok0 = (unsigned)p0 < (unsigned)npairs;
                const bool ok1 = v + 1 <= vlast && (unsigned)(p0 + 1) < (unsigned)npairs;
                const int first = ok0 ? 0 : 1;
                nb[o] = (ok0 ? 16u : 0u) + (ok1 ? 16u : 0u);
                src[o] = tabb + (o ? roff1 : roff0) + (long long)(p0 + first) * 16;
                dst[o] = ringb + (q + o * Q) * kRingSlots + (v & (kRingSlots - 1)) + first;
            }
            mbar_arrive_expect_tx(bar, nb[0] + nb[1]);
            if (nb[0]) bulk_copy_g2s(dst[0], src[0], nb[0], bar);
            if (nb[1]) bulk_copy_g2s(dst[1], src[1], nb[1], bar);
        };
        // BULK: wait for the oldest chunk not yet waited for (chunks are waited for in issue order,
        // and a barrier's next chunk is issued only after its previous one was waited for)
        auto chunk_wait = [&]() {
            unsigned long long *bar = wbar + (n_waited & 1);
            const unsigned parity = (n_waited >> 1) & 1;
            ++n_waited;
            if (bulk_failed || mbar_try_wait(bar, parity)) return;
            const long long t0 = clock64();
            while (!mbar_try_wait(bar, parity)) {
                if (clock64() - t0 > kBulkWaitCycles) {
                    bulk_failed = true;
                    if (a.status) atomicOr(a.status, 1);
                    break;
                }
            }
        };
        if (warp_active) {
            if (BULK) {
                ring_chunk(-4, -1);
                ring_chunk(-2, -1);
            } else {
                for (int u = -(X / 2); u < 0; ++u) ring_copy(u);
            }
            if (STAGE) {
                if (a.nextrap > 1) stage_idx(1);
                stage_kahan(0);
            }
        }
        cp_async_commit();
        const int srow0 = b * X + MP - M;  // row of input t = 0
        const int nmid = (L - X + 1) / 2;  // middle tap-loop iterations (two inputs each)

        for (int l = 0; l < a.nextrap; ++l) {
            const int par = l & 1;
            // this step's prologue pairs (copied at the end of the previous step) for the group
            cp_async_wait_all();
            if (BULK && warp_active) {
                chunk_wait();
                chunk_wait();
            }
            __syncwarp();  // control flow is warp-uniform here
            const long long pe = prow0 + (long long)l * a.nx;
            float cur_s0 = 0.f, cur_c0 = 0.f, cur_s1 = 0.f, cur_c1 = 0.f;
            if (!STAGE) {
                // this step's Kahan values and the next step's operator indices: the loads are
                // issued here and complete during the tap loop
                if (img0) {
                    cur_s0 = a.partial[pe];
                    cur_c0 = a.comp[pe];
                }
                if (img1) {
                    cur_s1 = a.partial[pe + Q];
                    cur_c1 = a.comp[pe + Q];
                }
                if (l + 1 < a.nextrap) {
                    const uint16_t *inext = idx_j + (long long)(l + 1) * a.idx_lstride;
                    nidx01 = (unsigned)inext[xq0] | ((unsigned)inext[xq1] << 16);
                }
            }
            // the partial-image rows of the next step into L2 (read at the end of this step by the
            // stage, or at the start of the next one)
            if (q == 0 && img0 && l + 1 < a.nextrap) {
                asm volatile("prefetch.global.L2 [%0];" ::"l"(a.partial + pe + a.nx));
                asm volatile("prefetch.global.L2 [%0];" ::"l"(a.comp + pe + a.nx));
            }
            float acc[X][8];
#pragma unroll
            for (int jj = 0; jj < X; ++jj)
#pragma unroll
                for (int e = 0; e < 8; ++e) acc[jj][e] = 0.f;
            if (warp_active) {  // warps past the CTA's share of the window skip the step's work
            float4 tp[X];
            // input t: row srow0 + t, columns wide_col(row, q, 0/1)
            auto load_in = [&](int row, float4 &va, float4 &vb) {
                const float4 *r = ext + (size_t)row * G + 2 * q;
                const int sw = (row >> 3) & 1;
                va = r[sw];
                vb = r[sw ^ 1];
            };

            // prologue: t = 0 .. X-2, outputs jj <= t are active
#pragma unroll
            for (int t = 0; t < X - 1; ++t) {
                float4 va, vb;
                load_in(srow0 + t, va, vb);
#pragma unroll
                for (int jj = 0; jj < X; ++jj) {
                    const int k = t - jj;
                    if (k >= 0) {
                        if ((k & 1) == 0)
                            tp[jj] = ringb[jj * kRingSlots + (((k >> 1) - ((X - jj) >> 1)) & (kRingSlots - 1))];
                        const float fr = (k & 1) ? tp[jj].z : tp[jj].x;
                        const float fi = (k & 1) ? tp[jj].w : tp[jj].y;
                        wide_mac<ARITH>(acc[jj], fr, fi, va, vb);
                    }
                }
                // after t = 2u the slot of iteration u - 4 has been read; copy iteration u
                if ((t & 1) == 0 && (t >> 1) < 3) {
                    if (BULK) {
                        if (t == 2) ring_chunk(0, nmid + 3);
                    } else {
                        ring_copy(t >> 1);
                        cp_async_commit();
                    }
                }
            }
            // middle: t = X-1 .. L-1 in steps of two (odd t, then even t+1)
            int row = srow0 + X - 1;
            for (int u = 0; u < nmid; ++u, row += 2) {
                const float4 *rs = ringb + (u & (kRingSlots - 1));
                // iteration u - 1 has read the slot of iteration u + 3; wait for iteration u
                if (BULK) {
                    if (!(u & 1)) {
                        ring_chunk(u + 2, nmid + 3);
                        chunk_wait();
                    }
                } else {
                    ring_copy(u + 3);
                    cp_async_commit();
                    cp_async_wait<3>();
                }
                __syncwarp();  // control flow is warp-uniform here
                {
                    float4 va, vb;
                    load_in(row, va, vb);
#pragma unroll
                    for (int jj = 0; jj < X; ++jj) {
                        if (jj & 1) tp[jj] = rs[jj * kRingSlots];
                        const float fr = (jj & 1) ? tp[jj].x : tp[jj].z;
                        const float fi = (jj & 1) ? tp[jj].y : tp[jj].w;
                        wide_mac<ARITH>(acc[jj], fr, fi, va, vb);
                    }
                }
                {
                    float4 va, vb;
                    load_in(row + 1, va, vb);
#pragma unroll
                    for (int jj = 0; jj < X; ++jj) {
                        if (!(jj & 1)) tp[jj] = rs[jj * kRingSlots];
                        const float fr = (jj & 1) ? tp[jj].z : tp[jj].x;
                        const float fi = (jj & 1) ? tp[jj].w : tp[jj].y;
                        wide_mac<ARITH>(acc[jj], fr, fi, va, vb);
                    }
                }
            }
            // epilogue: t = L .. L+X-2, outputs jj > t-L are active (k = t - jj <= L-1)
            if (BULK) {
                ring_chunk((nmid + 3) & ~1, nmid + 3);
            } else {
                ring_copy(nmid + 3);
                cp_async_commit();
            }
#pragma unroll
            for (int e = 0; e < X - 1; ++e) {
                float4 va, vb;
                load_in(srow0 + L + e, va, vb);
                if ((e & 1) == 0) {
                    // steps e and e + 1 read iteration nmid + e / 2; later iterations may be in flight
                    if (BULK) {
                        if (!((nmid + (e >> 1)) & 1)) chunk_wait();
                    } else {
                        switch (e >> 1) {
                            case 0: cp_async_wait<3>(); break;
                            case 1: cp_async_wait<2>(); break;
                            case 2: cp_async_wait<1>(); break;
                            default: cp_async_wait<0>(); break;
                        }
                    }
                    __syncwarp();  // control flow is warp-uniform here
                }
#pragma unroll
                for (int jj = 0; jj < X; ++jj) {
                    if (jj > e) {
                        // k = L + e - jj, parity of (1 + e - jj) since L is odd
                        const bool even = ((1 + e - jj) & 1) == 0;
                        if (even) tp[jj] = ringb[jj * kRingSlots + ((nmid + (e >> 1)) & (kRingSlots - 1))];
                        const float fr = even ? tp[jj].x : tp[jj].z;
                        const float fi = even ? tp[jj].y : tp[jj].w;
                        wide_mac<ARITH>(acc[jj], fr, fi, va, vb);
                    }
                }
            }
            // outputs outside every shot aperture of their slot stay zero; most lanes have none
            if ((in_a & in_b) != (1u << X) - 1u) {
#pragma unroll
                for (int jj = 0; jj < X; ++jj) {
                    if (!((in_a >> jj) & 1u)) acc[jj][0] = acc[jj][2] = acc[jj][4] = acc[jj][6] = 0.f;
                    if (!((in_b >> jj) & 1u)) acc[jj][1] = acc[jj][3] = acc[jj][5] = acc[jj][7] = 0.f;
                }
            }
            // halos of step l+1 into the neighbours' staging (parity par^1): left neighbour's right
            // halo rows are its ext rows PC + MP + x, right neighbour's left halo rows its rows x
            if (push_left) {
                float4 *dst = stg + ((size_t)((par ^ 1) * 2 + 1) * MP) * G;
#pragma unroll
                for (int jj = 0; jj < X; ++jj) {
                    const int x = b * X + jj;
                    if (x < MP) {
                        const int prow = NC + MP + x;
                        const unsigned ra = map_rank(dst + (size_t)x * G, crank - 1);
                        st_cluster(ra + wide_col(prow, q, 0) * 16, make_float4(acc[jj][0], acc[jj][1], acc[jj][2], acc[jj][3]));
                        st_cluster(ra + wide_col(prow, q, 1) * 16, make_float4(acc[jj][4], acc[jj][5], acc[jj][6], acc[jj][7]));
                    }
                }
            }
            if (push_right) {
                float4 *dst = stg + ((size_t)((par ^ 1) * 2 + 0) * MP) * G;
#pragma unroll
                for (int jj = 0; jj < X; ++jj) {
                    const int x = b * X + jj - (NC - MP);
                    if (x >= 0) {
                        const unsigned ra = map_rank(dst + (size_t)x * G, crank + 1);
                        st_cluster(ra + wide_col(x, q, 0) * 16, make_float4(acc[jj][0], acc[jj][1], acc[jj][2], acc[jj][3]));
                        st_cluster(ra + wide_col(x, q, 1) * 16, make_float4(acc[jj][4], acc[jj][5], acc[jj][6], acc[jj][7]));
                    }
                }
            }
            }  // warp_active
            // The neighbours read only their halo staging (the pushes above), never this CTA's ext[]:
            // arrive now, so the barrier's release covers the pushes but not the in-place writes.
            // The staging of parity par^1 is rewritten (step l+2) only after this CTA's arrival of
            // step l+1, which follows its copy of that staging at the end of this step.
            cluster_arrive();
            // every ring slot has been read: copy the next step's prologue pairs (u < 0) now, so
            // that they arrive during the halo exchange and the imaging
            if (warp_active && l + 1 < a.nextrap) {
                if (STAGE) {
                    const unsigned w0 = sst[0], w1 = sst[1];
                    roff0 = ((w0 >> (16 * (xq0 & 1))) & 0xffffu) * (unsigned)row_bytes;
                    roff1 = ((w1 >> (16 * (xq1 & 1))) & 0xffffu) * (unsigned)row_bytes;
                } else {
                    roff0 = (nidx01 & 0xffffu) * (unsigned)row_bytes;
                    roff1 = (nidx01 >> 16) * (unsigned)row_bytes;
                }
                if (BULK) {
                    ring_chunk(-4, -1);
                    ring_chunk(-2, -1);
                } else {
                    for (int u = -(X / 2); u < 0; ++u) ring_copy(u);
                }
                // the words just read are refilled for step l + 2 (their reads are complete: the
                // copies above used them)
                if (STAGE && l + 2 < a.nextrap) stage_idx(l + 2);
            }
            cp_async_commit();
            __syncthreads();  // every read of step l's values in ext[] is done
            if (warp_active) {
#pragma unroll
            for (int jj = 0; jj < X; ++jj) {
                const int prow = b * X + MP + jj;
                float4 *dst = ext + (size_t)prow * G;
                dst[wide_col(prow, q, 0)] = make_float4(acc[jj][0], acc[jj][1], acc[jj][2], acc[jj][3]);
                dst[wide_col(prow, q, 1)] = make_float4(acc[jj][4], acc[jj][5], acc[jj][6], acc[jj][7]);
            }
            // Re(S conj R) of both slots per output, summed over the group's 4 lanes by a reduce-scatter:
            // exchange across lanes q ^ 2 keeps the 4 outputs with (jj & 2) == (q & 2), exchange
            // across q ^ 1 keeps jj = q and q + 4 (6 shuffles instead of 8 x 2)
            float img[X];
#pragma unroll
            for (int jj = 0; jj < X; ++jj) {
                const float ia = acc[jj][0] * acc[jj][4] - acc[jj][2] * acc[jj][6];
                const float ib = acc[jj][1] * acc[jj][5] - acc[jj][3] * acc[jj][7];
                if (a.image_shots) {
                    // per-shot images (optional output): shot ids re-read from the owner table
                    const GroupDesc &g2 = a.groups[item.x];
                    const int16_t *orow = a.owner + g2.owner_off + c0 + b * X + jj;
                    if ((in_a >> jj) & 1u)
                        atomicAdd(a.image_shots + (long long)orow[(long long)q * g2.owner_stride] * a.img_sstride +
                                      (long long)l * a.nx + xg + jj, ia);
                    if ((in_b >> jj) & 1u)
                        atomicAdd(a.image_shots + (long long)orow[(long long)(q + Q) * g2.owner_stride] * a.img_sstride +
                                      (long long)l * a.nx + xg + jj, ib);
                }
                img[jj] = ia + ib;
            }
            const bool hi2 = (q & 2) != 0, hi1 = (q & 1) != 0;
            float r4[4];  // outputs {0, 1, 4, 5} ^ (q & 2)
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int base = (i & 1) | ((i & 2) << 1);
                const float keep = hi2 ? img[base ^ 2] : img[base];
                const float send = hi2 ? img[base] : img[base ^ 2];
                r4[i] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
            }
            float img_q[2];  // outputs q and q + 4
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const float keep = hi1 ? r4[2 * k + 1] : r4[2 * k];
                const float send = hi1 ? r4[2 * k] : r4[2 * k + 1];
                img_q[k] = keep + __shfl_xor_sync(0xffffffffu, send, 1);
            }
            const float img_q0 = img_q[0], img_q1 = img_q[1];
            // Kahan update (the operations of kahan_add) on the values loaded at the step's start
            if (STAGE) {
                cur_s0 = __uint_as_float(sst[2]);
                cur_c0 = __uint_as_float(sst[3]);
                cur_s1 = __uint_as_float(sst[4]);
                cur_c1 = __uint_as_float(sst[5]);
            }
            if (img0) {
                const float y = img_q0 - cur_c0;
                const float t = cur_s0 + y;
                a.partial[pe] = t;
                a.comp[pe] = (t - cur_s0) - y;
            }
            if (img1) {
                const float y = img_q1 - cur_c1;
                const float t = cur_s1 + y;
                a.partial[pe + Q] = t;
                a.comp[pe + Q] = (t - cur_s1) - y;
            }
            if (STAGE && l + 1 < a.nextrap) stage_kahan(l + 1);  // refilled for the next step
            }  // warp_active
            if (STAGE) cp_async_commit();  // the Kahan words, waited for at the next step's start
            cluster_wait();
            const float4 *hs = stg + (size_t)((par ^ 1) * 2) * MP * G;
            for (int i = threadIdx.x; i < 2 * MP * G; i += blockDim.x) {
                const int side = i / (MP * G), r = i % (MP * G);
                ext[(side ? (NC + MP) * G : 0) + r] = hs[i];
            }
            __syncthreads();
        }
        if (a.write_back) {
            for (int k = grp.seg_begin; k < grp.seg_begin + grp.nseg; ++k) {
                const int4 sg = a.segs[k];
                const int r0 = sg.z - u0;
                const int lo = max(r0, c0), hi = min(r0 + sg.w, c0 + own);
                cpx *ws = a.wave + a.shot_off[sg.x] + (long long)j * sg.w;
                cpx *rs = a.shot + a.shot_off[sg.x] + (long long)j * sg.w;
                const int sq = sg.y & (Q - 1), sh = sg.y / Q;
                for (int x = lo + (int)threadIdx.x; x < hi; x += blockDim.x) {
                    const int pos = x - c0 + MP;
                    const float *fa = extf + ((size_t)pos * G + wide_col(pos, sq, 0)) * 4;
                    const float *fb = extf + ((size_t)pos * G + wide_col(pos, sq, 1)) * 4;
                    ws[x - r0] = cpx{fa[sh], fa[2 + sh]};
                    rs[x - r0] = cpx{fb[sh], -fb[2 + sh]};
                }
            }
        }
        __syncthreads();
    }
    cluster_arrive();
    cluster_wait();
}

}  // namespace img2d
