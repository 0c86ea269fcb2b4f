// Cluster form of the migration kernel: one thread-block cluster of K CTAs owns one work item
// (group of 16 lane slots, one frequency) for the whole depth loop, each CTA holding 256
// consecutive positions of the group's window plus halos.  Same arithmetic and results as
// migrate_fixed_kernel (wlsq_kernels.cuh); see there for the reference semantics.
//
// Why a cluster: the operator row of a position is shared by every shot of the item, so the more
// shots an item carries the fewer operator loads per FMA.  Sixteen shots over a 2048-wide window
// need 2048*16*16 B = 512 KB of wavefield, more than one SM's shared memory; eight CTAs of a
// cluster hold 64 KB each and exchange only M halo positions per side and depth step through
// distributed shared memory.
//
// Per lane: two slots (shot q and shot q+8 of the item, each S and conj(R) as a float4) and a
// block of X=8 consecutive positions, so each 16-byte operator load (two taps) feeds 16 FMAs.
// Lanes 8p..8p+7 of a warp share position block p: operator rows are loaded once per block and
// broadcast to the 8 lanes.  Every lane group owns exactly one block per depth step, which lets
// the wavefield be updated in place: outputs stay in registers until all reads of the old values
// are done.
//
// Per depth step (l):
//   1. compute the block from ext[] (own positions + halo copies)
//   2. edge blocks store their outputs into the neighbour CTA's halo staging buffer [l+1 parity]
//   3. __syncthreads; write outputs in place; cluster barrier arrive (release)
//   4. imaging: Kahan add into the CTA's partial image row (global, private to the CTA)
//   5. cluster barrier wait (acquire); copy the staging halos into ext[]; __syncthreads
// The staging buffers are double-buffered by depth parity: a neighbour one step ahead writes the
// other parity (proof in the comments of the loop).
#pragma once
#include "wlsq_kernels.cuh"

namespace img2d {

__device__ __forceinline__ unsigned cluster_rank()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ unsigned cluster_size()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }

__device__ __forceinline__ unsigned map_rank(const void *p, unsigned rank)
{
    unsigned local = (unsigned)__cvta_generic_to_shared(p), remote;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(local), "r"(rank));
    return remote;
}

__device__ __forceinline__ void st_cluster(unsigned addr, float4 v)
{
    asm volatile("st.shared::cluster.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(v.x), "f"(v.y), "f"(v.z),
                 "f"(v.w)
                 : "memory");
}

__device__ __forceinline__ int ld_cluster_s32(unsigned addr)
{
    int v;
    asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
    return v;
}

struct ClusterShape {
    static constexpr int Q = 8;            // lanes per position group
    static constexpr int G = 2 * Q;        // lane slots per item (two per lane)
    static constexpr int P = 32 / Q;       // position groups per warp
    static constexpr int NW = 8;           // warps per CTA
    static constexpr int X = 8;            // positions per block
    static constexpr int PC = NW * P * X;  // positions per CTA
};

template <int L>
__host__ __device__ constexpr int cluster_mp()
{
    return (((L - 1) / 2 + ClusterShape::X - 1) / ClusterShape::X) * ClusterShape::X;
}

template <int L>
__host__ __device__ constexpr size_t cluster_smem_bytes()
{
    // ext[PC + 2 MP][G] + staging[2 parity][2 side][MP][G], float4 each
    return (size_t)((ClusterShape::PC + 2 * cluster_mp<L>()) + 4 * cluster_mp<L>()) * ClusterShape::G * 16;
}

template <int L>
__global__ void __launch_bounds__(256, 1) migrate_cluster_kernel(MigrateArgs a)
{
    using S = ClusterShape;
    constexpr int Q = S::Q, G = S::G, P = S::P, X = S::X, PC = S::PC;
    constexpr int M = (L - 1) / 2;
    constexpr int MP = cluster_mp<L>();
    constexpr int NEXT = PC + 2 * MP;
    extern __shared__ float4 smem[];
    float4 *ext = smem;                    // [NEXT][G]; local position x at index x + MP
    float4 *stg = smem + (size_t)NEXT * G;  // [parity][side][MP][G]; side 0 = left halo, 1 = right
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
    const unsigned rank0_item = map_rank(&s_item, 0);

    for (;;) {
        if (crank == 0 && threadIdx.x == 0) s_item = atomicAdd(a.counter, 1);
        cluster_arrive();
        cluster_wait();
        const int it = ld_cluster_s32(rank0_item);
        // every CTA has read the item before rank 0 may overwrite it
        cluster_arrive();
        cluster_wait();
        if (it >= a.n_items) break;
        const int2 item = a.items[it];
        const GroupDesc grp = a.groups[item.x];
        const int j = item.y, u0 = grp.u0, W = grp.W;

        for (int i = threadIdx.x; i < (NEXT + 4 * MP) * G; i += blockDim.x) smem[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        __syncthreads();
        // own positions and both halos from the input wavefields (relative window [c0-MP, c0+PC+MP))
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
        int16_t oa[X], ob[X];
        load_owner<X>(own_a, oa);
        load_owner<X>(own_b, ob);
        const uint16_t *idx_j = a.idx + (long long)j * a.idx_jstride;
        const int xg = u0 + c0 + b * X;  // model position of the block's first output

        for (int l = 0; l < a.nextrap; ++l) {
            const int par = l & 1;
            const uint16_t *idx_l = idx_j + (long long)l * a.idx_lstride;
            const float4 *row[X];
#pragma unroll
            for (int jj = 0; jj < X; ++jj) {
                const int xm = min(xg + jj, a.nx - 1);
                row[jj] = reinterpret_cast<const float4 *>(a.tabF + (long long)idx_l[xm] * a.tab_stride);
            }
            float acc[X][8];
#pragma unroll
            for (int jj = 0; jj < X; ++jj)
#pragma unroll
                for (int e = 0; e < 8; ++e) acc[jj][e] = 0.f;
            float4 tp[X];
            const float4 *src = ext + (size_t)(b * X + MP - M) * G + q;
#pragma unroll
            for (int t = 0; t < X + L - 1; ++t) {
                const float4 va = src[(size_t)t * G];
                const float4 vb = src[(size_t)t * G + Q];
#pragma unroll
                for (int jj = 0; jj < X; ++jj) {
                    const int k = t - jj;
                    if (k >= 0 && k < L) {
                        if ((k & 1) == 0) tp[jj] = __ldg(row[jj] + (k >> 1));
                        const float fr = (k & 1) ? tp[jj].z : tp[jj].x;
                        const float fi = (k & 1) ? tp[jj].w : tp[jj].y;
                        float *c = acc[jj];
                        c[0] = fmaf(fr, va.x, c[0]); c[0] = fmaf(-fi, va.y, c[0]);
                        c[1] = fmaf(fr, va.y, c[1]); c[1] = fmaf(fi, va.x, c[1]);
                        c[2] = fmaf(fr, va.z, c[2]); c[2] = fmaf(-fi, va.w, c[2]);
                        c[3] = fmaf(fr, va.w, c[3]); c[3] = fmaf(fi, va.z, c[3]);
                        c[4] = fmaf(fr, vb.x, c[4]); c[4] = fmaf(-fi, vb.y, c[4]);
                        c[5] = fmaf(fr, vb.y, c[5]); c[5] = fmaf(fi, vb.x, c[5]);
                        c[6] = fmaf(fr, vb.z, c[6]); c[6] = fmaf(-fi, vb.w, c[6]);
                        c[7] = fmaf(fr, vb.w, c[7]); c[7] = fmaf(fi, vb.z, c[7]);
                    }
                }
            }
            // mask to each shot's aperture
#pragma unroll
            for (int jj = 0; jj < X; ++jj) {
                if (oa[jj] < 0) acc[jj][0] = acc[jj][1] = acc[jj][2] = acc[jj][3] = 0.f;
                if (ob[jj] < 0) acc[jj][4] = acc[jj][5] = acc[jj][6] = acc[jj][7] = 0.f;
            }
            // Edge blocks feed the neighbours' halos for step l+1 (staging parity par^1).  A
            // neighbour reads that parity only after the cluster barrier of this step, and the
            // next write to it (step l+2) happens after this CTA has copied it out (step l+1's
            // barrier needs this CTA's arrival, which follows that copy).
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
            // imaging: Re(S conj R) of both slots, summed over the 8 lanes of the group
            float *prow = part ? part + (long long)l * a.nx : nullptr;
            float *crow = cmp ? cmp + (long long)l * a.nx : nullptr;
#pragma unroll
            for (int jj = 0; jj < X; ++jj) {
                const float ia = acc[jj][0] * acc[jj][2] - acc[jj][1] * acc[jj][3];
                const float ib = acc[jj][4] * acc[jj][6] - acc[jj][5] * acc[jj][7];
                if (a.image_shots) {
                    if (oa[jj] >= 0)
                        atomicAdd(a.image_shots + (long long)oa[jj] * a.img_sstride + (long long)l * a.nx + xg + jj, ia);
                    if (ob[jj] >= 0)
                        atomicAdd(a.image_shots + (long long)ob[jj] * a.img_sstride + (long long)l * a.nx + xg + jj, ib);
                }
                float img = ia + ib;
#pragma unroll
                for (int off = 1; off < Q; off <<= 1) img += __shfl_xor_sync(gmask, img, off);
                if (prow && q == 0 && c0 + b * X + jj < W) kahan_add(prow + xg + jj, crow + xg + jj, img);
            }
            cluster_wait();
            // halos for step l+1
            const float4 *hs = stg + (size_t)((par ^ 1) * 2) * MP * G;
            for (int i = threadIdx.x; i < 2 * MP * G; i += blockDim.x) {
                const int side = i / (MP * G), r = i % (MP * G);
                ext[(side ? (PC + MP) * G : 0) + r] = hs[i];
            }
            __syncthreads();
        }
        // final wavefields of this CTA's positions
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
    // no CTA leaves while a peer may still address its shared memory
    cluster_arrive();
    cluster_wait();
}

}  // namespace img2d
