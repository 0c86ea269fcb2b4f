// C ABI of the B200 extrapolation + imaging library: plans, kernel dispatch and the
// reference-compatible entry points.  Declarations and contracts: include/imaging2d_wlsq_b200.h.
#include <algorithm>
#include <atomic>
#include <map>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/imaging2d_wlsq_b200.h"
#include <cufft.h>
#include "wlsq_kernels.cuh"
#include "wlsq_cluster.cuh"
#include "wlsq_cluster2.cuh"
#include "wlsq_wide.cuh"
#include "wlsq_adjoint.cuh"
#include "wlsq_adjoint_cluster.cuh"
#include "wlsq_frontend.cuh"

namespace img2d {

static thread_local std::string g_err;

static int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

#define IMG2D_CUDA(call)                                                                   \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            cudaGetLastError();                                                            \
            return fail(e_ == cudaErrorMemoryAllocation ? IMG2D_ENOMEM : IMG2D_ECUDA,      \
                        std::string(#call) + ": " + cudaGetErrorString(e_));               \
        }                                                                                  \
    } while (0)

typedef void (*KernelFn)(MigrateArgs);

// ---------------------------------------------------------------------------------------
// Kernel tables.  The fixed-length kernel is instantiated for the operator lengths of the
// reference tests and of the benchmark configurations; any other length runs on the generic
// kernel.
// ---------------------------------------------------------------------------------------
constexpr int kX = 8;

template <int G, int L>
struct FixedEntry {
    static constexpr int g = G, l = L;
};

struct FixedKernel {
    int G, L;
    KernelFn fn;
};

#define IMG2D_FIXED(G, L) {G, L, migrate_fixed_kernel<G, kX, L, OP_CONJ>}
#define IMG2D_FIXED_L(L) IMG2D_FIXED(1, L), IMG2D_FIXED(2, L), IMG2D_FIXED(4, L), IMG2D_FIXED(8, L)

static const FixedKernel kFixed[] = {
    IMG2D_FIXED_L(3),  IMG2D_FIXED_L(5),  IMG2D_FIXED_L(11), IMG2D_FIXED_L(25),
    IMG2D_FIXED_L(31), IMG2D_FIXED_L(35), IMG2D_FIXED_L(43), IMG2D_FIXED_L(55),
};

static KernelFn find_fixed(int G, int L)
{
    for (const auto &k : kFixed)
        if (k.G == G && k.L == L) return k.fn;
    return nullptr;
}

static KernelFn find_generic(int G, int mode)
{
#define IMG2D_GEN(GG)                                                        \
    if (G == GG) {                                                           \
        if (mode == OP_CONJ) return migrate_generic_kernel<GG, OP_CONJ>;     \
        if (mode == OP_TWO) return migrate_generic_kernel<GG, OP_TWO>;       \
        return migrate_generic_kernel<GG, OP_DENSE>;                         \
    }
    IMG2D_GEN(1) IMG2D_GEN(2) IMG2D_GEN(4) IMG2D_GEN(8)
#undef IMG2D_GEN
    return nullptr;
}

struct ClusterKernel {
    int L;
    KernelFn fn;
    size_t smem;
};

static const ClusterKernel kCluster[] = {
    {25, migrate_cluster_kernel<25>, cluster_smem_bytes<25>()},
    {31, migrate_cluster_kernel<31>, cluster_smem_bytes<31>()},
    {35, migrate_cluster_kernel<35>, cluster_smem_bytes<35>()},
    {43, migrate_cluster_kernel<43>, cluster_smem_bytes<43>()},
    {55, migrate_cluster_kernel<55>, cluster_smem_bytes<55>()},
};

// Variants of the second-generation cluster kernel: warps per CTA (positions per CTA = 32 * warps),
// operator-pair prefetch into registers, next-step operator rows prefetched into L1.
struct Cluster2Variant {
    int nw;
    bool tap_pf, row_pf;
    KernelFn fn;
    bool stage = false;  // uses the step-ahead shared-memory stage (cluster2_stage_bytes)
    bool ring = false;   // reads operator taps from the per-lane-group ring (cluster2_ring_bytes)
};

static const Cluster2Variant kCluster2[] = {
    {16, false, false, migrate_cluster2_kernel<16, false, false>},
    {16, false, true, migrate_cluster2_kernel<16, false, true>},
    {12, true, false, migrate_cluster2_kernel<12, true, false>},
    {12, true, true, migrate_cluster2_kernel<12, true, true>},
    {8, true, false, migrate_cluster2_kernel<8, true, false>},
    {8, true, true, migrate_cluster2_kernel<8, true, true>},
    {16, false, false, migrate_cluster2_kernel<16, false, false, true>},  // packed FFMA2 arithmetic
    {16, false, false, migrate_cluster2_kernel<16, false, false, false, TAB_F32, 1>},  // grouped FMA order
    {16, false, false, migrate_cluster2_kernel<16, false, false, false, TAB_F32, 2>},  // index prefetch
    {16, false, false, migrate_cluster2_kernel<16, false, false, false, TAB_F32, 3>},  // both
    {16, false, false, migrate_cluster2_kernel<16, false, false, false, TAB_F32, 4>, true},  // step-ahead stage
    {16, false, false, migrate_cluster2_kernel<16, false, false, false, TAB_F32, 8>, false, true},  // tap-pair ring
};
constexpr int kCluster2Staged = 10;   // 16 warps with the step-ahead shared-memory stage
constexpr int kCluster2Default = 11;  // 16 warps, tap pairs through the shared-memory ring
constexpr int kNumCluster2 = (int)(sizeof(kCluster2) / sizeof(kCluster2[0]));

// Demigration kernels: G lane slots per item, compile-time operator length (0 = runtime length).
constexpr int kAdjWarps = 16;
typedef void (*DemigFn)(DemigrateArgs);
struct DemigKernel {
    int G, L;
    DemigFn fn;
};
#define IMG2D_DEMIG(G, L) {G, L, demigrate_kernel<G, L, kAdjWarps>}
#define IMG2D_DEMIG_G(G) IMG2D_DEMIG(G, 0), IMG2D_DEMIG(G, 25), IMG2D_DEMIG(G, 31), IMG2D_DEMIG(G, 35), IMG2D_DEMIG(G, 55)
static const DemigKernel kDemig[] = {IMG2D_DEMIG_G(2), IMG2D_DEMIG_G(4), IMG2D_DEMIG_G(8)};

struct DemigClusterKernel {
    int L;
    DemigFn fn;
    DemigFn ring;  // forward steps through the shared-memory tap-pair ring (compile-time L only)
};
static const DemigClusterKernel kDemigCluster[] = {
    {0, demigrate_cluster_kernel<0>, nullptr},
    {25, demigrate_cluster_kernel<25>, demigrate_cluster_kernel<25, true>},
    {31, demigrate_cluster_kernel<31>, demigrate_cluster_kernel<31, true>},
    {35, demigrate_cluster_kernel<35>, demigrate_cluster_kernel<35, true>},
    {55, demigrate_cluster_kernel<55>, demigrate_cluster_kernel<55, true>},
};

static DemigFn find_demig_cluster(int L, bool ring = false)
{
    DemigFn generic = nullptr;
    for (const auto &k : kDemigCluster) {
        if (k.L == L) return ring ? k.ring : k.fn;
        if (k.L == 0) generic = k.fn;
    }
    return ring ? nullptr : generic;
}

static DemigFn find_demig(int G, int L)
{
    DemigFn generic = nullptr;
    for (const auto &k : kDemig) {
        if (k.G != G) continue;
        if (k.L == L) return k.fn;
        if (k.L == 0) generic = k.fn;
    }
    return generic;
}

// Shared memory of the demigration kernel: one complex wavefield per slot, ping-pong.
static size_t demig_smem_bytes(int G, int W, int M)
{
    const int X = 8;
    const int Mp = ((M + X - 1) / X) * X;
    const int Wp = ((W + X - 1) / X) * X;
    return 2 * (size_t)((Mp + Wp + Mp) / X * (X + 1)) * G * sizeof(float2) +
           2 * (size_t)demig_idx_words(Wp, Mp) * sizeof(unsigned);
}

static const ClusterKernel *find_cluster(int L)
{
    for (const auto &k : kCluster)
        if (k.L == L) return &k;
    return nullptr;
}

// ---------------------------------------------------------------------------------------
// Naive comparison kernel: one launch per (shot, frequency, depth), one thread per position,
// wavefields and operators in global memory.
// ---------------------------------------------------------------------------------------
__global__ void naive_step_kernel(const float4 *__restrict__ cur, float4 *__restrict__ nxt, int w,
                                  int M, const cpx *__restrict__ tab, int tab_stride,
                                  const uint16_t *__restrict__ idx_row, int x0,
                                  float *__restrict__ image_row)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w) return;
    const cpx *t = tab + (long long)idx_row[x0 + i] * tab_stride;
    float sr = 0.f, si = 0.f, rr = 0.f, ri = 0.f;
    for (int k = 0; k <= 2 * M; ++k) {
        const float4 v = cur[i + k];
        const cpx f = t[k];
        sr = fmaf(f.re, v.x, sr); sr = fmaf(-f.im, v.y, sr);
        si = fmaf(f.re, v.y, si); si = fmaf(f.im, v.x, si);
        rr = fmaf(f.re, v.z, rr); rr = fmaf(-f.im, v.w, rr);
        ri = fmaf(f.re, v.w, ri); ri = fmaf(f.im, v.z, ri);
    }
    nxt[i + M] = make_float4(sr, si, rr, ri);
    atomicAdd(image_row + x0 + i, sr * rr - si * ri);
}

__global__ void naive_pack_kernel(const cpx *__restrict__ wave, const cpx *__restrict__ shot, int w,
                                  int M, float4 *__restrict__ buf, int to_buf)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w) return;
    if (to_buf) {
        const cpx S = wave[i], R = shot[i];
        buf[i + M] = make_float4(S.re, S.im, R.re, -R.im);
    }
}

__global__ void naive_unpack_kernel(const float4 *__restrict__ buf, int w, int M,
                                    cpx *__restrict__ wave, cpx *__restrict__ shot)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w) return;
    const float4 v = buf[i + M];
    wave[i] = cpx{v.x, v.y};
    shot[i] = cpx{v.z, -v.w};
}

// Dense operator table of the reference's legacy ABI from the compact table and the operator index:
// dense[l][j][x][k] = tab[idx[j][l][x]][k] (conjugated when conj != 0).  One block per (l, j) row of
// nx*L elements, written with coalesced stores; x and k advance incrementally with the block stride.
__global__ void dense_table_kernel(const uint16_t *__restrict__ idx, int nf, int nextrap, int nx, int lstride,
                                   const cpx *__restrict__ tab, int tab_stride, int L, int conj,
                                   cpx *__restrict__ dense)
{
    const int lj = blockIdx.x;  // l * nf + j
    const int l = lj / nf, j = lj - l * nf;
    const uint16_t *irow = idx + ((long long)j * nextrap + l) * lstride;
    cpx *out = dense + (long long)lj * nx * L;
    const int n = nx * L;
    const int sx = (int)blockDim.x / L, sk = (int)blockDim.x - sx * L;
    int x = (int)threadIdx.x / L, k = (int)threadIdx.x - x * L;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        cpx v = tab[(long long)irow[x] * tab_stride + k];
        if (conj) v.im = -v.im;
        out[e] = v;
        x += sx;
        k += sk;
        if (k >= L) {
            k -= L;
            ++x;
        }
    }
}

// L2 read probe: every thread streams float4 from an L2-resident buffer with ld.global.cg (L2 only,
// no L1 allocation); four independent accumulators keep many loads in flight.
__global__ void l2_read_probe_kernel(const float4 *__restrict__ buf, long long n4, int iters, float *out)
{
    float4 acc[4] = {};
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (int it = 0; it < iters; ++it) {
        long long i = t0;
        for (; i + 3 * stride < n4; i += 4 * stride) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const float4 v = __ldcg(buf + i + u * stride);
                acc[u].x += v.x; acc[u].y += v.y; acc[u].z += v.z; acc[u].w += v.w;
            }
        }
        for (; i < n4; i += stride) {
            const float4 v = __ldcg(buf + i);
            acc[0].x += v.x; acc[0].y += v.y; acc[0].z += v.z; acc[0].w += v.w;
        }
    }
    float s = 0.f;
#pragma unroll
    for (int u = 0; u < 4; ++u) s += acc[u].x + acc[u].y + acc[u].z + acc[u].w;
    out[t0] = s;
}

// FP32 FMA probe: 16 independent chains per thread so the FMA pipe, not latency, limits it.
__global__ void fma_probe_kernel(float *out, int iters)
{
    float a[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) a[i] = threadIdx.x * 1e-3f + i;
    const float b = 0.9999f, c = 1e-4f;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int r = 0; r < 8; ++r)
#pragma unroll
            for (int i = 0; i < 16; ++i) a[i] = fmaf(a[i], b, c);
    }
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < 16; ++i) s += a[i];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// ---------------------------------------------------------------------------------------
// Device allocation.  Every device buffer the library allocates goes through device_alloc, which
// refuses (IMG2D_ENOMEM, before calling cudaMalloc) any single allocation larger than the limit set
// by img2d_set_alloc_limit or, until that is called, by the environment variable
// IMG2D_ALLOC_LIMIT_BYTES (unset or 0: no limit).  The limit injects allocation failures on the
// host for tests of the error path, including through the void drop-in shims.
// ---------------------------------------------------------------------------------------
static std::mutex g_alloc_mu;
static bool g_alloc_limit_set = false;
static size_t g_alloc_limit = 0;

static size_t alloc_limit()
{
    std::lock_guard<std::mutex> lock(g_alloc_mu);
    if (!g_alloc_limit_set) {
        const char *e = getenv("IMG2D_ALLOC_LIMIT_BYTES");
        g_alloc_limit = e ? (size_t)strtoull(e, nullptr, 10) : 0;
        g_alloc_limit_set = true;
    }
    return g_alloc_limit;
}

static int device_alloc(void **p, size_t n)
{
    *p = nullptr;
    const size_t lim = alloc_limit();
    if (lim && n > lim)
        return fail(IMG2D_ENOMEM, "device allocation of " + std::to_string(n) + " bytes refused: above the " +
                                      std::to_string(lim) + "-byte allocation limit (IMG2D_ALLOC_LIMIT_BYTES)");
    cudaError_t e = cudaMalloc(p, n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(IMG2D_ENOMEM, "cudaMalloc(" + std::to_string(n) + " bytes): " + cudaGetErrorString(e));
    }
    return IMG2D_OK;
}

// ---------------------------------------------------------------------------------------
// Plan
// ---------------------------------------------------------------------------------------
// Bump allocator over a fixed device region (the no-allocation entry point's static scratch).
struct Carver {
    unsigned char *base = nullptr;
    size_t cap = 0, used = 0;
};

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    bool owned = false;
    Carver *carver = nullptr;  // when set, storage is carved from it and never freed
    ~DevBuf() { release(); }
    void release()
    {
        if (p && owned) cudaFree(p);
        p = nullptr;
        bytes = 0;
        owned = false;
    }
    int ensure(size_t n)
    {
        if (n <= bytes && p) return IMG2D_OK;
        release();
        if (carver) {
            const size_t off = (carver->used + 255) & ~(size_t)255;
            if (off + n > carver->cap)
                return fail(IMG2D_EINVAL, "problem needs more than the " + std::to_string(carver->cap >> 20) +
                                              " MiB of fixed scratch of the no-allocation entry point");
            p = carver->base + off;
            bytes = n;
            carver->used = off + n;
            return IMG2D_OK;
        }
        if (n == 0) n = 16;
        const int rc = device_alloc(&p, n);
        if (rc) return rc;
        owned = true;
        bytes = n;
        return IMG2D_OK;
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

}  // namespace img2d

struct img2d_plan {
    int ns = 0, nextrap = 0, nz = 0, nx = 0, nf = 0, nt = 0, M = 0, L = 0, nk = 0, flags = 0;
    int mode = img2d::OP_CONJ;
    int G = 1, grid = 0, n_items = 0, max_w = 0, tab_stride = 0, idx_lstride = 0;
    bool fixed = false;
    img2d::KernelFn fn = nullptr;
    size_t smem = 0;
    std::vector<int> x0, w;
    std::vector<long long> off;
    long long wave_elems = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool ev_recorded = false;
    bool launched = false;  // a migration kernel has been queued (its status word is initialised)
    // identity of this plan for caches keyed on it (a new plan may reuse a freed plan's address)
    const unsigned long long uid = next_uid();
    static unsigned long long next_uid()
    {
        static std::atomic<unsigned long long> n{0};
        return ++n;
    }
    const char *packing = "lines";  // how shots were packed into the wide kernel's items
    double pack_cost = 0.0;         // wide kernel: modelled cost of all items of one frequency, in CTA units
    double computed_per_useful = 0.0;  // computed (slot, position) pairs per aperture sample
    ~img2d_plan()
    {
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
    }
    int n_slots = 0;
    std::vector<int> group_order;  // migration groups, widest first (the order of the item queue)
    int cluster = 0;  // CTAs per cluster of the cluster kernel, 0 = single-CTA kernels
    int block = 256;                  // threads per CTA of the chosen kernel
    int variant = -1;                 // index into the cluster2 variant table
    int tab16 = 0;                    // operator table storage: 0 FP32, 1 FP16, 2 BF16
    const char *kname = "";           // name of the chosen kernel
    img2d::Carver *carver = nullptr;  // no-allocation mode: buffers carved from fixed scratch
    cudaStream_t upload_stream = 0;   // no-allocation mode: stream of the descriptor uploads
    bool timing = true;               // record events around the migration kernel
    img2d::DevBuf items, groups, segs, owner, shot_off, idx, tabF, tabB, tab16buf, partial, comp, counter, naive_buf;
    // dense tables (drop-in ABI) are owned by the caller of run_dense
    // lane-slot packing: shots of each slot, slots ordered by extent, right end of each slot
    std::vector<std::vector<int>> slots;
    std::vector<int> slot_order, slot_end;
    // demigration (adjoint) launch state, built on its first call
    int adj_G = 0, adj_grid = 0, adj_items_n = 0, adj_wmax = 0, adj_block = 0, adj_slab = 0, adj_nslab = 0;
    int adj_cluster = 0;               // CTAs per cluster of the cluster demigration kernel, 0 = single CTA
    bool adj_ring = false;             // its forward steps read operator pairs through the shared-memory ring
    bool model_set = false;            // set_model has built the padded tables and the operator index
    long long adj_work_cta = 0, adj_cache_item = 0;  // float2 elements: per-CTA work area, kept per item
    size_t adj_smem = 0;
    void (*adj_fn)(img2d::DemigrateArgs) = nullptr;
    img2d::DevBuf adj_items, adj_groups, adj_segs, adj_owner, adj_work, adj_counter;
    img2d::DevBuf adj_cache;   // source checkpoints kept per item (IMG2D_SOURCE_KEEP)
    bool adj_cache_valid = false;
};

namespace img2d {

static int check_device()
{
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(IMG2D_ENODEV, "no CUDA device visible to imaging2d_wlsq_b200");
    }
    return IMG2D_OK;
}

// Largest portable cluster is 8 CTAs; B200 runs up to 16 when the kernel opts in.
constexpr int kMaxCluster = 16;

// How many clusters of K CTAs (block threads, smem bytes each) of `fn` fit on the device at once;
// 0 when none does.  K > 8 sets the non-portable cluster-size attribute first.
static int clusters_that_fit(const void *fn, int K, int block, size_t smem)
{
    if (K > 8 && cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr{};
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = K;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.gridDim = dim3(K * 64, 1, 1);
    cfg.blockDim = dim3(block, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, fn, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

// Shared memory bytes of one CTA for groups of G shots over a union window of width W.
static size_t smem_bytes(int G, int W, int M, int X)
{
    const int Mp = ((M + X - 1) / X) * X;
    const int Wp = ((W + X - 1) / X) * X;
    const int npos = Mp + Wp + Mp;
    const size_t nslot = (size_t)npos / X * (X + 1);
    return 2 * nslot * G * sizeof(float4);
}

// One group from its lines (each a list of shots, in increasing x, separated by >= M zero samples).
static void emit_group(const img2d_plan *p, const std::vector<std::vector<int>> &lines, std::vector<GroupDesc> &groups,
                       std::vector<int4> &segs, std::vector<int16_t> &owner)
{
    int u0 = p->nx, u1 = 0;
    for (const auto &line : lines)
        for (int s : line) {
            u0 = std::min(u0, p->x0[s]);
            u1 = std::max(u1, p->x0[s] + p->w[s]);
        }
    GroupDesc gd{};
    gd.seg_begin = (int)segs.size();
    gd.u0 = u0;
    gd.W = u1 - u0;
    gd.nslots = (int)lines.size();
    gd.owner_stride = (gd.W + 7) / 8 * 8;
    gd.owner_off = (long long)owner.size();
    owner.resize(owner.size() + (size_t)gd.nslots * gd.owner_stride, (int16_t)-1);
    for (int k = 0; k < gd.nslots; ++k)
        for (int s : lines[k]) {
            segs.push_back(make_int4(s, k, p->x0[s], p->w[s]));
            int16_t *row = owner.data() + gd.owner_off + (size_t)k * gd.owner_stride;
            for (int x = p->x0[s]; x < p->x0[s] + p->w[s]; ++x) row[x - u0] = (int16_t)s;
        }
    gd.nseg = (int)segs.size() - gd.seg_begin;
    groups.push_back(gd);
}

// Slots of similar extent form groups of G that share a work item; returns the widest group.
static int pack_groups(const img2d_plan *p, int G, std::vector<GroupDesc> &groups, std::vector<int4> &segs,
                       std::vector<int16_t> &owner)
{
    groups.clear();
    segs.clear();
    owner.clear();
    int widest = 0;
    const std::vector<int> &sorder = p->slot_order;
    for (size_t g0 = 0; g0 < sorder.size(); g0 += G) {
        const int n = (int)std::min<size_t>(G, sorder.size() - g0);
        std::vector<std::vector<int>> lines;
        for (int k = 0; k < n; ++k) lines.push_back(p->slots[sorder[g0 + k]]);
        emit_group(p, lines, groups, segs, owner);
        widest = std::max(widest, groups.back().W);
    }
    return widest;
}

// Wide kernel (8 slots x 1024 positions per CTA, clusters of K CTAs, each item's window split
// evenly over the cluster in 256-position units): cost of one item of width W in CTA units (one
// CTA, one depth step, all 1024 positions), divided by the throughput of a CTA with NC/64 busy
// warps relative to 16.  The relative throughputs were measured on a B200 on equal work (full
// aperture shots, windows of 2048/1536/512/256 positions): 0.92 with 12 busy warps, 0.87 with 8,
// 0.62 with 4.  eff12 replaces the 12-warp figure (the packing's greedy also tries other values to
// steer its choices; costs are always compared with the measured one).
static double wide_item_cost(int W, int K, double eff12 = 0.92)
{
    const int NC = std::min(WideShape::PC, (W + K * 256 - 1) / (K * 256) * 256);
    const double eff = NC >= 1024 ? 1.0 : (NC >= 768 ? eff12 : (NC >= 512 ? 0.87 : 0.62));
    return (double)K * NC / WideShape::PC / eff;
}

// The shots of `pool` (sorted by aperture end) that lie inside [u0, u1), in that order; returns
// their total aperture width.
static long long window_shots(const img2d_plan *p, const std::vector<int> &pool, int u0, int u1,
                              std::vector<int> &cand)
{
    cand.clear();
    long long sum = 0;
    for (int s : pool)
        if (p->x0[s] >= u0 && p->x0[s] + p->w[s] <= u1) {
            cand.push_back(s);
            sum += p->w[s];
        }
    return sum;
}

// Up to G lines from the shots `cand` (sorted by aperture end): each line is the heaviest chain of
// shots (total aperture width) separated by >= M, taken in turn (weighted interval scheduling,
// repeated).  Returns the aperture width covered; the lines when asked.
static long long window_lines(const img2d_plan *p, std::vector<int> cand, int G,
                              std::vector<std::vector<int>> *lines_out)
{
    long long covered = 0;
    std::vector<long long> best, ends;
    std::vector<int> prev;
    std::vector<char> take;
    for (int line = 0; line < G && !cand.empty(); ++line) {
        const int n = (int)cand.size();
        ends.resize(n);
        best.assign(n + 1, 0);
        prev.resize(n);
        take.assign(n, 0);
        for (int i = 0; i < n; ++i) ends[i] = (long long)p->x0[cand[i]] + p->w[cand[i]] + p->M;
        for (int i = 0; i < n; ++i) {
            const int s = cand[i];
            // shots before i that end (with the M gap) at or before this one's start
            const int j = (int)(std::upper_bound(ends.begin(), ends.begin() + i, (long long)p->x0[s]) - ends.begin());
            prev[i] = j;
            const long long with = best[j] + p->w[s];
            if (with > best[i]) {
                best[i + 1] = with;
                take[i] = 1;
            } else {
                best[i + 1] = best[i];
            }
        }
        std::vector<int> chosen;
        std::vector<char> used(n, 0);
        for (int i = n; i > 0;) {
            if (take[i - 1]) {
                chosen.push_back(cand[i - 1]);
                used[i - 1] = 1;
                i = prev[i - 1];
            } else {
                --i;
            }
        }
        covered += best[n];
        if (lines_out) {
            std::reverse(chosen.begin(), chosen.end());
            lines_out->push_back(chosen);
        }
        std::vector<int> rest;
        for (int i = 0; i < n; ++i)
            if (!used[i]) rest.push_back(cand[i]);
        cand.swap(rest);
    }
    return covered;
}

// Window-first packing for the wide kernel: repeatedly take the window (a start on a 32-position
// grid or at an end of one of the 8 widest remaining shots, and a width of K x 256 x m positions,
// m = 1..4, the widths at which an item's cost steps) whose G best lines of the remaining shots
// cover the most aperture per unit of cost, until every shot is placed.  Narrow windows become narrow items, which the kernel runs with fewer busy warps
// instead of computing positions outside every aperture.  Returns the total cost in CTA units.
static double pack_groups_windows(const img2d_plan *p, int G, int K, std::vector<GroupDesc> &groups,
                                  std::vector<int4> &segs, std::vector<int16_t> &owner, double sel_eff12 = 0.92)
{
    groups.clear();
    segs.clear();
    owner.clear();
    std::vector<int> pool(p->ns);
    std::iota(pool.begin(), pool.end(), 0);
    std::stable_sort(pool.begin(), pool.end(),
                     [&](int a, int b) { return p->x0[a] + p->w[a] < p->x0[b] + p->w[b]; });
    const int nx = p->nx;
    const int step = std::max(32, (nx / 64 + 31) / 32 * 32);
    double total = 0.0;
    std::vector<int> starts, cand, prev;
    while (!pool.empty()) {
        double best_ratio = -1.0;
        int best_u0 = 0, best_w = 0;
        // the 8 widest remaining shots also get windows aligned to either of their ends, so that a
        // shot nearly as wide as a window still has one that holds it
        std::vector<int> widest(pool);
        std::stable_sort(widest.begin(), widest.end(), [&](int a, int b) { return p->w[a] > p->w[b]; });
        widest.resize(std::min<size_t>(8, widest.size()));
        for (int m = 1; m <= 4; ++m) {
            const int W = std::min(nx, K * 256 * m);
            const double c = wide_item_cost(W, K, sel_eff12);
            starts.clear();
            for (int u = 0; u <= std::max(nx - W, 0) + step - 1; u += step) starts.push_back(u);
            for (int s : widest) starts.push_back(p->x0[s]);
            for (int s : widest) starts.push_back(p->x0[s] + p->w[s] - W);
            prev.clear();
            for (int u : starts) {
                const int u0 = std::max(0, std::min(u, nx - W));
                // the total width of the shots inside bounds what G lines can cover; a window with
                // the same shots as the previous one of this width covers the same
                const long long bound = window_shots(p, pool, u0, u0 + W, cand);
                if (bound == 0 || bound / c <= best_ratio || cand == prev) continue;
                prev = cand;
                const long long cov = window_lines(p, cand, G, nullptr);
                if (cov > 0 && cov / c > best_ratio) {
                    best_ratio = cov / c;
                    best_u0 = u0;
                    best_w = W;
                }
            }
            if (W >= nx) break;
        }
        if (best_ratio <= 0.0) return -1.0;  // a shot wider than every window (not reached: K covers it)
        std::vector<std::vector<int>> lines;
        window_shots(p, pool, best_u0, best_u0 + best_w, cand);
        window_lines(p, cand, G, &lines);
        emit_group(p, lines, groups, segs, owner);
        total += wide_item_cost(groups.back().W, K);
        std::vector<char> placed(p->ns, 0);
        for (const auto &line : lines)
            for (int s : line) placed[s] = 1;
        std::vector<int> rest;
        for (int s : pool)
            if (!placed[s]) rest.push_back(s);
        pool.swap(rest);
    }
    return total;
}

// Pack shots into lane slots: shots sorted by aperture start go to the slot whose last shot ends
// furthest to the left while still leaving >= M zero samples before this one (interval colouring,
// best fit); full-aperture shots get a slot each.  Slots are then ordered by extent.  Needs x0, w
// and M of the plan.
static void colour_slots(img2d_plan *p)
{
    const int ns = (int)p->x0.size(), M = p->M;
    std::vector<int> order(ns);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        if (p->x0[a] != p->x0[b]) return p->x0[a] < p->x0[b];
        return p->w[a] < p->w[b];
    });
    std::vector<std::vector<int>> slots;
    std::vector<int> slot_end;
    for (int s : order) {
        int best = -1;
        for (size_t i = 0; i < slots.size(); ++i)
            if (slot_end[i] + M <= p->x0[s] && (best < 0 || slot_end[i] > slot_end[best])) best = (int)i;
        if (best < 0) {
            slots.push_back({s});
            slot_end.push_back(p->x0[s] + p->w[s]);
        } else {
            slots[best].push_back(s);
            slot_end[best] = p->x0[s] + p->w[s];
        }
    }
    std::vector<int> sorder(slots.size());
    std::iota(sorder.begin(), sorder.end(), 0);
    auto ext0 = [&](int i) { return p->x0[slots[i].front()]; };
    std::stable_sort(sorder.begin(), sorder.end(), [&](int a, int b) {
        if (ext0(a) != ext0(b)) return ext0(a) < ext0(b);
        return slot_end[a] < slot_end[b];
    });
    p->n_slots = (int)slots.size();
    p->slots = slots;
    p->slot_order = sorder;
    p->slot_end = slot_end;
}

// Surveys with more shots keep the line packing: the window greedy would take seconds per plan.
constexpr int kWindowPackingMaxShots = 2048;

// The window-first packing with three weightings of 12-warp items in the greedy's choices (the
// measured 0.92, then 0.95 and 1.0: a myopic greedy lands on different packings); keeps the one of
// lowest measured-model cost.  The greedy's time grows about as the square of the shot count
// (0.4 s for 1024 shots on one host core), so above 512 shots only the measured weighting runs.
static double pack_windows_best(const img2d_plan *p, int G, int K, std::vector<GroupDesc> &groups,
                                std::vector<int4> &segs, std::vector<int16_t> &owner)
{
    double best = -1.0;
    const double sels[3] = {0.92, 0.95, 1.0};
    const int nsel = p->ns > 512 ? 1 : 3;
    for (int i = 0; i < nsel; ++i) {
        const double sel = sels[i];
        std::vector<GroupDesc> g2;
        std::vector<int4> s2;
        std::vector<int16_t> o2;
        const double c = pack_groups_windows(p, G, K, g2, s2, o2, sel);
        if (c > 0.0 && (best < 0.0 || c < best - 1e-9)) {
            best = c;
            groups.swap(g2);
            segs.swap(s2);
            owner.swap(o2);
        }
    }
    return best;
}

static int build_plan(img2d_plan *p, int ns, int nextrap, int nz, int nx, int nf, int nt, int M,
                      int nk, const int *shot_x0, const int *shot_nx, int flags, int mode)
{
    if (ns <= 0 || nextrap <= 0 || nz < nextrap || nx <= 0 || nf <= 0 || nt < nf || M < 0)
        return fail(IMG2D_EINVAL, "invalid dimensions (need ns>0, 0<nextrap<=nz, nx>0, 0<nf<=nt, M>=0)");
    if (mode != OP_DENSE && (nk <= 0 || nk > 65535))
        return fail(IMG2D_EINVAL, "nk must be in [1, 65535]");
    if ((long long)nf * nextrap * nx > (1ll << 40)) return fail(IMG2D_EINVAL, "problem too large");
    if (ns > 32767) return fail(IMG2D_EINVAL, "at most 32767 shots per plan");
    p->ns = ns; p->nextrap = nextrap; p->nz = nz; p->nx = nx; p->nf = nf; p->nt = nt; p->M = M;
    p->L = 2 * M + 1; p->nk = nk; p->flags = flags; p->mode = mode;
    p->x0.assign(ns, 0);
    p->w.assign(ns, nx);
    for (int s = 0; s < ns; ++s) {
        if (shot_x0) p->x0[s] = shot_x0[s];
        if (shot_nx) p->w[s] = shot_nx[s];
        if (p->x0[s] < 0 || p->w[s] <= 0 || p->x0[s] + p->w[s] > nx)
            return fail(IMG2D_EINVAL, "shot " + std::to_string(s) + " aperture outside [0, nx)");
    }
    p->off.assign(ns, 0);
    long long acc = 0;
    for (int s = 0; s < ns; ++s) {
        p->off[s] = acc;
        acc += (long long)nt * p->w[s];
    }
    p->wave_elems = acc;

    int dev = 0;
    IMG2D_CUDA(cudaGetDevice(&dev));
    int smem_optin = 0, nsm = 0;
    IMG2D_CUDA(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    IMG2D_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int static_reserve = 1024;

    colour_slots(p);

    std::vector<GroupDesc> groups;
    std::vector<int4> segs;
    std::vector<int16_t> owner;
    auto make_groups = [&](int G) { return pack_groups(p, G, groups, segs, owner); };

    // Kernel choice.  The second-generation cluster kernel (16 slots per item, 512 positions per CTA,
    // clusters of up to 16 CTAs where they fit) when there are enough slots to fill it and the
    // operator has at least 7 taps; else the first-generation cluster kernel (256 positions per CTA,
    // up to 8 CTAs, compile-time operator lengths); otherwise the single-CTA kernels with the
    // largest power of two <= 8 slots whose ping-pong buffers fit in shared memory.
    p->cluster = 0;
    p->block = 256;
    const bool cluster_ok = mode == OP_CONJ && !(flags & (IMG2D_FLAG_GENERIC | IMG2D_FLAG_NO_CLUSTER)) &&
                            p->n_slots >= 12;
    int vsel = (flags >> IMG2D_FLAG_VARIANT_SHIFT) & 0xff;
    const bool explicit_variant = vsel >= 1 && vsel <= kNumCluster2;
    vsel = explicit_variant ? vsel - 1 : kCluster2Default;
    Cluster2Variant cv = kCluster2[vsel];
    const int tab16 = (flags & IMG2D_FLAG_TABLE_BF16) ? 2 : ((flags & IMG2D_FLAG_TABLE_FP16) ? 1 : 0);
    if (tab16) {
        // reduced-precision operator storage: the staged shape with 16-bit tap loads
        cv = {16, false, false,
              tab16 == 1 ? migrate_cluster2_kernel<16, false, false, false, TAB_F16, 4>
                         : migrate_cluster2_kernel<16, false, false, false, TAB_BF16, 4>,
              true};
        vsel = kCluster2Staged;
    }
    // Use variant v when its shared memory fits and, for windows wider than 8 CTAs, clusters of the
    // needed size fit on the device.
    auto try_cluster2 = [&](const Cluster2Variant &v, int index) {
        const int pc2 = v.nw * 32;
        const size_t smem2 = cluster2_smem_bytes(M, pc2) + (v.stage ? cluster2_stage_bytes(pc2) : 0) +
                             (v.ring ? cluster2_ring_bytes(pc2) : 0);
        if (smem2 + static_reserve > (size_t)smem_optin) return false;
        const int widest = make_groups(16);
        const int K = (widest + pc2 - 1) / pc2;
        if (!(K <= 8 || (K <= kMaxCluster && clusters_that_fit((const void *)v.fn, K, pc2, smem2) > 0))) return false;
        p->cluster = K;
        p->G = 16;
        p->fixed = true;
        p->fn = v.fn;
        p->smem = smem2;
        p->max_w = widest;
        p->block = pc2;
        p->variant = index;
        p->kname = "migrate_cluster2";
        return true;
    };
    // Wide cluster kernel (8 slots x 1024 positions per CTA, clusters of half the size, packed FMAs).
    // It is the default where the cluster2 kernel's clusters would leave SMs idle (clusters of 4 fit
    // 33 times on 148 SMs), and on request (IMG2D_FLAG_WIDE / _WIDE_SCALAR).
    auto try_wide = [&]() {
        // with the step-ahead stage where its 12 KB fit (operators up to 49 taps); the bulk-copy
        // ring adds 256 bytes of barriers
        const bool bulk = (flags & IMG2D_FLAG_WIDE_BULK) != 0;
        const size_t bars = bulk ? wide_bulk_smem_bytes(M, true) - wide_stage_smem_bytes(M) : 0;
        const bool stage = wide_stage_smem_bytes(M) + bars + static_reserve <= (size_t)smem_optin;
        KernelFn wf;
        if (bulk)
            wf = stage ? migrate_wide_kernel<1, true, true> : migrate_wide_kernel<1, false, true>;
        else if (flags & IMG2D_FLAG_WIDE_SCALAR)
            wf = stage ? migrate_wide_kernel<0, true> : migrate_wide_kernel<0, false>;
        else
            wf = stage ? migrate_wide_kernel<1, true> : migrate_wide_kernel<1, false>;
        const size_t smemw = (stage ? wide_stage_smem_bytes(M) : wide_smem_bytes(M)) + bars;
        if (smemw + static_reserve > (size_t)smem_optin) return false;
        int widest = make_groups(WideShape::G);
        int K = (widest + WideShape::PC - 1) / WideShape::PC;
        p->packing = "lines";
        p->pack_cost = 0.0;
        for (const GroupDesc &g : groups) p->pack_cost += wide_item_cost(g.W, K);
        if (!(flags & IMG2D_FLAG_LINE_PACKING) && p->ns <= kWindowPackingMaxShots) {
            // window-first packing where it costs at least 1% less, on clusters just wide enough for
            // the widest shot or one CTA wider (wider windows chain more shots per lane slot);
            // cluster sizes beyond the portable 8 only where the line packing needs them anyway
            const int Kw = (*std::max_element(p->w.begin(), p->w.end()) + WideShape::PC - 1) / WideShape::PC;
            const int Kline = K;
            for (int Kc = Kw; Kc <= Kw + 1; ++Kc) {
                if (Kc > 8 && Kc != Kline) continue;
                std::vector<GroupDesc> g2;
                std::vector<int4> s2;
                std::vector<int16_t> o2;
                const double cost2 = pack_windows_best(p, WideShape::G, Kc, g2, s2, o2);
                if (cost2 > 0.0 && cost2 < p->pack_cost * 0.99) {
                    groups.swap(g2);
                    segs.swap(s2);
                    owner.swap(o2);
                    K = Kc;
                    widest = 0;
                    for (const GroupDesc &g : groups) widest = std::max(widest, g.W);
                    p->packing = "windows";
                    p->pack_cost = cost2;
                }
            }
        }
        if (!(K <= 8 || (K <= kMaxCluster && clusters_that_fit((const void *)wf, K, WideShape::NW * 32, smemw) > 0)))
            return false;
        p->cluster = K;
        p->G = WideShape::G;
        p->fixed = true;
        p->fn = wf;
        p->smem = smemw;
        p->max_w = widest;
        p->block = WideShape::NW * 32;
        p->variant = ((flags & IMG2D_FLAG_WIDE_SCALAR) ? 0 : 1) + (stage ? 2 : 0) + (bulk ? 4 : 0);
        p->kname = "migrate_wide";
        return true;
    };
    const int wide_flags = IMG2D_FLAG_WIDE | IMG2D_FLAG_WIDE_SCALAR | IMG2D_FLAG_WIDE_BULK;
    if ((flags & IMG2D_FLAG_WIDE_BULK) && (flags & IMG2D_FLAG_WIDE_SCALAR))
        return fail(IMG2D_EINVAL, "IMG2D_FLAG_WIDE_BULK runs packed FMAs; it does not combine with "
                                  "IMG2D_FLAG_WIDE_SCALAR");
    const bool wide_requested = (flags & wide_flags) != 0;
    const bool wide_ok = mode == OP_CONJ && !tab16 && p->L >= 7 &&
                         !(flags & (IMG2D_FLAG_GENERIC | IMG2D_FLAG_NO_CLUSTER | IMG2D_FLAG_CLUSTER_V1 |
                                    IMG2D_FLAG_CLUSTER2)) &&
                         !explicit_variant && (wide_requested || p->n_slots >= 6);
    bool want_wide = wide_ok && wide_requested;
    if (wide_ok && !wide_requested) {
        // default choice: SMs the cluster2 kernel would keep busy on this geometry
        const int pc2 = cv.nw * 32;
        const size_t smem2 = cluster2_smem_bytes(M, pc2) + (cv.stage ? cluster2_stage_bytes(pc2) : 0) +
                             (cv.ring ? cluster2_ring_bytes(pc2) : 0);
        const int K2 = (make_groups(16) + pc2 - 1) / pc2;
        const int busy = smem2 + static_reserve <= (size_t)smem_optin && K2 <= kMaxCluster
                             ? clusters_that_fit((const void *)cv.fn, K2, pc2, smem2) * K2
                             : 0;
        want_wide = p->n_slots < 12 || busy < nsm * 96 / 100;
    }
    if (want_wide) try_wide();
    if (!p->cluster && cluster_ok && !(flags & (IMG2D_FLAG_CLUSTER_V1 | wide_flags)) &&
        p->L >= 7) {
        // the default ring variant needs 33 KB more shared memory than the staged one: long
        // operators or very wide windows fall back to the staged variant
        if (!try_cluster2(cv, vsel) && !explicit_variant && !tab16 && vsel != kCluster2Staged)
            try_cluster2(kCluster2[kCluster2Staged], kCluster2Staged);
    }
    if (tab16 && !p->cluster)
        return fail(IMG2D_EINVAL, "16-bit operator tables need the cluster kernel (>= 12 lane slots, 2M+1 >= 7, "
                                  "window <= 16 CTAs)");
    p->tab16 = tab16;
    const ClusterKernel *ck = cluster_ok ? find_cluster(p->L) : nullptr;
    if (!p->cluster && ck && ck->smem + static_reserve <= (size_t)smem_optin) {
        const int widest = make_groups(ClusterShape::G);
        const int K = (widest + ClusterShape::PC - 1) / ClusterShape::PC;
        if (K <= 8) {
            p->cluster = K == 1 ? 1 : (K <= 2 ? 2 : (K <= 4 ? 4 : 8));
            p->G = ClusterShape::G;
            p->fixed = true;
            p->fn = ck->fn;
            p->smem = ck->smem;
            p->max_w = widest;
            p->kname = "migrate_cluster";
        }
    }
    if (!p->cluster) {
        int nsp2 = 1;
        while (nsp2 < p->n_slots) nsp2 <<= 1;
        int G = 8;
        while (G > 1 && (G > nsp2 || smem_bytes(G, nx, M, kX) + static_reserve > (size_t)smem_optin)) G >>= 1;
        const bool use_fixed = (mode == OP_CONJ) && !(flags & IMG2D_FLAG_GENERIC) && find_fixed(G, p->L);
        const int X = use_fixed ? kX : 4;
        if (smem_bytes(G, nx, M, X) + static_reserve > (size_t)smem_optin)
            return fail(IMG2D_EINVAL, "aperture too wide for one CTA's shared memory");
        p->G = G;
        p->fixed = use_fixed;
        p->fn = use_fixed ? find_fixed(G, p->L) : find_generic(G, mode);
        p->max_w = make_groups(G);
        p->smem = smem_bytes(G, p->max_w, M, X);
        p->kname = use_fixed ? "migrate_fixed" : "migrate_generic";
    }
    // Items (group, frequency), widest groups first so the tail of the queue is short work.
    std::vector<int2> items;
    items.reserve(groups.size() * (size_t)nf);
    std::vector<int> gorder(groups.size());
    std::iota(gorder.begin(), gorder.end(), 0);
    std::stable_sort(gorder.begin(), gorder.end(), [&](int a, int b) { return groups[a].W > groups[b].W; });
    for (int g : gorder)
        for (int j = 0; j < nf; ++j) items.push_back(make_int2(g, j));
    p->n_items = (int)items.size();
    p->group_order = gorder;
    {
        // (slot, position) pairs the kernel computes per depth step and frequency, per useful one
        double computed = 0.0, useful = 0.0;
        for (int s = 0; s < ns; ++s) useful += p->w[s];
        const int K = std::max(1, p->cluster);
        for (const GroupDesc &g : groups) {
            if (!strcmp(p->kname, "migrate_wide"))
                computed += (double)K * std::min(WideShape::PC, (g.W + K * 256 - 1) / (K * 256) * 256) * p->G;
            else if (!strcmp(p->kname, "migrate_cluster2"))
                computed += (double)K * p->block * p->G;
            else
                computed += (double)g.W * p->G;
        }
        p->computed_per_useful = computed / useful;
    }
    IMG2D_CUDA(cudaFuncSetAttribute(p->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->smem));
    if (p->cluster) {
        cudaLaunchConfig_t cfg{};
        cudaLaunchAttribute attr{};
        attr.id = cudaLaunchAttributeClusterDimension;
        attr.val.clusterDim.x = p->cluster;
        attr.val.clusterDim.y = 1;
        attr.val.clusterDim.z = 1;
        cfg.gridDim = dim3(p->cluster * 64, 1, 1);
        cfg.blockDim = dim3(p->block, 1, 1);
        cfg.dynamicSmemBytes = p->smem;
        cfg.attrs = &attr;
        cfg.numAttrs = 1;
        int nclusters = 0;
        IMG2D_CUDA(cudaOccupancyMaxActiveClusters(&nclusters, (void *)p->fn, &cfg));
        if (nclusters <= 0) return fail(IMG2D_ECUDA, "no cluster of this size fits on the device");
        p->grid = std::min(p->n_items, nclusters) * p->cluster;
    } else {
        p->grid = std::min(p->n_items, nsm);
    }

    int rc;
    if ((rc = p->items.ensure(items.size() * sizeof(int2)))) return rc;
    if ((rc = p->groups.ensure(groups.size() * sizeof(GroupDesc)))) return rc;
    if ((rc = p->segs.ensure(segs.size() * sizeof(int4)))) return rc;
    if ((rc = p->owner.ensure(owner.size() * sizeof(int16_t)))) return rc;
    if ((rc = p->shot_off.ensure(p->off.size() * sizeof(long long)))) return rc;
    if ((rc = p->counter.ensure(2 * sizeof(int)))) return rc;  // work-queue counter, status word
    if (p->carver) {
        // ordered on the caller's stream after any earlier call that used the same scratch
        cudaStream_t us = p->upload_stream;
        IMG2D_CUDA(cudaMemcpyAsync(p->items.p, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice, us));
        IMG2D_CUDA(cudaMemcpyAsync(p->groups.p, groups.data(), groups.size() * sizeof(GroupDesc), cudaMemcpyHostToDevice, us));
        IMG2D_CUDA(cudaMemcpyAsync(p->segs.p, segs.data(), segs.size() * sizeof(int4), cudaMemcpyHostToDevice, us));
        IMG2D_CUDA(cudaMemcpyAsync(p->owner.p, owner.data(), owner.size() * sizeof(int16_t), cudaMemcpyHostToDevice, us));
        IMG2D_CUDA(cudaMemcpyAsync(p->shot_off.p, p->off.data(), p->off.size() * sizeof(long long), cudaMemcpyHostToDevice, us));
        // pageable sources: make sure the copies have read the host vectors before they go away
        IMG2D_CUDA(cudaStreamSynchronize(us));
    } else {
        IMG2D_CUDA(cudaMemcpy(p->items.p, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice));
        IMG2D_CUDA(cudaMemcpy(p->groups.p, groups.data(), groups.size() * sizeof(GroupDesc), cudaMemcpyHostToDevice));
        IMG2D_CUDA(cudaMemcpy(p->segs.p, segs.data(), segs.size() * sizeof(int4), cudaMemcpyHostToDevice));
        IMG2D_CUDA(cudaMemcpy(p->owner.p, owner.data(), owner.size() * sizeof(int16_t), cudaMemcpyHostToDevice));
        IMG2D_CUDA(cudaMemcpy(p->shot_off.p, p->off.data(), p->off.size() * sizeof(long long), cudaMemcpyHostToDevice));
    }
    const size_t plane = (size_t)nextrap * nx;
    if (p->carver) {
        // fixed scratch: fewer persistent CTAs when their private image partials would not fit
        const size_t idx_b = (size_t)nf * nextrap * ((nx + 7) / 8 * 8) * sizeof(uint16_t) + 256;
        const size_t tab_b = ((size_t)nk * ((p->L + 1) / 2 * 2) * sizeof(cpx) + 256) * (mode == OP_TWO ? 2 : 1);
        const size_t used = (p->carver->used + 255) & ~(size_t)255;
        const size_t left = p->carver->cap > used + idx_b + tab_b ? p->carver->cap - used - idx_b - tab_b : 0;
        const size_t fit = left / (2 * plane * sizeof(float) + 512);
        if (fit < 1)
            return fail(IMG2D_EINVAL, "problem needs more than the " + std::to_string(p->carver->cap >> 20) +
                                          " MiB of fixed scratch of the no-allocation entry point");
        p->grid = (int)std::min<size_t>((size_t)p->grid, fit);
    }
    if ((rc = p->partial.ensure((size_t)p->grid * plane * sizeof(float)))) return rc;
    if ((rc = p->comp.ensure((size_t)p->grid * plane * sizeof(float)))) return rc;
    if (mode != OP_DENSE) {
        p->idx_lstride = (nx + 7) / 8 * 8;
        if ((rc = p->idx.ensure((size_t)nf * nextrap * p->idx_lstride * sizeof(uint16_t)))) return rc;
        p->tab_stride = (p->L + 1) / 2 * 2;
        if ((rc = p->tabF.ensure((size_t)nk * p->tab_stride * sizeof(cpx)))) return rc;
        if (p->tab16 && (rc = p->tab16buf.ensure((size_t)nk * p->tab_stride * sizeof(unsigned)))) return rc;
        if (mode == OP_TWO && (rc = p->tabB.ensure((size_t)nk * p->tab_stride * sizeof(cpx)))) return rc;
    }
    return IMG2D_OK;
}

static MigrateArgs base_args(img2d_plan *p, cpx *wave, cpx *shot)
{
    MigrateArgs a{};
    a.nextrap = p->nextrap;
    a.nx = p->nx;
    a.nf = p->nf;
    a.M = p->M;
    a.tab_stride = p->tab_stride;
    a.n_items = p->n_items;
    a.items = p->items.as<int2>();
    a.groups = p->groups.as<GroupDesc>();
    a.segs = p->segs.as<int4>();
    a.owner = p->owner.as<int16_t>();
    a.shot_off = p->shot_off.as<long long>();
    a.tabF = p->tabF.as<cpx>();
    a.tabB = p->mode == OP_TWO ? p->tabB.as<cpx>() : p->tabF.as<cpx>();
    a.tab16 = p->tab16buf.p;
    a.idx = p->idx.as<uint16_t>();
    a.idx_jstride = (long long)p->nextrap * p->idx_lstride;
    a.idx_lstride = p->idx_lstride;
    a.wave = wave;
    a.shot = shot;
    a.write_back = 1;
    a.counter = p->counter.as<int>();
    return a;
}

// Status word of the last launch (after the work-queue counter), read on `st` after it.
static int read_status(img2d_plan *p, cudaStream_t st)
{
    int status = 0;
    IMG2D_CUDA(cudaMemcpyAsync(&status, p->counter.as<int>() + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    IMG2D_CUDA(cudaStreamSynchronize(st));
    if (status)
        return fail(IMG2D_ECUDA, "a bounded wait in the migration kernel gave up (status " + std::to_string(status) +
                                     "): the results of that launch are not valid");
    return IMG2D_OK;
}

// The plan's persistent migration kernel on `grid` CTAs (whole clusters) of stream st.
static int launch_kernel(img2d_plan *p, const MigrateArgs &a, int grid, cudaStream_t st)
{
    if (p->cluster) {
        cudaLaunchConfig_t cfg{};
        cudaLaunchAttribute attr{};
        attr.id = cudaLaunchAttributeClusterDimension;
        attr.val.clusterDim.x = p->cluster;
        attr.val.clusterDim.y = 1;
        attr.val.clusterDim.z = 1;
        cfg.gridDim = dim3(grid, 1, 1);
        cfg.blockDim = dim3(p->block, 1, 1);
        cfg.dynamicSmemBytes = p->smem;
        cfg.stream = st;
        cfg.attrs = &attr;
        cfg.numAttrs = 1;
        IMG2D_CUDA(cudaLaunchKernelEx(&cfg, p->fn, a));
    } else {
        p->fn<<<grid, 256, p->smem, st>>>(a);
    }
    IMG2D_CUDA(cudaGetLastError());
    return IMG2D_OK;
}

// Launch the persistent kernel and (optionally) reduce the stacked image.
static int launch(img2d_plan *p, MigrateArgs a, float *d_image, float *d_image_shots,
                  long long img_sstride, cudaStream_t st)
{
    const size_t plane = (size_t)p->nextrap * p->nx;
    IMG2D_CUDA(cudaMemsetAsync(p->counter.p, 0, 2 * sizeof(int), st));
    a.status = p->counter.as<int>() + 1;
    p->launched = true;
    if (d_image) {
        IMG2D_CUDA(cudaMemsetAsync(p->partial.p, 0, (size_t)p->grid * plane * sizeof(float), st));
        IMG2D_CUDA(cudaMemsetAsync(p->comp.p, 0, (size_t)p->grid * plane * sizeof(float), st));
        a.partial = p->partial.as<float>();
        a.comp = p->comp.as<float>();
    }
    if (d_image_shots) {
        IMG2D_CUDA(cudaMemset2DAsync(d_image_shots, img_sstride * sizeof(float), 0, plane * sizeof(float),
                                     p->ns, st));
        a.image_shots = d_image_shots;
        a.img_sstride = img_sstride;
    }
    if (p->timing && !p->ev0) {
        IMG2D_CUDA(cudaEventCreate(&p->ev0));
        IMG2D_CUDA(cudaEventCreate(&p->ev1));
    }
    if (p->timing) IMG2D_CUDA(cudaEventRecord(p->ev0, st));
    int rc;
    if ((rc = launch_kernel(p, a, p->grid, st))) return rc;
    if (p->timing) {
        IMG2D_CUDA(cudaEventRecord(p->ev1, st));
        p->ev_recorded = true;
    }
    if (d_image) {
        const int blocks = (int)std::min<size_t>((plane + 255) / 256, 148 * 8);
        reduce_partials_kernel<<<blocks, 256, 0, st>>>(p->partial.as<float>(), p->comp.as<float>(), p->grid,
                                                       (long long)plane, d_image);
        IMG2D_CUDA(cudaGetLastError());
    }
    return IMG2D_OK;
}

static int set_model(img2d_plan *p, const double *d_omega, const double *d_vel, double dk,
                     const cpx *d_tabF, const cpx *d_tabB, cudaStream_t st)
{
    p->adj_cache_valid = false;
    if (!d_omega || !d_vel || !d_tabF || !(dk > 0.0))
        return fail(IMG2D_EINVAL, "set_model needs omega, velocity, tab_forw and dk > 0");
    if (p->mode == OP_TWO && !d_tabB) return fail(IMG2D_EINVAL, "two-table mode needs tab_back");
    const size_t row = (size_t)p->L * sizeof(cpx), prow = (size_t)p->tab_stride * sizeof(cpx);
    IMG2D_CUDA(cudaMemsetAsync(p->tabF.p, 0, (size_t)p->nk * prow, st));
    IMG2D_CUDA(cudaMemcpy2DAsync(p->tabF.p, prow, d_tabF, row, row, p->nk, cudaMemcpyDeviceToDevice, st));
    if (p->mode == OP_TWO) {
        IMG2D_CUDA(cudaMemsetAsync(p->tabB.p, 0, (size_t)p->nk * prow, st));
        IMG2D_CUDA(cudaMemcpy2DAsync(p->tabB.p, prow, d_tabB, row, row, p->nk, cudaMemcpyDeviceToDevice, st));
    }
    if (p->tab16) {
        const long long n = (long long)p->nk * p->tab_stride;
        table_to_16bit_kernel<<<(int)std::min<long long>((n + 255) / 256, 148 * 8), 256, 0, st>>>(
            p->tabF.as<cpx>(), n, p->tab16 == 2, p->tab16buf.as<unsigned>());
        IMG2D_CUDA(cudaGetLastError());
    }
    const long long total = (long long)p->nf * p->nextrap * p->nx;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 16);
    index_table_kernel<<<blocks, 256, 0, st>>>(d_omega, d_vel, p->nf, p->nextrap, p->nx, p->idx_lstride, p->nk,
                                               dk, p->idx.as<uint16_t>());
    IMG2D_CUDA(cudaGetLastError());
    p->model_set = true;
    return IMG2D_OK;
}

// Launch state of the demigration: its own slot groups (one complex wavefield per slot, so up to
// 8 slots fit beside the halos), items, and the per-CTA checkpoint / slab / save planes.
static int demig_prepare(img2d_plan *p, int slab)
{
    if (slab <= 0) slab = 8;
    slab = std::min(slab, p->nextrap);
    const int nslab = (p->nextrap + slab - 1) / slab;
    if (p->adj_fn && p->adj_slab == slab) return IMG2D_OK;
    p->adj_cache_valid = false;  // the checkpoint layout depends on the slab depth
    int dev = 0, smem_optin = 0, nsm = 0;
    IMG2D_CUDA(cudaGetDevice(&dev));
    IMG2D_CUDA(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    IMG2D_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int static_reserve = 1024;
    std::vector<GroupDesc> groups;
    std::vector<int4> segs;
    std::vector<int16_t> owner;
    int G = 8, widest = 0, K = 0;
    bool ring = false;
    DemigFn fn = nullptr;
    size_t smem = 0;
    // Cluster kernel (16 slots per item, 512 positions per CTA) when there are enough slots to fill
    // it and the widest window fits 16 CTAs, with the forward steps' tap-pair ring where the operator
    // length has an instance and its shared memory fits; otherwise the single-CTA kernel.
    if (p->n_slots >= 12 && !(p->flags & IMG2D_FLAG_NO_CLUSTER)) {
        widest = pack_groups(p, 16, groups, segs, owner);
        const int k = (widest + kDcPC - 1) / kDcPC;
        auto try_fn = [&](DemigFn cfn, size_t csmem, bool is_ring) {
            if (!cfn || K || csmem + static_reserve > (size_t)smem_optin) return;
            if (k <= 8 || (k <= kMaxCluster && clusters_that_fit((const void *)cfn, k, kDcNW * 32, csmem) > 0)) {
                K = k;
                G = 16;
                fn = cfn;
                smem = csmem;
                ring = is_ring;
            }
        };
        if (!(p->flags & IMG2D_FLAG_DEMIG_NO_RING))
            try_fn(find_demig_cluster(p->L, true), demigc_ring_smem_bytes(p->M), true);
        try_fn(find_demig_cluster(p->L), demigc_smem_bytes(p->M), false);
    }
    if (!K) {
        for (;; G >>= 1) {
            widest = pack_groups(p, G, groups, segs, owner);
            if (demig_smem_bytes(G, widest, p->M) + static_reserve <= (size_t)smem_optin) break;
            if (G == 2) return fail(IMG2D_EINVAL, "aperture too wide for the demigration kernel's shared memory");
        }
        // fewer slots than lanes: smaller groups leave fewer idle lanes
        while (G > 2 && (int)p->slot_order.size() <= G / 2) G >>= 1;
        widest = pack_groups(p, G, groups, segs, owner);
        fn = find_demig(G, p->L);
        smem = demig_smem_bytes(G, widest, p->M);
    }
    if (!fn) return fail(IMG2D_EINVAL, "no demigration kernel for this configuration");
    IMG2D_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    std::vector<int2> items;
    std::vector<int> gorder(groups.size());
    std::iota(gorder.begin(), gorder.end(), 0);
    std::stable_sort(gorder.begin(), gorder.end(), [&](int a, int b) { return groups[a].W > groups[b].W; });
    for (int g : gorder)
        for (int j = 0; j < p->nf; ++j) items.push_back(make_int2(g, j));
    int grid = 0;
    long long work_cta = 0;   // float2 elements of per-CTA work area
    long long cache_item = 0; // float2 elements of kept checkpoints per item
    if (K) {
        cudaLaunchConfig_t cfg{};
        cudaLaunchAttribute attr{};
        attr.id = cudaLaunchAttributeClusterDimension;
        attr.val.clusterDim.x = K;
        attr.val.clusterDim.y = 1;
        attr.val.clusterDim.z = 1;
        cfg.gridDim = dim3(K * 64, 1, 1);
        cfg.blockDim = dim3(kDcNW * 32, 1, 1);
        cfg.dynamicSmemBytes = smem;
        cfg.attrs = &attr;
        cfg.numAttrs = 1;
        int nclusters = 0;
        IMG2D_CUDA(cudaOccupancyMaxActiveClusters(&nclusters, (void *)fn, &cfg));
        if (nclusters <= 0) return fail(IMG2D_ECUDA, "no demigration cluster of this size fits on the device");
        grid = (int)std::min<size_t>(items.size(), (size_t)nclusters) * K;
        const long long pe4 = (long long)kDcPC * kDcQ;  // float4 per plane
        work_cta = 2 * (long long)(nslab + slab + 1) * pe4;
        cache_item = 2 * (long long)K * nslab * pe4;
    } else {
        int bps = 0;
        IMG2D_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, fn, kAdjWarps * 32, smem));
        if (bps <= 0) return fail(IMG2D_ECUDA, "demigration kernel does not fit on an SM");
        grid = (int)std::min<size_t>(items.size(), (size_t)nsm * bps);
        work_cta = (long long)(nslab + slab + 1) * widest * G;
        cache_item = (long long)nslab * widest * G;
    }
    int rc;
    if ((rc = p->adj_items.ensure(items.size() * sizeof(int2)))) return rc;
    if ((rc = p->adj_groups.ensure(groups.size() * sizeof(GroupDesc)))) return rc;
    if ((rc = p->adj_segs.ensure(segs.size() * sizeof(int4)))) return rc;
    if ((rc = p->adj_owner.ensure(owner.size() * sizeof(int16_t)))) return rc;
    if ((rc = p->adj_counter.ensure(sizeof(int)))) return rc;
    if ((rc = p->adj_work.ensure((size_t)grid * work_cta * sizeof(float2)))) return rc;
    IMG2D_CUDA(cudaMemcpy(p->adj_items.p, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice));
    IMG2D_CUDA(cudaMemcpy(p->adj_groups.p, groups.data(), groups.size() * sizeof(GroupDesc), cudaMemcpyHostToDevice));
    IMG2D_CUDA(cudaMemcpy(p->adj_segs.p, segs.data(), segs.size() * sizeof(int4), cudaMemcpyHostToDevice));
    IMG2D_CUDA(cudaMemcpy(p->adj_owner.p, owner.data(), owner.size() * sizeof(int16_t), cudaMemcpyHostToDevice));
    p->adj_G = G;
    p->adj_grid = grid;
    p->adj_items_n = (int)items.size();
    p->adj_wmax = widest;
    p->adj_block = K ? kDcNW * 32 : kAdjWarps * 32;
    p->adj_cluster = K;
    p->adj_work_cta = work_cta;
    p->adj_cache_item = cache_item;
    p->adj_slab = slab;
    p->adj_nslab = nslab;
    p->adj_smem = smem;
    p->adj_fn = fn;
    p->adj_ring = ring;
    return IMG2D_OK;
}

// Scoped device allocation for the host entry points.
struct Scratch {
    std::vector<void *> ptrs;
    ~Scratch()
    {
        for (void *q : ptrs) cudaFree(q);
    }
    template <class T> int alloc(T **out, size_t n)
    {
        void *q = nullptr;
        const int rc = device_alloc(&q, n ? n : 16);
        if (rc) return rc;
        ptrs.push_back(q);
        *out = static_cast<T *>(q);
        return IMG2D_OK;
    }
};

// Dense-table drop-in: both argument orders come here.
// Sizes for which the reference's loops (cpp_src/extrapolation_cpu.cpp:39-99) do no extrapolation:
// ns, nx or nextrap zero leave every buffer as it was; nf zero writes zero image rows [0, nextrap).
// Handled on the host; returns 1 when the call is complete.
static int degenerate_call(int ns, int nextrap, int nz, int nx, int nf, float *image, int *rc)
{
    if (ns < 0 || nextrap < 0 || nz < 0 || nx < 0 || nf < 0 || nz < nextrap) {
        *rc = fail(IMG2D_EINVAL, "invalid dimensions (negative, or nz < nextrap)");
        return 1;
    }
    if (ns == 0 || nx == 0 || nextrap == 0) {
        *rc = IMG2D_OK;
        return 1;
    }
    if (nf == 0) {
        if (!image) {
            *rc = fail(IMG2D_EINVAL, "null image pointer");
            return 1;
        }
        for (int s = 0; s < ns; ++s)
            std::memset(image + (size_t)s * nz * nx, 0, (size_t)nextrap * nx * sizeof(float));
        *rc = IMG2D_OK;
        return 1;
    }
    return 0;
}

static int run_dense(int ns, int nextrap, int nz, int nx, int nf, int nt, int M, const cpx *opF,
                     const cpx *opB, cpx *wave, cpx *shot, float *image, int write_back)
{
    int rc;
    if (degenerate_call(ns, nextrap, nz, nx, nf, image, &rc)) return rc;
    if ((rc = check_device())) return rc;
    if (!opF || !opB || !wave || !shot || !image) return fail(IMG2D_EINVAL, "null pointer argument");
    img2d_plan plan;
    if ((rc = build_plan(&plan, ns, nextrap, nz, nx, nf, nt, M, 1, nullptr, nullptr, 0, OP_DENSE))) return rc;
    Scratch sc;
    const size_t L = 2 * (size_t)M + 1;
    const size_t tab = (size_t)nextrap * nf * nx * L;
    const size_t wel = (size_t)ns * nt * nx;
    const size_t plane = (size_t)nz * nx;
    cpx *dF, *dB, *dW, *dS;
    float *dI;
    if ((rc = sc.alloc(&dF, tab * sizeof(cpx)))) return rc;
    if ((rc = sc.alloc(&dB, tab * sizeof(cpx)))) return rc;
    if ((rc = sc.alloc(&dW, wel * sizeof(cpx)))) return rc;
    if ((rc = sc.alloc(&dS, wel * sizeof(cpx)))) return rc;
    if ((rc = sc.alloc(&dI, (size_t)ns * plane * sizeof(float)))) return rc;
    IMG2D_CUDA(cudaMemcpy(dF, opF, tab * sizeof(cpx), cudaMemcpyHostToDevice));
    IMG2D_CUDA(cudaMemcpy(dB, opB, tab * sizeof(cpx), cudaMemcpyHostToDevice));
    IMG2D_CUDA(cudaMemcpy(dW, wave, wel * sizeof(cpx), cudaMemcpyHostToDevice));
    IMG2D_CUDA(cudaMemcpy(dS, shot, wel * sizeof(cpx), cudaMemcpyHostToDevice));
    MigrateArgs a = base_args(&plan, dW, dS);
    a.denseF = dF;
    a.denseB = dB;
    if ((rc = launch(&plan, a, nullptr, dI, (long long)plane, 0))) return rc;
    IMG2D_CUDA(cudaDeviceSynchronize());
    // rows [0, nextrap) of every shot image
    IMG2D_CUDA(cudaMemcpy2D(image, plane * sizeof(float), dI, plane * sizeof(float),
                            (size_t)nextrap * nx * sizeof(float), ns, cudaMemcpyDeviceToHost));
    if (write_back) {
        // only the first nf rows of every (nt, nx) shot block carry data
        IMG2D_CUDA(cudaMemcpy2D(wave, (size_t)nt * nx * sizeof(cpx), dW, (size_t)nt * nx * sizeof(cpx),
                                (size_t)nf * nx * sizeof(cpx), ns, cudaMemcpyDeviceToHost));
        IMG2D_CUDA(cudaMemcpy2D(shot, (size_t)nt * nx * sizeof(cpx), dS, (size_t)nt * nx * sizeof(cpx),
                                (size_t)nf * nx * sizeof(cpx), ns, cudaMemcpyDeviceToHost));
    }
    return IMG2D_OK;
}

// Per device: one cached plan for the host compact entry point, reused while the geometry is
// unchanged, and its device buffers, kept between calls (grown on demand) so a call allocates
// nothing when the sizes repeat.  Everything in an entry belongs to that device and is only used
// (and freed) while it is the current device.
struct HostEntryBuffers {
    DevBuf omega, vel, tabF, tabB, wave, shot, image, image_shots;
    // frequency-chunked path: items per chunk, the two queue counters and two status words, its
    // streams (copies in, copies out, two for the kernels); its two sets of per-CTA image partials
    // are the plan's partial buffers, grown to twice the single-launch size
    DevBuf chunk_items, pipe_counter;
    unsigned long long chunk_plan = 0;       // uid of the plan and chunk count chunk_items was built for
    int chunks = 0;
    std::vector<int> chunk_first;            // first item of each chunk, chunks + 1 entries
    cudaStream_t st[4] = {nullptr, nullptr, nullptr, nullptr};
    std::vector<cudaEvent_t> ev;
    ~HostEntryBuffers()
    {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
        for (cudaStream_t x : st)
            if (x) cudaStreamDestroy(x);
    }
};

// img2d_migrate_compact in C frequency chunks.  Each chunk's spectra go to the device, its items
// run as one persistent launch and its final wavefields come back, on separate streams, so the
// copies of one chunk overlap the kernels of the others.  The launches alternate between two
// streams, each with its own work-queue counter and its own set of per-CTA image partials: a
// launch's clusters start on the SMs that the previous launch's last items leave free, and the two
// partial sets are summed once at the end.  Each launch is issued before the wavefields of the
// previous chunk are copied back, so the GPU has queued work while a pageable copy holds the host.
// The kernels and the per-item arithmetic are those of a single launch.
static int migrate_chunked(img2d_plan *p, HostEntryBuffers &hb, int C, img2d_c64 *wave_fs, img2d_c64 *shot_fs,
                           cpx *dW, cpx *dS, float *dI)
{
    int rc;
    const int nf = p->nf;
    const size_t plane = (size_t)p->nextrap * p->nx;
    auto fbegin = [&](int c) { return (int)((long long)c * nf / C); };
    if (hb.chunk_plan != p->uid || hb.chunks != C) {
        // within a chunk, widest groups first (the short items end the launch)
        std::vector<int2> items;
        hb.chunk_first.assign(1, 0);
        for (int c = 0; c < C; ++c) {
            for (int g : p->group_order)
                for (int j = fbegin(c); j < fbegin(c + 1); ++j) items.push_back(make_int2(g, j));
            hb.chunk_first.push_back((int)items.size());
        }
        if ((rc = hb.chunk_items.ensure(items.size() * sizeof(int2)))) return rc;
        IMG2D_CUDA(cudaMemcpy(hb.chunk_items.p, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice));
        hb.chunk_plan = p->uid;
        hb.chunks = C;
    }
    const size_t set_bytes = (size_t)p->grid * plane * sizeof(float);
    if ((rc = p->partial.ensure(2 * set_bytes))) return rc;
    if ((rc = p->comp.ensure(2 * set_bytes))) return rc;
    if ((rc = hb.pipe_counter.ensure(4 * sizeof(int)))) return rc;
    for (cudaStream_t &x : hb.st)
        if (!x) IMG2D_CUDA(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
    while ((int)hb.ev.size() < 2 * C + 1) {
        cudaEvent_t e;
        IMG2D_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        hb.ev.push_back(e);
    }
    cudaStream_t sin = hb.st[0], sout = hb.st[1], sk[2] = {hb.st[2], hb.st[3]};
    int *cnt = hb.pipe_counter.as<int>();
    float *part = p->partial.as<float>(), *comp = p->comp.as<float>();
    // zeroed partial sets, counters and status words before the first launch of either stream
    IMG2D_CUDA(cudaMemsetAsync(part, 0, 2 * set_bytes, sk[0]));
    IMG2D_CUDA(cudaMemsetAsync(comp, 0, 2 * set_bytes, sk[0]));
    IMG2D_CUDA(cudaMemsetAsync(cnt, 0, 4 * sizeof(int), sk[0]));
    IMG2D_CUDA(cudaEventRecord(hb.ev[2 * C], sk[0]));
    IMG2D_CUDA(cudaStreamWaitEvent(sk[1], hb.ev[2 * C], 0));
    auto copy_rows = [&](int c, bool in) -> int {
        const int f0 = fbegin(c), f1 = fbegin(c + 1);
        for (int s = 0; s < p->ns; ++s) {
            const long long off = p->off[s] + (long long)f0 * p->w[s];
            const size_t bytes = (size_t)(f1 - f0) * p->w[s] * sizeof(cpx);
            if (in) {
                IMG2D_CUDA(cudaMemcpyAsync(dW + off, wave_fs + off, bytes, cudaMemcpyHostToDevice, sin));
                IMG2D_CUDA(cudaMemcpyAsync(dS + off, shot_fs + off, bytes, cudaMemcpyHostToDevice, sin));
            } else {
                IMG2D_CUDA(cudaMemcpyAsync(wave_fs + off, dW + off, bytes, cudaMemcpyDeviceToHost, sout));
                IMG2D_CUDA(cudaMemcpyAsync(shot_fs + off, dS + off, bytes, cudaMemcpyDeviceToHost, sout));
            }
        }
        return IMG2D_OK;
    };
    const int K = std::max(1, p->cluster);
    for (int c = 0; c < C; ++c) {
        if ((rc = copy_rows(c, true))) return rc;
        IMG2D_CUDA(cudaEventRecord(hb.ev[2 * c], sin));
        cudaStream_t st = sk[c & 1];
        IMG2D_CUDA(cudaStreamWaitEvent(st, hb.ev[2 * c], 0));
        if (c >= 2) IMG2D_CUDA(cudaMemsetAsync(cnt + (c & 1), 0, sizeof(int), st));  // after launch c - 2
        MigrateArgs a = base_args(p, dW, dS);
        const int n = hb.chunk_first[c + 1] - hb.chunk_first[c];
        a.items = hb.chunk_items.as<int2>() + hb.chunk_first[c];
        a.n_items = n;
        a.counter = cnt + (c & 1);
        a.status = cnt + 2 + (c & 1);
        a.partial = dI ? part + (size_t)(c & 1) * p->grid * plane : nullptr;
        a.comp = dI ? comp + (size_t)(c & 1) * p->grid * plane : nullptr;
        if ((rc = launch_kernel(p, a, std::min(n, p->grid / K) * K, st))) return rc;
        IMG2D_CUDA(cudaEventRecord(hb.ev[2 * c + 1], st));
        if (c >= 1) {
            IMG2D_CUDA(cudaStreamWaitEvent(sout, hb.ev[2 * c - 1], 0));
            if ((rc = copy_rows(c - 1, false))) return rc;
        }
    }
    IMG2D_CUDA(cudaStreamWaitEvent(sout, hb.ev[2 * C - 1], 0));
    if ((rc = copy_rows(C - 1, false))) return rc;
    if (dI) {
        IMG2D_CUDA(cudaStreamWaitEvent(sk[0], hb.ev[2 * C - 1], 0));
        if (C >= 2) IMG2D_CUDA(cudaStreamWaitEvent(sk[0], hb.ev[2 * C - 3], 0));
        const int blocks = (int)std::min<size_t>((plane + 255) / 256, 148 * 8);
        reduce_partials_kernel<<<blocks, 256, 0, sk[0]>>>(part, comp, 2 * p->grid, (long long)plane, dI);
        IMG2D_CUDA(cudaGetLastError());
    }
    for (cudaStream_t x : hb.st) IMG2D_CUDA(cudaStreamSynchronize(x));
    int status[2] = {0, 0};
    IMG2D_CUDA(cudaMemcpy(status, cnt + 2, sizeof(status), cudaMemcpyDeviceToHost));
    if (status[0] || status[1])
        return fail(IMG2D_ECUDA, "a bounded wait in the migration kernel gave up: the results of that call are not valid");
    return IMG2D_OK;
}
struct HostCache {
    img2d_plan *plan = nullptr;
    std::vector<int> key;
    HostEntryBuffers *bufs = nullptr;
};
static std::mutex g_cache_mu;
static std::map<int, HostCache> g_host_cache;

}  // namespace img2d

// ---------------------------------------------------------------------------------------
// Fixed scratch for img2d_migrate_compact_noalloc.  A file-scope device array: every GPU that
// loads this library holds it (IMG2D_NOALLOC_SCRATCH_BYTES) until the process exits.  In host code
// the name g_noalloc_scratch is only a stand-in for the symbol, not a device address, so the
// address is looked up once per device with cudaGetSymbolAddress while that device is current.
// ---------------------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_noalloc_scratch[IMG2D_NOALLOC_SCRATCH_BYTES];

namespace img2d {

static std::mutex g_noalloc_mu;
static void *g_noalloc_addr[256];

static int noalloc_scratch(void **out)
{
    int dev = 0;
    IMG2D_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) return fail(IMG2D_EINVAL, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void *addr = nullptr;
        IMG2D_CUDA(cudaGetSymbolAddress(&addr, g_noalloc_scratch));
        g_noalloc_addr[dev] = addr;
    }
    *out = g_noalloc_addr[dev];
    return IMG2D_OK;
}

}  // namespace img2d

using namespace img2d;

extern "C" {

const char *img2d_last_error(void) { return g_err.c_str(); }

void img2d_set_alloc_limit(size_t max_bytes)
{
    std::lock_guard<std::mutex> lock(g_alloc_mu);
    g_alloc_limit = max_bytes;
    g_alloc_limit_set = true;
}

int img2d_version(void) { return 10000; }

int img2d_extrapolate_host_order(int ns, int nextrap, int nz, int nx, int nf, int nt, int M,
                                 const img2d_c64 *op_forw, const img2d_c64 *op_back,
                                 img2d_c64 *wave_fs, img2d_c64 *shot_fs, float *image)
{
    return run_dense(ns, nextrap, nz, nx, nf, nt, M, (const cpx *)op_forw, (const cpx *)op_back,
                     (cpx *)wave_fs, (cpx *)shot_fs, image, 1);
}

int img2d_extrapolate_device_order(int ns, int nextrap, int nz, int nt, int nf, int nx, int M,
                                   const img2d_c64 *op_forw, img2d_c64 *forw_pulse,
                                   const img2d_c64 *op_back, img2d_c64 *back_pulse, float *image,
                                   int write_back)
{
    return run_dense(ns, nextrap, nz, nx, nf, nt, M, (const cpx *)op_forw, (const cpx *)op_back,
                     (cpx *)forw_pulse, (cpx *)back_pulse, image, write_back);
}

int img2d_plan_create(img2d_plan **plan, int ns, int nextrap, int nz, int nx, int nf, int nt, int M,
                      int nk, const int *shot_x0, const int *shot_nx, int flags)
{
    if (!plan) return fail(IMG2D_EINVAL, "plan pointer is NULL");
    *plan = nullptr;
    int rc;
    if ((rc = check_device())) return rc;
    img2d_plan *p = new img2d_plan();
    const int mode = (flags & IMG2D_FLAG_TWO_TABLES) ? OP_TWO : OP_CONJ;
    if ((rc = build_plan(p, ns, nextrap, nz, nx, nf, nt, M, nk, shot_x0, shot_nx, flags, mode))) {
        delete p;
        return rc;
    }
    *plan = p;
    return IMG2D_OK;
}

int img2d_plan_set_model(img2d_plan *p, const double *d_omega, const double *d_velocity, double dk,
                         const img2d_c64 *d_tab_forw, const img2d_c64 *d_tab_back, void *stream)
{
    if (!p) return fail(IMG2D_EINVAL, "plan is NULL");
    return set_model(p, d_omega, d_velocity, dk, (const cpx *)d_tab_forw, (const cpx *)d_tab_back,
                     (cudaStream_t)stream);
}

int img2d_plan_execute(img2d_plan *p, img2d_c64 *d_wave, img2d_c64 *d_shot, float *d_image,
                       float *d_image_shots, void *stream)
{
    if (!p) return fail(IMG2D_EINVAL, "plan is NULL");
    if (!d_wave || !d_shot) return fail(IMG2D_EINVAL, "wavefield pointers are NULL");
    MigrateArgs a = base_args(p, (cpx *)d_wave, (cpx *)d_shot);
    return launch(p, a, d_image, d_image_shots, (long long)p->nz * p->nx, (cudaStream_t)stream);
}

int img2d_plan_demigrate(img2d_plan *p, const float *d_refl, const img2d_c64 *d_wave, img2d_c64 *d_data,
                         int slab_depth, int source_mode, void *stream)
{
    if (!p) return fail(IMG2D_EINVAL, "plan is NULL");
    if (!d_refl || !d_wave || !d_data) return fail(IMG2D_EINVAL, "null device pointer");
    if ((const void *)d_wave == (const void *)d_data) return fail(IMG2D_EINVAL, "data must not alias wave");
    if (p->mode != OP_CONJ) return fail(IMG2D_EINVAL, "demigration supports the single-table mode only");
    if (source_mode < IMG2D_SOURCE_RECOMPUTE || source_mode > IMG2D_SOURCE_REUSE)
        return fail(IMG2D_EINVAL, "source_mode must be IMG2D_SOURCE_RECOMPUTE, _KEEP or _REUSE");
    int rc;
    if ((rc = demig_prepare(p, slab_depth))) return rc;
    if (source_mode == IMG2D_SOURCE_REUSE && !p->adj_cache_valid)
        return fail(IMG2D_EINVAL, "no kept source checkpoints on this plan (call with IMG2D_SOURCE_KEEP first, "
                                  "after the last set_model, with the same slab depth)");
    const long long cache_elems = (long long)p->adj_items_n * p->adj_cache_item;  // float2
    if (source_mode == IMG2D_SOURCE_KEEP) {
        if ((rc = p->adj_cache.ensure((size_t)cache_elems * sizeof(float2)))) return rc;
    }
    cudaStream_t st = (cudaStream_t)stream;
    DemigrateArgs a{};
    a.nextrap = p->nextrap;
    a.nx = p->nx;
    a.M = p->M;
    a.tab_stride = p->tab_stride;
    a.n_items = p->adj_items_n;
    a.slab = p->adj_slab;
    a.nslab = p->adj_nslab;
    a.items = p->adj_items.as<int2>();
    a.groups = p->adj_groups.as<GroupDesc>();
    a.segs = p->adj_segs.as<int4>();
    a.owner = p->adj_owner.as<int16_t>();
    a.shot_off = p->shot_off.as<long long>();
    a.tab = p->tabF.as<cpx>();
    a.idx = p->idx.as<uint16_t>();
    a.idx_jstride = (long long)p->nextrap * p->idx_lstride;
    a.idx_lstride = p->idx_lstride;
    a.wave = (const cpx *)d_wave;
    a.refl = d_refl;
    a.data = (cpx *)d_data;
    a.work = p->adj_work.as<float2>();
    a.work_cta = p->adj_work_cta;
    a.wmax = p->adj_wmax;
    a.counter = p->adj_counter.as<int>();
    a.ckpt_mode = source_mode;
    a.ckpt_items = source_mode == IMG2D_SOURCE_RECOMPUTE ? nullptr : p->adj_cache.as<float2>();
    IMG2D_CUDA(cudaMemsetAsync(p->adj_counter.p, 0, sizeof(int), st));
    if (p->timing && !p->ev0) {
        IMG2D_CUDA(cudaEventCreate(&p->ev0));
        IMG2D_CUDA(cudaEventCreate(&p->ev1));
    }
    if (p->timing) IMG2D_CUDA(cudaEventRecord(p->ev0, st));
    if (p->adj_cluster) {
        cudaLaunchConfig_t cfg{};
        cudaLaunchAttribute attr{};
        attr.id = cudaLaunchAttributeClusterDimension;
        attr.val.clusterDim.x = p->adj_cluster;
        attr.val.clusterDim.y = 1;
        attr.val.clusterDim.z = 1;
        cfg.gridDim = dim3(p->adj_grid, 1, 1);
        cfg.blockDim = dim3(p->adj_block, 1, 1);
        cfg.dynamicSmemBytes = p->adj_smem;
        cfg.stream = st;
        cfg.attrs = &attr;
        cfg.numAttrs = 1;
        IMG2D_CUDA(cudaLaunchKernelEx(&cfg, p->adj_fn, a));
    } else {
        p->adj_fn<<<p->adj_grid, p->adj_block, p->adj_smem, st>>>(a);
    }
    IMG2D_CUDA(cudaGetLastError());
    if (p->timing) {
        IMG2D_CUDA(cudaEventRecord(p->ev1, st));
        p->ev_recorded = true;
    }
    if (source_mode == IMG2D_SOURCE_KEEP) p->adj_cache_valid = true;
    return IMG2D_OK;
}

int img2d_plan_describe_demigration(const img2d_plan *p, char *buf, int buflen)
{
    if (!p || !buf || buflen <= 0) return fail(IMG2D_EINVAL, "bad describe arguments");
    if (!p->adj_fn) return fail(IMG2D_EINVAL, "no demigration has run on this plan yet");
    snprintf(buf, buflen,
             "{\"kernel\": \"%s\", \"cluster\": %d, \"G\": %d, \"X\": 8, \"L\": %d, \"grid\": %d, \"block\": %d, "
             "\"smem\": %zu, \"items\": %d, \"max_union_width\": %d, \"slab\": %d, \"slabs\": %d, "
             "\"workspace_bytes\": %zu, \"source_cache_bytes\": %zu, \"ring\": %s}",
             p->adj_cluster ? "demigrate_cluster" : "demigrate", p->adj_cluster, p->adj_G, p->L, p->adj_grid,
             p->adj_block, p->adj_smem, p->adj_items_n, p->adj_wmax, p->adj_slab,
             p->adj_nslab, p->adj_work.bytes, p->adj_cache.bytes, p->adj_ring ? "true" : "false");
    return IMG2D_OK;
}

int img2d_plan_dense_table(const img2d_plan *p, int which, img2d_c64 *d_dense, void *stream)
{
    if (!p) return fail(IMG2D_EINVAL, "plan is NULL");
    if (!d_dense) return fail(IMG2D_EINVAL, "d_dense is NULL");
    if (which != 0 && which != 1) return fail(IMG2D_EINVAL, "which must be 0 (forward) or 1 (receiver)");
    if (p->mode == OP_DENSE) return fail(IMG2D_EINVAL, "a dense-table plan has no compact table");
    if (!p->model_set) return fail(IMG2D_EINVAL, "call img2d_plan_set_model first");
    if ((long long)p->nx * p->L >= (1ll << 31) || (long long)p->nextrap * p->nf >= (1ll << 31))
        return fail(IMG2D_EINVAL, "dense table rows too large");
    const bool back_rows = which == 1 && p->mode == OP_TWO;
    const cpx *tab = back_rows ? p->tabB.as<cpx>() : p->tabF.as<cpx>();
    const int conj = which == 1 && !back_rows;
    cudaStream_t st = (cudaStream_t)stream;
    dense_table_kernel<<<p->nextrap * p->nf, 256, 0, st>>>(p->idx.as<uint16_t>(), p->nf, p->nextrap, p->nx,
                                                          p->idx_lstride, tab, p->tab_stride, p->L, conj,
                                                          (cpx *)d_dense);
    IMG2D_CUDA(cudaGetLastError());
    return IMG2D_OK;
}

long long img2d_plan_shot_offset(const img2d_plan *p, int s)
{
    if (!p || s < 0 || s >= p->ns) return -1;
    return p->off[s];
}

long long img2d_plan_wavefield_elems(const img2d_plan *p) { return p ? p->wave_elems : -1; }

size_t img2d_plan_workspace_bytes(const img2d_plan *p)
{
    if (!p) return 0;
    return p->items.bytes + p->groups.bytes + p->segs.bytes + p->owner.bytes + p->shot_off.bytes +
           p->idx.bytes + p->tabF.bytes + p->tabB.bytes + p->tab16buf.bytes + p->partial.bytes + p->comp.bytes + p->counter.bytes +
           p->naive_buf.bytes + p->adj_items.bytes + p->adj_groups.bytes + p->adj_segs.bytes + p->adj_owner.bytes +
           p->adj_work.bytes + p->adj_counter.bytes + p->adj_cache.bytes;
}

int img2d_plan_describe(const img2d_plan *p, char *buf, int buflen)
{
    if (!p || !buf || buflen <= 0) return fail(IMG2D_EINVAL, "bad describe arguments");
    snprintf(buf, buflen,
             "{\"kernel\": \"%s\", \"cluster\": %d, \"G\": %d, \"X\": %d, \"L\": %d, \"grid\": %d, \"block\": %d, "
             "\"smem\": %zu, \"items\": %d, \"slots\": %d, \"max_union_width\": %d, \"mode\": %d, \"variant\": %d, "
             "\"table\": \"%s\", \"packing\": \"%s\", \"cost_units\": %.3f, \"computed_per_useful\": %.4f}",
             p->kname, p->cluster, p->G, p->fixed ? kX : 4, p->L, p->grid, p->block, p->smem,
             p->n_items, p->n_slots, p->max_w, p->mode, p->variant,
             p->tab16 == 2 ? "bf16" : (p->tab16 == 1 ? "fp16" : "fp32"), p->packing, p->pack_cost,
             p->computed_per_useful);
    return IMG2D_OK;
}

void img2d_plan_destroy(img2d_plan *p) { delete p; }

int img2d_plan_kernel_ms(img2d_plan *p, float *ms)
{
    if (!p || !ms) return fail(IMG2D_EINVAL, "bad arguments");
    if (!p->ev_recorded) return fail(IMG2D_EINVAL, "no kernel launched on this plan yet");
    IMG2D_CUDA(cudaEventSynchronize(p->ev1));
    IMG2D_CUDA(cudaEventElapsedTime(ms, p->ev0, p->ev1));
    return IMG2D_OK;
}

int img2d_pack_shots(int ns, int nx, int M, const int *shot_x0, const int *shot_nx, int windows, int K,
                     int *group_of_shot, int *slot_of_shot, int *group_u0, int *group_w, int *n_groups,
                     double *cost_units)
{
    if (ns <= 0 || nx <= 0 || M < 0 || !shot_x0 || !shot_nx || !group_of_shot || !slot_of_shot || !n_groups)
        return fail(IMG2D_EINVAL, "img2d_pack_shots: invalid arguments");
    if (ns > 32767) return fail(IMG2D_EINVAL, "at most 32767 shots");
    img2d_plan pl;
    pl.ns = ns;
    pl.nx = nx;
    pl.M = M;
    pl.x0.assign(shot_x0, shot_x0 + ns);
    pl.w.assign(shot_nx, shot_nx + ns);
    int wmax = 0;
    for (int s = 0; s < ns; ++s) {
        if (pl.x0[s] < 0 || pl.w[s] <= 0 || pl.x0[s] + pl.w[s] > nx)
            return fail(IMG2D_EINVAL, "shot " + std::to_string(s) + " aperture outside [0, nx)");
        wmax = std::max(wmax, pl.w[s]);
    }
    const int Kmin = (wmax + WideShape::PC - 1) / WideShape::PC;
    std::vector<GroupDesc> groups;
    std::vector<int4> segs;
    std::vector<int16_t> owner;
    double cost = 0.0;
    if (windows) {
        if (K < Kmin) return fail(IMG2D_EINVAL, "K too small for the widest shot");
        cost = pack_windows_best(&pl, WideShape::G, K, groups, segs, owner);
        if (cost < 0.0) return fail(IMG2D_EINVAL, "a shot fits no window");
    } else {
        colour_slots(&pl);
        const int widest = pack_groups(&pl, WideShape::G, groups, segs, owner);
        if (K <= 0) K = (widest + WideShape::PC - 1) / WideShape::PC;
        if (K * WideShape::PC < widest) return fail(IMG2D_EINVAL, "K too small for the widest group");
        for (const GroupDesc &g : groups) cost += wide_item_cost(g.W, K);
    }
    for (size_t g = 0; g < groups.size(); ++g) {
        if (group_u0) group_u0[g] = groups[g].u0;
        if (group_w) group_w[g] = groups[g].W;
        for (int k = groups[g].seg_begin; k < groups[g].seg_begin + groups[g].nseg; ++k) {
            group_of_shot[segs[k].x] = (int)g;
            slot_of_shot[segs[k].x] = segs[k].y;
        }
    }
    *n_groups = (int)groups.size();
    if (cost_units) *cost_units = cost;
    return IMG2D_OK;
}

int img2d_plan_status(img2d_plan *p, void *stream)
{
    if (!p) return fail(IMG2D_EINVAL, "plan is NULL");
    if (!p->launched) return fail(IMG2D_EINVAL, "no kernel launched on this plan yet");
    return img2d::read_status(p, (cudaStream_t)stream);
}

int img2d_measure_fp32_peak(double *tflops)
{
    if (!tflops) return fail(IMG2D_EINVAL, "tflops is NULL");
    int rc;
    if ((rc = check_device())) return rc;
    int dev = 0, nsm = 0;
    IMG2D_CUDA(cudaGetDevice(&dev));
    IMG2D_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    Scratch sc;
    float *out;
    const int blocks = nsm * 4, threads = 512, iters = 4096;
    if ((rc = sc.alloc(&out, (size_t)blocks * threads * sizeof(float)))) return rc;
    fma_probe_kernel<<<blocks, threads>>>(out, 64);
    IMG2D_CUDA(cudaGetLastError());
    cudaEvent_t e0, e1;
    IMG2D_CUDA(cudaEventCreate(&e0));
    IMG2D_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    for (int r = 0; r < 3; ++r) {
        cudaEventRecord(e0);
        fma_probe_kernel<<<blocks, threads>>>(out, iters);
        cudaEventRecord(e1);
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return fail(IMG2D_ECUDA, std::string("fma probe: ") + cudaGetErrorString(e));
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        best = std::min(best, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // 16 chains x 8 FMAs per iteration per thread, 2 flops per FMA
    *tflops = 2.0 * 128.0 * iters * (double)blocks * threads / (best * 1e-3) * 1e-12;
    return IMG2D_OK;
}

int img2d_ricker_sources(int ns, int nt, int nx, double dt, double x_first, double dx, double depth_offset,
                         double v, double fpeak, const double *src_x, float *d_out, void *stream)
{
    int rc;
    if ((rc = check_device())) return rc;
    if (ns <= 0 || nt <= 0 || nx <= 0 || !(dt > 0.0) || !(dx > 0.0) || !(v > 0.0))
        return fail(IMG2D_EINVAL, "invalid source-wavelet dimensions or spacing");
    if (!src_x || !d_out) return fail(IMG2D_EINVAL, "null pointer argument");
    cudaStream_t st = (cudaStream_t)stream;
    Scratch sc;
    double *d_sx;
    if ((rc = sc.alloc(&d_sx, (size_t)ns * sizeof(double)))) return rc;
    IMG2D_CUDA(cudaMemcpyAsync(d_sx, src_x, (size_t)ns * sizeof(double), cudaMemcpyHostToDevice, st));
    const long long total = (long long)ns * nt * nx;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 32);
    ricker_sources_kernel<<<blocks, 256, 0, st>>>(ns, nt, nx, dt, x_first, dx, depth_offset, v, fpeak, d_sx, d_out);
    IMG2D_CUDA(cudaGetLastError());
    IMG2D_CUDA(cudaStreamSynchronize(st));  // the source positions are freed on return
    return IMG2D_OK;
}

int img2d_records_to_spectra(int ns, int nt, int nx, int nf, int nt_rows, const float *d_records,
                             const int *shot_x0, const int *shot_nx, img2d_c64 *d_out, void *stream)
{
    int rc;
    if ((rc = check_device())) return rc;
    if (ns <= 0 || nt <= 0 || nx <= 0 || nf <= 0 || nf > nt || nt_rows < nf)
        return fail(IMG2D_EINVAL, "invalid dimensions (need ns, nt, nx > 0, 0 < nf <= nt, nt_rows >= nf)");
    if (!d_records || !d_out) return fail(IMG2D_EINVAL, "null pointer argument");
    std::vector<int> x0(ns, 0), w(ns, nx);
    std::vector<long long> off(ns, 0);
    long long acc = 0;
    for (int s = 0; s < ns; ++s) {
        if (shot_x0) x0[s] = shot_x0[s];
        if (shot_nx) w[s] = shot_nx[s];
        if (x0[s] < 0 || w[s] <= 0 || x0[s] + w[s] > nx)
            return fail(IMG2D_EINVAL, "shot " + std::to_string(s) + " aperture outside [0, nx)");
        off[s] = acc;
        acc += (long long)nt_rows * w[s];
    }
    cudaStream_t st = (cudaStream_t)stream;
    // shots per transform group: their spectra (nt/2+1 rows) in at most 512 MB of scratch
    const long long shot_spec = (long long)(nt / 2 + 1) * nx;
    const int group = (int)std::max<long long>(1, std::min<long long>(ns, (512ll << 20) / (shot_spec * 8)));
    int dev = 0;
    IMG2D_CUDA(cudaGetDevice(&dev));
    // One plan per (device, nt, nx), kept for the process: the nx transforms of length nt of one
    // shot, element (t, x) at x + t*nx in and at x + j*nx out; shots are issued one by one.  The
    // plans are shared, so the lock is held while this call issues its transforms.
    static std::mutex plan_mu;
    static std::map<std::vector<long long>, cufftHandle> plans;
    std::lock_guard<std::mutex> plan_lock(plan_mu);
    const std::vector<long long> key = {dev, nt, nx};
    auto itp = plans.find(key);
    if (itp == plans.end()) {
        int n[1] = {nt};
        int inembed[1] = {nt}, onembed[1] = {nt / 2 + 1};
        cufftHandle h;
        if (cufftCreate(&h) != CUFFT_SUCCESS) return fail(IMG2D_ECUDA, "cufftCreate failed");
        size_t ws = 0;
        if (cufftMakePlanMany(h, 1, n, inembed, nx, 1, onembed, nx, 1, CUFFT_R2C, nx, &ws) != CUFFT_SUCCESS) {
            cufftDestroy(h);
            return fail(IMG2D_ECUDA, "cufftMakePlanMany (real-to-complex along time) failed");
        }
        itp = plans.emplace(key, h).first;
    }
    const cufftHandle plan = itp->second;
    if (cufftSetStream(plan, st) != CUFFT_SUCCESS) return fail(IMG2D_ECUDA, "cufftSetStream failed");
    // the spectra scratch (up to 512 MB) is kept per device with the plans, grown on demand
    static std::map<int, DevBuf> spec_scratch;
    DevBuf &spec = spec_scratch[dev];
    if ((rc = spec.ensure((size_t)group * shot_spec * sizeof(cpx)))) return rc;
    cpx *d_spec = spec.as<cpx>();
    Scratch sc;
    int *d_x0, *d_w;
    long long *d_off;
    if ((rc = sc.alloc(&d_x0, ns * sizeof(int)))) return rc;
    if ((rc = sc.alloc(&d_w, ns * sizeof(int)))) return rc;
    if ((rc = sc.alloc(&d_off, ns * sizeof(long long)))) return rc;
    IMG2D_CUDA(cudaMemcpyAsync(d_x0, x0.data(), ns * sizeof(int), cudaMemcpyHostToDevice, st));
    IMG2D_CUDA(cudaMemcpyAsync(d_w, w.data(), ns * sizeof(int), cudaMemcpyHostToDevice, st));
    IMG2D_CUDA(cudaMemcpyAsync(d_off, off.data(), ns * sizeof(long long), cudaMemcpyHostToDevice, st));
    for (int s0 = 0; s0 < ns; s0 += group) {
        const int nsc = std::min(group, ns - s0);
        for (int k = 0; k < nsc; ++k) {
            cufftReal *in = const_cast<cufftReal *>(d_records + (long long)(s0 + k) * nt * nx);
            cufftComplex *o = reinterpret_cast<cufftComplex *>(d_spec + (long long)k * shot_spec);
            if (cufftExecR2C(plan, in, o) != CUFFT_SUCCESS) return fail(IMG2D_ECUDA, "cufftExecR2C failed");
        }
        const long long total = (long long)nsc * nf * nx;
        const int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 32);
        pack_spectra_kernel<<<blocks, 256, 0, st>>>(s0, nsc, nt, nx, nf, d_spec, d_x0, d_w, d_off, (cpx *)d_out);
        IMG2D_CUDA(cudaGetLastError());
    }
    IMG2D_CUDA(cudaStreamSynchronize(st));  // the descriptors are freed on return
    return IMG2D_OK;
}

int img2d_measure_l2_bandwidth(double *gbs)
{
    if (!gbs) return fail(IMG2D_EINVAL, "gbs is NULL");
    int rc;
    if ((rc = check_device())) return rc;
    int dev = 0, nsm = 0;
    IMG2D_CUDA(cudaGetDevice(&dev));
    IMG2D_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    Scratch sc;
    const long long bytes = 32ll << 20;  // resident in L2 (126 MB on B200)
    const long long n4 = bytes / 16;
    const int blocks = nsm * 4, threads = 512, iters = 64;
    float4 *buf;
    float *out;
    if ((rc = sc.alloc(&buf, (size_t)bytes))) return rc;
    if ((rc = sc.alloc(&out, (size_t)blocks * threads * sizeof(float)))) return rc;
    IMG2D_CUDA(cudaMemset(buf, 0, (size_t)bytes));
    l2_read_probe_kernel<<<blocks, threads>>>(buf, n4, 2, out);  // warm the lines into L2
    IMG2D_CUDA(cudaGetLastError());
    cudaEvent_t e0, e1;
    IMG2D_CUDA(cudaEventCreate(&e0));
    IMG2D_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    for (int r = 0; r < 3; ++r) {
        cudaEventRecord(e0);
        l2_read_probe_kernel<<<blocks, threads>>>(buf, n4, iters, out);
        cudaEventRecord(e1);
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return fail(IMG2D_ECUDA, std::string("l2 probe: ") + cudaGetErrorString(e));
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        best = std::min(best, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *gbs = (double)bytes * iters / (best * 1e-3) * 1e-9;
    return IMG2D_OK;
}

int img2d_plan_execute_naive(img2d_plan *p, img2d_c64 *d_wave, img2d_c64 *d_shot, float *d_image,
                             void *stream)
{
    if (!p) return fail(IMG2D_EINVAL, "plan is NULL");
    if (p->mode != OP_CONJ) return fail(IMG2D_EINVAL, "naive form supports the single-table mode only");
    if (!d_wave || !d_shot || !d_image) return fail(IMG2D_EINVAL, "null device pointer");
    cudaStream_t st = (cudaStream_t)stream;
    const int M = p->M;
    const int maxw = *std::max_element(p->w.begin(), p->w.end());
    int rc;
    if ((rc = p->naive_buf.ensure(2 * (size_t)(maxw + 2 * M) * sizeof(float4)))) return rc;
    float4 *b0 = p->naive_buf.as<float4>(), *b1 = b0 + (maxw + 2 * M);
    IMG2D_CUDA(cudaMemsetAsync(d_image, 0, (size_t)p->nextrap * p->nx * sizeof(float), st));
    for (int s = 0; s < p->ns; ++s) {
        const int w = p->w[s], x0 = p->x0[s];
        const int blocks = (w + 127) / 128;
        for (int j = 0; j < p->nf; ++j) {
            IMG2D_CUDA(cudaMemsetAsync(b0, 0, 2 * (size_t)(maxw + 2 * M) * sizeof(float4), st));
            cpx *ws = (cpx *)d_wave + p->off[s] + (long long)j * w;
            cpx *rs = (cpx *)d_shot + p->off[s] + (long long)j * w;
            naive_pack_kernel<<<blocks, 128, 0, st>>>(ws, rs, w, M, b0, 1);
            float4 *cur = b0, *nxt = b1;
            for (int l = 0; l < p->nextrap; ++l) {
                const uint16_t *idx_row = p->idx.as<uint16_t>() + ((long long)j * p->nextrap + l) * p->idx_lstride;
                naive_step_kernel<<<blocks, 128, 0, st>>>(cur, nxt, w, M, p->tabF.as<cpx>(), p->tab_stride, idx_row,
                                                          x0, d_image + (long long)l * p->nx);
                std::swap(cur, nxt);
            }
            naive_unpack_kernel<<<blocks, 128, 0, st>>>(cur, w, M, ws, rs);
        }
    }
    IMG2D_CUDA(cudaGetLastError());
    return IMG2D_OK;
}

int img2d_migrate_compact_noalloc(int ns, int nextrap, int nz, int nx, int nf, int nt, int M, int nk, double dk,
                                  const double *d_omega, const double *d_velocity, const img2d_c64 *d_tab_forw,
                                  const int *shot_x0, const int *shot_nx, img2d_c64 *d_wave, img2d_c64 *d_shot,
                                  float *d_image, void *stream)
{
    int rc;
    if ((rc = check_device())) return rc;
    if (!d_omega || !d_velocity || !d_tab_forw || !d_wave || !d_shot || !d_image)
        return fail(IMG2D_EINVAL, "null pointer argument");
    void *base = nullptr;
    if ((rc = noalloc_scratch(&base))) return rc;
    Carver carver;
    carver.base = static_cast<unsigned char *>(base);
    carver.cap = IMG2D_NOALLOC_SCRATCH_BYTES;
    img2d_plan plan;
    plan.carver = &carver;
    plan.upload_stream = (cudaStream_t)stream;
    plan.timing = false;
    for (DevBuf *b : {&plan.items, &plan.groups, &plan.segs, &plan.owner, &plan.shot_off, &plan.idx, &plan.tabF,
                      &plan.tabB, &plan.tab16buf, &plan.partial, &plan.comp, &plan.counter, &plan.naive_buf})
        b->carver = &carver;
    if ((rc = build_plan(&plan, ns, nextrap, nz, nx, nf, nt, M, nk, shot_x0, shot_nx, IMG2D_FLAG_NO_CLUSTER, OP_CONJ)))
        return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if ((rc = set_model(&plan, d_omega, d_velocity, dk, (const cpx *)d_tab_forw, nullptr, st))) return rc;
    MigrateArgs a = base_args(&plan, (cpx *)d_wave, (cpx *)d_shot);
    return launch(&plan, a, d_image, nullptr, 0, st);
}

void img2d_release_host_cache(void)
{
    std::lock_guard<std::mutex> lock(g_cache_mu);
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) {
        cudaGetLastError();
        cur = -1;
    }
    for (auto &kv : g_host_cache) {
        // free each device's plan and buffers with that device current
        if (cudaSetDevice(kv.first) != cudaSuccess) cudaGetLastError();
        delete kv.second.plan;
        delete kv.second.bufs;
    }
    g_host_cache.clear();
    if (cur >= 0 && cudaSetDevice(cur) != cudaSuccess) cudaGetLastError();
}

int img2d_host_cache_device_count(void)
{
    std::lock_guard<std::mutex> lock(g_cache_mu);
    return (int)g_host_cache.size();
}

int img2d_migrate_compact(int ns, int nextrap, int nz, int nx, int nf, int nt, int M, int nk, double dk,
                          const double *omega, const double *velocity, const img2d_c64 *tab_forw,
                          const img2d_c64 *tab_back, const int *shot_x0, const int *shot_nx,
                          img2d_c64 *wave_fs, img2d_c64 *shot_fs, float *image, float *image_shots, int flags)
{
    int rc;
    if ((rc = check_device())) return rc;
    if (!omega || !velocity || !tab_forw || !wave_fs || !shot_fs)
        return fail(IMG2D_EINVAL, "null pointer argument");
    if ((flags & IMG2D_FLAG_TWO_TABLES) && !tab_back) return fail(IMG2D_EINVAL, "two-table mode needs tab_back");
    std::lock_guard<std::mutex> lock(g_cache_mu);
    int dev = 0;
    IMG2D_CUDA(cudaGetDevice(&dev));
    HostCache &hc = g_host_cache[dev];
    std::vector<int> key = {ns, nextrap, nz, nx, nf, nt, M, nk, flags};
    for (int s = 0; s < ns; ++s) {
        key.push_back(shot_x0 ? shot_x0[s] : 0);
        key.push_back(shot_nx ? shot_nx[s] : nx);
    }
    if (!hc.plan || key != hc.key) {
        delete hc.plan;
        hc.plan = nullptr;
        hc.key.clear();
        img2d_plan *p = nullptr;
        if ((rc = img2d_plan_create(&p, ns, nextrap, nz, nx, nf, nt, M, nk, shot_x0, shot_nx, flags))) return rc;
        hc.plan = p;
        hc.key = key;
    }
    img2d_plan *p = hc.plan;
    if (!hc.bufs) hc.bufs = new HostEntryBuffers();
    HostEntryBuffers &hb = *hc.bufs;
    const size_t L = 2 * (size_t)M + 1;
    const size_t plane = (size_t)nz * nx;
    if ((rc = hb.omega.ensure(nf * sizeof(double)))) return rc;
    if ((rc = hb.vel.ensure((size_t)nextrap * nx * sizeof(double)))) return rc;
    if ((rc = hb.tabF.ensure(nk * L * sizeof(cpx)))) return rc;
    if ((flags & IMG2D_FLAG_TWO_TABLES) && (rc = hb.tabB.ensure(nk * L * sizeof(cpx)))) return rc;
    if ((rc = hb.wave.ensure(p->wave_elems * sizeof(cpx)))) return rc;
    if ((rc = hb.shot.ensure(p->wave_elems * sizeof(cpx)))) return rc;
    if (image && (rc = hb.image.ensure((size_t)nextrap * nx * sizeof(float)))) return rc;
    if (image_shots && (rc = hb.image_shots.ensure((size_t)ns * plane * sizeof(float)))) return rc;
    double *dO = hb.omega.as<double>(), *dV = hb.vel.as<double>();
    cpx *dTF = hb.tabF.as<cpx>(), *dTB = (flags & IMG2D_FLAG_TWO_TABLES) ? hb.tabB.as<cpx>() : nullptr;
    cpx *dW = hb.wave.as<cpx>(), *dS = hb.shot.as<cpx>();
    float *dI = image ? hb.image.as<float>() : nullptr, *dIS = image_shots ? hb.image_shots.as<float>() : nullptr;
    IMG2D_CUDA(cudaMemcpy(dO, omega, nf * sizeof(double), cudaMemcpyHostToDevice));
    IMG2D_CUDA(cudaMemcpy(dV, velocity, (size_t)nextrap * nx * sizeof(double), cudaMemcpyHostToDevice));
    IMG2D_CUDA(cudaMemcpy(dTF, tab_forw, nk * L * sizeof(cpx), cudaMemcpyHostToDevice));
    if (dTB) IMG2D_CUDA(cudaMemcpy(dTB, tab_back, nk * L * sizeof(cpx), cudaMemcpyHostToDevice));
    // large wavefields: frequency chunks whose copies overlap the other chunks' kernels
    const int chunks = std::min(8, nf);
    if (!image_shots && chunks >= 2 && p->wave_elems * sizeof(cpx) >= ((size_t)64 << 20)) {
        if ((rc = set_model(p, dO, dV, dk, dTF, dTB, 0))) return rc;
        IMG2D_CUDA(cudaDeviceSynchronize());
        if ((rc = migrate_chunked(p, hb, chunks, wave_fs, shot_fs, dW, dS, dI))) {
            // leave no queued work behind on the error path
            for (cudaStream_t x : hb.st)
                if (x && cudaStreamSynchronize(x) != cudaSuccess) cudaGetLastError();
            return rc;
        }
        if (image) IMG2D_CUDA(cudaMemcpy(image, dI, (size_t)nextrap * nx * sizeof(float), cudaMemcpyDeviceToHost));
        return IMG2D_OK;
    }
    IMG2D_CUDA(cudaMemcpy(dW, wave_fs, p->wave_elems * sizeof(cpx), cudaMemcpyHostToDevice));
    IMG2D_CUDA(cudaMemcpy(dS, shot_fs, p->wave_elems * sizeof(cpx), cudaMemcpyHostToDevice));
    if ((rc = set_model(p, dO, dV, dk, dTF, dTB, 0))) return rc;
    MigrateArgs a = base_args(p, dW, dS);
    if ((rc = launch(p, a, dI, dIS, (long long)plane, 0))) return rc;
    IMG2D_CUDA(cudaDeviceSynchronize());
    if ((rc = read_status(p, 0))) return rc;
    if (image) IMG2D_CUDA(cudaMemcpy(image, dI, (size_t)nextrap * nx * sizeof(float), cudaMemcpyDeviceToHost));
    if (image_shots)
        IMG2D_CUDA(cudaMemcpy2D(image_shots, plane * sizeof(float), dIS, plane * sizeof(float),
                                (size_t)nextrap * nx * sizeof(float), ns, cudaMemcpyDeviceToHost));
    IMG2D_CUDA(cudaMemcpy(wave_fs, dW, p->wave_elems * sizeof(cpx), cudaMemcpyDeviceToHost));
    IMG2D_CUDA(cudaMemcpy(shot_fs, dS, p->wave_elems * sizeof(cpx), cudaMemcpyDeviceToHost));
    return IMG2D_OK;
}

}  // extern "C"
