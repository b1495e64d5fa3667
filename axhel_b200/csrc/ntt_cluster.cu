// Single-launch NTT of small batches: one thread-block cluster per limb.
//
// A transform of N = 2^logn points runs as the two passes of the pass kernels
// (ntt_kernels.cuh) -- stages [0, LGA) on LGA-stage groups, then [LGA, logn)
// on LGB-stage groups -- but both passes run in one launch: the C = 2^c CTAs
// of a cluster each hold 1/C of the limb, run their share of the first pass,
// hand every element to the CTA that owns it in the second pass by a store
// into that CTA's shared memory (distributed shared memory), meet at one
// cluster barrier, and run their share of the second pass.  The limb crosses
// HBM once each way and the transform costs one launch instead of two, which
// is what bounds a transform of one or a few limbs (a few microseconds of
// work spread over C SMs instead of one).
//
// Forward: first pass = strided columns (stride 2^LGB), CTA k takes columns
// [k, k+1) * 2^(LGB-c); second pass = contiguous rows of 2^LGB, CTA k takes
// rows [k, k+1) * 2^(LGA-c), i.e. the contiguous chunk k of N/C words.
// Inverse: first pass = contiguous rows of 2^LGA (CTA k: chunk k), second
// pass = strided columns (stride 2^LGA), CTA k takes columns
// [k, k+1) * 2^(LGA-c).  Both passes have 2^(logn-c-LR) threads per CTA
// holding 2^LR elements each.
//
// Every butterfly is the pass kernels' (the reference's radix-2 butterflies
// applied to the same pairs, with the same twiddles, in the same stage
// order), so results are bit-identical to the two-launch form.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <mutex>

#include "launch.h"
#include "ntt_kernels.cuh"

namespace axhel_impl {

namespace cg = cooperative_groups;

namespace {

// Landing position of limb word p for the second pass of CTA `owner`:
// forward (contiguous second pass) chunk offset; inverse (strided second
// pass) row * 2^lgtgB + column-in-tile.
template <bool INV, int LGA>
__device__ __forceinline__ void landing_of(uint64_t p, uint32_t lgchunk, uint32_t lgtgB, uint32_t& owner,
                                           uint32_t& off)
{
    if constexpr (INV) {
        const uint32_t col = (uint32_t)p & ((1u << LGA) - 1), row = (uint32_t)(p >> LGA);
        owner = col >> lgtgB;
        off = (row << lgtgB) | (col & ((1u << lgtgB) - 1));
    } else {
        owner = (uint32_t)(p >> lgchunk);
        off = (uint32_t)p & ((1u << lgchunk) - 1);
    }
}

__device__ __forceinline__ void cluster_arrive_relaxed()
{
    asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait()
{
    asm volatile("barrier.cluster.wait.aligned;" ::: "memory");
}

}  // namespace

// One cluster of C CTAs per limb (grid = limbs * C, cluster dims C x 1 x 1);
// blockDim = 2^(logn - c - LR); dynamic shared memory = 2 * N/C words (the
// exchange scratch of the rounds, then the landing area of the second pass).
template <bool INV, int LGA, int LGB, int LR>
__global__ void __launch_bounds__(max_threads(LR)) ntt_cluster_kernel(const __grid_constant__ PassArgs a)
{
    extern __shared__ uint64_t sm[];
    constexpr int R = 1 << LR;
    constexpr uint32_t logn = LGA + LGB;
    cg::cluster_group cl = cg::this_cluster();
    // every CTA of the cluster must be running before its shared memory is
    // written by the others: arrive now, wait just before the first remote store
    cluster_arrive_relaxed();
    const uint32_t rank = cl.block_rank();
    const uint32_t c = __ffs(cl.num_blocks()) - 1;
    const uint64_t limb = blockIdx.x >> c;
    const uint32_t lgchunk = logn - c;
    const uint32_t lgtgA = LGB - c, lgtgB = LGA - c;
    uint64_t* scratch = sm;
    uint64_t* landing = sm + (1u << lgchunk);
    const ModCtx* cx = a.ctx[limb_mod(limb, a.nctx)];
    const uint64_t q = cx->q, q2 = cx->q2;
    const uint64_t n = 1ull << logn;
    const uint64_t* lsrc = a.src + (limb << logn);
    uint64_t* ldst = a.dst + (limb << logn);
    const bool vec_ok = ((reinterpret_cast<uintptr_t>(a.src) | reinterpret_cast<uintptr_t>(a.dst)) & 15) == 0;
    uint64_t v[R];

    // ---- first pass: stages [0, LGA)
    {
        constexpr int LO_FIRST = round_lo<INV, LGA, LR, 0>();
        constexpr int LO_LAST = round_lo<INV, LGA, LR, num_rounds<LGA, LR>() - 1>();
        const Tile t = make_tile<LGA>(INV ? 0u : (uint32_t)LGB, lgtgA, limb, rank);
        uint32_t gi, k;
        thread_role<LGA, LR>(t, gi, k);
        load_global<LGA, LR, LO_FIRST>(v, lsrc, t, gi, round_base<LR>(k, LO_FIRST), vec_ok);
        if (a.flags & kPreCsub2q) {
#pragma unroll
            for (int i = 0; i < R; ++i) v[i] = csub_lazy(v[i], q2);
        }
        run_rounds<INV, LGA, LR>(v, scratch + (gi << LGA), k, group_mask<LGA, LR>(t.strided, lgtgA, gi),
                                 lane_shift(t.strided, lgtgA), tile_blk<LGA>(t, gi), 0, n, cx, q, q2, false);
        // hand each element to its second-pass owner
        const uint32_t rb = round_base<LR>(k, LO_LAST);
        cluster_wait();
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const uint64_t r = rb + ((uint64_t)i << LO_LAST);
            const uint64_t p = t.strided ? t.base + gi + (r << t.lgS) : t.base + ((uint64_t)gi << LGA) + r;
            uint32_t owner, off;
            landing_of<INV, LGA>(p, lgchunk, lgtgB, owner, off);
            cl.map_shared_rank(landing, owner)[off] = v[i];
        }
    }
    // all remote stores of the cluster are visible after this barrier
    cl.sync();

    // ---- second pass: stages [LGA, logn)
    {
        constexpr int LO_FIRST = round_lo<INV, LGB, LR, 0>();
        constexpr int LO_LAST = round_lo<INV, LGB, LR, num_rounds<LGB, LR>() - 1>();
        const Tile t = make_tile<LGB>(INV ? (uint32_t)LGA : 0u, lgtgB, limb, rank);
        uint32_t gi, k;
        thread_role<LGB, LR>(t, gi, k);
        // the landing area is the tile itself, compacted: strided tiles as
        // rows of 2^lgtgB columns, contiguous ones as they are
        Tile tl = t;
        tl.base = 0;
        if (tl.strided) tl.lgS = lgtgB;
        load_global<LGB, LR, LO_FIRST>(v, landing, tl, gi, round_base<LR>(k, LO_FIRST), true);
        run_rounds<INV, LGB, LR>(v, scratch + (gi << LGB), k, group_mask<LGB, LR>(t.strided, lgtgB, gi),
                                 lane_shift(t.strided, lgtgB), tile_blk<LGB>(t, gi), LGA, n, cx, q, q2, INV);
        if (a.flags & kPostNorm) {
#pragma unroll
            for (int i = 0; i < R; ++i) v[i] = INV ? csub_lazy(v[i], q) : csub_lazy(csub_lazy(v[i], q2), q);
        }
        store_global<LGB, LR, LO_LAST>(v, ldst, t, gi, round_base<LR>(k, LO_LAST), vec_ok);
    }
}

// ------------------------------------------------------------------ host side

namespace {

using ClusterFn = void (*)(const PassArgs);

struct Entry {
    int lga, lgb, lr;
    ClusterFn fwd, inv;
};

template <int A, int B, int L>
Entry entry()
{
    return Entry{A, B, L, ntt_cluster_kernel<false, A, B, L>, ntt_cluster_kernel<true, A, B, L>};
}

// The compiled (first-pass stages, second-pass stages, register stages).
const Entry kEntries[] = {
    entry<6, 6, 2>(), entry<6, 6, 3>(), entry<5, 7, 3>(), entry<7, 5, 3>(), entry<6, 7, 3>(), entry<7, 6, 3>(),
    entry<7, 7, 3>(), entry<7, 8, 3>(), entry<8, 7, 3>(), entry<8, 8, 3>(), entry<8, 8, 4>(), entry<8, 9, 4>(),
    entry<9, 8, 4>(), entry<6, 7, 2>(), entry<7, 6, 2>(), entry<7, 7, 2>(), entry<7, 8, 2>(), entry<8, 7, 2>(),
    entry<5, 5, 2>(), entry<5, 6, 2>(), entry<6, 5, 2>(),
};
constexpr int kNumEntries = sizeof(kEntries) / sizeof(kEntries[0]);

const Entry* find_entry(int lga, int lgb, int lr)
{
    for (const Entry& e : kEntries)
        if (e.lga == lga && e.lgb == lgb && e.lr == lr) return &e;
    return nullptr;
}

// Built-in choice per direction and log2 N (10..17): first-pass stages,
// register stages, cluster size, and the largest limb count that takes the
// cluster form -- the fastest on a B200 by device time per transform
// (CUDA-graph replay): at N = 2^10 one limb takes 3.2 / 3.7 us (forward /
// inverse) against 6.5 / 4.6 us for the pass form, at 2^11 3.6 / 3.8 against
// 5.0 / 5.5, at 2^12 3.8 / 4.6 against 6.0 / 6.5 (two pass launches), at 2^13
// 3.9 / 4.6 against 6.6 / 7.2, at 2^14 4.9 / 5.3 against 7.1 / 7.8, at 2^15
// 6.8 / 7.1 against 7.6 / 7.4.  From 2^16 one limb's work needs more than the
// 16 SMs of a cluster and the pass form (all SMs) is faster, as it is from
// 16 / 4 limbs up at 2^14 / 2^15; at 2^10..2^13 the cluster form is still
// ahead at 64 limbs, the largest count measured.
ClusterCfg default_cfg(bool inverse, uint32_t logn)
{
    switch (logn) {
    case 10: return ClusterCfg{5, 2, 2, 64};
    case 11: return ClusterCfg{6, 2, 4, 64};
    case 12: return ClusterCfg{6, 2, 8, 64};
    case 13: return inverse ? ClusterCfg{7, 2, 16, 64} : ClusterCfg{6, 2, 16, 64};
    case 14: return ClusterCfg{7, 2, 16, 16};
    case 15: return inverse ? ClusterCfg{7, 2, 16, 4} : ClusterCfg{8, 2, 16, 4};
    case 16: return ClusterCfg{8, 3, 16, 0};
    case 17: return ClusterCfg{8, 4, 16, 0};
    default: return ClusterCfg{0, 0, 0, 0};
    }
}

std::mutex g_mu;
bool g_set[2][18] = {};
ClusterCfg g_over[2][18] = {};
// per entry and device: shared-memory / cluster-size attributes set
std::mutex g_attr_mu;
uint64_t g_attr_done[2][kNumEntries] = {};

int entry_index(const Entry* e) { return (int)(e - kEntries); }

}  // namespace

bool cluster_cfg_valid(uint32_t logn, const ClusterCfg& c)
{
    if (logn < 10 || logn > 17 || c.max_limbs == 0) return false;
    const int lgb = (int)logn - c.lga;
    if (!find_entry(c.lga, lgb, c.lr)) return false;
    if (c.csize < 2 || c.csize > 16 || (c.csize & (c.csize - 1))) return false;
    const int lc = __builtin_ctz(c.csize);
    if (lc > c.lga || lc > lgb) return false;
    const int lgthreads = (int)logn - lc - c.lr;
    if (lgthreads < 5 || (1 << lgthreads) > max_threads(c.lr)) return false;
    return 2 * (sizeof(uint64_t) << (logn - lc)) <= 227 * 1024;
}

bool cluster_plan(bool inverse, uint32_t logn, uint64_t count, ClusterCfg* out)
{
    if (logn < 10 || logn > 17) return false;
    ClusterCfg c;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        c = g_set[inverse][logn] ? g_over[inverse][logn] : default_cfg(inverse, logn);
    }
    if (count == 0 || count > c.max_limbs || !cluster_cfg_valid(logn, c)) return false;
    *out = c;
    return true;
}

void cluster_plan_override(bool inverse, uint32_t logn, const ClusterCfg* c)
{
    if (logn > 17) return;
    std::lock_guard<std::mutex> lk(g_mu);
    g_set[inverse][logn] = c != nullptr;
    if (c) g_over[inverse][logn] = *c;
}

ClusterCfg cluster_plan_current(bool inverse, uint32_t logn)
{
    if (logn > 17) return ClusterCfg{0, 0, 0, 0};
    std::lock_guard<std::mutex> lk(g_mu);
    return g_set[inverse][logn] ? g_over[inverse][logn] : default_cfg(inverse, logn);
}

cudaError_t launch_ntt_cluster(bool inverse, const ClusterCfg& c, const PassArgs& a, cudaStream_t s)
{
    if (!cluster_cfg_valid(a.logn, c)) return cudaErrorInvalidValue;
    const int lgb = (int)a.logn - c.lga;
    const Entry* e = find_entry(c.lga, lgb, c.lr);
    ClusterFn fn = inverse ? e->inv : e->fwd;
    const int lc = __builtin_ctz(c.csize);
    const size_t smem = 2 * (sizeof(uint64_t) << (a.logn - lc));
    const uint64_t blocks = a.count * (uint64_t)c.csize;
    if (a.count == 0) return cudaSuccess;
    if (blocks > 0x7fffffffull) return cudaErrorInvalidValue;
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    if (dev >= 64) return cudaErrorInvalidDevice;
    {
        std::lock_guard<std::mutex> lk(g_attr_mu);
        uint64_t& done = g_attr_done[inverse][entry_index(e)];
        if (!(done >> dev & 1)) {
            err = cudaFuncSetAttribute(reinterpret_cast<const void*>(fn),
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
            if (err == cudaSuccess)
                err = cudaFuncSetAttribute(reinterpret_cast<const void*>(fn),
                                           cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            if (err != cudaSuccess) return err;
            done |= 1ull << dev;
        }
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks, 1, 1);
    cfg.blockDim = dim3(1u << (a.logn - lc - c.lr), 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)c.csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    count_launch();
    ProfScope prof(s, "ntt_%s_cluster lga=%d lr=%d c=%d", inverse ? "inv" : "fwd", c.lga, c.lr, c.csize);
    void* args[] = {const_cast<PassArgs*>(&a)};
    err = cudaLaunchKernelExC(&cfg, reinterpret_cast<const void*>(fn), args);
    return err != cudaSuccess ? err : cudaGetLastError();
}

}  // namespace axhel_impl
