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
// order), so results are bit-identical to the two-launch form.  The
// transform kernel also applies the dyadic product of kPreMul / kPostMul (a
// MulMod on load / before the store), and the fused kernel further down runs
// the INTT -> op -> NTT chains and the NTT -> MulMod -> INTT product in one
// launch with two exchanges.  The host side picks the cluster shape per kind
// and degree (override > `K` lines of ntt_plans.txt > built-in choice) and
// takes this form up to a limb count beyond which the pass kernels, which
// use every SM, are faster.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <atomic>
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

// ---- rounds with their twiddles loaded ahead
//
// A cluster holds one limb on a few SMs with a handful of warps each, so
// every dependent load shows: a round that loads its twiddles after the
// exchange before it waits a full L2 round trip.  These variants of the pass
// kernels' rounds (fwd_stages / inv_stages: same butterflies, same twiddles,
// same order) take all of a pass's twiddles from registers filled before the
// pass starts, so their loads overlap the limb's own load (first pass) or
// the cluster exchange (second pass).

template <bool INV, int LG, int LR, int RD>
struct RoundShape {
    static constexpr int R = 1 << LR;
    static constexpr int LO = round_lo<INV, LG, LR, RD>();
    static constexpr int HI = LG - RD * LR;  // forward: stage bits HI-1 .. HI-NB
    static constexpr int NB = HI < LR ? HI : LR;
    static constexpr int B0 = RD * LR;  // inverse: stage bits B0 .. B1-1
    static constexpr int B1 = (B0 + LR < LG) ? B0 + LR : LG;
};

// Twiddles of a pass held in registers: at most 2^LR - 1 per round.
template <int NR, int LR>
struct PassTw {
    ulonglong2 w[NR][(1 << LR) - 1];
    uint64_t ninv, ninv_q, sr, sr_q;  // the inverse's final stage
};

template <bool INV, int LG, int LR, int RD, bool LAST>
__device__ __forceinline__ void load_round_tw(ulonglong2 (&w)[(1 << LR) - 1], uint32_t k, uint64_t blk, uint32_t s0,
                                              uint64_t n, const ulonglong2* __restrict__ tw)
{
    using S = RoundShape<INV, LG, LR, RD>;
    const uint32_t rbase = round_base<LR>(k, S::LO);
    int idx = 0;
    if constexpr (INV) {
#pragma unroll
        for (int b = S::B0; b < S::B1; ++b) {
            const int rb = b - S::LO;
            if (LAST && b == LG - 1) continue;
            const uint32_t s = s0 + b;
            const ulonglong2* tws = tw + (1 + n - (n >> s)) + (blk << (LG - b - 1)) + (rbase >> (b + 1));
#pragma unroll
            for (int j = 0; j < (S::R >> (rb + 1)); ++j) w[idx++] = __ldg(tws + j);
        }
    } else {
#pragma unroll
        for (int bb = 0; bb < S::NB; ++bb) {
            const int b = S::HI - 1 - bb;
            const int rb = b - S::LO;
            const uint32_t t = s0 + (LG - 1 - b);
            const ulonglong2* tws = tw + (1ull << t) + (blk << (LG - 1 - b)) + (rbase >> (b + 1));
#pragma unroll
            for (int j = 0; j < (S::R >> (rb + 1)); ++j) w[idx++] = __ldg(tws + j);
        }
    }
}

template <bool INV, int LG, int LR, int RD, bool LAST, int NR>
__device__ __forceinline__ void apply_round(uint64_t (&v)[1 << LR], const PassTw<NR, LR>& pt, uint64_t q,
                                            uint64_t q2)
{
    using S = RoundShape<INV, LG, LR, RD>;
    int idx = 0;
    if constexpr (INV) {
#pragma unroll
        for (int b = S::B0; b < S::B1; ++b) {
            const int rb = b - S::LO;
            if (LAST && b == LG - 1) {
#pragma unroll
                for (int j = 0; j < (S::R >> (rb + 1)); ++j)
#pragma unroll
                    for (int l = 0; l < (1 << rb); ++l) {
                        const int i0 = (j << (rb + 1)) | l;
                        inv_final_butterfly(v[i0], v[i0 | (1 << rb)], pt.ninv, pt.ninv_q, pt.sr, pt.sr_q, q, q2);
                    }
            } else {
#pragma unroll
                for (int j = 0; j < (S::R >> (rb + 1)); ++j) {
                    const ulonglong2 w = pt.w[RD][idx++];
#pragma unroll
                    for (int l = 0; l < (1 << rb); ++l) {
                        const int i0 = (j << (rb + 1)) | l;
                        inv_butterfly(v[i0], v[i0 | (1 << rb)], w.x, w.y, q, q2);
                    }
                }
            }
        }
    } else {
#pragma unroll
        for (int bb = 0; bb < S::NB; ++bb) {
            const int rb = S::HI - 1 - bb - S::LO;
#pragma unroll
            for (int j = 0; j < (S::R >> (rb + 1)); ++j) {
                const ulonglong2 w = pt.w[RD][idx++];
#pragma unroll
                for (int l = 0; l < (1 << rb); ++l) {
                    const int i0 = (j << (rb + 1)) | l;
                    fwd_butterfly(v[i0], v[i0 | (1 << rb)], w.x, w.y, q, q2);
                }
            }
        }
    }
}

template <bool INV, int LG, int LR, bool LAST, int NR, int... RD>
__device__ __forceinline__ void load_pass_tw(std::integer_sequence<int, RD...>, PassTw<NR, LR>& pt, uint32_t k,
                                             uint64_t blk, uint32_t s0, uint64_t n, const ModCtx* cx)
{
    (load_round_tw<INV, LG, LR, RD, LAST>(pt.w[RD], k, blk, s0, n, INV ? cx->inv : cx->fwd), ...);
    if constexpr (INV && LAST) {
        pt.ninv = cx->ninv;
        pt.ninv_q = cx->ninv_q;
        pt.sr = cx->sroot;
        pt.sr_q = cx->sroot_q;
    }
}

template <bool INV, int LG, int LR, int RD, bool LAST, int NR>
__device__ __forceinline__ void step(uint64_t (&v)[1 << LR], const PassTw<NR, LR>& pt, uint64_t* smg, uint32_t k,
                                     uint32_t hmask, uint32_t lsh, uint64_t q, uint64_t q2)
{
    if constexpr (RD > 0) exchange<INV, LG, LR, RD>(v, smg, k, hmask, lsh);
    apply_round<INV, LG, LR, RD, LAST, NR>(v, pt, q, q2);
}

template <bool INV, int LG, int LR, bool LAST, int NR, int... RD>
__device__ __forceinline__ void run_pass_tw(std::integer_sequence<int, RD...>, uint64_t (&v)[1 << LR],
                                            const PassTw<NR, LR>& pt, uint64_t* smg, uint32_t k, uint32_t hmask,
                                            uint32_t lsh, uint64_t q, uint64_t q2)
{
    (step<INV, LG, LR, RD, LAST, NR>(v, pt, smg, k, hmask, lsh, q, q2), ...);
}

// Prefetched twiddles fit the register budget when a pass has at most 12.
template <int LG, int LR>
constexpr bool prefetch_fits()
{
    return num_rounds<LG, LR>() * ((1 << LR) - 1) <= 12;
}

}  // namespace

// One cluster of C CTAs per limb (grid = limbs * C, cluster dims C x 1 x 1);
// blockDim = 2^(logn - c - LR); dynamic shared memory = 2 * N/C words (the
// exchange scratch of the rounds, then the landing area of the second pass).
template <bool INV, int LGA, int LGB, int LR, bool PREFETCH>
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
    // twiddles prefetched into registers: shorter dependent chains, more
    // registers (the launcher picks it when the grid is one wave)
    constexpr bool PRE = PREFETCH && prefetch_fits<LGA, LR>() && prefetch_fits<LGB, LR>();
    constexpr int NRA = num_rounds<LGA, LR>(), NRB = num_rounds<LGB, LR>();
    uint64_t v[R];

    // second-pass geometry (needed early to prefetch its twiddles)
    const Tile tB = make_tile<LGB>(INV ? (uint32_t)LGA : 0u, lgtgB, limb, rank);
    uint32_t giB, kB;
    thread_role<LGB, LR>(tB, giB, kB);
    const uint64_t blkB = tile_blk<LGB>(tB, giB);

    // ---- first pass: stages [0, LGA)
    {
        constexpr int LO_FIRST = round_lo<INV, LGA, LR, 0>();
        constexpr int LO_LAST = round_lo<INV, LGA, LR, NRA - 1>();
        const Tile t = make_tile<LGA>(INV ? 0u : (uint32_t)LGB, lgtgA, limb, rank);
        uint32_t gi, k;
        thread_role<LGA, LR>(t, gi, k);
        const uint64_t blk = tile_blk<LGA>(t, gi);
        load_global<LGA, LR, LO_FIRST>(v, lsrc, t, gi, round_base<LR>(k, LO_FIRST), vec_ok);
        if (a.flags & kPreMul)
            mul_operand<LGA, LR, LO_FIRST, false>(v, a.operand + (limb << logn), t, gi, k, cx, vec_ok);
        if constexpr (PRE) {
            PassTw<NRA, LR> pt;
            load_pass_tw<INV, LGA, LR, false>(std::make_integer_sequence<int, NRA>{}, pt, k, blk, 0, n, cx);
            if (a.flags & kPreCsub2q) {
#pragma unroll
                for (int i = 0; i < R; ++i) v[i] = csub_lazy(v[i], q2);
            }
            run_pass_tw<INV, LGA, LR, false>(std::make_integer_sequence<int, NRA>{}, v, pt, scratch + (gi << LGA), k,
                                             group_mask<LGA, LR>(t.strided, lgtgA, gi), lane_shift(t.strided, lgtgA),
                                             q, q2);
        } else {
            if (a.flags & kPreCsub2q) {
#pragma unroll
                for (int i = 0; i < R; ++i) v[i] = csub_lazy(v[i], q2);
            }
            run_rounds<INV, LGA, LR>(v, scratch + (gi << LGA), k, group_mask<LGA, LR>(t.strided, lgtgA, gi),
                                     lane_shift(t.strided, lgtgA), blk, 0, n, cx, q, q2, false);
        }
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

    // ---- second pass: stages [LGA, logn)
    constexpr int LO_FIRST = round_lo<INV, LGB, LR, 0>();
    constexpr int LO_LAST = round_lo<INV, LGB, LR, NRB - 1>();
    // the landing area is the tile itself, compacted: strided tiles as rows
    // of 2^lgtgB columns, contiguous ones as they are
    Tile tl = tB;
    tl.base = 0;
    if (tl.strided) tl.lgS = lgtgB;
    if constexpr (PRE) {
        PassTw<NRB, LR> pt;
        load_pass_tw<INV, LGB, LR, INV>(std::make_integer_sequence<int, NRB>{}, pt, kB, blkB, LGA, n, cx);
        // all remote stores of the cluster are visible after this barrier
        cl.sync();
        load_global<LGB, LR, LO_FIRST>(v, landing, tl, giB, round_base<LR>(kB, LO_FIRST), true);
        run_pass_tw<INV, LGB, LR, INV>(std::make_integer_sequence<int, NRB>{}, v, pt, scratch + (giB << LGB), kB,
                                       group_mask<LGB, LR>(tB.strided, lgtgB, giB), lane_shift(tB.strided, lgtgB),
                                       q, q2);
    } else {
        cl.sync();
        load_global<LGB, LR, LO_FIRST>(v, landing, tl, giB, round_base<LR>(kB, LO_FIRST), true);
        run_rounds<INV, LGB, LR>(v, scratch + (giB << LGB), kB, group_mask<LGB, LR>(tB.strided, lgtgB, giB),
                                 lane_shift(tB.strided, lgtgB), blkB, LGA, n, cx, q, q2, INV);
    }
    if (a.flags & kPostNorm) {
#pragma unroll
        for (int i = 0; i < R; ++i) v[i] = INV ? csub_lazy(v[i], q) : csub_lazy(csub_lazy(v[i], q2), q);
    }
    if (a.flags & kPostMul)
        mul_operand<LGB, LR, LO_LAST, false>(v, a.operand + (limb << logn), tB, giB, kB, cx, vec_ok);
    store_global<LGB, LR, LO_LAST>(v, ldst, tB, giB, round_base<LR>(kB, LO_LAST), vec_ok);
}

// ---- fused chains in one launch
//
// INTT -> MulMod/FMAMod -> NTT (the chain kernels' job) and NTT -> MulMod ->
// INTT (the product kernels' job) of one limb per cluster, in three phases
// with two exchanges through distributed shared memory.  With N = 2^(LGR +
// LGC), "rows" are the 2^LGC contiguous groups of 2^LGR words and "columns"
// the 2^LGR groups of stride 2^LGR; CTA k holds row chunk k or the columns
// [k, k+1) * 2^(LGR-c).
//   chain:   inverse rows (stages 0..LGR-1) | columns: inverse stages
//            LGR..logn-1 with N^-1, the op, forward stages 0..LGC-1 | forward
//            rows (stages LGC..logn-1)
//   product: forward columns (stages 0..LGC-1) | rows: forward stages
//            LGC..logn-1, MulMod<4>, inverse stages 0..LGR-1 | inverse columns
//            (stages LGR..logn-1 with N^-1)
// The middle phase is the chain / product tile's (the inverse's last round
// and the forward's first hold the same register bits, and the reverse), so
// every result equals the three-launch chains and the call sequences they
// replace.  Shared memory: 3 * N/C words (round exchanges, the first landing
// area, the second landing area).

namespace {

// Registers of round LO of tile t (LG-stage groups) into the landing area of
// their owners in the next phase: rows (chunk owners) or columns.
template <int LG, int LR, int LO, bool TO_COLUMNS, int LGR>
__device__ __forceinline__ void scatter(const uint64_t (&v)[1 << LR], const Tile& t, uint32_t gi, uint32_t k,
                                        uint32_t lgchunk, uint32_t lgtg_cols, uint64_t* landing,
                                        cg::cluster_group& cl)
{
    const uint32_t rb = round_base<LR>(k, LO);
#pragma unroll
    for (int i = 0; i < (1 << LR); ++i) {
        const uint64_t r = rb + ((uint64_t)i << LO);
        const uint64_t p = t.strided ? t.base + gi + (r << t.lgS) : t.base + ((uint64_t)gi << LG) + r;
        uint32_t owner, off;
        landing_of<TO_COLUMNS, LGR>(p, lgchunk, lgtg_cols, owner, off);
        cl.map_shared_rank(landing, owner)[off] = v[i];
    }
}

// The tile itself, compacted, as a landing area: columns as rows of
// 2^lgtg_cols words, row chunks as they are.
__device__ __forceinline__ Tile landing_tile(Tile t, uint32_t lgtg_cols)
{
    t.base = 0;
    if (t.strided) t.lgS = lgtg_cols;
    return t;
}

}  // namespace

template <bool PRODUCT, int LGR, int LGC, int LR>
__global__ void __launch_bounds__(max_threads(LR)) ntt_cluster_fused_kernel(const __grid_constant__ ChainArgs c)
{
    extern __shared__ uint64_t sm[];
    constexpr int R = 1 << LR;
    constexpr uint32_t logn = LGR + LGC;
    constexpr int NRR = num_rounds<LGR, LR>(), NRC = num_rounds<LGC, LR>();
    const PassArgs& a = c.pass;
    cg::cluster_group cl = cg::this_cluster();
    cluster_arrive_relaxed();
    const uint32_t rank = cl.block_rank();
    const uint32_t lc = __ffs(cl.num_blocks()) - 1;
    const uint64_t limb = blockIdx.x >> lc;
    const uint32_t lgchunk = logn - lc;
    const uint32_t lgtgR = LGC - lc, lgtgC = LGR - lc;  // rows / columns per CTA (log2)
    uint64_t* scratch = sm;
    uint64_t* landing1 = sm + (1u << lgchunk);
    uint64_t* landing2 = sm + (2u << lgchunk);
    const uint32_t mi = limb_mod(limb, a.nctx);
    const ModCtx* cx = a.ctx[mi];
    const uint64_t q = cx->q, q2 = cx->q2, mu = cx->mu;
    const uint32_t shift = cx->shift;
    const uint64_t n = 1ull << logn;
    const uint64_t* lsrc = a.src + (limb << logn);
    uint64_t* ldst = a.dst + (limb << logn);
    const uint64_t* lop = c.operand ? c.operand + (limb << logn) : nullptr;
    const bool vec_ok = ((reinterpret_cast<uintptr_t>(a.src) | reinterpret_cast<uintptr_t>(a.dst) |
                          reinterpret_cast<uintptr_t>(c.operand)) & 15) == 0;
    const Tile tR = make_tile<LGR>(0, lgtgR, limb, rank);
    const Tile tC = make_tile<LGC>(LGR, lgtgC, limb, rank);
    uint64_t v[R];
    uint32_t gi, k;

    static_assert(prefetch_fits<LGR, LR>() && prefetch_fits<LGC, LR>(), "fused shapes hold a pass's twiddles");
    // Each half-transform's twiddles are loaded into registers ahead of it
    // (with the limb, before a cluster barrier, or beside the operand): the
    // phases run one after another, so this adds no registers to the peak.
    if constexpr (!PRODUCT) {
        // ---- inverse rows: stages [0, LGR)
        thread_role<LGR, LR>(tR, gi, k);
        load_global<LGR, LR, round_lo<true, LGR, LR, 0>()>(v, lsrc, tR, gi,
                                                           round_base<LR>(k, round_lo<true, LGR, LR, 0>()), vec_ok);
        {
            PassTw<NRR, LR> pt;
            load_pass_tw<true, LGR, LR, false>(std::make_integer_sequence<int, NRR>{}, pt, k, tile_blk<LGR>(tR, gi), 0,
                                               n, cx);
            if (a.flags & kPreCsub2q) {
#pragma unroll
                for (int i = 0; i < R; ++i) v[i] = csub_lazy(v[i], q2);
            }
            run_pass_tw<true, LGR, LR, false>(std::make_integer_sequence<int, NRR>{}, v, pt, scratch + (gi << LGR), k,
                                              group_mask<LGR, LR>(false, lgtgR, gi), lane_shift(false, lgtgR), q, q2);
        }
        cluster_wait();
        scatter<LGR, LR, round_lo<true, LGR, LR, NRR - 1>(), true, LGR>(v, tR, gi, k, lgchunk, lgtgC, landing1, cl);

        // ---- columns: inverse stages [LGR, logn) with N^-1, the op, forward stages [0, LGC)
        constexpr int LO_IN = round_lo<true, LGC, LR, 0>();
        constexpr int LO_MID = round_lo<true, LGC, LR, NRC - 1>();
        static_assert(LO_MID == round_lo<false, LGC, LR, 0>(), "inverse last round and forward first round differ");
        thread_role<LGC, LR>(tC, gi, k);
        uint64_t* smg = scratch + (gi << LGC);
        const uint32_t hmask = group_mask<LGC, LR>(true, lgtgC, gi), lsh = lane_shift(true, lgtgC);
        {
            PassTw<NRC, LR> pt;
            load_pass_tw<true, LGC, LR, true>(std::make_integer_sequence<int, NRC>{}, pt, k, tile_blk<LGC>(tC, gi), LGR,
                                              n, cx);
            cl.sync();
            load_global<LGC, LR, LO_IN>(v, landing1, landing_tile(tC, lgtgC), gi, round_base<LR>(k, LO_IN), true);
            run_pass_tw<true, LGC, LR, true>(std::make_integer_sequence<int, NRC>{}, v, pt, smg, k, hmask, lsh, q, q2);
        }
        {
            PassTw<NRC, LR> pt;
            load_pass_tw<false, LGC, LR, false>(std::make_integer_sequence<int, NRC>{}, pt, k, 0, 0, n, cx);
            const uint32_t rb = round_base<LR>(k, LO_MID);
            // EltwiseMulModNative<2> / EltwiseFMAModNative<2> on the inverse's [0, 2q) output
            if (c.op == kChainMul) {
                uint64_t m[R];
                load_global<LGC, LR, LO_MID>(m, lop, tC, gi, rb, vec_ok);
#pragma unroll
                for (int i = 0; i < R; ++i)
                    v[i] = barrett_mul(reduce_input<2>(v[i], q), reduce_input<2>(m[i], q), q, mu, shift);
            } else if (c.op == kChainFma) {
                const uint64_t sc = reduce_input<2>(c.scalar[mi], q);
#pragma unroll
                for (int i = 0; i < R; ++i) v[i] = barrett_mul(reduce_input<2>(v[i], q), sc, q, mu, shift);
                if (lop) {
                    uint64_t m[R];
                    load_global<LGC, LR, LO_MID>(m, lop, tC, gi, rb, vec_ok);
#pragma unroll
                    for (int i = 0; i < R; ++i) v[i] = csub(v[i] + reduce_input<2>(m[i], q), q);
                }
            }
            run_pass_tw<false, LGC, LR, false>(std::make_integer_sequence<int, NRC>{}, v, pt, smg, k, hmask, lsh, q,
                                               q2);
        }
        scatter<LGC, LR, round_lo<false, LGC, LR, NRC - 1>(), false, LGR>(v, tC, gi, k, lgchunk, lgtgC, landing2,
                                                                           cl);

        // ---- forward rows: stages [LGC, logn)
        thread_role<LGR, LR>(tR, gi, k);
        {
            PassTw<NRR, LR> pt;
            load_pass_tw<false, LGR, LR, false>(std::make_integer_sequence<int, NRR>{}, pt, k, tile_blk<LGR>(tR, gi),
                                                LGC, n, cx);
            cl.sync();
            load_global<LGR, LR, round_lo<false, LGR, LR, 0>()>(
                v, landing2, landing_tile(tR, lgtgC), gi, round_base<LR>(k, round_lo<false, LGR, LR, 0>()), true);
            run_pass_tw<false, LGR, LR, false>(std::make_integer_sequence<int, NRR>{}, v, pt, scratch + (gi << LGR),
                                               k, group_mask<LGR, LR>(false, lgtgR, gi), lane_shift(false, lgtgR), q,
                                               q2);
        }
        if (a.flags & kPostNorm) {
#pragma unroll
            for (int i = 0; i < R; ++i) v[i] = csub_lazy(csub_lazy(v[i], q2), q);
        }
        store_global<LGR, LR, round_lo<false, LGR, LR, NRR - 1>()>(
            v, ldst, tR, gi, round_base<LR>(k, round_lo<false, LGR, LR, NRR - 1>()), vec_ok);
    } else {
        // ---- forward columns: stages [0, LGC)
        thread_role<LGC, LR>(tC, gi, k);
        load_global<LGC, LR, round_lo<false, LGC, LR, 0>()>(v, lsrc, tC, gi,
                                                            round_base<LR>(k, round_lo<false, LGC, LR, 0>()), vec_ok);
        {
            PassTw<NRC, LR> pt;
            load_pass_tw<false, LGC, LR, false>(std::make_integer_sequence<int, NRC>{}, pt, k, tile_blk<LGC>(tC, gi), 0,
                                                n, cx);
            run_pass_tw<false, LGC, LR, false>(std::make_integer_sequence<int, NRC>{}, v, pt, scratch + (gi << LGC), k,
                                               group_mask<LGC, LR>(true, lgtgC, gi), lane_shift(true, lgtgC), q, q2);
        }
        cluster_wait();
        scatter<LGC, LR, round_lo<false, LGC, LR, NRC - 1>(), false, LGR>(v, tC, gi, k, lgchunk, lgtgC, landing1,
                                                                           cl);

        // ---- rows: forward stages [LGC, logn), MulMod<4>, inverse stages [0, LGR)
        constexpr int LO_IN = round_lo<false, LGR, LR, 0>();
        constexpr int LO_MID = round_lo<false, LGR, LR, NRR - 1>();
        static_assert(LO_MID == round_lo<true, LGR, LR, 0>(), "forward last round and inverse first round differ");
        thread_role<LGR, LR>(tR, gi, k);
        uint64_t* smg = scratch + (gi << LGR);
        const uint32_t hmask = group_mask<LGR, LR>(false, lgtgR, gi), lsh = lane_shift(false, lgtgR);
        const uint64_t blk = tile_blk<LGR>(tR, gi);
        {
            PassTw<NRR, LR> pt;
            load_pass_tw<false, LGR, LR, false>(std::make_integer_sequence<int, NRR>{}, pt, k, blk, LGC, n, cx);
            cl.sync();
            load_global<LGR, LR, LO_IN>(v, landing1, landing_tile(tR, lgtgC), gi, round_base<LR>(k, LO_IN), true);
            run_pass_tw<false, LGR, LR, false>(std::make_integer_sequence<int, NRR>{}, v, pt, smg, k, hmask, lsh, q,
                                               q2);
        }
        {
            PassTw<NRR, LR> pt;
            load_pass_tw<true, LGR, LR, false>(std::make_integer_sequence<int, NRR>{}, pt, k, blk, 0, n, cx);
            uint64_t m[R];
            load_global<LGR, LR, LO_MID>(m, lop, tR, gi, round_base<LR>(k, LO_MID), vec_ok);
#pragma unroll
            for (int i = 0; i < R; ++i)
                v[i] = barrett_mul(reduce_input<4>(v[i], q), reduce_input<4>(m[i], q), q, mu, shift);
            run_pass_tw<true, LGR, LR, false>(std::make_integer_sequence<int, NRR>{}, v, pt, smg, k, hmask, lsh, q, q2);
        }
        scatter<LGR, LR, round_lo<true, LGR, LR, NRR - 1>(), true, LGR>(v, tR, gi, k, lgchunk, lgtgC, landing2, cl);

        // ---- inverse columns: stages [LGR, logn) with N^-1
        constexpr int LO_C = round_lo<true, LGC, LR, 0>();
        constexpr int LO_OUT = round_lo<true, LGC, LR, NRC - 1>();
        thread_role<LGC, LR>(tC, gi, k);
        {
            PassTw<NRC, LR> pt;
            load_pass_tw<true, LGC, LR, true>(std::make_integer_sequence<int, NRC>{}, pt, k, tile_blk<LGC>(tC, gi), LGR,
                                              n, cx);
            cl.sync();
            load_global<LGC, LR, LO_C>(v, landing2, landing_tile(tC, lgtgC), gi, round_base<LR>(k, LO_C), true);
            run_pass_tw<true, LGC, LR, true>(std::make_integer_sequence<int, NRC>{}, v, pt, scratch + (gi << LGC), k,
                                             group_mask<LGC, LR>(true, lgtgC, gi), lane_shift(true, lgtgC), q, q2);
        }
        if (a.flags & kPostNorm) {
#pragma unroll
            for (int i = 0; i < R; ++i) v[i] = csub_lazy(v[i], q);
        }
        store_global<LGC, LR, LO_OUT>(v, ldst, tC, gi, round_base<LR>(k, LO_OUT), vec_ok);
    }
}

// ------------------------------------------------------------------ host side

namespace {

using ClusterFn = void (*)(const PassArgs);
using FusedFn = void (*)(const ChainArgs);

struct Entry {
    int lga, lgb, lr;
    ClusterFn fn[2][2];  // [inverse][prefetching twiddles]; [.][1] null where it does not fit
};

template <int A, int B, int L>
Entry entry()
{
    constexpr bool pre = prefetch_fits<A, L>() && prefetch_fits<B, L>();
    Entry e{A, B, L, {{ntt_cluster_kernel<false, A, B, L, false>, nullptr},
                      {ntt_cluster_kernel<true, A, B, L, false>, nullptr}}};
    if constexpr (pre) {
        e.fn[0][1] = ntt_cluster_kernel<false, A, B, L, true>;
        e.fn[1][1] = ntt_cluster_kernel<true, A, B, L, true>;
    }
    return e;
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

// The fused chain / product kernels: (row stages, column stages, register stages).
struct FusedEntry {
    int lgr, lgc, lr;
    FusedFn fn[2];  // [product]
};

template <int A, int B, int L>
FusedEntry fused_entry()
{
    return FusedEntry{A, B, L, {ntt_cluster_fused_kernel<false, A, B, L>, ntt_cluster_fused_kernel<true, A, B, L>}};
}

const FusedEntry kFused[] = {
    fused_entry<5, 5, 2>(), fused_entry<6, 5, 2>(), fused_entry<5, 6, 2>(), fused_entry<6, 6, 2>(),
    fused_entry<7, 6, 2>(), fused_entry<6, 7, 2>(), fused_entry<7, 7, 2>(), fused_entry<8, 7, 2>(),
    fused_entry<7, 8, 2>(),
};
constexpr int kNumFused = sizeof(kFused) / sizeof(kFused[0]);

const FusedEntry* find_fused(int lgr, int lgc, int lr)
{
    for (const FusedEntry& e : kFused)
        if (e.lgr == lgr && e.lgc == lgc && e.lr == lr) return &e;
    return nullptr;
}

// Built-in choice (where ntt_plans.txt has no `K` line for it; the
// autotuner's lines reproduce it within noise) per kind and log2 N (10..17):
// first-pass (transforms) or
// row (fused chains) stages, register stages, cluster size, and the largest
// limb count that takes the cluster form -- the fastest on a B200 by device
// time per call (CUDA-graph replay).  Transforms of one limb, forward /
// inverse, against the pass form: 2^10 3.0 / 3.2 us (6.7 / 4.7), 2^11 3.2 /
// 3.3 (5.0 / 5.6), 2^12 3.4 / 3.5 (6.5 / 6.6), 2^13 3.7 / 3.7 (6.7 / 7.2),
// 2^14 4.7 / 4.9 (7.1 / 7.7), 2^15 7.0 / 7.3 (7.6 / 7.5).  From 2^16 one
// limb's work needs more than the 16 SMs of a cluster and the pass form (all
// SMs) is faster, as it is from 16 / 4 limbs up at 2^14 / 2^15; at
// 2^10..2^13 the cluster form is still ahead at 64 limbs, the largest count
// measured.
ClusterCfg default_cfg(int kind, uint32_t logn)
{
    // Fused chain / product of one limb against the three pass launches:
    // 2^10 5.0 / 5.2 us (7.7 / 7.2), 2^11 5.4 / 5.2 (9.6 / 9.0), 2^12 5.7 /
    // 5.8 (12.1 / 12.0), 2^13 6.2 / 5.6 (12.2 / 13.0), 2^14 8.2 / 8.1 (13.6 /
    // 15.2), 2^15 12.3 / 12.6 (13.7 / 14.3); still ahead at 64 limbs up to
    // 2^12, behind from about 32 / 8 / 8 limbs at 2^13 / 2^14 / 2^15.
    if (kind == kClusterChain || kind == kClusterProduct) {
        switch (logn) {
        case 10: return ClusterCfg{5, 2, 4, 64};
        case 11: return ClusterCfg{6, 2, 8, 64};
        case 12: return ClusterCfg{6, 2, 8, 64};
        case 13: return ClusterCfg{7, 2, 16, 16};
        case 14: return ClusterCfg{7, 2, 16, 8};
        case 15: return ClusterCfg{7, 2, 16, 4};
        default: return ClusterCfg{0, 0, 0, 0};
        }
    }
    const bool inverse = kind == kClusterInverse;
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

// Overrides (axhel_cuda_cluster_plan_set); g_set is read without the lock
// on every call, the configuration under it only when an override exists.
std::mutex g_mu;
std::atomic<bool> g_set[4][18] = {};
ClusterCfg g_over[4][18] = {};
// the autotuner's table (ntt_plans.txt), same scheme
std::atomic<bool> g_tab_set[4][18] = {};
ClusterCfg g_tab[4][18] = {};

// The configuration for (kind, logn): override > table > built-in.
ClusterCfg current_cfg(int kind, uint32_t logn)
{
    plan_table_ensure();
    ClusterCfg c = default_cfg(kind, logn);
    if (g_set[kind][logn].load(std::memory_order_acquire) || g_tab_set[kind][logn].load(std::memory_order_acquire)) {
        std::lock_guard<std::mutex> lk(g_mu);
        if (g_set[kind][logn].load(std::memory_order_relaxed))
            c = g_over[kind][logn];
        else if (g_tab_set[kind][logn].load(std::memory_order_relaxed))
            c = g_tab[kind][logn];
    }
    return c;
}
// per kernel and device: shared-memory / cluster-size attributes set (bit
// `device`), read without the lock once set
std::mutex g_attr_mu;
std::atomic<uint64_t> g_attr_done[kNumEntries][2][2] = {};
std::atomic<uint64_t> g_fused_attr_done[kNumFused][2] = {};

int entry_index(const Entry* e) { return (int)(e - kEntries); }
int fused_index(const FusedEntry* e) { return (int)(e - kFused); }

bool fused_kind(int kind) { return kind == kClusterChain || kind == kClusterProduct; }

// Sets the launch attributes of `fn` once per device (bit `dev` of `done`).
cudaError_t ensure_attrs(const void* fn, std::atomic<uint64_t>& done, int dev)
{
    if (done.load(std::memory_order_acquire) >> dev & 1) return cudaSuccess;
    std::lock_guard<std::mutex> lk(g_attr_mu);
    if (done.load(std::memory_order_relaxed) >> dev & 1) return cudaSuccess;
    cudaError_t err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (err == cudaSuccess) err = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (err == cudaSuccess) done.fetch_or(1ull << dev, std::memory_order_release);
    return err;
}

cudaError_t launch_cluster(const void* fn, void* args, uint64_t blocks, uint32_t threads, size_t smem, int csize,
                           cudaStream_t s)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks, 1, 1);
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void* argv[] = {args};
    const cudaError_t err = cudaLaunchKernelExC(&cfg, fn, argv);
    return err != cudaSuccess ? err : cudaGetLastError();
}

}  // namespace

bool cluster_cfg_valid(int kind, uint32_t logn, const ClusterCfg& c)
{
    if (kind < 0 || kind > 3 || logn < 10 || logn > 17 || c.max_limbs == 0) return false;
    const int lgb = (int)logn - c.lga;
    const bool fused = fused_kind(kind);
    if (fused ? !find_fused(c.lga, lgb, c.lr) : !find_entry(c.lga, lgb, c.lr)) return false;
    if (c.csize < 2 || c.csize > 16 || (c.csize & (c.csize - 1))) return false;
    const int lc = __builtin_ctz(c.csize);
    if (lc > c.lga || lc > lgb) return false;
    const int lgthreads = (int)logn - lc - c.lr;
    if (lgthreads < 5 || (1 << lgthreads) > max_threads(c.lr)) return false;
    return (fused ? 3 : 2) * (sizeof(uint64_t) << (logn - lc)) <= 227 * 1024;
}

bool cluster_plan(int kind, uint32_t logn, uint64_t count, ClusterCfg* out)
{
    if (kind < 0 || kind > 3 || logn < 10 || logn > 17) return false;
    const ClusterCfg c = current_cfg(kind, logn);
    if (count == 0 || count > c.max_limbs || !cluster_cfg_valid(kind, logn, c)) return false;
    *out = c;
    return true;
}

void cluster_plan_override(int kind, uint32_t logn, const ClusterCfg* c)
{
    if (kind < 0 || kind > 3 || logn > 17) return;
    std::lock_guard<std::mutex> lk(g_mu);
    if (c) g_over[kind][logn] = *c;
    g_set[kind][logn].store(c != nullptr, std::memory_order_release);
}

ClusterCfg cluster_plan_current(int kind, uint32_t logn)
{
    if (kind < 0 || kind > 3 || logn > 17) return ClusterCfg{0, 0, 0, 0};
    return current_cfg(kind, logn);
}

void cluster_plan_table_set(int kind, uint32_t logn, const ClusterCfg& c)
{
    if (kind < 0 || kind > 3 || logn > 17) return;
    std::lock_guard<std::mutex> lk(g_mu);
    g_tab[kind][logn] = c;
    g_tab_set[kind][logn].store(true, std::memory_order_release);
}

cudaError_t launch_ntt_cluster(bool inverse, const ClusterCfg& c, const PassArgs& a, cudaStream_t s)
{
    if (!cluster_cfg_valid(inverse ? kClusterInverse : kClusterForward, a.logn, c)) return cudaErrorInvalidValue;
    const Entry* e = find_entry(c.lga, (int)a.logn - c.lga, c.lr);
    const int lc = __builtin_ctz(c.csize);
    const uint64_t blocks = a.count * (uint64_t)c.csize;
    if (a.count == 0) return cudaSuccess;
    if (blocks > 0x7fffffffull) return cudaErrorInvalidValue;
    // Twiddles prefetched into registers shorten each round's dependent
    // chain but cost occupancy: worth it while the grid is one wave of at
    // most one CTA per SM (measured faster there up to N = 2^14, slower with
    // several clusters per SM and at 2^15).
    const bool pre = e->fn[inverse][1] && a.logn <= 14 && blocks <= (uint64_t)sm_count();
    const void* fn = reinterpret_cast<const void*>(e->fn[inverse][pre]);
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    if (dev >= 64) return cudaErrorInvalidDevice;
    err = ensure_attrs(fn, g_attr_done[entry_index(e)][inverse][pre], dev);
    if (err != cudaSuccess) return err;
    count_launch();
    ProfScope prof(s, "ntt_%s_cluster lga=%d lr=%d c=%d%s", inverse ? "inv" : "fwd", c.lga, c.lr, c.csize,
                   pre ? " prefetch" : "");
    return launch_cluster(fn, const_cast<PassArgs*>(&a), blocks, 1u << (a.logn - lc - c.lr),
                          2 * (sizeof(uint64_t) << (a.logn - lc)), c.csize, s);
}

cudaError_t launch_ntt_cluster_fused(bool product, const ClusterCfg& c, const ChainArgs& a, cudaStream_t s)
{
    const uint32_t logn = a.pass.logn;
    if (!cluster_cfg_valid(product ? kClusterProduct : kClusterChain, logn, c)) return cudaErrorInvalidValue;
    const FusedEntry* e = find_fused(c.lga, (int)logn - c.lga, c.lr);
    const int lc = __builtin_ctz(c.csize);
    const uint64_t blocks = a.pass.count * (uint64_t)c.csize;
    if (a.pass.count == 0) return cudaSuccess;
    if (blocks > 0x7fffffffull) return cudaErrorInvalidValue;
    const void* fn = reinterpret_cast<const void*>(e->fn[product]);
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    if (dev >= 64) return cudaErrorInvalidDevice;
    err = ensure_attrs(fn, g_fused_attr_done[fused_index(e)][product], dev);
    if (err != cudaSuccess) return err;
    count_launch();
    ProfScope prof(s, "ntt_%s_cluster lgr=%d lr=%d c=%d", product ? "product" : "chain", c.lga, c.lr, c.csize);
    return launch_cluster(fn, const_cast<ChainArgs*>(&a), blocks, 1u << (logn - lc - c.lr),
                          3 * (sizeof(uint64_t) << (logn - lc)), c.csize, s);
}

}  // namespace axhel_impl
