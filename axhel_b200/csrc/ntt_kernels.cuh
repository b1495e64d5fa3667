// NTT pass kernels for sm_100a.
//
// A transform of N = 2^logn points is split into passes; a pass runs the
// reference's radix-2 stages [s0, s0 + LG) on "groups" of G = 2^LG elements
// that only interact with each other inside those stages:
//
//   element r of group (blk, col) sits at  p = blk*G*S + r*S + col
//
// with stride S = 2^(logn - s0 - LG) for the forward (Cooley-Tukey, large gaps
// first) and S = 2^s0 for the inverse (Gentleman-Sande, small gaps first).
// A CTA takes TG consecutive groups (a "tile"): TG adjacent columns of one
// block when S > 1 (coalesced rows of TG words), or TG adjacent contiguous
// blocks when S == 1.  The tile is staged in shared memory (padded, XOR
// swizzled), then processed in rounds: each thread holds R = 2^LR elements in
// registers and applies LR consecutive stages to them before the next
// shared-memory exchange.
//
// Every butterfly is exactly the reference's (ForwardButterflyNative /
// InverseButterflyNative, axhel/ntt/ntt-internal.hpp:20-49, and the final
// inverse stage of axhel/ntt/ntt-native.cpp:126-141), applied to the same
// element pairs with the same twiddles in the same stage order, so outputs
// are bit-identical, lazy ranges included.  Twiddle indices:
//   forward stage t, position p : fwd[2^t + (p >> (logn - t))]      (ntt-native.cpp:39)
//   inverse stage s, position p : inv[1 + N - N/2^s + (p >> (s+1))]  (ntt-native.cpp:84, sequential
//                                 root_index over blocks i of each stage)
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <utility>

#include "internal.h"
#include "modarith.cuh"

namespace axhel_impl {

using namespace axhel_dev;

// XOR swizzle of the in-group index: flips the low 4 bits by bits 4..7 so
// that both unit-stride and stride-16 register fetches hit distinct banks.
__device__ __forceinline__ uint32_t swz(uint32_t r) { return r ^ ((r >> 4) & 15u); }

template <int LG>
struct Geo {
    static constexpr int G = 1 << LG;
    static constexpr int GP = G + 1;  // padded group pitch in words
};

// Per-CTA tile geometry, shared by the plain and the fused chain kernels.
struct Tile {
    uint64_t limb;       // limb index in the batch
    uint64_t g0;         // first group of the tile within the limb
    uint64_t base;       // word offset (in the limb) of element (gi = 0, r = 0)
    uint64_t S;          // group stride in words
    uint32_t lgS;
    uint32_t lgtg;       // log2 groups per tile
    bool strided;        // S > 1
};

template <int LG>
__device__ __forceinline__ Tile make_tile(uint32_t logn, uint32_t lgS, uint32_t lgtg)
{
    Tile t;
    const uint64_t groups_per_limb = 1ull << (logn - LG);
    const uint64_t tiles_per_limb = groups_per_limb >> lgtg;
    const uint64_t tile = blockIdx.x;
    t.limb = tile / tiles_per_limb;
    t.g0 = (tile - t.limb * tiles_per_limb) << lgtg;
    t.lgS = lgS;
    t.S = 1ull << lgS;
    t.lgtg = lgtg;
    t.strided = lgS != 0;
    if (t.strided) {
        const uint64_t blk = t.g0 >> lgS, col = t.g0 & (t.S - 1);
        t.base = (blk << (LG + lgS)) + col;
    } else {
        t.base = t.g0 << LG;
    }
    return t;
}

// Word offset in the limb of element (gi, r), and the group's block index.
template <int LG>
__device__ __forceinline__ uint64_t tile_addr(const Tile& t, uint32_t gi, uint32_t r)
{
    return t.strided ? t.base + ((uint64_t)r << t.lgS) + gi : t.base + ((uint64_t)gi << LG) + r;
}
template <int LG>
__device__ __forceinline__ uint64_t tile_blk(const Tile& t, uint32_t gi)
{
    return t.strided ? (t.g0 >> t.lgS) : (t.g0 + gi);
}

// Element e of the tile in memory order -> (gi, r).
template <int LG>
__device__ __forceinline__ void tile_elem(const Tile& t, uint32_t e, uint32_t& gi, uint32_t& r)
{
    if (t.strided) {
        gi = e & ((1u << t.lgtg) - 1);
        r = e >> t.lgtg;
    } else {
        gi = e >> LG;
        r = e & ((1u << LG) - 1);
    }
}

// Thread -> (group in tile, thread in group).  Column-fastest when strided so
// a warp reads consecutive columns; thread-in-group-fastest otherwise.
template <int LG, int LR>
__device__ __forceinline__ void thread_role(const Tile& t, uint32_t& gi, uint32_t& k)
{
    constexpr uint32_t KT = 1u << (LG - LR);
    const uint32_t tid = threadIdx.x;
    if (t.strided) {
        gi = tid & ((1u << t.lgtg) - 1);
        k = tid >> t.lgtg;
    } else {
        gi = tid / KT;
        k = tid % KT;
    }
}

// ------------------------------------------------------------------ rounds

// Forward round RD: stage bits hi-1 .. hi-nb of the in-group index (largest
// gap first).  Registers hold bits [lo, lo + LR) of the index.
template <int LG, int LR, int RD>
__device__ __forceinline__ void fwd_round(uint64_t* smg, uint32_t k, uint64_t blk, uint32_t s0,
                                          const ulonglong2* __restrict__ tw, uint64_t q, uint64_t q2)
{
    constexpr int R = 1 << LR;
    constexpr int hi = LG - RD * LR;
    constexpr int nb = hi < LR ? hi : LR;
    constexpr int lo = hi - LR > 0 ? hi - LR : 0;
    const uint32_t rbase = ((k >> lo) << (lo + LR)) | (k & ((1u << lo) - 1));
    uint64_t v[R];
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = smg[swz(rbase | ((uint32_t)i << lo))];
#pragma unroll
    for (int bb = 0; bb < nb; ++bb) {
        const int b = hi - 1 - bb;  // in-group bit = butterfly span
        const int rb = b - lo;      // register bit
        const uint32_t t = s0 + (LG - 1 - b);
#pragma unroll
        for (int j = 0; j < (R >> (rb + 1)); ++j) {
            const uint32_t rrep = rbase | ((uint32_t)(j << (rb + 1)) << lo);
            const uint64_t idx = (1ull << t) + (blk << (LG - 1 - b)) + (rrep >> (b + 1));
            const ulonglong2 w = __ldg(tw + idx);
#pragma unroll
            for (int l = 0; l < (1 << rb); ++l) {
                const int i0 = (j << (rb + 1)) | l;
                fwd_butterfly(v[i0], v[i0 | (1 << rb)], w.x, w.y, q, q2);
            }
        }
    }
#pragma unroll
    for (int i = 0; i < R; ++i) smg[swz(rbase | ((uint32_t)i << lo))] = v[i];
}

// Inverse round RD: stage bits b0 .. b1-1 (smallest gap first).  When `last`
// is set the pass holds global stage logn-1, which runs the N^-1 final stage.
template <int LG, int LR, int RD>
__device__ __forceinline__ void inv_round(uint64_t* smg, uint32_t k, uint64_t blk, uint32_t s0, uint64_t n,
                                          const ulonglong2* __restrict__ tw, uint64_t q, uint64_t q2, bool last,
                                          uint64_t ninv, uint64_t ninv_q, uint64_t sr, uint64_t sr_q)
{
    constexpr int R = 1 << LR;
    constexpr int b0 = RD * LR;
    constexpr int b1 = (b0 + LR < LG) ? b0 + LR : LG;
    constexpr int lo = (b0 < LG - LR) ? b0 : LG - LR;
    const uint32_t rbase = ((k >> lo) << (lo + LR)) | (k & ((1u << lo) - 1));
    uint64_t v[R];
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = smg[swz(rbase | ((uint32_t)i << lo))];
#pragma unroll
    for (int b = b0; b < b1; ++b) {
        const int rb = b - lo;
        if (b == LG - 1 && last) {
#pragma unroll
            for (int j = 0; j < (R >> (rb + 1)); ++j)
#pragma unroll
                for (int l = 0; l < (1 << rb); ++l) {
                    const int i0 = (j << (rb + 1)) | l;
                    inv_final_butterfly(v[i0], v[i0 | (1 << rb)], ninv, ninv_q, sr, sr_q, q, q2);
                }
        } else {
            const uint32_t s = s0 + b;
            const uint64_t stage_base = 1 + n - (n >> s);
#pragma unroll
            for (int j = 0; j < (R >> (rb + 1)); ++j) {
                const uint32_t rrep = rbase | ((uint32_t)(j << (rb + 1)) << lo);
                const uint64_t idx = stage_base + (blk << (LG - b - 1)) + (rrep >> (b + 1));
                const ulonglong2 w = __ldg(tw + idx);
#pragma unroll
                for (int l = 0; l < (1 << rb); ++l) {
                    const int i0 = (j << (rb + 1)) | l;
                    inv_butterfly(v[i0], v[i0 | (1 << rb)], w.x, w.y, q, q2);
                }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < R; ++i) smg[swz(rbase | ((uint32_t)i << lo))] = v[i];
}

template <int LG, int LR, int... RD>
__device__ __forceinline__ void fwd_rounds(std::integer_sequence<int, RD...>, uint64_t* smg, uint32_t k,
                                           uint64_t blk, uint32_t s0, const ulonglong2* tw, uint64_t q, uint64_t q2)
{
    ((__syncthreads(), fwd_round<LG, LR, RD>(smg, k, blk, s0, tw, q, q2)), ...);
}

template <int LG, int LR, int... RD>
__device__ __forceinline__ void inv_rounds(std::integer_sequence<int, RD...>, uint64_t* smg, uint32_t k,
                                           uint64_t blk, uint32_t s0, uint64_t n, const ulonglong2* tw, uint64_t q,
                                           uint64_t q2, bool last, uint64_t ninv, uint64_t ninv_q, uint64_t sr,
                                           uint64_t sr_q)
{
    ((__syncthreads(), inv_round<LG, LR, RD>(smg, k, blk, s0, n, tw, q, q2, last, ninv, ninv_q, sr, sr_q)), ...);
}

// Threads per CTA allowed for a register depth: 32 elements per thread need
// more than the 128 registers a 512-thread launch bound leaves.
constexpr int max_threads(int LR) { return LR >= 5 ? 256 : 512; }

template <int LG, int LR>
constexpr int num_rounds()
{
    return (LG + LR - 1) / LR;
}

// ------------------------------------------------------------------ kernels

template <bool INV, int LG, int LR>
__global__ void __launch_bounds__(max_threads(LR)) ntt_pass_kernel(const __grid_constant__ PassArgs a)
{
    extern __shared__ uint64_t sm[];
    constexpr int GP = Geo<LG>::GP;
    const uint32_t logn = a.logn;
    const uint32_t lgS = INV ? a.s0 : (logn - a.s0 - LG);
    const uint32_t lgtg = __ffs(a.tg) - 1;
    const Tile t = make_tile<LG>(logn, lgS, lgtg);
    const ModCtx* cx = a.ctx[t.limb % a.nctx];
    const uint64_t q = cx->q, q2 = cx->q2;
    const uint64_t n = 1ull << logn;
    const uint64_t* src = a.src + t.limb * n;
    uint64_t* dst = a.dst + t.limb * n;
    const uint32_t nel = a.tg << LG;
    const bool pre = a.flags & kPreCsub2q;

    for (uint32_t e = threadIdx.x; e < nel; e += blockDim.x) {
        uint32_t gi, r;
        tile_elem<LG>(t, e, gi, r);
        uint64_t x = src[tile_addr<LG>(t, gi, r)];
        if (pre) x = csub(x, q2);
        sm[gi * GP + swz(r)] = x;
    }

    uint32_t gi, k;
    thread_role<LG, LR>(t, gi, k);
    uint64_t* smg = sm + gi * GP;
    const uint64_t blk = tile_blk<LG>(t, gi);
    if constexpr (INV) {
        const bool last = a.flags & kLastPass;
        inv_rounds<LG, LR>(std::make_integer_sequence<int, num_rounds<LG, LR>()>{}, smg, k, blk, a.s0, n, cx->inv,
                           q, q2, last, cx->ninv, cx->ninv_q, cx->sroot, cx->sroot_q);
    } else {
        fwd_rounds<LG, LR>(std::make_integer_sequence<int, num_rounds<LG, LR>()>{}, smg, k, blk, a.s0, cx->fwd, q,
                           q2);
    }
    __syncthreads();

    const bool norm = a.flags & kPostNorm;
    for (uint32_t e = threadIdx.x; e < nel; e += blockDim.x) {
        uint32_t g2, r;
        tile_elem<LG>(t, e, g2, r);
        uint64_t x = sm[g2 * GP + swz(r)];
        if (norm) x = INV ? csub(x, q) : csub(csub(x, q2), q);
        dst[tile_addr<LG>(t, g2, r)] = x;
    }
}

// Fused column pass of an INTT -> op -> NTT chain: the inverse's last pass
// (stages logn-LG .. logn-1, incl. the N^-1 final stage) and the forward's
// first pass (stages 0 .. LG-1) act on the same groups p = r*S + col, so the
// element-wise op runs on the tile in shared memory between them.
template <int LG, int LR>
__global__ void __launch_bounds__(max_threads(LR)) ntt_chain_kernel(const __grid_constant__ ChainArgs c)
{
    extern __shared__ uint64_t sm[];
    constexpr int GP = Geo<LG>::GP;
    const PassArgs& a = c.pass;
    const uint32_t logn = a.logn;
    const uint32_t lgS = logn - LG;
    const uint32_t lgtg = __ffs(a.tg) - 1;
    const Tile t = make_tile<LG>(logn, lgS, lgtg);
    const uint32_t mi = t.limb % a.nctx;
    const ModCtx* cx = a.ctx[mi];
    const uint64_t q = cx->q, q2 = cx->q2;
    const uint64_t n = 1ull << logn;
    const uint64_t* src = a.src + t.limb * n;
    uint64_t* dst = a.dst + t.limb * n;
    const uint32_t nel = a.tg << LG;
    const bool pre = a.flags & kPreCsub2q;

    for (uint32_t e = threadIdx.x; e < nel; e += blockDim.x) {
        uint32_t gi, r;
        tile_elem<LG>(t, e, gi, r);
        uint64_t x = src[tile_addr<LG>(t, gi, r)];
        if (pre) x = csub(x, q2);
        sm[gi * GP + swz(r)] = x;
    }
    uint32_t gi, k;
    thread_role<LG, LR>(t, gi, k);
    uint64_t* smg = sm + gi * GP;
    const uint64_t blk = tile_blk<LG>(t, gi);
    inv_rounds<LG, LR>(std::make_integer_sequence<int, num_rounds<LG, LR>()>{}, smg, k, blk, logn - LG, n, cx->inv,
                       q, q2, true, cx->ninv, cx->ninv_q, cx->sroot, cx->sroot_q);
    __syncthreads();

    // Element-wise op on the inverse output (lazy [0, 2q)), factor-2 inputs.
    const uint64_t* opnd = c.operand ? c.operand + t.limb * n : nullptr;
    const uint64_t mu = cx->mu;
    const uint32_t shift = cx->shift;
    if (c.op == kChainMul) {
        for (uint32_t e = threadIdx.x; e < nel; e += blockDim.x) {
            uint32_t g2, r;
            tile_elem<LG>(t, e, g2, r);
            uint64_t* s = &sm[g2 * GP + swz(r)];
            const uint64_t m = opnd[tile_addr<LG>(t, g2, r)];
            *s = barrett_mul(reduce_input<2>(*s, q), reduce_input<2>(m, q), q, mu, shift);
        }
    } else if (c.op == kChainFma) {
        const uint64_t sc = reduce_input<2>(c.scalar[mi], q);
        for (uint32_t e = threadIdx.x; e < nel; e += blockDim.x) {
            uint32_t g2, r;
            tile_elem<LG>(t, e, g2, r);
            uint64_t* s = &sm[g2 * GP + swz(r)];
            uint64_t v = barrett_mul(reduce_input<2>(*s, q), sc, q, mu, shift);
            if (opnd) {
                v += reduce_input<2>(opnd[tile_addr<LG>(t, g2, r)], q);
                v = csub(v, q);
            }
            *s = v;
        }
    }

    fwd_rounds<LG, LR>(std::make_integer_sequence<int, num_rounds<LG, LR>()>{}, smg, k, 0, 0, cx->fwd, q, q2);
    __syncthreads();

    const bool norm = a.flags & kPostNorm;
    for (uint32_t e = threadIdx.x; e < nel; e += blockDim.x) {
        uint32_t g2, r;
        tile_elem<LG>(t, e, g2, r);
        uint64_t x = sm[g2 * GP + swz(r)];
        if (norm) x = csub(csub(x, q2), q);
        dst[tile_addr<LG>(t, g2, r)] = x;
    }
}

}  // namespace axhel_impl
