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
// block when S > 1, or TG adjacent contiguous blocks when S == 1.
//
// Each thread holds R = 2^LR elements of one group in registers and applies
// LR consecutive stages to them per round.  The first round loads straight
// from global memory and the last round stores straight back; shared memory
// (XOR-swizzled, bank-conflict free) is used only to exchange elements between rounds,
// with one barrier per exchange.  Global accesses are coalesced: in strided
// tiles consecutive lanes take consecutive columns; in contiguous tiles a
// round whose register bits are the low bits reads R consecutive words per
// thread as 16-byte vectors, and the other rounds read runs of 2^lo words.
//
// Every butterfly is exactly the reference's (ForwardButterflyNative /
// InverseButterflyNative, axhel/ntt/ntt-internal.hpp:20-49, and the final
// inverse stage of axhel/ntt/ntt-native.cpp:126-141), applied to the same
// element pairs with the same twiddles in the same stage order, so outputs
// are bit-identical, lazy ranges included.  Twiddle indices:
//   forward stage t, position p : fwd[2^t + (p >> (logn - t))]      (ntt-native.cpp:39)
//   inverse stage s, position p : inv[1 + N - N/2^s + (p >> (s+1))]  (ntt-native.cpp:84, the
//                                 sequential root_index over the blocks of each stage)
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <utility>

#include "internal.h"
#include "modarith.cuh"

namespace axhel_impl {

using namespace axhel_dev;

// Threads per CTA allowed for a register depth: 32 elements per thread need
// more than the 128 registers a 512-thread launch bound leaves.
constexpr int max_threads(int LR) { return LR >= 5 ? 256 : 512; }

template <int LG, int LR>
constexpr int num_rounds()
{
    return (LG + LR - 1) / LR;
}

// Lowest in-group bit held in registers during round RD.  Forward rounds walk
// the bits from the top, inverse rounds from the bottom; a short final round
// re-covers already processed bits so every round holds LR bits.
template <bool INV, int LG, int LR, int RD>
constexpr int round_lo()
{
    if constexpr (INV) {
        return (RD * LR < LG - LR) ? RD * LR : LG - LR;
    } else {
        return (LG - (RD + 1) * LR > 0) ? LG - (RD + 1) * LR : 0;
    }
}

// XOR swizzle of the in-group index for register depth LR: the low 4 bits
// (the 8-byte bank pair among 16) are flipped by index bits LR..LR+3.  In a
// round whose register bits start at lo < 4, the 16 lanes of a half-warp vary
// in index bits [0, lo) and [lo + LR, LR + 4); the shift by LR lands the
// latter on [lo, 4), so every round's access hits 16 distinct bank pairs.
// (A bijection: each flipped bit is flipped by bits above it.)
template <int LR>
__device__ __forceinline__ uint32_t swz(uint32_t r)
{
    return r ^ ((r >> LR) & 15u);
}

// Shared-memory slot of in-group index r: groups are stored unpadded, G words
// each; `hmask` (per thread, below) XORs the group's varying bits into the
// bank pairs the element bits leave free, so half-warps that span several
// groups stay conflict-free too.
template <int LG, int LR>
__device__ __forceinline__ uint32_t slot(uint32_t r, uint32_t hmask)
{
    if constexpr (LG < 4) return r;
    return swz<LR>(r) ^ hmask;
}

// Group bits of a half-warp's lanes sit above the element bits: strided tiles
// put the group first in the lane index (lgtg bits), contiguous tiles the
// thread-in-group first (LG - LR bits).
template <int LG, int LR>
__device__ __forceinline__ uint32_t group_mask(bool strided, uint32_t lgtg, uint32_t gi)
{
    const uint32_t nk = strided ? (lgtg >= 4 ? 0u : 4u - lgtg) : ((LG - LR) >= 4 ? 4u : (uint32_t)(LG - LR));
    return (gi << nk) & 15u;
}

// Per-CTA tile geometry.
struct Tile {
    uint64_t limb;  // limb index in the batch
    uint64_t g0;    // first group of the tile within the limb
    uint64_t base;  // word offset (in the limb) of element (gi = 0, r = 0)
    uint32_t lgS;   // log2 group stride in words
    uint32_t lgtg;  // log2 groups per tile
    bool strided;   // S > 1
};

// Tile `tile_in_limb` of limb `limb` for a pass with group stride 2^lgS and
// 2^lgtg groups per tile.
template <int LG>
__device__ __forceinline__ Tile make_tile(uint32_t lgS, uint32_t lgtg, uint64_t limb, uint64_t tile_in_limb)
{
    Tile t;
    t.limb = limb;
    t.g0 = tile_in_limb << lgtg;
    t.lgS = lgS;
    t.lgtg = lgtg;
    t.strided = lgS != 0;
    if (t.strided) {
        const uint64_t blk = t.g0 >> lgS, col = t.g0 & ((1ull << lgS) - 1);
        t.base = (blk << (LG + lgS)) + col;
    } else {
        t.base = t.g0 << LG;
    }
    return t;
}

template <int LG>
__device__ __forceinline__ uint64_t tile_blk(const Tile& t, uint32_t gi)
{
    return t.strided ? (t.g0 >> t.lgS) : (t.g0 + gi);
}

// Thread -> (group in tile, thread in group).  Column-fastest when strided so
// a warp touches consecutive columns; thread-in-group-fastest otherwise.
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

// Highest thread-in-group bit (k) whose in-group bit changes between rounds
// RD-1 and RD (-1 if none).  Element r sits in thread k(r) = r's bits below
// the register window, then those above it shifted down by LR; bits move
// between k and the registers, or between k positions, only up to here.
template <bool INV, int LG, int LR, int RD>
constexpr int exchange_max_pos()
{
    constexpr int lp = round_lo<INV, LG, LR, RD - 1>(), ln = round_lo<INV, LG, LR, RD>();
    int m = -1;
    for (int b = 0; b < LG; ++b) {
        const bool rp = b >= lp && b < lp + LR, rn = b >= ln && b < ln + LR;
        const int pp = rp ? -1 : (b < lp ? b : b - LR), pn = rn ? -1 : (b < ln ? b : b - LR);
        if (pp != pn) m = (pp > m ? pp : m) > pn ? (pp > m ? pp : m) : pn;
    }
    return m;
}

// limb mod n, the limb's modulus context.  Limb indexes below 2^32 (every
// real batch) take the 32-bit division, a fraction of the 64-bit one's
// instructions.
__device__ __forceinline__ uint32_t limb_mod(uint64_t limb, uint32_t n)
{
    return (limb >> 32) == 0 ? (uint32_t)limb % n : (uint32_t)(limb % n);
}

// Lane shift of k in the thread index: 0 for contiguous tiles (thread =
// group * threads-per-group + k), log2 groups per tile for strided ones
// (thread = group + k * groups); 32 for CTAs under one warp, which always
// synchronize the whole CTA.
__device__ __forceinline__ uint32_t lane_shift(bool strided, uint32_t lgtg)
{
    return blockDim.x >= 32 ? (strided ? lgtg : 0u) : 32u;
}

// In-group index of register 0 for register bits [lo, lo + LR).
template <int LR>
__device__ __forceinline__ uint32_t round_base(uint32_t k, int lo)
{
    return ((k >> lo) << (lo + LR)) | (k & ((1u << lo) - 1));
}

// ------------------------------------------------------- global <-> registers

// Loads with CG = true bypass L1 (ld.global.cg): used when the data was
// written by other CTAs of the same launch (the persistent batch kernel).
template <bool CG>
__device__ __forceinline__ uint64_t ld64(const uint64_t* p)
{
    if constexpr (CG) return __ldcg(reinterpret_cast<const unsigned long long*>(p));
    return *p;
}
template <bool CG>
__device__ __forceinline__ ulonglong2 ld128(const ulonglong2* p)
{
    if constexpr (CG) return __ldcg(p);
    return *p;
}

template <int LG, int LR, int LO, bool CG = false>
__device__ __forceinline__ void load_global(uint64_t (&v)[1 << LR], const uint64_t* __restrict__ limb_src,
                                            const Tile& t, uint32_t gi, uint32_t rb, bool vec_ok)
{
    constexpr int R = 1 << LR;
    if (t.strided) {
        const uint64_t* p = limb_src + t.base + gi + ((uint64_t)rb << t.lgS);
#pragma unroll
        for (int i = 0; i < R; ++i) v[i] = ld64<CG>(p + ((uint64_t)i << (LO + t.lgS)));
    } else if (LO == 0 && vec_ok) {
        const ulonglong2* p = reinterpret_cast<const ulonglong2*>(limb_src + t.base + ((uint64_t)gi << LG) + rb);
#pragma unroll
        for (int i = 0; i < R / 2; ++i) {
            const ulonglong2 w = ld128<CG>(p + i);
            v[2 * i] = w.x;
            v[2 * i + 1] = w.y;
        }
    } else {
        const uint64_t* p = limb_src + t.base + ((uint64_t)gi << LG) + rb;
#pragma unroll
        for (int i = 0; i < R; ++i) v[i] = ld64<CG>(p + (i << LO));
    }
}

template <int LG, int LR, int LO>
__device__ __forceinline__ void store_global(const uint64_t (&v)[1 << LR], uint64_t* __restrict__ limb_dst,
                                             const Tile& t, uint32_t gi, uint32_t rb, bool vec_ok)
{
    constexpr int R = 1 << LR;
    if (t.strided) {
        uint64_t* p = limb_dst + t.base + gi + ((uint64_t)rb << t.lgS);
#pragma unroll
        for (int i = 0; i < R; ++i) p[(uint64_t)i << (LO + t.lgS)] = v[i];
    } else if (LO == 0 && vec_ok) {
        ulonglong2* p = reinterpret_cast<ulonglong2*>(limb_dst + t.base + ((uint64_t)gi << LG) + rb);
#pragma unroll
        for (int i = 0; i < R / 2; ++i) p[i] = make_ulonglong2(v[2 * i], v[2 * i + 1]);
    } else {
        uint64_t* p = limb_dst + t.base + ((uint64_t)gi << LG) + rb;
#pragma unroll
        for (int i = 0; i < R; ++i) p[i << LO] = v[i];
    }
}

// ------------------------------------------------------------------ stages

// Forward round RD on registers: stage bits hi-1 .. hi-nb of the in-group
// index (largest gap first); registers hold bits [lo, lo + LR).
template <int LG, int LR, int RD>
__device__ __forceinline__ void fwd_stages(uint64_t (&v)[1 << LR], uint32_t rbase, uint64_t blk, uint32_t s0,
                                           const ulonglong2* __restrict__ tw, uint64_t q, uint64_t q2)
{
    constexpr int R = 1 << LR;
    constexpr int hi = LG - RD * LR;
    constexpr int nb = hi < LR ? hi : LR;
    constexpr int lo = round_lo<false, LG, LR, RD>();
#pragma unroll
    for (int bb = 0; bb < nb; ++bb) {
        const int b = hi - 1 - bb;  // in-group bit = butterfly span
        const int rb = b - lo;      // register bit
        const uint32_t t = s0 + (LG - 1 - b);
        // the twiddles of this stage are consecutive: rbase's register bits
        // are zero, so (rbase | j << (b+1)) >> (b+1) = (rbase >> (b+1)) + j
        const ulonglong2* tws = tw + (1ull << t) + (blk << (LG - 1 - b)) + (rbase >> (b + 1));
#pragma unroll
        for (int j = 0; j < (R >> (rb + 1)); ++j) {
            const ulonglong2 w = __ldg(tws + j);
#pragma unroll
            for (int l = 0; l < (1 << rb); ++l) {
                const int i0 = (j << (rb + 1)) | l;
                fwd_butterfly(v[i0], v[i0 | (1 << rb)], w.x, w.y, q, q2);
            }
        }
    }
}

// Inverse round RD on registers: stage bits b0 .. b1-1 (smallest gap first).
// With `last` set the pass holds global stage logn-1, the N^-1 final stage.
template <int LG, int LR, int RD>
__device__ __forceinline__ void inv_stages(uint64_t (&v)[1 << LR], uint32_t rbase, uint64_t blk, uint32_t s0,
                                           uint64_t n, const ulonglong2* __restrict__ tw, uint64_t q, uint64_t q2,
                                           bool last, const ModCtx* cx)
{
    constexpr int R = 1 << LR;
    constexpr int b0 = RD * LR;
    constexpr int b1 = (b0 + LR < LG) ? b0 + LR : LG;
    constexpr int lo = round_lo<true, LG, LR, RD>();
#pragma unroll
    for (int b = b0; b < b1; ++b) {
        const int rb = b - lo;
        if (b == LG - 1 && last) {
            const uint64_t ninv = cx->ninv, ninv_q = cx->ninv_q, sr = cx->sroot, sr_q = cx->sroot_q;
#pragma unroll
            for (int j = 0; j < (R >> (rb + 1)); ++j)
#pragma unroll
                for (int l = 0; l < (1 << rb); ++l) {
                    const int i0 = (j << (rb + 1)) | l;
                    inv_final_butterfly(v[i0], v[i0 | (1 << rb)], ninv, ninv_q, sr, sr_q, q, q2);
                }
        } else {
            const uint32_t s = s0 + b;
            const ulonglong2* tws = tw + (1 + n - (n >> s)) + (blk << (LG - b - 1)) + (rbase >> (b + 1));
#pragma unroll
            for (int j = 0; j < (R >> (rb + 1)); ++j) {
                const ulonglong2 w = __ldg(tws + j);
#pragma unroll
                for (int l = 0; l < (1 << rb); ++l) {
                    const int i0 = (j << (rb + 1)) | l;
                    inv_butterfly(v[i0], v[i0 | (1 << rb)], w.x, w.y, q, q2);
                }
            }
        }
    }
}

// Register exchange between rounds RD-1 and RD through shared memory.  Each
// thread writes back the slots it held and reads its next slots; the slot
// sets of one round are disjoint across threads, so one barrier suffices.
template <bool INV, int LG, int LR, int RD>
__device__ __forceinline__ void exchange(uint64_t (&v)[1 << LR], uint64_t* smg, uint32_t k, uint32_t hmask,
                                         uint32_t lsh)
{
    constexpr int R = 1 << LR;
    constexpr int lp = round_lo<INV, LG, LR, RD - 1>();
    constexpr int ln = round_lo<INV, LG, LR, RD>();
    constexpr int mp = exchange_max_pos<INV, LG, LR, RD>();
    const uint32_t bp = round_base<LR>(k, lp), bn = round_base<LR>(k, ln);
#pragma unroll
    for (int i = 0; i < R; ++i) smg[slot<LG, LR>(bp | ((uint32_t)i << lp), hmask)] = v[i];
    // Every thread writes the slots it read at the previous exchange, so when
    // all changed k bits are lane bits (the inner stages) the elements only
    // move inside a warp and a warp barrier orders them.  (Uniform branch.)
    if (mp + (int)lsh < 5)
        __syncwarp();
    else
        __syncthreads();
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = smg[slot<LG, LR>(bn | ((uint32_t)i << ln), hmask)];
}

// Rounds 1 .. NR-1 (round 0 runs on the freshly loaded registers).
template <int LG, int LR, int... RD>
__device__ __forceinline__ void fwd_rest(std::integer_sequence<int, RD...>, uint64_t (&v)[1 << LR], uint64_t* smg,
                                         uint32_t k, uint32_t hmask, uint32_t lsh, uint64_t blk, uint32_t s0,
                                         const ulonglong2* tw, uint64_t q, uint64_t q2)
{
    ((exchange<false, LG, LR, RD + 1>(v, smg, k, hmask, lsh),
      fwd_stages<LG, LR, RD + 1>(v, round_base<LR>(k, round_lo<false, LG, LR, RD + 1>()), blk, s0, tw, q, q2)),
     ...);
}

template <int LG, int LR, int... RD>
__device__ __forceinline__ void inv_rest(std::integer_sequence<int, RD...>, uint64_t (&v)[1 << LR], uint64_t* smg,
                                         uint32_t k, uint32_t hmask, uint32_t lsh, uint64_t blk, uint32_t s0,
                                         uint64_t n, const ulonglong2* tw, uint64_t q, uint64_t q2, bool last,
                                         const ModCtx* cx)
{
    ((exchange<true, LG, LR, RD + 1>(v, smg, k, hmask, lsh),
      inv_stages<LG, LR, RD + 1>(v, round_base<LR>(k, round_lo<true, LG, LR, RD + 1>()), blk, s0, n, tw, q, q2,
                                 last, cx)),
     ...);
}

template <bool INV, int LG, int LR>
__device__ __forceinline__ void run_rounds(uint64_t (&v)[1 << LR], uint64_t* smg, uint32_t k, uint32_t hmask,
                                           uint32_t lsh, uint64_t blk, uint32_t s0, uint64_t n, const ModCtx* cx,
                                           uint64_t q, uint64_t q2, bool last)
{
    constexpr int NR = num_rounds<LG, LR>();
    if constexpr (INV) {
        inv_stages<LG, LR, 0>(v, round_base<LR>(k, round_lo<true, LG, LR, 0>()), blk, s0, n, cx->inv, q, q2, last,
                              cx);
        inv_rest<LG, LR>(std::make_integer_sequence<int, NR - 1>{}, v, smg, k, hmask, lsh, blk, s0, n, cx->inv, q,
                         q2, last, cx);
    } else {
        fwd_stages<LG, LR, 0>(v, round_base<LR>(k, round_lo<false, LG, LR, 0>()), blk, s0, cx->fwd, q, q2);
        fwd_rest<LG, LR>(std::make_integer_sequence<int, NR - 1>{}, v, smg, k, hmask, lsh, blk, s0, cx->fwd, q, q2);
    }
}

// ------------------------------------------------------------------ kernels

// Dyadic product of the registers (round with register bits at LO) with the
// multiplicand at the same positions: EltwiseMulModNative<4>
// (eltwise-mul-mod.cpp:40-60), both operands in [0, 4q), result in [0, q).
template <int LG, int LR, int LO, bool CG>
__device__ __forceinline__ void mul_operand(uint64_t (&v)[1 << LR], const uint64_t* __restrict__ limb_m,
                                            const Tile& t, uint32_t gi, uint32_t k, const ModCtx* cx, bool vec_ok)
{
    uint64_t m[1 << LR];
    load_global<LG, LR, LO, CG>(m, limb_m, t, gi, round_base<LR>(k, LO),
                                vec_ok && (reinterpret_cast<uintptr_t>(limb_m) & 15) == 0);
    const uint64_t q = cx->q, mu = cx->mu;
    const uint32_t shift = cx->shift;
#pragma unroll
    for (int i = 0; i < (1 << LR); ++i)
        v[i] = barrett_mul(reduce_input<4>(v[i], q), reduce_input<4>(m[i], q), q, mu, shift);
}

// One tile of a pass: stages [s0, s0 + LG) of limb `limb`.  `sm` holds
// 2^lgtg groups of 2^LG words; all threads of the CTA take part.  With MUL,
// flags kPreMul / kPostMul multiply by `operand` (MulMod<4>) after the load /
// before the store.
template <bool INV, int LG, int LR, bool CG, bool MUL = false>
__device__ __forceinline__ void pass_tile(const uint64_t* src, uint64_t* dst, const ModCtx* cx, uint32_t logn,
                                          uint32_t s0, uint32_t lgtg, uint64_t limb, uint64_t tile_in_limb,
                                          uint32_t flags, uint64_t* sm, const uint64_t* operand = nullptr)
{
    constexpr int R = 1 << LR;
    constexpr int NR = num_rounds<LG, LR>();
    constexpr int LO_FIRST = round_lo<INV, LG, LR, 0>();
    constexpr int LO_LAST = round_lo<INV, LG, LR, NR - 1>();
    const uint32_t lgS = INV ? s0 : (logn - s0 - LG);
    const Tile t = make_tile<LG>(lgS, lgtg, limb, tile_in_limb);
    const uint64_t q = cx->q, q2 = cx->q2;
    const uint64_t n = 1ull << logn;
    const uint64_t* lsrc = src + (limb << logn);
    uint64_t* ldst = dst + (limb << logn);
    const bool vec_ok = ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0;

    uint32_t gi, k;
    thread_role<LG, LR>(t, gi, k);
    const uint64_t blk = tile_blk<LG>(t, gi);

    uint64_t v[R];
    load_global<LG, LR, LO_FIRST, CG>(v, lsrc, t, gi, round_base<LR>(k, LO_FIRST), vec_ok);
    if (flags & kPreCsub2q) {
#pragma unroll
        for (int i = 0; i < R; ++i) v[i] = csub_lazy(v[i], q2);
    }
    if constexpr (MUL)
        if (flags & kPreMul) mul_operand<LG, LR, LO_FIRST, CG>(v, operand + (limb << logn), t, gi, k, cx, vec_ok);
    run_rounds<INV, LG, LR>(v, sm + (gi << LG), k, group_mask<LG, LR>(t.strided, lgtg, gi),
                            lane_shift(t.strided, lgtg), blk, s0, n, cx, q, q2, (flags & kLastPass) != 0);
    if (flags & kPostNorm) {
#pragma unroll
        for (int i = 0; i < R; ++i) v[i] = INV ? csub_lazy(v[i], q) : csub_lazy(csub_lazy(v[i], q2), q);
    }
    if constexpr (MUL)
        if (flags & kPostMul) mul_operand<LG, LR, LO_LAST, CG>(v, operand + (limb << logn), t, gi, k, cx, vec_ok);
    store_global<LG, LR, LO_LAST>(v, ldst, t, gi, round_base<LR>(k, LO_LAST), vec_ok);
}

template <bool INV, int LG, int LR>
__global__ void __launch_bounds__(max_threads(LR)) ntt_pass_kernel(const __grid_constant__ PassArgs a)
{
    extern __shared__ uint64_t sm[];
    const uint32_t lgtg = __ffs(a.tg) - 1;
    const uint32_t lg_tiles = a.logn - LG - lgtg;  // log2 tiles per limb
    const uint64_t tile = blockIdx.x;
    const uint64_t limb = tile >> lg_tiles;
    pass_tile<INV, LG, LR, false>(a.src, a.dst, a.ctx[limb_mod(limb, a.nctx)], a.logn, a.s0, lgtg, limb,
                                  tile & ((1ull << lg_tiles) - 1), a.flags, sm);
}

// The same pass with the dyadic product of kPreMul / kPostMul: a kernel of
// its own, so that the product's registers do not count against the plain
// passes.
template <bool INV, int LG, int LR>
__global__ void __launch_bounds__(max_threads(LR)) ntt_pass_mul_kernel(const __grid_constant__ PassArgs a)
{
    extern __shared__ uint64_t sm[];
    const uint32_t lgtg = __ffs(a.tg) - 1;
    const uint32_t lg_tiles = a.logn - LG - lgtg;
    const uint64_t tile = blockIdx.x;
    const uint64_t limb = tile >> lg_tiles;
    pass_tile<INV, LG, LR, false, true>(a.src, a.dst, a.ctx[limb_mod(limb, a.nctx)], a.logn, a.s0, lgtg, limb,
                                        tile & ((1ull << lg_tiles) - 1), a.flags, sm, a.operand);
}

// Fused column pass of an INTT -> op -> NTT chain: the inverse's last pass
// (stages logn-LG .. logn-1, incl. the N^-1 final stage) and the forward's
// first pass (stages 0 .. LG-1) act on the same groups p = r*S + col, and the
// inverse's last round holds the same register bits as the forward's first
// round, so the element-wise op runs in registers between them.
template <int LG, int LR, bool CG>
__device__ __forceinline__ void chain_tile(const uint64_t* src, uint64_t* dst, const uint64_t* operand,
                                           const ModCtx* cx, uint32_t op, uint64_t scalar, uint32_t logn,
                                           uint32_t lgtg, uint64_t limb, uint64_t tile_in_limb, uint32_t flags,
                                           uint64_t* sm)
{
    constexpr int R = 1 << LR;
    constexpr int NR = num_rounds<LG, LR>();
    constexpr int LO_FIRST = round_lo<true, LG, LR, 0>();
    constexpr int LO_MID = round_lo<true, LG, LR, NR - 1>();
    constexpr int LO_LAST = round_lo<false, LG, LR, NR - 1>();
    static_assert(LO_MID == round_lo<false, LG, LR, 0>(), "inverse last round and forward first round differ");
    const Tile t = make_tile<LG>(logn - LG, lgtg, limb, tile_in_limb);
    const uint64_t q = cx->q, q2 = cx->q2;
    const uint64_t n = 1ull << logn;
    const uint64_t* lsrc = src + (limb << logn);
    uint64_t* ldst = dst + (limb << logn);
    const bool vec_ok = ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst) |
                          reinterpret_cast<uintptr_t>(operand)) & 15) == 0;

    uint32_t gi, k;
    thread_role<LG, LR>(t, gi, k);
    const uint64_t blk = tile_blk<LG>(t, gi);
    uint64_t* smg = sm + (gi << LG);
    const uint32_t hmask = group_mask<LG, LR>(t.strided, lgtg, gi);
    const uint32_t lsh = lane_shift(t.strided, lgtg);

    uint64_t v[R];
    load_global<LG, LR, LO_FIRST, CG>(v, lsrc, t, gi, round_base<LR>(k, LO_FIRST), vec_ok);
    if (flags & kPreCsub2q) {
#pragma unroll
        for (int i = 0; i < R; ++i) v[i] = csub_lazy(v[i], q2);
    }
    run_rounds<true, LG, LR>(v, smg, k, hmask, lsh, blk, logn - LG, n, cx, q, q2, true);

    // Element-wise op on the inverse output (lazy [0, 2q)) with factor-2
    // inputs: EltwiseMulModNative<2> / EltwiseFMAModNative<2> formulas.
    const uint64_t mu = cx->mu;
    const uint32_t shift = cx->shift;
    const uint32_t rb = round_base<LR>(k, LO_MID);
    if (op == kChainMul) {
        uint64_t m[R];
        load_global<LG, LR, LO_MID, false>(m, operand + (limb << logn), t, gi, rb, vec_ok);
#pragma unroll
        for (int i = 0; i < R; ++i)
            v[i] = barrett_mul(reduce_input<2>(v[i], q), reduce_input<2>(m[i], q), q, mu, shift);
    } else if (op == kChainFma) {
        const uint64_t sc = reduce_input<2>(scalar, q);
#pragma unroll
        for (int i = 0; i < R; ++i) v[i] = barrett_mul(reduce_input<2>(v[i], q), sc, q, mu, shift);
        if (operand) {
            uint64_t m[R];
            load_global<LG, LR, LO_MID, false>(m, operand + (limb << logn), t, gi, rb, vec_ok);
#pragma unroll
            for (int i = 0; i < R; ++i) v[i] = csub(v[i] + reduce_input<2>(m[i], q), q);
        }
    }

    // The forward's first pass: stages 0 .. LG-1 of block 0.
    fwd_stages<LG, LR, 0>(v, rb, 0, 0, cx->fwd, q, q2);
    fwd_rest<LG, LR>(std::make_integer_sequence<int, NR - 1>{}, v, smg, k, hmask, lsh, 0, 0, cx->fwd, q, q2);
    if (flags & kPostNorm) {
#pragma unroll
        for (int i = 0; i < R; ++i) v[i] = csub_lazy(csub_lazy(v[i], q2), q);
    }
    store_global<LG, LR, LO_LAST>(v, ldst, t, gi, round_base<LR>(k, LO_LAST), vec_ok);
}

// Fused row pass of an NTT -> MulMod -> INTT product (the polynomial product
// in evaluation form, SEAL's multiply_plain): the forward's last pass (stages
// logn-LG .. logn-1) and the inverse's first pass (stages 0 .. LG-1) act on
// the same contiguous groups of 2^LG words, and the forward's last round
// holds the same register bits as the inverse's first round (the low LR
// bits), so the dyadic product runs in registers between them.  The product
// is EltwiseMulModNative<4> (axhel/eltwise/eltwise-mul-mod.cpp:18-63) of the
// forward's lazy output and the multiplicand, both in [0, 4q).  With LG ==
// logn (one pass each way) the tile also holds the inverse's N^-1 stage.
template <int LG, int LR>
__device__ __forceinline__ void product_tile(const uint64_t* src, uint64_t* dst, const uint64_t* operand,
                                             const ModCtx* cx, uint32_t logn, uint32_t lgtg, uint64_t limb,
                                             uint64_t tile_in_limb, uint32_t flags, uint64_t* sm)
{
    constexpr int R = 1 << LR;
    constexpr int NR = num_rounds<LG, LR>();
    constexpr int LO_FIRST = round_lo<false, LG, LR, 0>();
    constexpr int LO_MID = round_lo<false, LG, LR, NR - 1>();
    constexpr int LO_LAST = round_lo<true, LG, LR, NR - 1>();
    static_assert(LO_MID == round_lo<true, LG, LR, 0>(), "forward last round and inverse first round differ");
    const Tile t = make_tile<LG>(0, lgtg, limb, tile_in_limb);
    const uint64_t q = cx->q, q2 = cx->q2;
    const uint64_t n = 1ull << logn;
    const bool vec_ok = ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst) |
                          reinterpret_cast<uintptr_t>(operand)) & 15) == 0;
    uint32_t gi, k;
    thread_role<LG, LR>(t, gi, k);
    const uint64_t blk = tile_blk<LG>(t, gi);
    uint64_t* smg = sm + (gi << LG);
    const uint32_t hmask = group_mask<LG, LR>(t.strided, lgtg, gi);
    const uint32_t lsh = lane_shift(t.strided, lgtg);

    uint64_t v[R];
    load_global<LG, LR, LO_FIRST, false>(v, src + (limb << logn), t, gi, round_base<LR>(k, LO_FIRST), vec_ok);
    run_rounds<false, LG, LR>(v, smg, k, hmask, lsh, blk, logn - LG, n, cx, q, q2, false);
    {
        uint64_t m[R];
        load_global<LG, LR, LO_MID, false>(m, operand + (limb << logn), t, gi, round_base<LR>(k, LO_MID), vec_ok);
        const uint64_t mu = cx->mu;
        const uint32_t shift = cx->shift;
#pragma unroll
        for (int i = 0; i < R; ++i)
            v[i] = barrett_mul(reduce_input<4>(v[i], q), reduce_input<4>(m[i], q), q, mu, shift);
    }
    run_rounds<true, LG, LR>(v, smg, k, hmask, lsh, blk, 0, n, cx, q, q2, (flags & kLastPass) != 0);
    if (flags & kPostNorm) {
#pragma unroll
        for (int i = 0; i < R; ++i) v[i] = csub_lazy(v[i], q);
    }
    store_global<LG, LR, LO_LAST>(v, dst + (limb << logn), t, gi, round_base<LR>(k, LO_LAST), vec_ok);
}

// Kernel of the fused product pass: one CTA per tile of product_tile above.
template <int LG, int LR>
__global__ void __launch_bounds__(max_threads(LR)) ntt_product_kernel(const __grid_constant__ ChainArgs c)
{
    extern __shared__ uint64_t sm[];
    const PassArgs& a = c.pass;
    const uint32_t lgtg = __ffs(a.tg) - 1;
    const uint32_t lg_tiles = a.logn - LG - lgtg;
    const uint64_t tile = blockIdx.x;
    const uint64_t limb = tile >> lg_tiles;
    product_tile<LG, LR>(a.src, a.dst, c.operand, a.ctx[limb_mod(limb, a.nctx)], a.logn, lgtg, limb,
                         tile & ((1ull << lg_tiles) - 1), a.flags, sm);
}

// Kernel of the fused chain pass: one CTA per tile of chain_tile above; the
// modulus context and the FMA scalar follow the limb.
template <int LG, int LR>
__global__ void __launch_bounds__(max_threads(LR)) ntt_chain_kernel(const __grid_constant__ ChainArgs c)
{
    extern __shared__ uint64_t sm[];
    const PassArgs& a = c.pass;
    const uint32_t lgtg = __ffs(a.tg) - 1;
    const uint32_t lg_tiles = a.logn - LG - lgtg;
    const uint64_t tile = blockIdx.x;
    const uint64_t limb = tile >> lg_tiles;
    const uint32_t mi = limb_mod(limb, a.nctx);
    chain_tile<LG, LR, false>(a.src, a.dst, c.operand, a.ctx[mi], c.op, c.scalar[mi], a.logn, lgtg, limb,
                              tile & ((1ull << lg_tiles) - 1), a.flags, sm);
}

}  // namespace axhel_impl
