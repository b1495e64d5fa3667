// Uneven batches: one persistent launch, or ordinary launches phase by phase.
//
// A batch mixes jobs of different degree N (2^10 .. 2^17), limb count and
// kind: forward NTT, inverse NTT, the fused INTT -> MulMod/FMAMod -> NTT
// chain, and the element-wise Add/Sub/Mul/FMA/ReduceMod.  Every job runs as
// one to three phases of tiles:
//
//   forward : column pass (stages 0..A-1)  -> row pass (stages A..n-1)
//   inverse : row pass (stages 0..B-1)     -> column pass (stages B..n-1, N^-1)
//   chain   : inverse row pass -> fused [inverse column pass, op, forward
//             column pass] -> forward row pass
//   element-wise : one phase, the op on 1024 residues of one limb per tile
//
// with B stages in the contiguous pass, from the autotuner's table per degree
// (default min(9, n - 5): as wide as a tile allows), and A = n - B.  The kernel is persistent (one wave of CTAs
// sized to the device); CTAs take tiles from one atomic counter in
// phase-major order (every phase-0 tile of every job before any phase-1
// tile), so by the time a phase-p tile is taken, every tile it depends on is
// already held by a running CTA.  A CTA claims its next tile while it works
// on the current one (the counter's latency is hidden); the lowest unfinished
// tile is then still always runnable, because everything it waits for has a
// lower index and every CTA holding a tile is resident.  A tile of phase p >= 1 of limb l waits for
// the phase p-1 tiles of the same limb (per-limb completion counters,
// release/acquire at device scope); the wait is bounded and, if it ever runs
// out, the CTA records AXHEL's timeout status in the batch's error word and
// stops.  Data written by other CTAs of the launch is read through L2
// (ld.global.cg), never through a possibly stale L1 line.  A finished tile
// is published as a grid barrier publishes arrival: CTA barrier, then one
// thread's device-scope release increment (cumulative over the stores the
// barrier ordered before it), by a thread of another warp than the one that
// claims and checks the next tile, which waits on nothing before it.
//
// Each tile is 1024 residues: 2^(10-LG) groups of 2^LG for the pass widths
// LG = 5..9 of the degrees 2^10 .. 2^17 (a tile never spans two limbs or two
// blocks), handled by 128 threads x 8 registers (LR = 3) in the persistent
// kernel.  The per-phase launches run one kernel per tile class and pass
// width (64 threads x 16 registers for the 7-stage transform passes), each
// phase's largest entries in launches of their own that take the entry as a
// kernel parameter, side by side on extra streams.
// The same tile functions as the plain kernels run the butterflies
// (ntt_kernels.cuh), so every job's result equals the per-limb calls bit for
// bit.
#include <cuda/atomic>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/axhel_cuda.h"
#include "internal.h"
#include "launch.h"
#include "batch.h"
#include "eltwise_ops.cuh"
#include "ntt_kernels.cuh"

namespace axhel_impl {

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Per-phase pass of a transform job: direction, width and first stage
// (chain: inverse row pass, fused column pass, forward row pass).
struct PhaseCfg {
    bool inv, chain;
    uint32_t lg, s0;
};

inline PhaseCfg phase_cfg(const BatchJob& j, uint32_t p)
{
    PhaseCfg c{false, false, 0, 0};
    if (j.kind == kJobForward) {
        c.lg = p == 0 ? j.lg_col : j.lg_row;
        c.s0 = p == 0 ? 0 : j.lg_col;
    } else if (j.kind == kJobInverse) {
        c.inv = true;
        c.lg = p == 0 ? j.lg_row : j.lg_col;
        c.s0 = p == 0 ? 0 : j.lg_row;
    } else {  // chain
        if (p == 0) {
            c.inv = true;
            c.lg = j.lg_row;
            c.s0 = 0;
        } else if (p == 1) {
            c.chain = true;
            c.lg = j.lg_col;
            c.s0 = j.lg_row;
        } else {
            c.lg = j.lg_row;
            c.s0 = j.lg_col;
        }
    }
    return c;
}

// Element-wise job tile: 1024 residues of one limb, 8 per thread at a
// stride of the CTA width (every warp access is 256 contiguous bytes); all
// loads are issued before the first store.
template <bool HAS_B, class Op>
__device__ __forceinline__ void elt_tile(const ClassEntry& j, uint64_t base, const Op& op)
{
    constexpr int kPer = kBatchTileWords / kBatchThreads;
    uint64_t a[kPer], b[kPer];
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        a[k] = j.src[base + (uint64_t)k * kBatchThreads];
        b[k] = HAS_B ? j.vec[base + (uint64_t)k * kBatchThreads] : 0;
    }
#pragma unroll
    for (int k = 0; k < kPer; ++k) j.dst[base + (uint64_t)k * kBatchThreads] = op(a[k], b[k]);
}

template <bool ADD>
__device__ __forceinline__ void elt_fma(const ClassEntry& j, uint64_t base, uint64_t q, uint64_t mu, uint64_t s,
                                        uint32_t sh)
{
    switch (j.ef) {
    case 1: elt_tile<ADD>(j, base, OpFma<1, ADD>{q, mu, s, sh}); break;
    case 2: elt_tile<ADD>(j, base, OpFma<2, ADD>{q, mu, s, sh}); break;
    case 4: elt_tile<ADD>(j, base, OpFma<4, ADD>{q, mu, s, sh}); break;
    default: elt_tile<ADD>(j, base, OpFma<8, ADD>{q, mu, s, sh}); break;
    }
}

// The element-wise job's op on one tile, with limb `limb`'s modulus.
__device__ __forceinline__ void run_elt_tile(const ClassEntry& j, uint64_t limb, uint64_t til)
{
    const uint32_t mi = limb_mod(limb, j.nmods);
    const ModCtx* cx = j.ctx[mi];
    const uint64_t q = cx->q, mu = cx->mu;
    const uint32_t sh = cx->shift;
    const uint64_t s = j.scalars ? j.scalars[mi] : 0;
    const uint64_t base = (limb << j.logn) + til * kBatchTileWords + threadIdx.x;
    switch (j.eop) {
    case kEltAddVV: elt_tile<true>(j, base, OpAddVV{q}); break;
    case kEltAddVS: elt_tile<false>(j, base, OpAddVS{q, s}); break;
    case kEltSubVV: elt_tile<true>(j, base, OpSubVV{q}); break;
    case kEltSubVS: elt_tile<false>(j, base, OpSubVS{q, s}); break;
    case kEltMul:
        if (j.ef == 1) elt_tile<true>(j, base, OpMul<1>{q, mu, sh});
        else if (j.ef == 2) elt_tile<true>(j, base, OpMul<2>{q, mu, sh});
        else elt_tile<true>(j, base, OpMul<4>{q, mu, sh});
        break;
    case kEltFma: elt_fma<false>(j, base, q, mu, s, sh); break;
    case kEltFmaAdd: elt_fma<true>(j, base, q, mu, s, sh); break;
    default:  // kEltReduce
        switch (j.ef) {
        case 0: elt_tile<false>(j, base, OpReduce<0>{q, mu, sh}); break;
        case 1: elt_tile<false>(j, base, OpReduce<1>{q, mu, sh}); break;
        case 2: elt_tile<false>(j, base, OpReduce<2>{q, mu, sh}); break;
        case 3: elt_tile<false>(j, base, OpReduce<3>{q, mu, sh}); break;
        default: elt_tile<false>(j, base, OpReduce<4>{q, mu, sh}); break;
        }
        break;
    }
}

// One tile of class CLS and pass width LG with LR register stages; the
// entry carries the pass's operands, first stage and flags (built on the
// host from the job).  With LR = 4 a 1024-residue tile takes 64 threads x 16
// registers.  CG: loads bypass L1, for
// data written by other CTAs of the same launch (the persistent kernel); the
// per-phase launches read what an earlier launch wrote and load plainly.
template <int CLS, int LG, int LR, bool CG>
__device__ __forceinline__ void run_class_tile(const ClassEntry& c, uint64_t limb, uint64_t tile_in_limb,
                                               uint64_t* sm)
{
    constexpr uint32_t lgtg = 10 - LG;
    const uint32_t mi = limb_mod(limb, c.nmods);
    const ModCtx* cx = c.ctx[mi];
    if constexpr (CLS == kClsChain) {
        chain_tile<LG, LR, CG>(c.src, c.dst, c.vec, cx, c.op, c.scalars ? c.scalars[mi] : 0, c.logn, lgtg, limb,
                               tile_in_limb, c.flags, sm);
    } else {
        pass_tile<CLS == kClsInv, LG, LR, CG>(c.src, c.dst, cx, c.logn, c.s0, lgtg, limb, tile_in_limb, c.flags,
                                              sm);
    }
}

// One tile of any class (the persistent kernel: 128 threads x 8 registers).
__device__ __forceinline__ void run_any_tile(const ClassEntry& c, uint64_t limb, uint64_t til, uint64_t* sm)
{
    switch (c.cls_lg) {
#define AXHEL_TILE_CASE(CLS, LG) \
    case (CLS << 8) | LG: run_class_tile<CLS, LG, kBatchLR, true>(c, limb, til, sm); break;
#define AXHEL_TILE_CASES(CLS) \
    AXHEL_TILE_CASE(CLS, 5) AXHEL_TILE_CASE(CLS, 6) AXHEL_TILE_CASE(CLS, 7) AXHEL_TILE_CASE(CLS, 8) AXHEL_TILE_CASE(CLS, 9)
    AXHEL_TILE_CASES(kClsFwd)
    AXHEL_TILE_CASES(kClsInv)
    AXHEL_TILE_CASES(kClsChain)
#undef AXHEL_TILE_CASES
#undef AXHEL_TILE_CASE
    default: run_elt_tile(c, limb, til); break;  // kClsElt << 8
    }
}

// Last entry at or after `from` whose first tile is <= tile (tiles are
// claimed in increasing order, so a CTA's next tile is at or after its
// previous entry): gallop forward, then bisect.
__device__ __forceinline__ uint32_t find_entry(const BatchArgs& a, uint64_t tile, uint32_t from)
{
    uint32_t lo = from, step = 1;
    while (lo + step < a.nentries && a.entries[lo + step].tile_begin <= tile) {
        lo += step;
        step <<= 1;
    }
    uint32_t hi = lo + step < a.nentries ? lo + step : a.nentries;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a.entries[mid].tile_begin <= tile) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(kBatchThreads, kBatchMinBlocks) batch_kernel(const __grid_constant__ BatchArgs a)
{
    __shared__ uint64_t sm[kBatchTileWords + 128];
    __shared__ unsigned long long s_tile[2];
    __shared__ uint32_t s_entry;
    __shared__ int s_abort;
    uint32_t entry = 0;  // thread 0: entry of the CTA's latest tile
    if (threadIdx.x == 0) {
        s_tile[0] = atomicAdd(a.next_tile, 1ull);
        s_abort = 0;
    }
    __syncthreads();
    for (uint32_t it = 0;; ++it) {
        const uint64_t tile = s_tile[it & 1];
        if (tile >= a.total_tiles) break;
        unsigned long long nxt = 0;  // the next tile, claimed now, announced after this one
        if (threadIdx.x == 0) {
            nxt = atomicAdd(a.next_tile, 1ull);
            entry = find_entry(a, tile, entry);
            s_entry = entry;
            const BatchEntry e = a.entries[entry];
            if (e.phase > 0) {
                const BatchJob& j = a.jobs[e.job];
                const uint64_t limb = (tile - e.tile_begin) >> (j.logn - kBatchTileLog);
                cuda::atomic_ref<unsigned int, cuda::thread_scope_device> dep(
                    a.done[j.done_off + (uint64_t)(e.phase - 1) * j.count + limb]);
                const unsigned need = j.tiles_per_limb[e.phase - 1] + j.wait_extra;
                const uint64_t t0 = global_ns();
                uint32_t polls = 0;
                while (dep.load(cuda::memory_order_acquire) < need) {
                    // bounded in wall time and in polls
                    if (++polls > (1u << 24) || global_ns() - t0 > a.wait_ns) {
                        atomicExch(a.error, AXHEL_ERR_TIMEOUT);
                        s_abort = 1;
                        break;
                    }
                    __nanosleep(100);
                }
            }
        }
        __syncthreads();
        if (s_abort) break;
        const uint32_t cur = s_entry;
        const ClassEntry& c = a.tile_args[cur];
        const uint64_t lt = tile - c.tile0;
        const uint32_t lgt = c.logn - kBatchTileLog;  // tiles per limb: a power of two
        const uint64_t limb = lt >> lgt;
        run_any_tile(c, limb, lt & ((1ull << lgt) - 1), sm);
        if (threadIdx.x == 0) s_tile[(it + 1) & 1] = nxt;
        __syncthreads();
        // The finished tile is published by a thread of another warp than the
        // claiming thread 0, so its release fence overlaps the next tile's
        // lookup and dependency check instead of preceding them.
        if (threadIdx.x == kBatchPublisher) {
            const BatchEntry e = a.entries[cur];
            const BatchJob& j = a.jobs[e.job];
            if (e.phase + 1 < j.nphase) {
                // release at device scope, cumulative over the stores the
                // barrier ordered before it
                cuda::atomic_ref<unsigned int, cuda::thread_scope_device> done(
                    a.done[j.done_off + (uint64_t)e.phase * j.count + limb]);
                done.fetch_add(1u, cuda::memory_order_release);
            }
        }
    }
}

template <int CLS, int LR>
constexpr int class_min_blocks()
{
    return CLS == kClsChain ? 6 : (LR == 4 ? (CLS == kClsInv ? 12 : 16) : kBatchMinBlocks);
}

template <int CLS, int LG, int LR>
__device__ __forceinline__ void run_class_entry(const ClassEntry& c, uint64_t t, uint64_t* sm)
{
    const uint64_t lt = t - c.tile0;
    const uint32_t lgt = c.logn - kBatchTileLog;  // tiles per limb: a power of two
    const uint64_t limb = lt >> lgt;
    const uint64_t til = lt & ((1ull << lgt) - 1);
    if constexpr (CLS == kClsElt)
        run_elt_tile(c, limb, til);
    else
        run_class_tile<CLS, LG, LR, false>(c, limb, til, sm);
}

// One class launch: CTA b runs the class's tile b (entries in tile order),
// held to class_min_blocks CTAs per SM.
template <int CLS, int LG, int LR>
__global__ void __launch_bounds__(kBatchTileWords >> LR, class_min_blocks<CLS, LR>())
    batch_class_kernel(const ClassEntry* __restrict__ ce, uint32_t n_ce)
{
    __shared__ uint64_t sm[kBatchTileWords + 128];
    const uint64_t t = blockIdx.x;
    uint32_t lo = 0, hi = n_ce;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (ce[mid].tile0 <= t) lo = mid; else hi = mid;
    }
    run_class_entry<CLS, LG, LR>(ce[lo], t, sm);
}

// A class launch of one entry reads it from the kernel parameters, as the
// pass kernels read theirs: no dependent load ahead of the tile's data, and
// its fields stay out of the registers.  Without a CTAs-per-SM bound the
// compiler settles at 56-64 registers without spills, which measured 4 %
// faster than the bounded form.
template <int CLS, int LG, int LR>
__global__ void __launch_bounds__(kBatchTileWords >> LR) batch_class_one_kernel(const __grid_constant__ ClassEntry one)
{
    __shared__ uint64_t sm[kBatchTileWords + 128];
    run_class_entry<CLS, LG, LR>(one, blockIdx.x, sm);
}

}  // namespace axhel_impl

using namespace axhel_impl;

// ------------------------------------------------------------------ host

struct axhel_batch {
    int device = 0;
    void* mem = nullptr;  // descriptors | entries | ctx tables | scalars | done | counter | error
    size_t bytes = 0;
    size_t zero_off = 0, zero_bytes = 0;  // counters cleared before every launch
    BatchArgs args{};
    std::vector<ClassLaunch> classes;        // the per-phase launches
    LaunchLanes lanes;                       // their side-by-side streams
    unsigned grid = 0;
    std::vector<axhel_ntt_t> held;  // table contexts kept alive while the batch exists
    cudaGraphExec_t graph = nullptr;
    cudaStream_t graph_stream = nullptr;
};

namespace {

thread_local std::string t_batch_error;

axhel_status_t bfail(axhel_status_t st, const std::string& m)
{
    t_batch_error = m;
    return st;
}

}  // namespace

void axhel_impl::batch_set_error(const std::string& msg) { t_batch_error = msg; }

namespace {

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Persistent grid of the current device: resident CTAs per SM x SMs, kept
// per device index (threads that race on the first call store the same
// value).
int batch_grid()
{
    static std::atomic<int> cached[64];
    int dev = 0;
    cudaGetDevice(&dev);
    const bool keep = dev >= 0 && dev < 64;
    int g = keep ? cached[dev].load(std::memory_order_relaxed) : 0;
    if (!g) {
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel, kBatchThreads, 0);
        if (per_sm < 1) per_sm = 1;
        g = per_sm * sm_count();
        if (keep) cached[dev].store(g, std::memory_order_relaxed);
    }
    return g;
}

}  // namespace

namespace {

// Branch of EltwiseReduceModNative (eltwise-reduce-mod.cpp:35-127) taken for
// (in_f, out_f): 0 copy, 1 [0,2q)->[0,q), 2 [0,4q)->[0,q), 3 [0,4q)->[0,2q),
// 4 Barrett (in_f equal to the modulus); -1 for a pair that does nothing.
int reduce_branch(uint64_t in_f, uint64_t out_f)
{
    if (in_f == AXHEL_FACTOR_MODULUS) return 4;
    if (in_f == 1 || (out_f == 2 && in_f <= 2)) return 0;
    if (in_f == 2 && out_f == 1) return 1;
    if (in_f == 4 && out_f == 1) return 2;
    if (in_f == 4 && out_f == 2) return 3;
    return -1;
}

}  // namespace

namespace axhel_impl {

axhel_status_t batch_check_job(const axhel_job_t& J, const std::string& who, std::string* err)
{
    const std::string job = who + ": ";
    if (J.kind < AXHEL_JOB_FORWARD || J.kind > AXHEL_JOB_REDUCE) {
        *err = job + "unknown kind";
        return AXHEL_ERR_INVALID;
    }
    if (!J.ntts || J.n_ntts == 0 || J.n_ntts > 1024) {
        *err = job + "1..1024 NTT handles needed";
        return AXHEL_ERR_INVALID;
    }
    const uint64_t n = J.ntts[0] ? J.ntts[0]->n : 0;
    for (uint32_t m = 0; m < J.n_ntts; ++m) {
        if (!J.ntts[m] || J.ntts[m]->n != n) {
            *err = job + "handles must share one degree";
            return AXHEL_ERR_INVALID;
        }
    }
    const uint32_t logn = J.ntts[0]->logn;
    if (logn < 10 || logn > 17) {
        *err = job + "batched degree must be in [2^10, 2^17]";
        return AXHEL_ERR_UNSUPPORTED;
    }
    if (J.count && (!J.result || !J.operand)) {
        *err = job + "null data pointer";
        return AXHEL_ERR_INVALID;
    }
    const uint64_t f = J.input_mod_factor;
    switch (J.kind) {
    case AXHEL_JOB_CHAIN_MUL:
        if (J.count && !J.vector) {
            *err = job + "chain multiplicand missing";
            return AXHEL_ERR_INVALID;
        }
        break;
    case AXHEL_JOB_CHAIN_FMA:
        if (!J.scalars) {
            *err = job + "chain scalars missing";
            return AXHEL_ERR_INVALID;
        }
        break;
    case AXHEL_JOB_ADD:
    case AXHEL_JOB_SUB:
        if (!J.vector && !J.scalars) {
            *err = job + "a vector or per-modulus scalars needed";
            return AXHEL_ERR_INVALID;
        }
        break;
    case AXHEL_JOB_MUL:
        if (J.count && !J.vector) {
            *err = job + "multiplicand missing";
            return AXHEL_ERR_INVALID;
        }
        if (f != 1 && f != 2 && f != 4) {
            *err = job + "MulMod input factor must be 1, 2 or 4";
            return AXHEL_ERR_INVALID;
        }
        break;
    case AXHEL_JOB_FMA:
        if (!J.scalars) {
            *err = job + "FMAMod scalars missing";
            return AXHEL_ERR_INVALID;
        }
        if (f != 1 && f != 2 && f != 4 && f != 8) {
            *err = job + "FMAMod input factor must be 1, 2, 4 or 8";
            return AXHEL_ERR_INVALID;
        }
        break;
    case AXHEL_JOB_REDUCE:
        if (reduce_branch(f, J.output_mod_factor) < 0) {
            *err = job + "ReduceMod factor pair (" + std::to_string(f) + ", " + std::to_string(J.output_mod_factor) +
                   ") is not one the reference reduces";
            return AXHEL_ERR_INVALID;
        }
        break;
    default:
        break;
    }
    return AXHEL_OK;
}

// Host layout of a batch: fills `host` (to be copied to the device at `base`)
// and the kernel arguments.  Shared by the allocating and the static-scratch
// entry points.
// The specialized kernel for a launch of one transform or chain entry: the
// pass of the tuned plan (plan_for) that covers the same stages with the
// same width, with its register depth and tile width; a chain's fused pass
// as the chain kernel over the inverse plan's last pass (register depth at
// most 3, as the chain entry point runs it).  Left as a class launch when no
// tuned pass matches the batch's split.
static void set_specialized(ClassLaunch& L, const BatchJob& b, const std::vector<const ModCtx*>& ctx,
                     const std::vector<uint64_t>& sc, uint32_t phase)
{
    L.spec = 0;
    if (L.cls == kClsElt || ctx.empty() || ctx.size() > (size_t)kMaxInlineMods || b.count == 0) return;
    const PhaseCfg pc = phase_cfg(b, phase);
    PassArgs a{};
    a.src = L.first.src;
    a.dst = L.first.dst;
    a.count = b.count;
    a.logn = b.logn;
    a.s0 = pc.s0;
    a.flags = L.first.flags;
    a.nctx = (uint32_t)ctx.size();
    for (size_t m = 0; m < ctx.size(); ++m) a.ctx[m] = ctx[m];
    const NttPlan inv = plan_for(true, b.logn, b.count);
    if (pc.chain) {
        if (inv.npass < 2) return;
        PassCfg fc = inv.pass[inv.npass - 1];
        if (fc.lg != (int)pc.lg) return;
        if (fc.lr > 3 && fc.lg >= 4 && ((uint64_t)fc.tg << (fc.lg - 3)) <= 512) fc.lr = 3;
        if (fc.lr > 3) return;
        a.tg = (uint32_t)fc.tg;
        L.spec_args = ChainArgs{};
        L.spec_args.pass = a;
        L.spec_args.operand = L.first.vec;
        L.spec_args.op = L.first.op;
        L.spec_args.op_factor = 2;
        if (L.first.op == kChainFma) {
            if (sc.size() != ctx.size()) return;
            for (size_t m = 0; m < sc.size(); ++m) L.spec_args.scalar[m] = sc[m];
        }
        L.spec_cfg = fc;
        L.spec = 2;
        return;
    }
    const NttPlan pl = pc.inv ? inv : plan_for(false, b.logn, b.count);
    uint32_t s0 = 0;
    for (int i = 0; i < pl.npass; ++i) {
        if (s0 == pc.s0 && pl.pass[i].lg == (int)pc.lg) {
            a.tg = (uint32_t)pl.pass[i].tg;
            L.spec_args = ChainArgs{};
            L.spec_args.pass = a;
            L.spec_cfg = pl.pass[i];
            L.spec_inv = pc.inv;
            L.spec = 1;
            return;
        }
        s0 += (uint32_t)pl.pass[i].lg;
    }
}

axhel_status_t batch_build(const axhel_job_t* jobs, uint64_t n_jobs, unsigned char* base,
                           std::vector<unsigned char>& host, size_t* zero_off, size_t* zero_bytes, BatchArgs* args,
                           std::vector<axhel_ntt_t>* held, std::string* err, std::vector<ClassLaunch>* classes)
{
    if (!jobs || n_jobs == 0) {
        *err = "empty batch";
        return AXHEL_ERR_INVALID;
    }
    std::vector<BatchJob> bj(n_jobs);
    std::vector<std::vector<const ModCtx*>> ctxs(n_jobs);
    std::vector<std::vector<uint64_t>> scal(n_jobs);
    uint64_t done_total = 0;
    for (uint64_t i = 0; i < n_jobs; ++i) {
        const axhel_job_t& J = jobs[i];
        BatchJob& b = bj[i];
        std::memset(&b, 0, sizeof b);
        const axhel_status_t st = batch_check_job(J, "job " + std::to_string(i), err);
        if (st) return st;
        for (uint32_t m = 0; m < J.n_ntts; ++m) {
            ctxs[i].push_back(J.ntts[m]->dctx);
            if (held) held->push_back(J.ntts[m]);
        }
        const uint32_t logn = J.ntts[0]->logn;
        b.kind = J.kind;
        b.logn = logn;
        b.count = J.count;
        b.nmods = J.n_ntts;
        b.src = J.operand;
        b.dst = J.result;
        b.vec = J.vector;
        if (J.kind >= AXHEL_JOB_ADD) {
            // element-wise: one phase of 1024-residue tiles, no dependencies
            const uint64_t f = J.input_mod_factor;
            b.nphase = 1;
            b.tiles_per_limb[0] = (uint32_t)((1ull << logn) / kBatchTileWords);
            if (J.kind == AXHEL_JOB_ADD || J.kind == AXHEL_JOB_SUB) {
                const bool vv = J.vector != nullptr;
                b.eop = J.kind == AXHEL_JOB_ADD ? (vv ? kEltAddVV : kEltAddVS) : (vv ? kEltSubVV : kEltSubVS);
                if (!vv) scal[i].assign(J.scalars, J.scalars + J.n_ntts);
            } else if (J.kind == AXHEL_JOB_MUL) {
                b.eop = kEltMul;
                b.ef = (uint32_t)f;
            } else if (J.kind == AXHEL_JOB_FMA) {
                b.eop = J.vector ? kEltFmaAdd : kEltFma;
                b.ef = (uint32_t)f;
                // the scalar enters reduced by ReduceInput<F> (eltwise-fma-mod.cpp:33)
                for (uint32_t m = 0; m < J.n_ntts; ++m) {
                    uint64_t v = J.scalars[m];
                    const uint64_t q = J.ntts[m]->q;
                    if (f == 8 && v >= 4 * q) v -= 4 * q;
                    if (f >= 4 && v >= 2 * q) v -= 2 * q;
                    if (f >= 2 && v >= q) v -= q;
                    scal[i].push_back(v);
                }
            } else {
                b.eop = kEltReduce;
                b.ef = reduce_branch(f, J.output_mod_factor);
            }
            b.done_off = done_total;
            continue;
        }
        if (J.kind == AXHEL_JOB_CHAIN_FMA) scal[i].assign(J.scalars, J.scalars + J.n_ntts);
        b.lg_row = (uint32_t)batch_row_stages(logn);
        b.lg_col = logn - b.lg_row;
        const bool inv_first = J.kind != AXHEL_JOB_FORWARD;
        b.pre = inv_first && J.input_mod_factor == 4;
        b.norm = (J.kind == AXHEL_JOB_INVERSE) ? (J.output_mod_factor != 2) : (J.output_mod_factor != 4);
        b.nphase = (J.kind == AXHEL_JOB_CHAIN_MUL || J.kind == AXHEL_JOB_CHAIN_FMA) ? 3 : 2;
        for (uint32_t p = 0; p < b.nphase; ++p) {
            const uint32_t lg = phase_cfg(b, p).lg;
            if (lg < (uint32_t)kBatchMinLG || lg > (uint32_t)kBatchMaxLG || (1ull << logn) % kBatchTileWords) {
                *err = "job " + std::to_string(i) + ": degree outside the batched range";
                return AXHEL_ERR_UNSUPPORTED;
            }
            b.tiles_per_limb[p] = (uint32_t)((1ull << logn) / kBatchTileWords);
        }
        b.done_off = done_total;
        done_total += (uint64_t)(b.nphase - 1) * b.count;
    }
    // phase-major tile order
    std::vector<BatchEntry> ent;
    uint64_t tiles = 0;
    for (uint32_t p = 0; p < 3; ++p) {
        for (uint64_t i = 0; i < n_jobs; ++i) {
            if (p >= bj[i].nphase || bj[i].count == 0) continue;
            ent.push_back(BatchEntry{tiles, (uint32_t)i, p});
            tiles += bj[i].count * bj[i].tiles_per_limb[p];
        }
    }
    if (classes) classes->clear();
    if (ent.empty()) {
        *err = "";
        args->total_tiles = 0;
        return AXHEL_OK;
    }
    // every entry's tile class and pass width
    std::vector<uint32_t> ent_cls(ent.size()), ent_lg(ent.size());
    for (size_t k = 0; k < ent.size(); ++k) {
        const BatchJob& b = bj[ent[k].job];
        if (b.kind >= kJobAdd) {
            ent_cls[k] = kClsElt;
            ent_lg[k] = 0;
            continue;
        }
        const PhaseCfg pc = phase_cfg(b, ent[k].phase);
        ent_cls[k] = pc.chain ? kClsChain : (pc.inv ? kClsInv : kClsFwd);
        ent_lg[k] = pc.lg;
    }
    // per (phase, class, pass width): the entries, in order, with their
    // first tile in that launch's numbering
    std::vector<ClassLaunch> cl;
    std::vector<std::vector<ClassEntry>> cl_ent;
    std::vector<std::vector<uint32_t>> cl_idx;  // the batch entry of each class entry
    std::vector<ClassLaunch> alone;             // launches of one large entry
    std::vector<uint32_t> alone_idx;
    if (classes) {
        // The largest entries of each phase (at least kAloneMinTiles tiles,
        // up to kAloneMax) get launches of their own, which take the entry
        // as a kernel parameter; the rest are grouped by class and width.
        constexpr uint64_t kAloneMinTiles = 512;
        constexpr size_t kAloneMax = 128;
        const auto ent_tiles = [&](uint32_t k) { return bj[ent[k].job].count * bj[ent[k].job].tiles_per_limb[ent[k].phase]; };
        std::vector<char> is_alone(ent.size(), 0);
        for (uint32_t p = 0; p < 3; ++p) {
            std::vector<uint32_t> big;
            for (uint32_t k = 0; k < (uint32_t)ent.size(); ++k)
                if (ent[k].phase == p && ent_tiles(k) >= kAloneMinTiles) big.push_back(k);
            std::stable_sort(big.begin(), big.end(), [&](uint32_t x, uint32_t y) { return ent_tiles(x) > ent_tiles(y); });
            for (size_t i = 0; i < big.size() && i < kAloneMax; ++i) is_alone[big[i]] = 1;
        }
        std::map<std::tuple<uint32_t, uint32_t, uint32_t>, size_t> at;
        for (uint32_t k = 0; k < (uint32_t)ent.size(); ++k) {
            const BatchEntry& e = ent[k];
            const BatchJob& b = bj[e.job];
            const uint32_t cls = ent_cls[k], lg = ent_lg[k];
            if (is_alone[k]) {
                alone.push_back(ClassLaunch{e.phase, cls, lg, 1, nullptr, ent_tiles(k), ClassEntry{}});
                alone_idx.push_back(k);
                continue;
            }
            const auto key = std::make_tuple(e.phase, cls, lg);
            auto it = at.find(key);
            if (it == at.end()) {
                it = at.emplace(key, cl.size()).first;
                cl.push_back(ClassLaunch{e.phase, cls, lg, 0, nullptr, 0, ClassEntry{}});
                cl_ent.emplace_back();
                cl_idx.emplace_back();
            }
            ClassLaunch& L = cl[it->second];
            ClassEntry x{};
            x.tile0 = L.tiles;
            cl_ent[it->second].push_back(x);
            cl_idx[it->second].push_back(k);
            L.tiles += b.count * b.tiles_per_limb[e.phase];
            ++L.n_ce;
        }
    }
    // device image
    size_t off = 0;
    const size_t jobs_off = off;
    off = align_up(off + n_jobs * sizeof(BatchJob), 256);
    const size_t ent_off = off;
    off = align_up(off + ent.size() * sizeof(BatchEntry), 256);
    const size_t targ_off = off;
    off = align_up(off + ent.size() * sizeof(ClassEntry), 256);
    std::vector<size_t> ctx_off(n_jobs), sc_off(n_jobs, 0);
    for (uint64_t i = 0; i < n_jobs; ++i) {
        ctx_off[i] = off;
        off = align_up(off + ctxs[i].size() * sizeof(void*), 16);
        if (!scal[i].empty()) {
            sc_off[i] = off;
            off = align_up(off + scal[i].size() * 8, 16);
        }
    }
    std::vector<size_t> ce_off(cl.size());
    for (size_t c = 0; c < cl.size(); ++c) {
        off = align_up(off, 16);
        ce_off[c] = off;
        off += cl_ent[c].size() * sizeof(ClassEntry);
    }
    off = align_up(off, 256);
    *zero_off = off;
    const size_t done_off = off;
    off = align_up(off + done_total * sizeof(unsigned), 16);
    const size_t ctr_off = off;
    off += 16;
    const size_t err_off = off;
    off = align_up(off + 16, 256);
    *zero_bytes = off - *zero_off;
    host.assign(off, 0);
    for (uint64_t i = 0; i < n_jobs; ++i) {
        bj[i].ctx = reinterpret_cast<const ModCtx* const*>(base + ctx_off[i]);
        bj[i].scalars = scal[i].empty() ? nullptr : reinterpret_cast<const uint64_t*>(base + sc_off[i]);
        std::memcpy(host.data() + ctx_off[i], ctxs[i].data(), ctxs[i].size() * sizeof(void*));
        if (!scal[i].empty()) std::memcpy(host.data() + sc_off[i], scal[i].data(), scal[i].size() * 8);
    }
    std::memcpy(host.data() + jobs_off, bj.data(), n_jobs * sizeof(BatchJob));
    std::memcpy(host.data() + ent_off, ent.data(), ent.size() * sizeof(BatchEntry));
    // each entry's tile arguments: operands, first stage and the tile
    // functions' flags (the first tile of a class launch's entry is in that
    // launch's numbering, of the persistent kernel's entry the global one)
    std::vector<ClassEntry> targ(ent.size());
    for (size_t k = 0; k < ent.size(); ++k) {
        ClassEntry& x = targ[k];
        const uint32_t p = ent[k].phase, cls = ent_cls[k];
        const BatchJob& b = bj[ent[k].job];
        const bool first = p == 0, last = p + 1 == b.nphase;
        x.tile0 = ent[k].tile_begin;
        x.src = first ? b.src : b.dst;
        x.dst = b.dst;
        x.vec = b.vec;
        x.ctx = b.ctx;
        x.scalars = (b.kind == kJobChainFma || b.kind >= kJobAdd) ? b.scalars : nullptr;
        x.nmods = b.nmods;
        x.logn = b.logn;
        x.eop = b.eop;
        x.ef = b.ef;
        x.cls_lg = cls << 8 | ent_lg[k];
        if (cls == kClsElt) continue;
        const PhaseCfg pc = phase_cfg(b, p);
        x.s0 = pc.s0;
        if (cls == kClsChain) {
            x.op = b.kind == kJobChainMul ? kChainMul : kChainFma;
            x.flags = (first && b.pre ? kPreCsub2q : 0) | (last && b.norm ? kPostNorm : 0);
        } else {
            x.flags = (first && b.pre) ? kPreCsub2q : 0;
            if (last) x.flags |= kLastPass | (b.norm ? kPostNorm : 0);
            // the inverse's last pass holds the N^-1 stage even inside a chain
            if (cls == kClsInv && pc.s0 + ent_lg[k] == b.logn) x.flags |= kLastPass;
        }
    }
    std::memcpy(host.data() + targ_off, targ.data(), targ.size() * sizeof(ClassEntry));
    for (size_t c = 0; c < cl.size(); ++c) {
        for (size_t i = 0; i < cl_ent[c].size(); ++i) {
            const uint64_t t0 = cl_ent[c][i].tile0;
            cl_ent[c][i] = targ[cl_idx[c][i]];
            cl_ent[c][i].tile0 = t0;
        }
        std::memcpy(host.data() + ce_off[c], cl_ent[c].data(), cl_ent[c].size() * sizeof(ClassEntry));
        cl[c].ce = reinterpret_cast<const ClassEntry*>(base + ce_off[c]);
        cl[c].first = cl_ent[c][0];
    }
    if (classes) {
        for (size_t i = 0; i < alone.size(); ++i) {
            alone[i].first = targ[alone_idx[i]];
            alone[i].first.tile0 = 0;
            const uint32_t j = ent[alone_idx[i]].job;
            set_specialized(alone[i], bj[j], ctxs[j], scal[j], ent[alone_idx[i]].phase);
        }
        cl.insert(cl.end(), alone.begin(), alone.end());
        // phase by phase, the largest launches first (spread over the lanes)
        std::stable_sort(cl.begin(), cl.end(), [](const ClassLaunch& x, const ClassLaunch& y) {
            return x.phase != y.phase ? x.phase < y.phase : x.tiles > y.tiles;
        });
        *classes = cl;
    }
    args->jobs = reinterpret_cast<const BatchJob*>(base + jobs_off);
    args->entries = reinterpret_cast<const BatchEntry*>(base + ent_off);
    args->tile_args = reinterpret_cast<const ClassEntry*>(base + targ_off);
    args->nentries = (uint32_t)ent.size();
    args->total_tiles = tiles;
    args->done = reinterpret_cast<unsigned*>(base + done_off);
    args->next_tile = reinterpret_cast<unsigned long long*>(base + ctr_off);
    args->error = reinterpret_cast<int*>(base + err_off);
    args->wait_ns = 2000000000ull;  // 2 s
    return AXHEL_OK;
}

namespace {

struct ClassKernel {
    void (*one)(const ClassEntry) = nullptr;
    void (*many)(const ClassEntry*, uint32_t) = nullptr;
    unsigned threads = 0;
};

// Register depth per class and width: 4 (64 threads per tile) for the
// 7-stage transform passes, 3 (128 threads) otherwise -- measured per width
// on the per-phase launches: 4 is 5 % faster at 7 stages, 3 is 8 % faster
// at 8 stages and 15-22 % faster at 5 and 6.
template <int CLS, int LG>
ClassKernel class_kernel()
{
    constexpr int LR = (CLS == kClsFwd || CLS == kClsInv) && LG == 7 ? 4 : 3;
    return ClassKernel{batch_class_one_kernel<CLS, LG, LR>, batch_class_kernel<CLS, LG, LR>,
                       (unsigned)(kBatchTileWords >> LR)};
}

ClassKernel pick_class_kernel(uint32_t cls, uint32_t lg)
{
    if (cls == kClsElt) return class_kernel<kClsElt, 5>();
    if (lg < (uint32_t)kBatchMinLG || lg > (uint32_t)kBatchMaxLG) return ClassKernel{};
    static const ClassKernel table[3][5] = {
        {class_kernel<kClsFwd, 5>(), class_kernel<kClsFwd, 6>(), class_kernel<kClsFwd, 7>(), class_kernel<kClsFwd, 8>(),
         class_kernel<kClsFwd, 9>()},
        {class_kernel<kClsInv, 5>(), class_kernel<kClsInv, 6>(), class_kernel<kClsInv, 7>(), class_kernel<kClsInv, 8>(),
         class_kernel<kClsInv, 9>()},
        {class_kernel<kClsChain, 5>(), class_kernel<kClsChain, 6>(), class_kernel<kClsChain, 7>(),
         class_kernel<kClsChain, 8>(), class_kernel<kClsChain, 9>()}};
    return cls < 3 ? table[cls][lg - kBatchMinLG] : ClassKernel{};
}

}  // namespace

cudaError_t lanes_create(LaunchLanes* l, int priority)
{
    for (int i = 0; i < kLaunchLanes - 1; ++i) {
        cudaError_t e = cudaStreamCreateWithPriority(&l->st[i], cudaStreamNonBlocking, priority);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&l->join[i], cudaEventDisableTiming);
        if (e != cudaSuccess) return e;
    }
    return cudaEventCreateWithFlags(&l->fork, cudaEventDisableTiming);
}

void lanes_destroy(LaunchLanes* l)
{
    for (int i = 0; i < kLaunchLanes - 1; ++i) {
        if (l->st[i]) cudaStreamDestroy(l->st[i]);
        if (l->join[i]) cudaEventDestroy(l->join[i]);
        l->st[i] = nullptr;
        l->join[i] = nullptr;
    }
    if (l->fork) cudaEventDestroy(l->fork);
    l->fork = nullptr;
}

cudaError_t batch_launch_classes(const std::vector<ClassLaunch>& classes, cudaStream_t s, const LaunchLanes* lanes,
                                 bool specialized)
{
    for (size_t i = 0; i < classes.size();) {
        size_t j = i;
        while (j < classes.size() && classes[j].phase == classes[i].phase) ++j;
        // this phase's launches, round-robin over the caller's stream and
        // the lanes forked from it
        const int nl = lanes ? (int)std::min<size_t>(kLaunchLanes, j - i) : 1;
        cudaError_t e = cudaSuccess;
        if (nl > 1) {
            e = cudaEventRecord(lanes->fork, s);
            for (int l = 1; l < nl && e == cudaSuccess; ++l) e = cudaStreamWaitEvent(lanes->st[l - 1], lanes->fork, 0);
        }
        for (size_t k = i; k < j && e == cudaSuccess; ++k) {
            const ClassLaunch& L = classes[k];
            if (L.tiles == 0) continue;
            if (L.tiles > 0x7fffffffull) return cudaErrorInvalidValue;
            const ClassKernel kn = pick_class_kernel(L.cls, L.lg);
            if (!kn.one) return cudaErrorInvalidValue;
            const int l = (int)((k - i) % nl);
            cudaStream_t ls = l == 0 ? s : lanes->st[l - 1];
            if (specialized && L.spec == 1) {
                e = launch_ntt_pass(L.spec_inv, L.spec_cfg, L.spec_args.pass, ls);
                continue;
            }
            if (specialized && L.spec == 2) {
                e = launch_chain_pass(L.spec_cfg, L.spec_args, ls);
                continue;
            }
            count_launch();
            ProfScope prof(ls, "batch_class_kernel cls=%u lg=%u", L.cls, L.lg);
            if (L.n_ce == 1)
                kn.one<<<(unsigned)L.tiles, kn.threads, 0, ls>>>(L.first);
            else
                kn.many<<<(unsigned)L.tiles, kn.threads, 0, ls>>>(L.ce, L.n_ce);
            e = cudaGetLastError();
        }
        for (int l = 1; l < nl && e == cudaSuccess; ++l) {
            e = cudaEventRecord(lanes->join[l - 1], lanes->st[l - 1]);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(s, lanes->join[l - 1], 0);
        }
        if (e != cudaSuccess) return e;
        i = j;
    }
    return cudaSuccess;
}

cudaError_t batch_launch_args(const BatchArgs& a, cudaStream_t s)
{
    if (a.total_tiles == 0) return cudaSuccess;
    uint64_t grid = (uint64_t)batch_grid();
    if (grid > a.total_tiles) grid = a.total_tiles;
    count_launch();
    ProfScope prof(s, "batch_kernel");
    batch_kernel<<<(unsigned)grid, kBatchThreads, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace axhel_impl

extern "C" {

axhel_status_t axhel_cuda_batch_create(const axhel_job_t* jobs, uint64_t n_jobs, axhel_batch_t* out)
{
    if (!out) return bfail(AXHEL_ERR_INVALID, "null output");
    *out = nullptr;
    auto b = std::make_unique<axhel_batch>();
    cudaGetDevice(&b->device);
    // first pass for the size, then with the real base address
    std::vector<unsigned char> img;
    BatchArgs args{};
    std::string err;
    std::vector<axhel_ntt_t> held;
    std::vector<ClassLaunch> sizing;
    axhel_status_t st =
        batch_build(jobs, n_jobs, nullptr, img, &b->zero_off, &b->zero_bytes, &args, nullptr, &err, &sizing);
    if (st) return bfail(st, err);
    b->bytes = img.size();
    if (b->bytes) {
        cudaError_t e = cudaMalloc(&b->mem, b->bytes);
        if (e != cudaSuccess) return bfail(AXHEL_ERR_NOMEM, std::string("cudaMalloc(batch): ") + cudaGetErrorString(e));
        st = batch_build(jobs, n_jobs, static_cast<unsigned char*>(b->mem), img, &b->zero_off, &b->zero_bytes,
                         &b->args, &held, &err, &b->classes);
        if (st) {
            cudaFree(b->mem);
            return bfail(st, err);
        }
        e = cudaMemcpy(b->mem, img.data(), img.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(b->mem);
            return bfail(AXHEL_ERR_CUDA, std::string("cudaMemcpy(batch): ") + cudaGetErrorString(e));
        }
    } else {
        b->args = args;
    }
    for (axhel_ntt_t h : held) axhel_cuda_ntt_retain(h);
    b->held = std::move(held);
    *out = b.release();
    return AXHEL_OK;
}

axhel_status_t axhel_cuda_batch_launch(axhel_batch_t b, void* stream)
{
    if (!b) return bfail(AXHEL_ERR_INVALID, "null batch");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (b->args.total_tiles == 0) return AXHEL_OK;
    cudaError_t e = cudaMemsetAsync(static_cast<unsigned char*>(b->mem) + b->zero_off, 0, b->zero_bytes, s);
    if (e == cudaSuccess) e = batch_launch_args(b->args, s);
    if (e != cudaSuccess) return bfail(AXHEL_ERR_CUDA, std::string("batch launch: ") + cudaGetErrorString(e));
    return AXHEL_OK;
}

axhel_status_t axhel_cuda_batch_launch_phased(axhel_batch_t b, void* stream)
{
    if (!b) return bfail(AXHEL_ERR_INVALID, "null batch");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (b->args.total_tiles == 0) return AXHEL_OK;
    // the error word is cleared as before a persistent launch (no wait can fail here)
    cudaError_t e = cudaMemsetAsync(static_cast<unsigned char*>(b->mem) + b->zero_off, 0, b->zero_bytes, s);
    if (e == cudaSuccess && !b->lanes.fork) {
        // the lanes are made on the first launch outside a stream capture
        // (no stream may be created while one is captured); until then a
        // phase's launches queue on the caller's stream
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone &&
            lanes_create(&b->lanes, 0) != cudaSuccess) {
            lanes_destroy(&b->lanes);
            cudaGetLastError();
        }
    }
    if (e == cudaSuccess) e = batch_launch_classes(b->classes, s, b->lanes.fork ? &b->lanes : nullptr, true);
    if (e != cudaSuccess) return bfail(AXHEL_ERR_CUDA, std::string("batch launch: ") + cudaGetErrorString(e));
    return AXHEL_OK;
}

axhel_status_t axhel_cuda_batch_graph_launch(axhel_batch_t b, void* stream)
{
    if (!b) return bfail(AXHEL_ERR_INVALID, "null batch");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (b->args.total_tiles == 0) return AXHEL_OK;
    if (!b->graph) {
        cudaStream_t cap;
        if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess)
            return bfail(AXHEL_ERR_CUDA, "stream create");
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaMemsetAsync(static_cast<unsigned char*>(b->mem) + b->zero_off, 0, b->zero_bytes, cap);
            batch_launch_args(b->args, cap);
            e = cudaStreamEndCapture(cap, &g);
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&b->graph, g, 0);
        if (g) cudaGraphDestroy(g);
        cudaStreamDestroy(cap);
        if (e != cudaSuccess) return bfail(AXHEL_ERR_CUDA, std::string("batch graph: ") + cudaGetErrorString(e));
    }
    count_launch();
    cudaError_t e = cudaGraphLaunch(b->graph, s);
    if (e != cudaSuccess) return bfail(AXHEL_ERR_CUDA, std::string("graph launch: ") + cudaGetErrorString(e));
    return AXHEL_OK;
}

axhel_status_t axhel_cuda_batch_status(axhel_batch_t b, void* stream)
{
    if (!b) return bfail(AXHEL_ERR_INVALID, "null batch");
    if (b->args.total_tiles == 0) return AXHEL_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int err = 0;
    cudaError_t e = cudaMemcpyAsync(&err, b->args.error, sizeof err, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return bfail(AXHEL_ERR_CUDA, std::string("batch status: ") + cudaGetErrorString(e));
    if (err) return bfail(err, "a dependency wait in the batch kernel timed out");
    return AXHEL_OK;
}

axhel_status_t axhel_cuda_batch_destroy(axhel_batch_t b)
{
    if (!b) return AXHEL_OK;
    if (b->graph) cudaGraphExecDestroy(b->graph);
    lanes_destroy(&b->lanes);
    if (b->mem) cudaFree(b->mem);
    for (axhel_ntt_t h : b->held) axhel_cuda_ntt_release(h);
    delete b;
    return AXHEL_OK;
}

axhel_status_t axhel_cuda_batch_run(const axhel_job_t* jobs, uint64_t n_jobs, void* stream)
{
    axhel_batch_t b = nullptr;
    axhel_status_t st = axhel_cuda_batch_create(jobs, n_jobs, &b);
    if (st) return st;
    st = axhel_cuda_batch_launch(b, stream);
    if (!st) st = axhel_cuda_batch_status(b, stream);
    axhel_cuda_batch_destroy(b);
    return st;
}

const char* axhel_cuda_batch_last_error(void) { return t_batch_error.c_str(); }

axhel_status_t axhel_cuda_batch_set_wait_ns(axhel_batch_t b, uint64_t ns)
{
    if (!b) return bfail(AXHEL_ERR_INVALID, "null batch");
    if (ns < 1000000ull || ns > 10000000000ull) return bfail(AXHEL_ERR_INVALID, "wait bound must be 1 ms .. 10 s");
    b->args.wait_ns = ns;
    if (b->graph) {  // the captured launch holds the old arguments
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return AXHEL_OK;
}

axhel_status_t axhel_cuda_batch_debug_unreachable(axhel_batch_t b, uint64_t job)
{
    if (!b || b->args.total_tiles == 0) return bfail(AXHEL_ERR_INVALID, "empty batch");
    // the job descriptors sit at the start of the batch allocation
    BatchJob* d = const_cast<BatchJob*>(b->args.jobs) + job;
    BatchJob host;
    cudaError_t e = cudaMemcpy(&host, d, sizeof host, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return bfail(AXHEL_ERR_CUDA, cudaGetErrorString(e));
    host.wait_extra = 1;
    e = cudaMemcpy(d, &host, sizeof host, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return bfail(AXHEL_ERR_CUDA, cudaGetErrorString(e));
    return AXHEL_OK;
}

}  // extern "C"
