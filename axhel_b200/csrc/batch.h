// Descriptors of the uneven-batch engine (batch.cu), shared with the
// static-scratch entry point (batch_static.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/axhel_cuda.h"
#include "internal.h"

namespace axhel_impl {

constexpr int kBatchThreads = 128;
constexpr int kBatchLR = 3;
constexpr int kBatchTileWords = kBatchThreads << kBatchLR;  // 1024 residues
constexpr int kBatchTileLog = 10;                           // tiles per limb: 2^(logn - 10)
static_assert(kBatchTileWords == 1 << kBatchTileLog, "tile size");
constexpr int kBatchPublisher = 32;                         // persistent kernel: the thread that publishes tiles
static_assert(kBatchThreads > kBatchPublisher, "publisher in a second warp");
constexpr int kBatchMinLG = 5, kBatchMaxLG = 9;
// CTAs per SM the persistent kernel (and the grouped per-phase launches of
// 128 threads) are compiled for: 64 registers (128 without the bound) and
// some spills, which cost less than the latency the extra resident warps
// hide -- measured on the 512-polynomial uneven batch with the generic
// kernels: 5 CTAs 1.08 M / 1.28 M limb-transforms/s (persistent / per
// phase), 7 CTAs 1.25 M / 1.36 M, 8 CTAs 1.29 M / 1.46 M.
constexpr int kBatchMinBlocks = 8;

enum BatchKind : uint32_t {
    kJobForward = 1, kJobInverse = 2, kJobChainMul = 3, kJobChainFma = 4,
    kJobAdd = 5, kJobSub = 6, kJobMul = 7, kJobFma = 8, kJobReduce = 9  // element-wise, one phase
};

// Element-wise operation of an element-wise job, resolved on the host.
enum EltOp : uint32_t {
    kEltAddVV, kEltAddVS, kEltSubVV, kEltSubVS, kEltMul, kEltFma, kEltFmaAdd, kEltReduce
};

struct BatchJob {
    const uint64_t* src;
    uint64_t* dst;
    const uint64_t* vec;              // chain multiplicand / addend (may be null for FMA)
    const ModCtx* const* ctx;         // nmods device pointers
    const uint64_t* scalars;          // chain FMA scalars (nmods), device
    uint64_t count;                   // limbs
    uint64_t done_off;                // first completion counter of this job (count per phase)
    uint32_t kind, logn, nmods, nphase;
    uint32_t lg_col, lg_row;          // pass widths A (strided) and B (contiguous)
    uint32_t tiles_per_limb[3];
    uint32_t pre, norm;               // fuse ReduceMod(4,2) on load / normalize the output
    uint32_t wait_extra;              // added to every dependency target (0; a test sets 1 to force a timeout)
    uint32_t eop, ef;                 // element-wise jobs: EltOp, and its factor (ReduceMod: branch 0..4)
};

struct BatchEntry {
    uint64_t tile_begin;  // first global tile of (job, phase)
    uint32_t job, phase;
};

// Tile classes of the per-phase launches: each class runs in a kernel of its
// own (its own register budget and register depth).
enum TileClass : uint32_t { kClsFwd = 0, kClsInv = 1, kClsChain = 2, kClsElt = 3 };

// One entry of a class launch: a (job, phase) with what its tiles read, and
// its first tile in the launch's numbering.
struct ClassEntry {
    uint64_t tile0;
    const uint64_t* src;               // the job's operand in phase 0, its result after
    uint64_t* dst;
    const uint64_t* vec;               // chain multiplicand / addend, element-wise second operand
    const ModCtx* const* ctx;          // nmods device pointers
    const uint64_t* scalars;           // per modulus: chain FMA, element-wise scalar ops; else null
    uint32_t nmods, logn, s0, flags;   // transform passes: first stage, the tile functions' flags
    uint32_t op, eop, ef;              // chain op; element-wise op and factor
    uint32_t cls_lg;                   // tile class << 8 | pass width
};

// One launch of a phase: the tiles of one class and pass width, from
// every job of the batch, in entry order; or one large entry alone.
struct ClassLaunch {
    uint32_t phase, cls, lg, n_ce;
    const ClassEntry* ce;  // device address, n_ce entries
    uint64_t tiles;
    ClassEntry first;      // host copy of ce[0]: a launch of one entry takes it as a kernel parameter
    // A launch of one transform or chain entry can instead run as the
    // specialized pass / chain kernel with the tuned plan's tile shape for
    // its pass (spec 1: pass kernel, 2: chain kernel; 0: class kernel only).
    uint32_t spec = 0;
    bool spec_inv = false;
    PassCfg spec_cfg{};
    ChainArgs spec_args{};
};

struct BatchArgs {
    const BatchJob* jobs;
    const BatchEntry* entries;
    const ClassEntry* tile_args;        // per entry: what its tiles read (tile0: its first global tile)
    uint32_t nentries;
    uint64_t total_tiles;
    unsigned int* done;                 // per (job, phase, limb) completed tiles
    unsigned long long* next_tile;      // work counter
    int* error;                         // AXHEL_OK or AXHEL_ERR_TIMEOUT
    uint64_t wait_ns;                   // a dependency wait gives up after this long
};

// Checks one job against the batch engine's contract (kinds, degrees,
// pointers, factors); `who` names it in the message.
axhel_status_t batch_check_job(const axhel_job_t& job, const std::string& who, std::string* err);

// Lays out the device image of a batch for the device address `base`:
// fills `host` (to be copied to `base`), the range of counters that must be
// zero before a launch, and the kernel arguments.  NTT handles referenced by
// the jobs are appended to `held` when it is not null.  Tiles are numbered
// phase-major.  `classes`, when not null, receives the per-phase launches
// (batch_launch_classes) and the image then holds their entry tables: give
// it to the sizing pass and to the final build alike.
axhel_status_t batch_build(const axhel_job_t* jobs, uint64_t n_jobs, unsigned char* base,
                           std::vector<unsigned char>& host, size_t* zero_off, size_t* zero_bytes, BatchArgs* args,
                           std::vector<axhel_ntt_t>* held, std::string* err,
                           std::vector<ClassLaunch>* classes = nullptr);

// Launches the persistent batch kernel for prepared arguments.
cudaError_t batch_launch_args(const BatchArgs& a, cudaStream_t s);

// Streams that run one phase's launches side by side: forked from the
// caller's stream by an event and joined back into it before the next phase.
constexpr int kLaunchLanes = 4;  // the caller's stream and three more
struct LaunchLanes {
    cudaStream_t st[kLaunchLanes - 1] = {};
    cudaEvent_t fork = nullptr, join[kLaunchLanes - 1] = {};
};
cudaError_t lanes_create(LaunchLanes* l, int priority);
void lanes_destroy(LaunchLanes* l);

// Runs a prepared batch as ordinary (non-persistent) launches, one per
// (phase, tile class, pass width) plus one for each of a phase's largest
// entries, one CTA per tile and no waits inside a launch; a phase's launches
// run side by side on `lanes` (when given) and the phases are ordered by the
// stream.  Each class runs in a kernel specialized for it (register depth
// and budget).  Concurrent batches on other streams share the SMs tile by
// tile.  `classes` as filled by batch_build.
cudaError_t batch_launch_classes(const std::vector<ClassLaunch>& classes, cudaStream_t s,
                                 const LaunchLanes* lanes, bool specialized = false);

// Records the message returned by axhel_cuda_batch_last_error on this thread.
void batch_set_error(const std::string& msg);

}  // namespace axhel_impl
