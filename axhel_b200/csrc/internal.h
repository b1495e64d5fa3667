// Internal declarations shared by the CUDA kernels, the C-ABI layer and the
// C++ drop-in.  Nothing here is part of the public interface.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <string>

#include "../../include/axhel_cuda.h"

namespace axhel_impl {

// Device-resident constants of one (N, q) transform context; the twiddle
// tables follow it in the same allocation.  One per distinct (N, q, tables).
struct ModCtx {
    uint64_t q, q2;
    uint64_t ninv, ninv_q;    // N^-1 mod q and its Shoup quotient
    uint64_t sroot, sroot_q;  // reduce2->1(Shoup(inv[N-1], N^-1)) and quotient (ntt-native.cpp:109-113)
    uint64_t mu;              // Barrett factor floor(2^(k+62)/q), k = BitWidth(q)
    uint32_t shift;           // k - 2
    uint32_t logn;
    const ulonglong2* fwd;    // N entries {w, floor(w 2^64 / q)}, bit-reversed (ntt-tables.cpp:96-106)
    const ulonglong2* inv;    // N entries, inverse order (ntt-tables.cpp:113-129)
};
static_assert(sizeof(ModCtx) == 80, "ModCtx layout");

constexpr int kMaxInlineMods = 64;

// Pass-level flags, uniform per launch.
enum PassFlags : uint32_t {
    kPreCsub2q = 1u,     // x <- csub(x, 2q) on load (fuses EltwiseReduceMod 4->2 ahead of an inverse)
    kPostNorm = 2u,      // forward: 4->1 after the last stage; inverse: 2->1 after the final stage
    kLastPass = 4u,      // this pass holds global stage logN-1 (inverse: runs the N^-1 final stage)
    kPreMul = 8u,        // x <- MulMod<4>(x, operand) on load (a dyadic product ahead of an inverse)
    kPostMul = 16u,      // x <- MulMod<4>(x, operand) before the store (a dyadic product after a forward)
};

// Geometry of one pass: stages [s0, s0 + lg) of an N = 2^logn transform, on
// `count` limbs stored back to back (limb stride = N words).  Limb i uses
// ctx[i % nctx].
struct PassArgs {
    const uint64_t* src;
    uint64_t* dst;
    const uint64_t* operand;  // multiplicand of kPreMul / kPostMul, laid out like the data
    uint64_t count;
    uint32_t logn, s0, tg, flags;
    uint32_t nctx;
    const ModCtx* ctx[kMaxInlineMods];
};

// Chain operation applied between the inverse and the forward transform of a
// fused INTT -> op -> NTT job (per element at natural-order position p).
enum ChainOp : uint32_t { kChainNone = 0, kChainMul = 1, kChainFma = 2 };

struct ChainArgs {
    PassArgs pass;                // geometry of the shared column pass (inverse last pass == forward first pass)
    const uint64_t* operand;      // MulMod operand / FMA addend, laid out like the data (count x N), may be null for FMA
    const uint64_t* scalars;      // FMA scalar per modulus context (nctx entries, host-visible copy inlined below)
    uint64_t scalar[kMaxInlineMods];
    uint32_t op, op_factor;       // ChainOp and the MulMod/FMAMod input mod_factor
};

// One pass configuration chosen by the planner / autotuner.
struct PassCfg {
    int lg, lr, tg;
};
struct NttPlan {
    int npass;
    PassCfg pass[3];
};

// Kernel launchers (ntt.cu / eltwise.cu).  All return cudaError_t of launch.
cudaError_t launch_ntt_pass(bool inverse, const PassCfg& cfg, const PassArgs& a, cudaStream_t s);
cudaError_t launch_chain_pass(const PassCfg& inv_cfg, const ChainArgs& a, cudaStream_t s);
// The fused row pass of an NTT -> MulMod -> INTT product (contiguous groups;
// register depth at most 3).
cudaError_t launch_product_pass(const PassCfg& cfg, const ChainArgs& a, cudaStream_t s);
bool pass_supported(const PassCfg& cfg);

// Single-launch forms of a few limbs, one thread-block cluster per limb
// (ntt_cluster.cu): first-pass (transforms) or row (fused chains) stages,
// register stages, CTAs per cluster, and the largest limb count that takes
// this form; per kind: forward, inverse, INTT -> op -> NTT chain, NTT ->
// MulMod -> INTT product.
enum ClusterKind : int { kClusterForward = 0, kClusterInverse = 1, kClusterChain = 2, kClusterProduct = 3 };
struct ClusterCfg {
    int lga, lr, csize;
    uint64_t max_limbs;
};
bool cluster_cfg_valid(int kind, uint32_t logn, const ClusterCfg& c);
// The cluster form for (kind, logN, limbs), if it applies.
bool cluster_plan(int kind, uint32_t logn, uint64_t count, ClusterCfg* out);
void cluster_plan_override(int kind, uint32_t logn, const ClusterCfg* c);  // nullptr clears
ClusterCfg cluster_plan_current(int kind, uint32_t logn);
// The autotuner's table entry (`K` lines of ntt_plans.txt), between the
// override and the built-in choice.
void cluster_plan_table_set(int kind, uint32_t logn, const ClusterCfg& c);
cudaError_t launch_ntt_cluster(bool inverse, const ClusterCfg& c, const PassArgs& a, cudaStream_t s);
cudaError_t launch_ntt_cluster_fused(bool product, const ClusterCfg& c, const ChainArgs& a, cudaStream_t s);

// Planner (plan.cpp): default plan for (dir, logN, limbs); autotuned table if loaded.
NttPlan plan_for(bool inverse, uint32_t logn, uint64_t limbs);
bool plan_valid(const NttPlan& p, uint32_t logn, bool inverse);
int plan_load(const char* path);
void plan_override(bool inverse, uint32_t logn, const NttPlan* p);  // nullptr clears
bool plan_overridden(bool inverse, uint32_t logn);
void plan_table_ensure();  // loads ntt_plans.txt beside the library once
// Uneven-batch engine: stages of the contiguous pass of an N = 2^logn job
// (override > table > default); the strided pass takes the rest.
bool batch_row_valid(uint32_t logn, int row);
int batch_row_stages(uint32_t logn);
void batch_row_override(uint32_t logn, int row);  // 0 clears

// Bytes reserved for the ModCtx header in front of the twiddle tables.
constexpr size_t kCtxHeaderBytes = 256;

}  // namespace axhel_impl

// One (N, q) transform context: device allocation ModCtx | fwd[N] | inv[N].
struct axhel_ntt_ctx {
    std::atomic<int> refs{1};
    uint64_t n = 0, q = 0, root = 0;
    uint32_t logn = 0;
    int device = 0;
    bool cached = false;
    void* mem = nullptr;                       // device allocation
    bool shared_mem = false;                   // mem lies in one block with the contexts created beside it
    bool external = false;                     // tables supplied by the caller (axhel_cuda_ntt_create_external)
    const axhel_impl::ModCtx* dctx = nullptr;  // device address of the ModCtx header
};
