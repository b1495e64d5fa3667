// C-ABI entry points (include/axhel_cuda.h): argument checking, the
// device-resident NTT table cache, and pass sequencing for the transforms.
#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/axhel_cuda.h"
#include "internal.h"
#include "tables.h"
#include "launch.h"

using namespace axhel_impl;

// ------------------------------------------------------------ bookkeeping

namespace {

thread_local std::string t_last_error;

axhel_status_t fail(axhel_status_t st, const std::string& msg)
{
    t_last_error = msg;
    return st;
}

axhel_status_t cuda_fail(cudaError_t e, const char* where)
{
    return fail(AXHEL_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

inline uint64_t bit_width(uint64_t x) { return x ? 64 - __builtin_clzll(x) : 0; }
typedef unsigned __int128 u128;

inline uint64_t shoup_quotient(uint64_t w, uint64_t q) { return (uint64_t)(((u128)w << 64) / q); }
inline uint64_t shoup_lazy(uint64_t v, uint64_t w, uint64_t wq, uint64_t q)
{
    return v * w - (uint64_t)(((u128)v * wq) >> 64) * q;
}
inline uint64_t mulmod(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((u128)a * b) % q); }
uint64_t powmod(uint64_t b, uint64_t e, uint64_t q)
{
    uint64_t r = 1;
    b %= q;
    while (e) {
        if (e & 1) r = mulmod(r, b, q);
        e >>= 1;
        if (e) b = mulmod(b, b, q);
    }
    return r;
}

}  // namespace

namespace axhel_impl {

int sm_count()
{
    static std::atomic<int> cache[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return 148;
    int n = cache[dev].load(std::memory_order_relaxed);
    if (!n) {
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cache[dev].store(n, std::memory_order_relaxed);
    }
    return n;
}

}  // namespace axhel_impl

// -------------------------------------------------------- table contexts

namespace {

std::mutex g_cache_mu;
std::map<std::tuple<int, uint64_t, uint64_t, uint64_t>, axhel_ntt_ctx*> g_cache;

constexpr size_t kHeader = kCtxHeaderBytes;

// The context header (ModCtx) for tables at `base`: N^-1 with its quotient,
// and the scaled root of the final inverse stage computed from the last
// inverse twiddle exactly as ntt-native.cpp:101-113.
ModCtx make_header(const axhel_ntt_ctx* c, unsigned char* base, uint64_t inv_last, uint64_t ninv, uint64_t ninv_q)
{
    ModCtx h{};
    h.q = c->q;
    h.q2 = c->q << 1;
    h.ninv = ninv;
    h.ninv_q = ninv_q;
    uint64_t sr = shoup_lazy(inv_last, ninv, ninv_q, c->q);
    if (sr >= c->q) sr -= c->q;
    h.sroot = sr;
    h.sroot_q = shoup_quotient(sr, c->q);
    barrett_params(c->q, &h.mu, &h.shift);
    h.logn = c->logn;
    h.fwd = reinterpret_cast<const ulonglong2*>(base + kHeader);
    h.inv = reinterpret_cast<const ulonglong2*>(base + kHeader + c->n * 16);
    return h;
}

// Caller-provided tables (the external-table constructor, ntt.cpp:124-133):
// copied into one device allocation behind their header.
axhel_status_t upload(axhel_ntt_ctx* c, const uint64_t* fwd, const uint64_t* inv, const uint64_t* ninv)
{
    const size_t tab = c->n * 16;
    const size_t total = kHeader + 2 * tab;
    std::vector<unsigned char> img(total, 0);
    cudaError_t e = cudaMalloc(&c->mem, total);
    if (e != cudaSuccess) return fail(AXHEL_ERR_NOMEM, std::string("cudaMalloc(tables): ") + cudaGetErrorString(e));
    unsigned char* base = static_cast<unsigned char*>(c->mem);
    const ModCtx h = make_header(c, base, inv[2 * (c->n - 1)], ninv[0], ninv[1]);
    std::memcpy(img.data(), &h, sizeof h);
    std::memcpy(img.data() + kHeader, fwd, tab);
    std::memcpy(img.data() + kHeader + tab, inv, tab);
    e = cudaMemcpy(c->mem, img.data(), total, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(c->mem);
        c->mem = nullptr;
        return cuda_fail(e, "cudaMemcpy(tables)");
    }
    c->dctx = reinterpret_cast<const ModCtx*>(base);
    return AXHEL_OK;
}

// Header and Montgomery constants for generating the tables of (N, q, psi)
// on the device (tables.cu) into c->mem.  GenerateNTTTables'
// host-side scalars (ntt-tables.cpp:109, 132-136): psi^-1 = psi^(q-2),
// N^-1 = (N mod q)^(q-2).
void gen_job(const axhel_ntt_ctx* c, uint64_t psi, TableGenJob* j)
{
    const uint64_t q = c->q, n = c->n;
    const uint64_t psi_inv = powmod(psi, q - 2, q);
    const uint64_t ninv = powmod(n % q, q - 2, q);
    uint64_t rev = 0;  // bitrev(n - 2): the last inverse entry is psi^-(bitrev(n-2)+1)
    for (uint32_t b = 0; b < c->logn; ++b) rev |= (((n - 2) >> b) & 1) << (c->logn - 1 - b);
    unsigned char* base = static_cast<unsigned char*>(c->mem);
    j->hdr = make_header(c, base, powmod(psi_inv, rev + 1, q), ninv, shoup_quotient(ninv, q));
    j->base = base;
    j->q = q;
    uint64_t x = q;  // q^-1 mod 2^64 by Newton's iteration (q odd)
    for (int k = 0; k < 6; ++k) x *= 2 - q * x;
    j->mninv = 0 - x;
    j->one_m = (uint64_t)(((u128)1 << 64) % q);
    j->r2m = (uint64_t)(((u128)j->one_m * j->one_m) % q);
    j->psi_m = (uint64_t)(((u128)(psi % q) << 64) % q);
    j->psiinv_m = (uint64_t)(((u128)psi_inv << 64) % q);
    j->n = n;
    j->logn = c->logn;
    j->pad = 0;
}

axhel_status_t check_modulus(uint64_t q, uint64_t limit_bits)
{
    if (q < 2 || bit_width(q) > limit_bits)
        return fail(AXHEL_ERR_INVALID, "modulus out of range (need 2 <= q < 2^" + std::to_string(limit_bits) + ")");
    return AXHEL_OK;
}

axhel_status_t check_degree(uint64_t n, uint32_t* logn)
{
    if (n < AXHEL_MIN_DEGREE || n > AXHEL_MAX_DEGREE || (n & (n - 1)))
        return fail(AXHEL_ERR_UNSUPPORTED, "degree must be a power of two in [2, 131072]");
    uint32_t l = 0;
    while ((1ull << l) < n) ++l;
    *logn = l;
    return AXHEL_OK;
}

inline cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }

}  // namespace

extern "C" {

const char* axhel_status_string(axhel_status_t st)
{
    switch (st) {
    case AXHEL_OK: return "ok";
    case AXHEL_ERR_INVALID: return "invalid argument";
    case AXHEL_ERR_CUDA: return "CUDA error";
    case AXHEL_ERR_NOMEM: return "out of memory";
    case AXHEL_ERR_UNSUPPORTED: return "unsupported configuration";
    case AXHEL_ERR_BUSY: return "busy";
    case AXHEL_ERR_TIMEOUT: return "timeout";
    case AXHEL_ERR_REJECTED: return "rejected";
    case AXHEL_ERR_CANCELLED: return "cancelled";
    default: return "unknown status";
    }
}

const char* axhel_last_error(void) { return t_last_error.c_str(); }
int axhel_version(void) { return 100; }

int axhel_cuda_is_device_pointer(const void* p)
{
    if (!p) return 0;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

axhel_status_t axhel_cuda_ntt_create(uint64_t degree, uint64_t modulus, uint64_t root, axhel_ntt_t* out)
{
    return axhel_cuda_ntt_create_many(1, &degree, &modulus, &root, out);
}

axhel_status_t axhel_cuda_ntt_create_many(uint64_t count, const uint64_t* degrees, const uint64_t* moduli,
                                          const uint64_t* roots, axhel_ntt_t* out)
{
    if (!out || (count && (!degrees || !moduli || !roots))) return fail(AXHEL_ERR_INVALID, "null argument");
    for (uint64_t i = 0; i < count; ++i) out[i] = nullptr;
    std::vector<uint32_t> logn(count);
    for (uint64_t i = 0; i < count; ++i) {
        axhel_status_t st = check_degree(degrees[i], &logn[i]);
        if (st) return st;
        if ((st = check_modulus(moduli[i], 62))) return st;
        if (!(moduli[i] & 1))
            return fail(AXHEL_ERR_INVALID, "the modulus must be odd (an NTT modulus is a prime q = 1 mod 2N)");
        if (roots[i] == 0 || roots[i] >= moduli[i]) return fail(AXHEL_ERR_INVALID, "root of unity must be in [1, q)");
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    std::lock_guard<std::mutex> lk(g_cache_mu);
    // cache hits take a reference; misses (each distinct key once) get an
    // allocation and a generation job
    std::map<std::tuple<int, uint64_t, uint64_t, uint64_t>, axhel_ntt_ctx*> fresh;
    std::vector<axhel_ntt_ctx*> order;  // the fresh contexts, in creation order
    std::vector<TableGenJob> jobs;
    void* block = nullptr;
    auto undo = [&](axhel_status_t st, const std::string& m) {
        for (uint64_t i = 0; i < count; ++i)
            if (out[i] && out[i]->cached && !fresh.count(std::make_tuple(dev, degrees[i], moduli[i], roots[i])))
                out[i]->refs.fetch_sub(1);
        for (auto& kv : fresh) delete kv.second;
        if (block) cudaFree(block);
        for (uint64_t i = 0; i < count; ++i) out[i] = nullptr;
        return fail(st, m);
    };
    for (uint64_t i = 0; i < count; ++i) {
        const auto key = std::make_tuple(dev, degrees[i], moduli[i], roots[i]);
        auto it = g_cache.find(key);
        if (it != g_cache.end()) {
            it->second->refs.fetch_add(1);
            out[i] = it->second;
            continue;
        }
        auto f = fresh.find(key);
        if (f != fresh.end()) {
            f->second->refs.fetch_add(1);
            out[i] = f->second;
            continue;
        }
        auto* c = new axhel_ntt_ctx();
        c->n = degrees[i];
        c->q = moduli[i];
        c->root = roots[i];
        c->logn = logn[i];
        c->device = dev;
        c->cached = true;
        c->refs.store(2);  // the cache keeps one reference: tables stay resident for the process
        fresh[key] = c;
        out[i] = c;
        order.push_back(c);
    }
    // One device block for all the fresh contexts' headers and tables: cached
    // contexts stay resident for the process, and one cudaMalloc instead of
    // one per context is most of a cold start's host time.
    std::vector<size_t> offs(order.size());
    size_t total = 0;
    for (size_t k = 0; k < order.size(); ++k) {
        offs[k] = total;
        total += (kHeader + 2 * order[k]->n * 16 + 255) / 256 * 256;
    }
    if (total && (e = cudaMalloc(&block, total)) != cudaSuccess) {
        block = nullptr;
        return undo(AXHEL_ERR_NOMEM, std::string("cudaMalloc(tables): ") + cudaGetErrorString(e));
    }
    for (size_t k = 0; k < order.size(); ++k) {
        axhel_ntt_ctx* c = order[k];
        c->mem = static_cast<unsigned char*>(block) + offs[k];
        c->shared_mem = true;
        c->dctx = reinterpret_cast<const ModCtx*>(c->mem);
        jobs.emplace_back();
        gen_job(c, c->root, &jobs.back());
    }
    // one launch per 96 contexts, then wait: the tables are complete when
    // this returns, for any stream of any thread
    const cudaStream_t s = cudaStreamPerThread;
    for (size_t k = 0; k < jobs.size(); k += kTableGenJobsPerLaunch) {
        TableGenArgs a{};
        uint64_t max_n = 0;
        for (size_t m = k; m < jobs.size() && a.njobs < (uint32_t)kTableGenJobsPerLaunch; ++m) {
            a.job[a.njobs++] = jobs[m];
            max_n = std::max<uint64_t>(max_n, jobs[m].n);
        }
        if ((e = launch_gen_tables(a, max_n, s)) != cudaSuccess) return undo(AXHEL_ERR_CUDA, cudaGetErrorString(e));
    }
    if (!jobs.empty() && (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return undo(AXHEL_ERR_CUDA, std::string("table generation: ") + cudaGetErrorString(e));
    for (auto& kv : fresh) g_cache[kv.first] = kv.second;
    return AXHEL_OK;
}

axhel_status_t axhel_cuda_ntt_create_external(uint64_t degree, uint64_t modulus, const uint64_t* fwd,
                                              const uint64_t* inv, const uint64_t* ninv, axhel_ntt_t* out)
{
    if (!out) return fail(AXHEL_ERR_INVALID, "null output handle");
    *out = nullptr;
    uint32_t logn;
    axhel_status_t st = check_degree(degree, &logn);
    if (st) return st;
    if ((st = check_modulus(modulus, 62))) return st;
    if (!fwd || !inv || !ninv) return fail(AXHEL_ERR_INVALID, "null table pointer");
    auto c = std::make_unique<axhel_ntt_ctx>();
    c->n = degree;
    c->q = modulus;
    c->logn = logn;
    cudaGetDevice(&c->device);
    if ((st = upload(c.get(), fwd, inv, ninv))) return st;
    c->external = true;
    *out = c.release();
    return AXHEL_OK;
}

axhel_status_t axhel_cuda_ntt_refresh_external(axhel_ntt_t h, const uint64_t* fwd, const uint64_t* inv,
                                               const uint64_t* ninv, void* stream)
{
    if (!h || !h->external) return fail(AXHEL_ERR_INVALID, "not a handle made from external tables");
    if (inv && !ninv) return fail(AXHEL_ERR_INVALID, "the inverse table needs its N^-1 pair");
    const size_t tab = h->n * 16;
    unsigned char* base = static_cast<unsigned char*>(h->mem);
    cudaStream_t s = S(stream);
    // Pageable sources: each copy has read its source when the call returns.
    cudaError_t e = cudaSuccess;
    if (fwd) e = cudaMemcpyAsync(base + kHeader, fwd, tab, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && inv) {
        const ModCtx hd = make_header(h, base, inv[2 * (h->n - 1)], ninv[0], ninv[1]);
        e = cudaMemcpyAsync(base + kHeader + tab, inv, tab, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(base, &hd, sizeof hd, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the header copy reads this stack frame
    }
    if (e != cudaSuccess) return cuda_fail(e, "refresh external tables");
    return AXHEL_OK;
}

axhel_status_t axhel_cuda_ntt_retain(axhel_ntt_t h)
{
    if (!h) return fail(AXHEL_ERR_INVALID, "null handle");
    h->refs.fetch_add(1);
    return AXHEL_OK;
}

axhel_status_t axhel_cuda_ntt_release(axhel_ntt_t h)
{
    if (!h) return AXHEL_OK;
    if (h->refs.fetch_sub(1) == 1) {
        if (h->mem && !h->shared_mem) cudaFree(h->mem);
        delete h;
    }
    return AXHEL_OK;
}

uint64_t axhel_cuda_ntt_degree(axhel_ntt_t h) { return h ? h->n : 0; }
uint64_t axhel_cuda_ntt_modulus(axhel_ntt_t h) { return h ? h->q : 0; }

axhel_status_t axhel_cuda_ntt_read_tables(axhel_ntt_t h, uint64_t* fwd, uint64_t* inv, uint64_t* ninv)
{
    if (!h || !fwd || !inv || !ninv) return fail(AXHEL_ERR_INVALID, "null argument");
    const unsigned char* base = static_cast<const unsigned char*>(h->mem);
    cudaError_t e = cudaMemcpy(fwd, base + kHeader, h->n * 16, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(inv, base + kHeader + h->n * 16, h->n * 16, cudaMemcpyDeviceToHost);
    ModCtx m;
    if (e == cudaSuccess) e = cudaMemcpy(&m, base, sizeof m, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy(read tables)");
    ninv[0] = m.ninv;
    ninv[1] = m.ninv_q;
    return AXHEL_OK;
}

}  // extern "C"

// ------------------------------------------------------------ transforms

namespace {

axhel_status_t collect(const axhel_ntt_t* ntts, uint64_t n_ntts, PassArgs& a, uint64_t* n_out)
{
    if (!ntts || n_ntts == 0) return fail(AXHEL_ERR_INVALID, "no NTT handles");
    if (n_ntts > (uint64_t)kMaxInlineMods) return fail(AXHEL_ERR_UNSUPPORTED, "at most 64 moduli per batch");
    const uint64_t n = ntts[0] ? ntts[0]->n : 0;
    for (uint64_t i = 0; i < n_ntts; ++i) {
        if (!ntts[i]) return fail(AXHEL_ERR_INVALID, "null NTT handle");
        if (ntts[i]->n != n) return fail(AXHEL_ERR_INVALID, "all limbs of a batch need one degree");
        a.ctx[i] = ntts[i]->dctx;
    }
    a.nctx = (uint32_t)n_ntts;
    a.logn = ntts[0]->logn;
    *n_out = n;
    return AXHEL_OK;
}

// Runs the passes of `plan` in order; pass i reads `src` (first pass) or
// `dst`, writes `dst`.
axhel_status_t run_plan(bool inverse, const NttPlan& plan, PassArgs a, const uint64_t* src, uint64_t* dst,
                        uint32_t first_flags, uint32_t last_flags, cudaStream_t s)
{
    uint32_t s0 = 0;
    for (int i = 0; i < plan.npass; ++i) {
        const PassCfg& c = plan.pass[i];
        a.src = i == 0 ? src : dst;
        a.dst = dst;
        a.s0 = s0;
        a.tg = (uint32_t)c.tg;
        a.flags = (i == 0 ? first_flags : 0) | (i == plan.npass - 1 ? (last_flags | kLastPass) : 0);
        cudaError_t e = launch_ntt_pass(inverse, c, a, s);
        if (e != cudaSuccess) return cuda_fail(e, inverse ? "inverse NTT pass" : "forward NTT pass");
        s0 += (uint32_t)c.lg;
    }
    return AXHEL_OK;
}

// `mul` (optional): the dyadic product with it fused into the transform --
// ahead of an inverse (MulMod<4> on load, so inputs in [0, 4q)) or after a
// forward (MulMod<4> of the lazy [0, 4q) output; canonical result).
// A cluster launch the GPU cannot place (a cluster needs its CTAs on the SMs
// of one GPC at once; a partitioned or smaller GPU may not have them): the
// caller falls back to the pass kernels.  Clears the error.
bool cluster_unschedulable(cudaError_t e)
{
    if (e != cudaErrorInvalidClusterSize) return false;  // "cluster misconfiguration"
    cudaGetLastError();
    return true;
}

axhel_status_t transform(bool inverse, const axhel_ntt_t* ntts, uint64_t n_ntts, uint64_t* result,
                         const uint64_t* operand, uint64_t count, uint64_t in_f, uint64_t out_f, bool batch_api,
                         void* stream, const uint64_t* mul = nullptr)
{
    PassArgs a{};
    uint64_t n;
    axhel_status_t st = collect(ntts, n_ntts, a, &n);
    if (st) return st;
    if (count == 0) return AXHEL_OK;
    if (!result || !operand) return fail(AXHEL_ERR_INVALID, "null data pointer");
    a.count = count;
    a.operand = mul;
    uint32_t first = 0, last = 0;
    if (mul) {
        if (inverse) {
            first |= kPreMul;
            if (out_f != 2) last |= kPostNorm;
        } else {
            last |= kPostMul;
        }
    } else if (inverse) {
        if (batch_api && in_f == 4) first |= kPreCsub2q;
        if (out_f != 2) last |= kPostNorm;  // ntt.cpp:198-203
    } else {
        if (out_f != 4) last |= kPostNorm;  // ntt.cpp:180-185
    }
    // a few limbs: both passes in one launch, one cluster per limb (unless a
    // pass plan was set explicitly for this degree)
    ClusterCfg cc;
    if (!plan_overridden(inverse, a.logn) &&
        cluster_plan(inverse ? kClusterInverse : kClusterForward, a.logn, count, &cc)) {
        a.src = operand;
        a.dst = result;
        a.s0 = 0;
        a.tg = 0;
        a.flags = first | last | kLastPass;
        const cudaError_t e = launch_ntt_cluster(inverse, cc, a, S(stream));
        if (e == cudaSuccess) return AXHEL_OK;
        if (!cluster_unschedulable(e))
            return cuda_fail(e, inverse ? "inverse NTT (cluster)" : "forward NTT (cluster)");
        // the GPU cannot place the cluster (fewer SMs per GPC): the pass form
    }
    const NttPlan plan = plan_for(inverse, a.logn, count);
    return run_plan(inverse, plan, a, operand, result, first, last, S(stream));
}

axhel_status_t chain(const axhel_ntt_t* ntts, uint64_t n_ntts, uint64_t* result, const uint64_t* operand,
                     const uint64_t* vec, const uint64_t* scalars, uint32_t op, uint64_t count, uint64_t in_f,
                     uint64_t out_f, void* stream)
{
    ChainArgs c{};
    uint64_t n;
    axhel_status_t st = collect(ntts, n_ntts, c.pass, &n);
    if (st) return st;
    if (count == 0) return AXHEL_OK;
    if (!result || !operand) return fail(AXHEL_ERR_INVALID, "null data pointer");
    if (op == kChainMul && !vec) return fail(AXHEL_ERR_INVALID, "null multiplicand");
    if (op == kChainFma && !scalars) return fail(AXHEL_ERR_INVALID, "null scalars");
    c.pass.count = count;
    const uint32_t logn = c.pass.logn;
    // a few limbs: the whole chain in one launch, one cluster per limb
    ClusterCfg cc;
    if (!plan_overridden(true, logn) && cluster_plan(kClusterChain, logn, count, &cc)) {
        c.pass.src = operand;
        c.pass.dst = result;
        c.pass.flags = (in_f == 4 ? (uint32_t)kPreCsub2q : 0u) | (out_f != 4 ? (uint32_t)kPostNorm : 0u);
        c.operand = vec;
        c.op = op;
        c.op_factor = 2;
        if (op == kChainFma)
            for (uint64_t i = 0; i < n_ntts; ++i) c.scalar[i] = scalars[i];
        const cudaError_t e = launch_ntt_cluster_fused(false, cc, c, S(stream));
        if (e == cudaSuccess) return AXHEL_OK;
        if (!cluster_unschedulable(e)) return cuda_fail(e, "chain (cluster)");
    }
    const NttPlan inv = plan_for(true, logn, count);
    // forward passes after the fused one: the inverse's earlier passes, reversed
    NttPlan fwd{};
    fwd.npass = inv.npass;
    for (int i = 0; i < inv.npass; ++i) fwd.pass[i] = inv.pass[inv.npass - 1 - i];
    cudaStream_t s = S(stream);
    // inverse passes before the fused column pass
    uint32_t s0 = 0;
    const uint64_t* src = operand;
    for (int i = 0; i + 1 < inv.npass; ++i) {
        PassArgs a = c.pass;
        a.src = src;
        a.dst = result;
        a.s0 = s0;
        a.tg = (uint32_t)inv.pass[i].tg;
        a.flags = (i == 0 && in_f == 4) ? (uint32_t)kPreCsub2q : 0u;
        cudaError_t e = launch_ntt_pass(true, inv.pass[i], a, s);
        if (e != cudaSuccess) return cuda_fail(e, "chain inverse pass");
        s0 += (uint32_t)inv.pass[i].lg;
        src = result;
    }
    // fused: inverse last pass -> op -> forward first pass.  It holds both
    // transforms' rounds and the op's operand, so with 16 registers per
    // thread (LR = 4) it needs 128 registers; 8 (LR = 3) keep it at 76 and
    // measured 3 % faster at N = 2^16, 768 limbs.
    PassCfg fc = inv.pass[inv.npass - 1];
    if (fc.lr > 3 && fc.lg >= 4 && ((uint64_t)fc.tg << (fc.lg - 3)) <= 512) fc.lr = 3;
    c.pass.src = src;
    c.pass.dst = result;
    c.pass.s0 = s0;
    c.pass.tg = (uint32_t)fc.tg;
    c.pass.flags = (inv.npass == 1 && in_f == 4 ? (uint32_t)kPreCsub2q : 0u) |
                   (fwd.npass == 1 && out_f != 4 ? (uint32_t)kPostNorm : 0u);
    c.operand = vec;
    c.op = op;
    c.op_factor = 2;
    if (op == kChainFma)
        for (uint64_t i = 0; i < n_ntts; ++i) c.scalar[i] = scalars[i];
    cudaError_t e = launch_chain_pass(fc, c, s);
    if (e != cudaSuccess) return cuda_fail(e, "chain fused pass");
    // remaining forward passes
    uint32_t f0 = (uint32_t)fc.lg;
    for (int i = 1; i < fwd.npass; ++i) {
        PassArgs a = c.pass;
        a.src = result;
        a.dst = result;
        a.s0 = f0;
        a.tg = (uint32_t)fwd.pass[i].tg;
        a.flags = (i == fwd.npass - 1) ? ((uint32_t)kLastPass | (out_f != 4 ? (uint32_t)kPostNorm : 0u)) : 0u;
        e = launch_ntt_pass(false, fwd.pass[i], a, s);
        if (e != cudaSuccess) return cuda_fail(e, "chain forward pass");
        f0 += (uint32_t)fwd.pass[i].lg;
    }
    return AXHEL_OK;
}

// NTT -> MulMod -> INTT over a batch: the forward's passes up to its last
// (contiguous) one, that pass fused with the dyadic product and the
// inverse's first pass, then the inverse's remaining passes.  The forward
// runs the inverse plan's passes in reverse order, so its last pass is the
// inverse's first (the same groups).
axhel_status_t product(const axhel_ntt_t* ntts, uint64_t n_ntts, uint64_t* result, const uint64_t* operand,
                       const uint64_t* vec, uint64_t count, uint64_t out_f, void* stream)
{
    ChainArgs c{};
    uint64_t n;
    axhel_status_t st = collect(ntts, n_ntts, c.pass, &n);
    if (st) return st;
    if (count == 0) return AXHEL_OK;
    if (!result || !operand || !vec) return fail(AXHEL_ERR_INVALID, "null data pointer");
    if (vec == result) return fail(AXHEL_ERR_INVALID, "the multiplicand must not be the result buffer");
    c.pass.count = count;
    const uint32_t logn = c.pass.logn;
    // a few limbs: the whole product in one launch, one cluster per limb
    ClusterCfg cc;
    if (!plan_overridden(true, logn) && cluster_plan(kClusterProduct, logn, count, &cc)) {
        c.pass.src = operand;
        c.pass.dst = result;
        c.pass.flags = out_f != 2 ? (uint32_t)kPostNorm : 0u;
        c.operand = vec;
        c.op = kChainMul;
        c.op_factor = 4;
        const cudaError_t e = launch_ntt_cluster_fused(true, cc, c, S(stream));
        if (e == cudaSuccess) return AXHEL_OK;
        if (!cluster_unschedulable(e)) return cuda_fail(e, "product (cluster)");
    }
    const NttPlan inv = plan_for(true, logn, count);
    cudaStream_t s = S(stream);
    // forward passes before the fused one: the inverse plan's passes npass-1 .. 1
    uint32_t f0 = 0;
    const uint64_t* src = operand;
    for (int i = inv.npass - 1; i >= 1; --i) {
        PassArgs a = c.pass;
        a.src = src;
        a.dst = result;
        a.s0 = f0;
        a.tg = (uint32_t)inv.pass[i].tg;
        a.flags = 0;
        cudaError_t e = launch_ntt_pass(false, inv.pass[i], a, s);
        if (e != cudaSuccess) return cuda_fail(e, "product forward pass");
        f0 += (uint32_t)inv.pass[i].lg;
        src = result;
    }
    // fused: forward last pass -> MulMod -> inverse first pass (register depth 3:
    // the pass holds both transforms' rounds and the multiplicand)
    PassCfg fc = inv.pass[0];
    if (fc.lr > 3 && fc.lg >= 4 && ((uint64_t)fc.tg << (fc.lg - 3)) <= 512) fc.lr = 3;
    if (fc.lr > 3) return fail(AXHEL_ERR_UNSUPPORTED, "no fused product pass for this plan");
    c.pass.src = src;
    c.pass.dst = result;
    c.pass.s0 = 0;
    c.pass.tg = (uint32_t)fc.tg;
    c.pass.flags = inv.npass == 1 ? ((uint32_t)kLastPass | (out_f != 2 ? (uint32_t)kPostNorm : 0u)) : 0u;
    c.operand = vec;
    c.op = kChainMul;
    c.op_factor = 4;
    cudaError_t e = launch_product_pass(fc, c, s);
    if (e != cudaSuccess) return cuda_fail(e, "product fused pass");
    // the inverse's remaining passes
    uint32_t i0 = (uint32_t)fc.lg;
    for (int i = 1; i < inv.npass; ++i) {
        PassArgs a = c.pass;
        a.src = result;
        a.dst = result;
        a.s0 = i0;
        a.tg = (uint32_t)inv.pass[i].tg;
        a.flags = (i == inv.npass - 1) ? ((uint32_t)kLastPass | (out_f != 2 ? (uint32_t)kPostNorm : 0u)) : 0u;
        e = launch_ntt_pass(true, inv.pass[i], a, s);
        if (e != cudaSuccess) return cuda_fail(e, "product inverse pass");
        i0 += (uint32_t)inv.pass[i].lg;
    }
    return AXHEL_OK;
}

}  // namespace

extern "C" {

axhel_status_t axhel_cuda_ntt_product_batch(const axhel_ntt_t* ntts, uint64_t n_ntts, uint64_t* result,
                                            const uint64_t* operand, const uint64_t* multiplicand, uint64_t count,
                                            uint64_t input_mod_factor, uint64_t output_mod_factor, void* stream)
{
    (void)input_mod_factor;  // the forward accepts [0, 4q) whatever the factor (ntt.cpp:173-186)
    return product(ntts, n_ntts, result, operand, multiplicand, count, output_mod_factor, stream);
}

axhel_status_t axhel_cuda_ntt_forward(axhel_ntt_t h, uint64_t* r, const uint64_t* x, uint64_t in_f, uint64_t out_f,
                                      void* stream)
{
    return transform(false, &h, 1, r, x, 1, in_f, out_f, false, stream);
}

axhel_status_t axhel_cuda_ntt_inverse(axhel_ntt_t h, uint64_t* r, const uint64_t* x, uint64_t in_f, uint64_t out_f,
                                      void* stream)
{
    return transform(true, &h, 1, r, x, 1, in_f, out_f, false, stream);
}

axhel_status_t axhel_cuda_ntt_forward_batch(const axhel_ntt_t* ntts, uint64_t n_ntts, uint64_t* r, const uint64_t* x,
                                            uint64_t count, uint64_t in_f, uint64_t out_f, void* stream)
{
    return transform(false, ntts, n_ntts, r, x, count, in_f, out_f, true, stream);
}

axhel_status_t axhel_cuda_ntt_inverse_batch(const axhel_ntt_t* ntts, uint64_t n_ntts, uint64_t* r, const uint64_t* x,
                                            uint64_t count, uint64_t in_f, uint64_t out_f, void* stream)
{
    return transform(true, ntts, n_ntts, r, x, count, in_f, out_f, true, stream);
}

axhel_status_t axhel_cuda_ntt_forward_mul_batch(const axhel_ntt_t* ntts, uint64_t n_ntts, uint64_t* r,
                                                const uint64_t* x, const uint64_t* m, uint64_t count, void* stream)
{
    if (count && !m) return fail(AXHEL_ERR_INVALID, "null multiplicand");
    if (count && m == r) return fail(AXHEL_ERR_INVALID, "the multiplicand must not be the result buffer");
    return transform(false, ntts, n_ntts, r, x, count, 4, 4, true, stream, m);
}

axhel_status_t axhel_cuda_ntt_mul_inverse_batch(const axhel_ntt_t* ntts, uint64_t n_ntts, uint64_t* r,
                                                const uint64_t* x, const uint64_t* m, uint64_t count, uint64_t out_f,
                                                void* stream)
{
    if (count && !m) return fail(AXHEL_ERR_INVALID, "null multiplicand");
    if (count && m == r) return fail(AXHEL_ERR_INVALID, "the multiplicand must not be the result buffer");
    return transform(true, ntts, n_ntts, r, x, count, 4, out_f, true, stream, m);
}

axhel_status_t axhel_cuda_ntt_chain_mul_batch(const axhel_ntt_t* ntts, uint64_t n_ntts, uint64_t* r,
                                              const uint64_t* x, const uint64_t* m, uint64_t count, uint64_t in_f,
                                              uint64_t out_f, void* stream)
{
    return chain(ntts, n_ntts, r, x, m, nullptr, kChainMul, count, in_f, out_f, stream);
}

axhel_status_t axhel_cuda_ntt_chain_fma_batch(const axhel_ntt_t* ntts, uint64_t n_ntts, uint64_t* r,
                                              const uint64_t* x, const uint64_t* scalars, const uint64_t* addend,
                                              uint64_t count, uint64_t in_f, uint64_t out_f, void* stream)
{
    return chain(ntts, n_ntts, r, x, addend, scalars, kChainFma, count, in_f, out_f, stream);
}

// ------------------------------------------------------------- eltwise

#define AXHEL_CHECK_PTRS(cond)                                                      \
    do {                                                                             \
        if (n == 0) return AXHEL_OK;                                                 \
        if (!(cond)) return fail(AXHEL_ERR_INVALID, "null data pointer");            \
    } while (0)

#define AXHEL_RET(expr, what)                                 \
    do {                                                      \
        cudaError_t e_ = (expr);                              \
        return e_ == cudaSuccess ? AXHEL_OK : cuda_fail(e_, what); \
    } while (0)

axhel_status_t axhel_cuda_eltwise_add_vv(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q,
                                         void* s)
{
    AXHEL_CHECK_PTRS(r && a && b);
    if (axhel_status_t st = check_modulus(q, 63)) return st;
    AXHEL_RET(eltwise_add(r, a, b, n, q, S(s)), "EltwiseAddMod");
}
axhel_status_t axhel_cuda_eltwise_add_vs(uint64_t* r, const uint64_t* a, uint64_t b, uint64_t n, uint64_t q, void* s)
{
    AXHEL_CHECK_PTRS(r && a);
    if (axhel_status_t st = check_modulus(q, 63)) return st;
    AXHEL_RET(eltwise_add_scalar(r, a, b, n, q, S(s)), "EltwiseAddMod");
}
axhel_status_t axhel_cuda_eltwise_sub_vv(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q,
                                         void* s)
{
    AXHEL_CHECK_PTRS(r && a && b);
    if (axhel_status_t st = check_modulus(q, 63)) return st;
    AXHEL_RET(eltwise_sub(r, a, b, n, q, S(s)), "EltwiseSubMod");
}
axhel_status_t axhel_cuda_eltwise_sub_vs(uint64_t* r, const uint64_t* a, uint64_t b, uint64_t n, uint64_t q, void* s)
{
    AXHEL_CHECK_PTRS(r && a);
    if (axhel_status_t st = check_modulus(q, 63)) return st;
    AXHEL_RET(eltwise_sub_scalar(r, a, b, n, q, S(s)), "EltwiseSubMod");
}
axhel_status_t axhel_cuda_eltwise_mul(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q,
                                      uint64_t f, void* s)
{
    AXHEL_CHECK_PTRS(r && a && b);
    if (axhel_status_t st = check_modulus(q, 62)) return st;
    AXHEL_RET(eltwise_mul(r, a, b, n, q, f, S(s)), "EltwiseMulMod");
}
axhel_status_t axhel_cuda_eltwise_fma(uint64_t* r, const uint64_t* a, uint64_t sc, const uint64_t* c, uint64_t n,
                                      uint64_t q, uint64_t f, void* s)
{
    AXHEL_CHECK_PTRS(r && a);
    if (axhel_status_t st = check_modulus(q, 62)) return st;
    AXHEL_RET(eltwise_fma(r, a, sc, c, n, q, f, S(s)), "EltwiseFMAMod");
}
axhel_status_t axhel_cuda_eltwise_reduce(uint64_t* r, const uint64_t* a, uint64_t n, uint64_t q, uint64_t in_f,
                                         uint64_t out_f, void* s)
{
    AXHEL_CHECK_PTRS(r && a);
    if (axhel_status_t st = check_modulus(q, 62)) return st;
    AXHEL_RET(eltwise_reduce(r, a, n, q, in_f, out_f, S(s)), "EltwiseReduceMod");
}

axhel_status_t axhel_cuda_tensor_product(uint64_t* r0, uint64_t* r1, uint64_t* r2, const uint64_t* c0,
                                         const uint64_t* c1, const uint64_t* d0, const uint64_t* d1, uint64_t n,
                                         uint64_t count, const uint64_t* moduli, uint64_t n_moduli,
                                         uint64_t mod_factor, void* s)
{
    if (n == 0 || count == 0) return AXHEL_OK;
    if (!r0 || !r1 || !r2 || !c0 || !c1 || !d0 || !d1 || !moduli) return fail(AXHEL_ERR_INVALID, "null pointer");
    if (n_moduli == 0 || n_moduli > (uint64_t)kMaxInlineMods) return fail(AXHEL_ERR_UNSUPPORTED, "1..64 moduli");
    if (n & 1) return fail(AXHEL_ERR_UNSUPPORTED, "limb length must be even");
    if (mod_factor != 1 && mod_factor != 2 && mod_factor != 4) return fail(AXHEL_ERR_INVALID, "mod_factor 1, 2 or 4");
    const uintptr_t al = (uintptr_t)r0 | (uintptr_t)r1 | (uintptr_t)r2 | (uintptr_t)c0 | (uintptr_t)c1 |
                         (uintptr_t)d0 | (uintptr_t)d1;
    if (al & 15) return fail(AXHEL_ERR_INVALID, "tensor product buffers must be 16-byte aligned");
    if (count > 65535) return fail(AXHEL_ERR_UNSUPPORTED, "at most 65535 limbs per call");
    for (uint64_t i = 0; i < n_moduli; ++i)
        if (axhel_status_t st = check_modulus(moduli[i], 62)) return st;
    AXHEL_RET(tensor_product(r0, r1, r2, c0, c1, d0, d1, n, count, moduli, n_moduli, mod_factor, S(s)),
              "tensor product");
}

// --------------------------------------------------------------- plans

axhel_status_t axhel_cuda_plan_set(int inverse, uint32_t logn, uint32_t npass, const uint32_t* lg, const uint32_t* lr,
                                   const uint32_t* tg)
{
    if (npass == 0) {
        plan_override(inverse != 0, logn, nullptr);
        return AXHEL_OK;
    }
    if (npass > 3 || !lg || !lr || !tg) return fail(AXHEL_ERR_INVALID, "bad plan");
    NttPlan p{};
    p.npass = (int)npass;
    for (uint32_t i = 0; i < npass; ++i) p.pass[i] = PassCfg{(int)lg[i], (int)lr[i], (int)tg[i]};
    if (!plan_valid(p, logn, inverse != 0)) return fail(AXHEL_ERR_UNSUPPORTED, "plan not valid for this degree");
    plan_override(inverse != 0, logn, &p);
    return AXHEL_OK;
}

axhel_status_t axhel_cuda_plan_get(int inverse, uint32_t logn, uint64_t count, uint32_t* npass, uint32_t* lg,
                                   uint32_t* lr, uint32_t* tg)
{
    if (!npass || !lg || !lr || !tg) return fail(AXHEL_ERR_INVALID, "null output");
    if (logn < 1 || logn > 17) return fail(AXHEL_ERR_UNSUPPORTED, "log degree out of range");
    const NttPlan p = plan_for(inverse != 0, logn, count);
    *npass = (uint32_t)p.npass;
    for (int i = 0; i < p.npass; ++i) {
        lg[i] = (uint32_t)p.pass[i].lg;
        lr[i] = (uint32_t)p.pass[i].lr;
        tg[i] = (uint32_t)p.pass[i].tg;
    }
    return AXHEL_OK;
}

axhel_status_t axhel_cuda_cluster_plan_set(int kind, uint32_t logn, uint32_t lga, uint32_t lr, uint32_t csize,
                                           uint64_t max_limbs)
{
    if (kind < 0 || kind > 3) return fail(AXHEL_ERR_INVALID, "cluster kind: 0 forward, 1 inverse, 2 chain, 3 product");
    if (logn < 10 || logn > 17) return fail(AXHEL_ERR_UNSUPPORTED, "cluster form covers log degree 10..17");
    if (lga == 0) {
        cluster_plan_override(kind, logn, nullptr);
        return AXHEL_OK;
    }
    const ClusterCfg c{(int)lga, (int)lr, (int)csize, max_limbs};
    if (max_limbs && !cluster_cfg_valid(kind, logn, c))
        return fail(AXHEL_ERR_UNSUPPORTED, "cluster configuration not compiled or not valid for this degree");
    cluster_plan_override(kind, logn, &c);
    return AXHEL_OK;
}

axhel_status_t axhel_cuda_cluster_plan_get(int kind, uint32_t logn, uint32_t* lga, uint32_t* lr, uint32_t* csize,
                                           uint64_t* max_limbs)
{
    if (!lga || !lr || !csize || !max_limbs) return fail(AXHEL_ERR_INVALID, "null output");
    if (kind < 0 || kind > 3) return fail(AXHEL_ERR_INVALID, "cluster kind: 0 forward, 1 inverse, 2 chain, 3 product");
    const ClusterCfg c = cluster_plan_current(kind, logn);
    *lga = (uint32_t)c.lga;
    *lr = (uint32_t)c.lr;
    *csize = (uint32_t)c.csize;
    *max_limbs = c.max_limbs;
    return AXHEL_OK;
}

axhel_status_t axhel_cuda_plan_load(const char* path, uint32_t* loaded)
{
    const int n = plan_load(path);
    if (loaded) *loaded = n < 0 ? 0 : (uint32_t)n;
    if (n < 0) return fail(AXHEL_ERR_INVALID, "cannot open plan table");
    return AXHEL_OK;
}

axhel_status_t axhel_cuda_batch_split_set(uint32_t logn, uint32_t row)
{
    if (row && !batch_row_valid(logn, (int)row))
        return fail(AXHEL_ERR_INVALID, "batch split: need log N in [10, 17] and contiguous stages in "
                                       "[max(5, log N - 9), min(9, log N - 5)]");
    batch_row_override(logn, (int)row);
    return AXHEL_OK;
}

axhel_status_t axhel_cuda_batch_split_get(uint32_t logn, uint32_t* row)
{
    if (!row || logn < 10 || logn > 17) return fail(AXHEL_ERR_INVALID, "batch split: log N in [10, 17]");
    *row = (uint32_t)batch_row_stages(logn);
    return AXHEL_OK;
}

}  // extern "C"
