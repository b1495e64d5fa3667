// Instantiations and launchers of the NTT pass kernels (ntt_kernels.cuh).
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <tuple>

#include "launch.h"
#include "ntt_kernels.cuh"

namespace axhel_impl {

namespace {

using PassFn = void (*)(const PassArgs);
using ChainFn = void (*)(const ChainArgs);

constexpr int kMaxLG = 13;
constexpr int kMaxLR = 5;

// Prefetching pass kernels are compiled for the group sizes of the passes
// of N >= 2^10 transforms (a pass of 5..10 stages) and register depths 3, 4.
constexpr int kPfMinLG = 5, kPfMaxLG = 10, kPfMaxLR = 4;

struct KernelTable {
    PassFn fwd[kMaxLG + 1][kMaxLR + 1] = {};
    PassFn inv[kMaxLG + 1][kMaxLR + 1] = {};
    PassFn fwd_pf[kMaxLG + 1][kMaxLR + 1] = {};
    PassFn inv_pf[kMaxLG + 1][kMaxLR + 1] = {};
    ChainFn chain[kMaxLG + 1][kMaxLR + 1] = {};
    bool smem_set[5][kMaxLG + 1][kMaxLR + 1] = {};
};

template <int LG, int LR>
void add_one(KernelTable& t)
{
    if constexpr (LR <= LG) {
        t.fwd[LG][LR] = ntt_pass_kernel<false, LG, LR>;
        t.inv[LG][LR] = ntt_pass_kernel<true, LG, LR>;
        t.chain[LG][LR] = ntt_chain_kernel<LG, LR>;
        if constexpr (LG >= kPfMinLG && LG <= kPfMaxLG && LR >= 3 && LR <= kPfMaxLR) {
            t.fwd_pf[LG][LR] = ntt_pass_pf_kernel<false, LG, LR>;
            t.inv_pf[LG][LR] = ntt_pass_pf_kernel<true, LG, LR>;
        }
    }
}

// Register-stage counts compiled for each group size: LR = LG for tiny groups,
// otherwise 3, 4 and 5.
template <int LG>
void add_lg(KernelTable& t)
{
    if constexpr (LG <= 3) {
        add_one<LG, LG>(t);
    } else {
        add_one<LG, 3>(t);
        add_one<LG, 4>(t);
        add_one<LG, 5>(t);
    }
}

template <int... LG>
void add_all(KernelTable& t, std::integer_sequence<int, LG...>)
{
    (add_lg<LG + 1>(t), ...);
}

KernelTable& table()
{
    static KernelTable t = [] {
        KernelTable k;
        add_all(k, std::make_integer_sequence<int, kMaxLG>{});
        return k;
    }();
    return t;
}

std::mutex g_attr_mu;

// Exchange space of a tile; the prefetching kernel adds two staging buffers
// of the same size.
size_t smem_bytes(const PassCfg& c) { return (size_t)c.tg * (size_t(1) << c.lg) * sizeof(uint64_t) * (c.pf ? 3 : 1); }

template <class Fn>
cudaError_t ensure_smem(Fn fn, int kind, const PassCfg& c)
{
    const size_t bytes = smem_bytes(c);
    if (bytes <= 48 * 1024) return cudaSuccess;
    std::lock_guard<std::mutex> lk(g_attr_mu);
    // Set to the maximum once per kernel; cheaper than tracking each size.
    bool& done = table().smem_set[kind][c.lg][c.lr];
    if (done) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(reinterpret_cast<const void*>(fn),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e == cudaSuccess) done = true;
    return e;
}

bool geometry_ok(const PassCfg& c, uint32_t logn, uint32_t lgS)
{
    if (c.lg < 1 || c.lg > kMaxLG || c.lr < 1 || c.lr > kMaxLR || c.lr > c.lg) return false;
    if (c.tg < 1 || (c.tg & (c.tg - 1))) return false;
    if ((uint32_t)c.lg > logn) return false;
    const uint64_t groups = 1ull << (logn - c.lg);
    if ((uint64_t)c.tg > groups) return false;
    if (lgS > 0 && (uint64_t)c.tg > (1ull << lgS)) return false;
    const uint64_t threads = (uint64_t)c.tg << (c.lg - c.lr);
    if (threads > (uint64_t)max_threads(c.lr) || threads < 1) return false;
    if (smem_bytes(c) > 227 * 1024) return false;
    return true;
}

}  // namespace

bool pass_supported(const PassCfg& c)
{
    if (c.lg < 1 || c.lg > kMaxLG || c.lr < 1 || c.lr > kMaxLR) return false;
    if (c.pf) return table().fwd_pf[c.lg][c.lr] != nullptr && smem_bytes(c) <= 227 * 1024;
    return table().fwd[c.lg][c.lr] != nullptr;
}

namespace {

// Resident CTAs of a prefetching pass kernel on the whole device (its grid),
// per (direction, width, depth, tile groups), computed once.
unsigned pf_grid(PassFn fn, bool inverse, const PassCfg& c, unsigned threads)
{
    static std::mutex mu;
    static std::map<std::tuple<int, int, int, int, int>, unsigned> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    const auto key = std::make_tuple(dev, inverse ? 1 : 0, c.lg, c.lr, c.tg);
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reinterpret_cast<const void*>(fn), (int)threads,
                                                  smem_bytes(c));
    const unsigned g = (unsigned)(per_sm < 1 ? 1 : per_sm) * (unsigned)sm_count();
    cache.emplace(key, g);
    return g;
}

}  // namespace

cudaError_t launch_ntt_pass(bool inverse, const PassCfg& c, const PassArgs& a, cudaStream_t s)
{
    if (!pass_supported(c)) return cudaErrorInvalidValue;
    const uint32_t lgS = inverse ? a.s0 : (a.logn - a.s0 - c.lg);
    if (!geometry_ok(c, a.logn, lgS) || (uint32_t)c.tg != a.tg) return cudaErrorInvalidValue;
    PassFn fn = c.pf ? (inverse ? table().inv_pf[c.lg][c.lr] : table().fwd_pf[c.lg][c.lr])
                     : (inverse ? table().inv[c.lg][c.lr] : table().fwd[c.lg][c.lr]);
    cudaError_t e = ensure_smem(fn, (inverse ? 1 : 0) + (c.pf ? 3 : 0), c);
    if (e != cudaSuccess) return e;
    const uint64_t tiles = a.count * ((1ull << (a.logn - c.lg)) / c.tg);
    if (tiles == 0) return cudaSuccess;
    if (tiles > 0x7fffffffull) return cudaErrorInvalidValue;
    const unsigned threads = (unsigned)c.tg << (c.lg - c.lr);
    unsigned grid = (unsigned)tiles;
    if (c.pf) {
        const unsigned g = pf_grid(fn, inverse, c, threads);
        if (g < grid) grid = g;
    }
    count_launch();
    ProfScope prof(s, "ntt_%s_pass lg=%d lr=%d tg=%d%s", inverse ? "inv" : "fwd", c.lg, c.lr, c.tg,
                   c.pf ? " pf" : "");
    fn<<<grid, threads, smem_bytes(c), s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_chain_pass(const PassCfg& c, const ChainArgs& a, cudaStream_t s)
{
    if (!pass_supported(c)) return cudaErrorInvalidValue;
    if (!geometry_ok(c, a.pass.logn, a.pass.logn - c.lg) || (uint32_t)c.tg != a.pass.tg)
        return cudaErrorInvalidValue;
    ChainFn fn = table().chain[c.lg][c.lr];
    cudaError_t e = ensure_smem(fn, 2, c);
    if (e != cudaSuccess) return e;
    const uint64_t tiles = a.pass.count * ((1ull << (a.pass.logn - c.lg)) / c.tg);
    if (tiles == 0) return cudaSuccess;
    if (tiles > 0x7fffffffull) return cudaErrorInvalidValue;
    const unsigned threads = (unsigned)c.tg << (c.lg - c.lr);
    count_launch();
    ProfScope prof(s, "ntt_chain_pass lg=%d lr=%d tg=%d", c.lg, c.lr, c.tg);
    fn<<<(unsigned)tiles, threads, smem_bytes(c), s>>>(a);
    return cudaGetLastError();
}

}  // namespace axhel_impl
