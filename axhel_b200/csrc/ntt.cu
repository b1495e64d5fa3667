// Instantiations and launchers of the NTT pass kernels (ntt_kernels.cuh).
#include <cuda_runtime.h>

#include <mutex>

#include "launch.h"
#include "ntt_kernels.cuh"

namespace axhel_impl {

namespace {

using PassFn = void (*)(const PassArgs);
using ChainFn = void (*)(const ChainArgs);

constexpr int kMaxLG = 13;
constexpr int kMaxLR = 5;

struct KernelTable {
    PassFn fwd[kMaxLG + 1][kMaxLR + 1] = {};
    PassFn inv[kMaxLG + 1][kMaxLR + 1] = {};
    PassFn fwd_mul[kMaxLG + 1][kMaxLR + 1] = {};  // with the dyadic product (kPreMul / kPostMul)
    PassFn inv_mul[kMaxLG + 1][kMaxLR + 1] = {};
    ChainFn chain[kMaxLG + 1][kMaxLR + 1] = {};
    ChainFn product[kMaxLG + 1][kMaxLR + 1] = {};
    bool smem_set[6][kMaxLG + 1][kMaxLR + 1] = {};
};

template <int LG, int LR>
void add_one(KernelTable& t)
{
    if constexpr (LR <= LG) {
        t.fwd[LG][LR] = ntt_pass_kernel<false, LG, LR>;
        t.inv[LG][LR] = ntt_pass_kernel<true, LG, LR>;
        t.fwd_mul[LG][LR] = ntt_pass_mul_kernel<false, LG, LR>;
        t.inv_mul[LG][LR] = ntt_pass_mul_kernel<true, LG, LR>;
        t.chain[LG][LR] = ntt_chain_kernel<LG, LR>;
        if constexpr (LR <= 3) t.product[LG][LR] = ntt_product_kernel<LG, LR>;
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

size_t smem_bytes(const PassCfg& c) { return (size_t)c.tg * (size_t(1) << c.lg) * sizeof(uint64_t); }

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
    return table().fwd[c.lg][c.lr] != nullptr;
}

cudaError_t launch_ntt_pass(bool inverse, const PassCfg& c, const PassArgs& a, cudaStream_t s)
{
    if (!pass_supported(c)) return cudaErrorInvalidValue;
    const uint32_t lgS = inverse ? a.s0 : (a.logn - a.s0 - c.lg);
    if (!geometry_ok(c, a.logn, lgS) || (uint32_t)c.tg != a.tg) return cudaErrorInvalidValue;
    const bool mul = (a.flags & (kPreMul | kPostMul)) != 0;
    PassFn fn = mul ? (inverse ? table().inv_mul[c.lg][c.lr] : table().fwd_mul[c.lg][c.lr])
                    : (inverse ? table().inv[c.lg][c.lr] : table().fwd[c.lg][c.lr]);
    cudaError_t e = ensure_smem(fn, (inverse ? 1 : 0) + (mul ? 4 : 0), c);
    if (e != cudaSuccess) return e;
    const uint64_t tiles = a.count * ((1ull << (a.logn - c.lg)) / c.tg);
    if (tiles == 0) return cudaSuccess;
    if (tiles > 0x7fffffffull) return cudaErrorInvalidValue;
    const unsigned threads = (unsigned)c.tg << (c.lg - c.lr);
    count_launch();
    ProfScope prof(s, "ntt_%s%s_pass lg=%d lr=%d tg=%d", inverse ? "inv" : "fwd", mul ? "_mul" : "", c.lg, c.lr,
                   c.tg);
    fn<<<(unsigned)tiles, threads, smem_bytes(c), s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_product_pass(const PassCfg& c, const ChainArgs& a, cudaStream_t s)
{
    if (!pass_supported(c) || c.lr > 3) return cudaErrorInvalidValue;
    if (!geometry_ok(c, a.pass.logn, 0) || (uint32_t)c.tg != a.pass.tg) return cudaErrorInvalidValue;
    ChainFn fn = table().product[c.lg][c.lr];
    if (!fn) return cudaErrorInvalidValue;
    cudaError_t e = ensure_smem(fn, 3, c);
    if (e != cudaSuccess) return e;
    const uint64_t tiles = a.pass.count * ((1ull << (a.pass.logn - c.lg)) / c.tg);
    if (tiles == 0) return cudaSuccess;
    if (tiles > 0x7fffffffull) return cudaErrorInvalidValue;
    const unsigned threads = (unsigned)c.tg << (c.lg - c.lr);
    count_launch();
    ProfScope prof(s, "ntt_product_pass lg=%d lr=%d tg=%d", c.lg, c.lr, c.tg);
    fn<<<(unsigned)tiles, threads, smem_bytes(c), s>>>(a);
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
