// Element-wise modular kernels for sm_100a (EltwiseAdd/Sub/Mul/FMA/ReduceMod).
//
// HBM-bound streaming kernels: a grid sized to a multiple of the SM count
// walks the vector in chunks of four 16-byte loads per operand and thread,
// each warp access 512 contiguous bytes (all pointers 16-byte aligned), or
// in scalar 8-byte accesses otherwise.  The
// arithmetic of each element is the reference native backend's formula
// (axhel/eltwise/eltwise-*-mod.cpp), so every output is bit-identical.
// result may alias any operand: each element is read before it is written by
// the same thread.
#include <cuda_runtime.h>

#include <cstdint>

#include "internal.h"
#include "launch.h"
#include "eltwise_ops.cuh"
#include "modarith.cuh"

namespace axhel_impl {
using namespace axhel_dev;

// ---------------------------------------------------------------- kernels

template <class Op, bool HAS_B>
__global__ void __launch_bounds__(256) eltwise_vec_kernel(uint64_t* r, const uint64_t* a, const uint64_t* b,
                                                          uint64_t n, const Op op)
{
    // 16-byte aligned path.  A CTA takes chunks of V * blockDim 16-byte
    // vectors; vector k of a chunk is read by thread t at k * blockDim + t,
    // so every warp access covers 512 contiguous bytes, and all loads of a
    // chunk are issued before its first store (V loads per operand in flight
    // per thread).
    constexpr int V = 4;
    const uint64_t nv = n >> 1;  // 16-byte vectors
    const ulonglong2* a2 = reinterpret_cast<const ulonglong2*>(a);
    const ulonglong2* b2 = reinterpret_cast<const ulonglong2*>(b);
    ulonglong2* r2 = reinterpret_cast<ulonglong2*>(r);
    const uint64_t chunk = (uint64_t)V * blockDim.x;
    for (uint64_t c = (uint64_t)blockIdx.x * chunk + threadIdx.x; c < nv; c += (uint64_t)gridDim.x * chunk) {
        ulonglong2 x[V], y[V];
#pragma unroll
        for (int k = 0; k < V; ++k) {
            const uint64_t i = c + (uint64_t)k * blockDim.x;
            x[k] = i < nv ? a2[i] : make_ulonglong2(0, 0);
            y[k] = (HAS_B && i < nv) ? b2[i] : make_ulonglong2(0, 0);
        }
#pragma unroll
        for (int k = 0; k < V; ++k) {
            const uint64_t i = c + (uint64_t)k * blockDim.x;
            if (i < nv) r2[i] = make_ulonglong2(op(x[k].x, y[k].x), op(x[k].y, y[k].y));
        }
    }
    // the odd last element by thread 0 of block 0
    if (blockIdx.x == 0 && threadIdx.x == 0 && (n & 1)) r[n - 1] = op(a[n - 1], HAS_B ? b[n - 1] : 0);
}

template <class Op, bool HAS_B>
__global__ void __launch_bounds__(256) eltwise_scalar_kernel(uint64_t* r, const uint64_t* a, const uint64_t* b,
                                                             uint64_t n, const Op op)
{
    // 8-byte aligned path: a CTA takes chunks of kPer * blockDim elements;
    // element k of a chunk is handled by thread t at k * blockDim + t (every
    // warp access 256 contiguous bytes), all loaded before the first store.
    // Two elements per thread measured 1-19 % faster than one (reduce the
    // most) and than four or eight.  Each result depends on its own operands
    // only, so in-place calls hold.
    constexpr int kPer = 2;
    const uint64_t chunk = (uint64_t)kPer * blockDim.x;
    for (uint64_t base = (uint64_t)blockIdx.x * chunk; base < n; base += (uint64_t)gridDim.x * chunk) {
        const uint64_t i = base + threadIdx.x;
        if (base + chunk <= n) {
            uint64_t x[kPer], y[kPer];
#pragma unroll
            for (int k = 0; k < kPer; ++k) {
                x[k] = a[i + (uint64_t)k * blockDim.x];
                y[k] = HAS_B ? b[i + (uint64_t)k * blockDim.x] : 0;
            }
#pragma unroll
            for (int k = 0; k < kPer; ++k) r[i + (uint64_t)k * blockDim.x] = op(x[k], y[k]);
        } else {
            for (int k = 0; k < kPer; ++k) {
                const uint64_t j = i + (uint64_t)k * blockDim.x;
                if (j < n) r[j] = op(a[j], HAS_B ? b[j] : 0);
            }
        }
    }
}

template <class Op, bool HAS_B>
static cudaError_t run(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, const Op& op, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    const int threads = 256;
    const uintptr_t align = reinterpret_cast<uintptr_t>(r) | reinterpret_cast<uintptr_t>(a) |
                            (HAS_B ? reinterpret_cast<uintptr_t>(b) : 0);
    const bool vec = (align & 15) == 0;
    const uint64_t work = vec ? (n >> 3) : ((n + 1) >> 1);  // elements per thread per chunk: 8 (vector), 2
    uint64_t blocks = (work + threads - 1) / threads;
    const uint64_t cap = (uint64_t)sm_count() * 8;  // 8 resident CTAs of 256 threads per SM
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    count_launch();
    ProfScope prof(s, "eltwise_%s%s", Op::kName, vec ? "" : "_unaligned");
    if (vec)
        eltwise_vec_kernel<Op, HAS_B><<<(unsigned)blocks, threads, 0, s>>>(r, a, b, n, op);
    else
        eltwise_scalar_kernel<Op, HAS_B><<<(unsigned)blocks, threads, 0, s>>>(r, a, b, n, op);
    return cudaGetLastError();
}

// ------------------------------------------------------------- launchers

static inline uint64_t bit_width(uint64_t x) { return x ? 64 - __builtin_clzll(x) : 0; }

void barrett_params(uint64_t q, uint64_t* mu, uint32_t* shift)
{
    const uint64_t k = bit_width(q);
    const unsigned __int128 num = (unsigned __int128)((uint64_t)1 << (k - 2)) << 64;
    *mu = (uint64_t)(num / q);
    *shift = (uint32_t)(k - 2);
}

cudaError_t eltwise_add(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q, cudaStream_t s)
{
    return run<OpAddVV, true>(r, a, b, n, OpAddVV{q}, s);
}
cudaError_t eltwise_add_scalar(uint64_t* r, const uint64_t* a, uint64_t b, uint64_t n, uint64_t q, cudaStream_t s)
{
    return run<OpAddVS, false>(r, a, nullptr, n, OpAddVS{q, b}, s);
}
cudaError_t eltwise_sub(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q, cudaStream_t s)
{
    return run<OpSubVV, true>(r, a, b, n, OpSubVV{q}, s);
}
cudaError_t eltwise_sub_scalar(uint64_t* r, const uint64_t* a, uint64_t b, uint64_t n, uint64_t q, cudaStream_t s)
{
    return run<OpSubVS, false>(r, a, nullptr, n, OpSubVS{q, b}, s);
}

cudaError_t eltwise_mul(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q, uint64_t f,
                        cudaStream_t s)
{
    uint64_t mu;
    uint32_t sh;
    barrett_params(q, &mu, &sh);
    switch (f) {
    case 1: return run<OpMul<1>, true>(r, a, b, n, OpMul<1>{q, mu, sh}, s);
    case 2: return run<OpMul<2>, true>(r, a, b, n, OpMul<2>{q, mu, sh}, s);
    case 4: return run<OpMul<4>, true>(r, a, b, n, OpMul<4>{q, mu, sh}, s);
    default: return cudaSuccess;  // unsupported factor: no-op, eltwise-mul-mod.cpp:83-93
    }
}

static uint64_t host_reduce_input(uint64_t x, uint64_t q, uint64_t f)
{
    if (f == 8 && x >= 4 * q) x -= 4 * q;
    if (f >= 4 && x >= 2 * q) x -= 2 * q;
    if (f >= 2 && x >= q) x -= q;
    return x;
}

template <int F>
static cudaError_t fma_f(uint64_t* r, const uint64_t* a, uint64_t sc, const uint64_t* c, uint64_t n, uint64_t q,
                         uint64_t mu, uint32_t sh, cudaStream_t s)
{
    const uint64_t sr = host_reduce_input(sc, q, F);  // eltwise-fma-mod.cpp:33
    if (c) return run<OpFma<F, true>, true>(r, a, c, n, OpFma<F, true>{q, mu, sr, sh}, s);
    return run<OpFma<F, false>, false>(r, a, nullptr, n, OpFma<F, false>{q, mu, sr, sh}, s);
}

cudaError_t eltwise_fma(uint64_t* r, const uint64_t* a, uint64_t sc, const uint64_t* c, uint64_t n, uint64_t q,
                        uint64_t f, cudaStream_t s)
{
    uint64_t mu;
    uint32_t sh;
    barrett_params(q, &mu, &sh);
    switch (f) {
    case 1: return fma_f<1>(r, a, sc, c, n, q, mu, sh, s);
    case 2: return fma_f<2>(r, a, sc, c, n, q, mu, sh, s);
    case 4: return fma_f<4>(r, a, sc, c, n, q, mu, sh, s);
    case 8: return fma_f<8>(r, a, sc, c, n, q, mu, sh, s);
    default: return cudaSuccess;  // eltwise-fma-mod.cpp:98-111
    }
}

cudaError_t eltwise_reduce(uint64_t* r, const uint64_t* a, uint64_t n, uint64_t q, uint64_t in_f, uint64_t out_f,
                           cudaStream_t s)
{
    uint64_t mu = 0;
    uint32_t sh = 0;
    // Branch order of EltwiseReduceModNative (eltwise-reduce-mod.cpp:35-127).
    if (in_f == 1 || (out_f == 2 && in_f <= 2)) {
        if (r == a) return cudaSuccess;
        return run<OpReduce<0>, false>(r, a, nullptr, n, OpReduce<0>{q, 0, 0}, s);
    }
    if (in_f == 2 && out_f == 1) return run<OpReduce<1>, false>(r, a, nullptr, n, OpReduce<1>{q, 0, 0}, s);
    if (in_f == 4 && out_f == 1) return run<OpReduce<2>, false>(r, a, nullptr, n, OpReduce<2>{q, 0, 0}, s);
    if (in_f == 4 && out_f == 2) return run<OpReduce<3>, false>(r, a, nullptr, n, OpReduce<3>{q, 0, 0}, s);
    if (in_f == q) {
        barrett_params(q, &mu, &sh);
        return run<OpReduce<4>, false>(r, a, nullptr, n, OpReduce<4>{q, mu, sh}, s);
    }
    return cudaSuccess;  // unmatched pair writes nothing
}

// ------------------------------------------------------ fused tensor product

struct ModConst {
    uint64_t q, mu;
    uint32_t shift, pad;
};
struct TensorArgs {
    uint64_t *r0, *r1, *r2;
    const uint64_t *c0, *c1, *d0, *d1;
    uint64_t n, count;
    uint32_t nmod, factor;
    ModConst m[kMaxInlineMods];
};

// Per element of limb i (modulus m[i % nmod]):
//   r0 = Mul(c0,d0); r1 = Add(Mul(c0,d1), Mul(c1,d0)); r2 = Mul(c1,d1)
// with EltwiseMulMod<F> / EltwiseAddMod semantics (canonical results, so the
// middle term's evaluation order is free); the trailing EltwiseReduceMod(4,1)
// is the identity on these canonical values.
template <int F>
__global__ void __launch_bounds__(256) tensor_product_kernel(const __grid_constant__ TensorArgs a)
{
    // grid: x = chunks of one limb, y = limb.  Two elements per thread step.
    const uint64_t limb = blockIdx.y;
    const ModConst mc = a.m[limb % a.nmod];
    const uint64_t q = mc.q;
    const OpMul<1> mul{q, mc.mu, mc.shift};  // on inputs already reduced to [0, q)
    const OpAddVV add{q};
    const OpSubVV sub{q};
    const uint64_t off = limb * a.n;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x * 2;
    // Every output is a canonical residue, so the middle term may be formed
    // as (c0 + c1)(d0 + d1) - c0 d0 - c1 d1: three Barrett products per
    // coefficient instead of four, the same bits.
    auto three = [&](uint64_t c0, uint64_t c1, uint64_t d0, uint64_t d1, uint64_t& r0, uint64_t& r1,
                     uint64_t& r2) {
        c0 = reduce_input<F>(c0, q);
        c1 = reduce_input<F>(c1, q);
        d0 = reduce_input<F>(d0, q);
        d1 = reduce_input<F>(d1, q);
        r0 = mul(c0, d0);
        r2 = mul(c1, d1);
        r1 = sub(sub(mul(add(c0, c1), add(d0, d1)), r0), r2);
    };
    for (uint64_t e = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * 2; e < a.n; e += stride) {
        const ulonglong2 x0 = *reinterpret_cast<const ulonglong2*>(a.c0 + off + e);
        const ulonglong2 x1 = *reinterpret_cast<const ulonglong2*>(a.c1 + off + e);
        const ulonglong2 y0 = *reinterpret_cast<const ulonglong2*>(a.d0 + off + e);
        const ulonglong2 y1 = *reinterpret_cast<const ulonglong2*>(a.d1 + off + e);
        uint64_t r[2][3];
        three(x0.x, x1.x, y0.x, y1.x, r[0][0], r[0][1], r[0][2]);
        three(x0.y, x1.y, y0.y, y1.y, r[1][0], r[1][1], r[1][2]);
        const ulonglong2 o0 = make_ulonglong2(r[0][0], r[1][0]);
        const ulonglong2 o1 = make_ulonglong2(r[0][1], r[1][1]);
        const ulonglong2 o2 = make_ulonglong2(r[0][2], r[1][2]);
        *reinterpret_cast<ulonglong2*>(a.r0 + off + e) = o0;
        *reinterpret_cast<ulonglong2*>(a.r1 + off + e) = o1;
        *reinterpret_cast<ulonglong2*>(a.r2 + off + e) = o2;
    }
}

cudaError_t tensor_product(uint64_t* r0, uint64_t* r1, uint64_t* r2, const uint64_t* c0, const uint64_t* c1,
                           const uint64_t* d0, const uint64_t* d1, uint64_t n, uint64_t count, const uint64_t* moduli,
                           uint64_t nmod, uint64_t factor, cudaStream_t s)
{
    TensorArgs a{};
    a.r0 = r0; a.r1 = r1; a.r2 = r2;
    a.c0 = c0; a.c1 = c1; a.d0 = d0; a.d1 = d1;
    a.n = n; a.count = count;
    a.nmod = (uint32_t)nmod;
    a.factor = (uint32_t)factor;
    for (uint64_t i = 0; i < nmod; ++i) {
        a.m[i].q = moduli[i];
        barrett_params(moduli[i], &a.m[i].mu, &a.m[i].shift);
    }
    if (n == 0 || count == 0) return cudaSuccess;
    const int threads = 256;
    uint64_t bx = (n / 2 + threads - 1) / threads;
    // enough CTAs for ~8 per SM in total, at least one per limb
    uint64_t want = ((uint64_t)sm_count() * 8 + count - 1) / count;
    if (want < 1) want = 1;
    if (bx > want) bx = want;
    const dim3 grid((unsigned)bx, (unsigned)count);
    count_launch();
    ProfScope prof(s, "tensor_product f=%d", (int)factor);
    switch (factor) {
    case 1: tensor_product_kernel<1><<<grid, threads, 0, s>>>(a); break;
    case 2: tensor_product_kernel<2><<<grid, threads, 0, s>>>(a); break;
    case 4: tensor_product_kernel<4><<<grid, threads, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace axhel_impl
