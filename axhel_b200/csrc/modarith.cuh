// Device-side modular arithmetic on 64-bit residues (q < 2^62).
//
// Every routine reproduces, operation for operation, the reference native
// backend's formula it names, so results are bit-identical including the lazy
// representatives in [0, 2q) / [0, 4q).  64x64->128 products use
// __umul64hi / 64-bit mul.lo; no floating point, no tensor cores.
#pragma once

#include <cstdint>

namespace axhel_dev {

// ConditionalSubtractNative (axhel/include/axhel/number-theory/modular-reduction.hpp:22-25)
__device__ __forceinline__ uint64_t csub(uint64_t x, uint64_t bound)
{
    return x >= bound ? x - bound : x;
}

// ReduceInputNative<F> (modular-reduction.hpp:48-67): cascade 8q -> 4q -> 2q -> q.
template <int F>
__device__ __forceinline__ uint64_t reduce_input(uint64_t x, uint64_t q)
{
    if constexpr (F == 8) x = csub(x, q << 2);
    if constexpr (F >= 4) x = csub(x, q << 1);
    if constexpr (F >= 2) x = csub(x, q);
    return x;
}

// MultiplyUIntModLazy (axhel/include/axhel/number-theory/uint-arith.hpp:48-52):
// value * w - floor(value * w' / 2^64) * q  (mod 2^64), in [0, 2q).
__device__ __forceinline__ uint64_t shoup_lazy(uint64_t v, uint64_t w, uint64_t wq, uint64_t q)
{
    const uint64_t est = __umul64hi(v, wq);
    return v * w - est * q;
}

// Barrett product of EltwiseMulModNative (axhel/eltwise/eltwise-mul-mod.cpp:40-60),
// alpha = 62, beta = -2: x, y in [0, q); mu = floor(2^(k+62) / q); shift = k - 2.
__device__ __forceinline__ uint64_t barrett_mul(uint64_t x, uint64_t y, uint64_t q, uint64_t mu,
                                                uint32_t shift)
{
    const uint64_t lo = x * y;
    const uint64_t hi = __umul64hi(x, y);
    const uint64_t c1 = shift ? (lo >> shift) | (hi << (64 - shift)) : lo;
    const uint64_t qhat = __umul64hi(c1, mu);
    const uint64_t z = lo - qhat * q;
    return reduce_input<4>(z, q);
}

// BarrettReduceUInt64Native (axhel/eltwise/eltwise-reduce-mod.cpp:19-29).
__device__ __forceinline__ uint64_t barrett_reduce64(uint64_t x, uint64_t q, uint64_t mu, uint32_t shift)
{
    const uint64_t qhat = __umul64hi(x >> shift, mu);
    return reduce_input<4>(x - qhat * q, q);
}

// ForwardButterflyNative (axhel/ntt/ntt-internal.hpp:20-31).
__device__ __forceinline__ void fwd_butterfly(uint64_t& x, uint64_t& y, uint64_t w, uint64_t wq, uint64_t q,
                                              uint64_t q2)
{
    const uint64_t gx = csub(x, q2);
    const uint64_t t = shoup_lazy(y, w, wq, q);
    x = gx + t;
    y = gx + q2 - t;
}

// InverseButterflyNative (axhel/ntt/ntt-internal.hpp:37-49).
__device__ __forceinline__ void inv_butterfly(uint64_t& x, uint64_t& y, uint64_t w, uint64_t wq, uint64_t q,
                                              uint64_t q2)
{
    const uint64_t u = x, v = y;
    x = csub(u + v, q2);
    y = shoup_lazy(u + q2 - v, w, wq, q);
}

// Final inverse stage (axhel/ntt/ntt-native.cpp:126-141): upper branch times
// N^-1, lower branch times scaled_root = N^-1 * w_last.
__device__ __forceinline__ void inv_final_butterfly(uint64_t& x, uint64_t& y, uint64_t ninv, uint64_t ninv_q,
                                                    uint64_t sr, uint64_t sr_q, uint64_t q, uint64_t q2)
{
    const uint64_t gx = csub(x, q2);
    const uint64_t v = y;
    x = shoup_lazy(gx + v, ninv, ninv_q, q);
    y = shoup_lazy(gx + q2 - v, sr, sr_q, q);
}

}  // namespace axhel_dev
