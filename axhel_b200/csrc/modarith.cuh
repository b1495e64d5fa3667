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

// Conditional subtract for the NTT's bounded ranges: the same function as
// csub() whenever |x - bound| < 2^63, which holds for every value a transform
// handles (x < 4q, bound <= 2q, q < 2^62).  Testing the sign of the
// difference takes one compare on its high word instead of a 64-bit compare.
__device__ __forceinline__ uint64_t csub_lazy(uint64_t x, uint64_t bound)
{
    const uint64_t d = x - bound;
    return static_cast<int64_t>(d) < 0 ? x : d;
}

// floor(a * b / 2^64) through a 32-bit multiply-add carry chain (seven
// integer multiply-adds and one add).
__device__ __forceinline__ uint64_t mul_hi64(uint64_t a, uint64_t b)
{
    uint64_t r;
    asm("{\n\t"
        ".reg .u32 a0, a1, b0, b1, t0, t1, t2, r0, r1;\n\t"
        "mov.b64 {a0, a1}, %1;\n\t"
        "mov.b64 {b0, b1}, %2;\n\t"
        "mul.hi.u32 t0, a0, b0;\n\t"
        "mad.lo.cc.u32 t0, a0, b1, t0;\n\t"
        "madc.hi.u32 t1, a0, b1, 0;\n\t"
        "mad.lo.cc.u32 t0, a1, b0, t0;\n\t"
        "madc.hi.cc.u32 t1, a1, b0, t1;\n\t"
        "addc.u32 t2, 0, 0;\n\t"
        "mad.lo.cc.u32 r0, a1, b1, t1;\n\t"
        "madc.hi.u32 r1, a1, b1, t2;\n\t"
        "mov.b64 %0, {r0, r1};\n\t"
        "}"
        : "=l"(r)
        : "l"(a), "l"(b));
    return r;
}

// (v * w + e * nq) mod 2^64 with 32-bit multiply-adds; nq = 2^64 - q turns
// the Shoup subtraction v*w - e*q into one accumulation chain.
__device__ __forceinline__ uint64_t mul_lo_acc(uint64_t v, uint64_t w, uint64_t e, uint64_t nq)
{
    uint64_t r;
    asm("{\n\t"
        ".reg .u32 v0, v1, w0, w1, e0, e1, n0, n1, r0, r1;\n\t"
        "mov.b64 {v0, v1}, %1;\n\t"
        "mov.b64 {w0, w1}, %2;\n\t"
        "mov.b64 {e0, e1}, %3;\n\t"
        "mov.b64 {n0, n1}, %4;\n\t"
        "mul.lo.u32 r0, v0, w0;\n\t"
        "mul.hi.u32 r1, v0, w0;\n\t"
        "mad.lo.u32 r1, v0, w1, r1;\n\t"
        "mad.lo.u32 r1, v1, w0, r1;\n\t"
        "mad.lo.u32 r1, e0, n1, r1;\n\t"
        "mad.lo.u32 r1, e1, n0, r1;\n\t"
        "mad.lo.cc.u32 r0, e0, n0, r0;\n\t"
        "madc.hi.u32 r1, e0, n0, r1;\n\t"
        "mov.b64 %0, {r0, r1};\n\t"
        "}"
        : "=l"(r)
        : "l"(v), "l"(w), "l"(e), "l"(nq));
    return r;
}

// MultiplyUIntModLazy (axhel/include/axhel/number-theory/uint-arith.hpp:48-52):
// value * w - floor(value * w' / 2^64) * q  (mod 2^64), in [0, 2q).
__device__ __forceinline__ uint64_t shoup_lazy(uint64_t v, uint64_t w, uint64_t wq, uint64_t q)
{
    return mul_lo_acc(v, w, mul_hi64(v, wq), 0 - q);
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
    const uint64_t gx = csub_lazy(x, q2);
    const uint64_t t = shoup_lazy(y, w, wq, q);
    x = gx + t;
    y = gx + q2 - t;
}

// InverseButterflyNative (axhel/ntt/ntt-internal.hpp:37-49).
__device__ __forceinline__ void inv_butterfly(uint64_t& x, uint64_t& y, uint64_t w, uint64_t wq, uint64_t q,
                                              uint64_t q2)
{
    const uint64_t u = x, v = y;
    x = csub_lazy(u + v, q2);
    y = shoup_lazy(u + q2 - v, w, wq, q);
}

// Final inverse stage (axhel/ntt/ntt-native.cpp:126-141): upper branch times
// N^-1, lower branch times scaled_root = N^-1 * w_last.
__device__ __forceinline__ void inv_final_butterfly(uint64_t& x, uint64_t& y, uint64_t ninv, uint64_t ninv_q,
                                                    uint64_t sr, uint64_t sr_q, uint64_t q, uint64_t q2)
{
    const uint64_t gx = csub_lazy(x, q2);
    const uint64_t v = y;
    x = shoup_lazy(gx + v, ninv, ninv_q, q);
    y = shoup_lazy(gx + q2 - v, sr, sr_q, q);
}

}  // namespace axhel_dev
