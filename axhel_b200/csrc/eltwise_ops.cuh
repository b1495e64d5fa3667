// Per-element formulas of the reference's element-wise kernels
// (axhel/eltwise/eltwise-*-mod.cpp), shared by the streaming kernels
// (eltwise.cu) and the batch engine's element-wise jobs (batch.cu), so both
// compute the same bits.
#pragma once

#include <cstdint>

#include "modarith.cuh"

namespace axhel_impl {
using namespace axhel_dev;

// -------------------------------------------------------------------- ops
// Each op maps (a, b) -> result for one element.

struct OpAddVV {  // eltwise-add-mod.cpp:15-30
    static constexpr const char* kName = "add_vv";
    uint64_t q;
    __device__ uint64_t operator()(uint64_t a, uint64_t b) const
    {
        const uint64_t s = a + b;
        return s >= q ? s - q : s;
    }
};
struct OpAddVS {  // eltwise-add-mod.cpp:33-47
    static constexpr const char* kName = "add_vs";
    uint64_t q, s;
    __device__ uint64_t operator()(uint64_t a, uint64_t) const
    {
        const uint64_t t = a + s;
        return t >= q ? t - q : t;
    }
};
struct OpSubVV {  // eltwise-sub-mod.cpp:15-30
    static constexpr const char* kName = "sub_vv";
    uint64_t q;
    __device__ uint64_t operator()(uint64_t a, uint64_t b) const { return a - b + (a < b ? q : 0); }
};
struct OpSubVS {  // eltwise-sub-mod.cpp:33-47
    static constexpr const char* kName = "sub_vs";
    uint64_t q, s;
    __device__ uint64_t operator()(uint64_t a, uint64_t) const { return a - s + (a < s ? q : 0); }
};
template <int F>
struct OpMul {  // EltwiseMulModNative<F>, eltwise-mul-mod.cpp:18-63
    static constexpr const char* kName = "mul";
    uint64_t q, mu;
    uint32_t shift;
    __device__ uint64_t operator()(uint64_t a, uint64_t b) const
    {
        return barrett_mul(reduce_input<F>(a, q), reduce_input<F>(b, q), q, mu, shift);
    }
};
template <int F, bool ADD>
struct OpFma {  // EltwiseFMAModNative<F>, eltwise-fma-mod.cpp:18-78 (b = op3[i] when ADD)
    static constexpr const char* kName = "fma";
    uint64_t q, mu, s;  // s already reduced by ReduceInput<F>
    uint32_t shift;
    __device__ uint64_t operator()(uint64_t a, uint64_t b) const
    {
        uint64_t v = barrett_mul(reduce_input<F>(a, q), s, q, mu, shift);
        if constexpr (ADD) {
            v += reduce_input<F>(b, q);
            if (v >= q) v -= q;
        }
        return v;
    }
};
template <int KIND>
struct OpReduce {  // EltwiseReduceModNative branches, eltwise-reduce-mod.cpp:32-128
    static constexpr const char* kName = "reduce";
    uint64_t q, mu;
    uint32_t shift;
    __device__ uint64_t operator()(uint64_t a, uint64_t) const
    {
        if constexpr (KIND == 0) return a;                               // copy branches (:35-52)
        if constexpr (KIND == 1) return csub(a, q);                      // 2 -> 1 (:55-64)
        if constexpr (KIND == 2) return csub(csub(a, q << 1), q);        // 4 -> 1 (:67-86)
        if constexpr (KIND == 3) return csub(a, q << 1);                 // 4 -> 2 (:89-106)
        if constexpr (KIND == 4) return barrett_reduce64(a, q, mu, shift);  // in == q (:109-127)
        return a;
    }
};

}  // namespace axhel_impl
