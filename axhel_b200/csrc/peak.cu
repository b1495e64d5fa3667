// Integer-pipe ceiling probe: the reference forward butterfly
// (ForwardButterflyNative, axhel/ntt/ntt-internal.hpp:20-31) and inverse
// butterfly (ntt-internal.hpp:37-49) applied to values held in registers,
// with no memory traffic in the timed loop.  The measured butterflies per
// second are the compute roofline the NTT kernels are reported against
// (a transform of N points needs (N/2) log2 N butterflies).
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/axhel_cuda.h"
#include "internal.h"
#include "launch.h"
#include "modarith.cuh"

namespace axhel_impl {
using namespace axhel_dev;

template <bool INV>
__global__ void __launch_bounds__(256) butterfly_peak_kernel(uint64_t* sink, const ulonglong2* tw, uint64_t q,
                                                             uint32_t iters)
{
    constexpr int R = 8;
    const uint64_t q2 = q << 1;
    uint64_t v[R];
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = (tid * 0x9E3779B97F4A7C15ull + i * 0xBF58476D1CE4E5B9ull) % q;
    ulonglong2 w[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) w[i] = tw[(tid + i) & 7];
    for (uint32_t it = 0; it < iters; ++it) {
        // three radix-2 stages over 8 registers: 12 butterflies
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            const int h = 1 << s;
#pragma unroll
            for (int i = 0; i < R; ++i) {
                if (i & h) continue;
                const ulonglong2 ww = w[(i + s) & 3];
                if (INV)
                    inv_butterfly(v[i], v[i | h], ww.x, ww.y, q, q2);
                else
                    fwd_butterfly(v[i], v[i | h], ww.x, ww.y, q, q2);
            }
        }
    }
    uint64_t acc = 0;
#pragma unroll
    for (int i = 0; i < R; ++i) acc ^= v[i];
    if (acc == 0x5555555555555555ull) sink[tid] = acc;  // keeps the loop live
}

}  // namespace axhel_impl

using namespace axhel_impl;

extern "C" axhel_status_t axhel_cuda_butterfly_peak(axhel_ntt_t ntt, int inverse, double* butterflies_per_s,
                                                    void* stream)
{
    if (!ntt || !butterflies_per_s || ntt->n < 8) return AXHEL_ERR_INVALID;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int blocks = sm_count() * 8;  // 8 CTAs of 256 threads per SM (as many as the registers allow stay resident)
    uint64_t* sink = nullptr;
    if (cudaMalloc(&sink, sizeof(uint64_t) * blocks * 256) != cudaSuccess) return AXHEL_ERR_NOMEM;
    const uint32_t iters = 4096;
    const uint64_t modulus = ntt->q;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const ulonglong2* tw = reinterpret_cast<const ulonglong2*>(static_cast<const unsigned char*>(ntt->mem) + 256);
    // warm-up, then timed
    if (inverse)
        butterfly_peak_kernel<true><<<blocks, 256, 0, s>>>(sink, tw, modulus, 64);
    else
        butterfly_peak_kernel<false><<<blocks, 256, 0, s>>>(sink, tw, modulus, 64);
    cudaEventRecord(a, s);
    if (inverse)
        butterfly_peak_kernel<true><<<blocks, 256, 0, s>>>(sink, tw, modulus, iters);
    else
        butterfly_peak_kernel<false><<<blocks, 256, 0, s>>>(sink, tw, modulus, iters);
    cudaEventRecord(b, s);
    cudaError_t e = cudaEventSynchronize(b);
    float ms = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    if (e != cudaSuccess || ms <= 0) return AXHEL_ERR_CUDA;
    const double bfly = (double)blocks * 256.0 * iters * 12.0;
    *butterflies_per_s = bfly / (ms * 1e-3);
    return AXHEL_OK;
}
