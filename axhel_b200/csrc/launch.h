// Launch bookkeeping and kernel-launcher declarations (internal).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace axhel_impl {

// SM count of the current device (cached per device).
int sm_count();
// Counts one kernel launch of this library (reported by axhel_cuda_launch_count).
void count_launch();

// Brackets one launch with CUDA events on its stream while profiling is on
// (axhel_cuda_profile_enable), and with an NVTX range named like the kernel
// configuration when the environment variable AXHEL_NVTX is set (non-zero);
// a no-op otherwise.  `fmt` names the kernel configuration.
class ProfScope {
public:
    ProfScope(cudaStream_t s, const char* fmt, ...) __attribute__((format(printf, 3, 4)));
    ~ProfScope();
    ProfScope(const ProfScope&) = delete;
    ProfScope& operator=(const ProfScope&) = delete;

private:
    cudaStream_t s_;
    bool on_;
    bool nvtx_;
};

// Whether AXHEL_NVTX asks for NVTX ranges (read once).
bool nvtx_enabled();

void barrett_params(uint64_t q, uint64_t* mu, uint32_t* shift);

cudaError_t eltwise_add(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q, cudaStream_t s);
cudaError_t eltwise_add_scalar(uint64_t* r, const uint64_t* a, uint64_t b, uint64_t n, uint64_t q, cudaStream_t s);
cudaError_t eltwise_sub(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q, cudaStream_t s);
cudaError_t eltwise_sub_scalar(uint64_t* r, const uint64_t* a, uint64_t b, uint64_t n, uint64_t q, cudaStream_t s);
cudaError_t eltwise_mul(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q, uint64_t f,
                        cudaStream_t s);
cudaError_t eltwise_fma(uint64_t* r, const uint64_t* a, uint64_t sc, const uint64_t* c, uint64_t n, uint64_t q,
                        uint64_t f, cudaStream_t s);
cudaError_t eltwise_reduce(uint64_t* r, const uint64_t* a, uint64_t n, uint64_t q, uint64_t in_f, uint64_t out_f,
                           cudaStream_t s);
cudaError_t tensor_product(uint64_t* r0, uint64_t* r1, uint64_t* r2, const uint64_t* c0, const uint64_t* c1,
                           const uint64_t* d0, const uint64_t* d1, uint64_t n, uint64_t count, const uint64_t* moduli,
                           uint64_t nmod, uint64_t factor, cudaStream_t s);

}  // namespace axhel_impl
