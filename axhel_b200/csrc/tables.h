// Device generation of twiddle tables (tables.cu), driven by the context
// constructors in capi.cpp.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "internal.h"

namespace axhel_impl {

// One context to fill: its header (written verbatim at `base`) and the
// Montgomery constants of its modulus; the tables follow the header.
struct TableGenJob {
    ModCtx hdr;
    unsigned char* base;  // device allocation: header | fwd[n] | inv[n]
    uint64_t q;
    uint64_t mninv;       // -q^-1 mod 2^64
    uint64_t r2m;         // 2^128 mod q
    uint64_t one_m;       // 2^64 mod q (1 in Montgomery form)
    uint64_t psi_m;       // psi 2^64 mod q
    uint64_t psiinv_m;    // psi^-1 2^64 mod q
    uint64_t n;
    uint32_t logn, pad;
};

constexpr int kTableGenJobsPerLaunch = 96;  // the argument block stays under 15 KB

struct TableGenArgs {
    uint32_t njobs;
    TableGenJob job[kTableGenJobsPerLaunch];
};

// One launch filling every job's header and tables; `max_n` is the largest n.
cudaError_t launch_gen_tables(const TableGenArgs& a, uint64_t max_n, cudaStream_t s);

}  // namespace axhel_impl
