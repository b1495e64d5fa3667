// Twiddle tables generated on the device.
//
// GenerateNTTTables (axhel/ntt/ntt-tables.cpp:81-140) fills, for one (N, q, psi):
//   fwd[i] = {w, floor(w 2^64 / q)} with w = psi^bitrev(i)             (:96-106)
//   inv[0] = {0, 0}, inv[i] = {w, ...} with w = psi^-(bitrev(i-1) + 1)  (:113-129)
// from sequential powers, one u128 multiply-and-divide per entry on the host.
// The values are unique (canonical residues and exact quotients), so any
// exact method gives the same tables.  Here every entry is one thread:
//
//   * w = psi^e mod q by square-and-multiply in Montgomery form (R = 2^64;
//     q odd, q < 2^62, so every REDC result is below 2q and one conditional
//     subtract makes it canonical);
//   * the Shoup quotient Q = floor(w 2^64 / q) from r = w 2^64 mod q (one
//     Montgomery product with R^2 mod q): Q q = w 2^64 - r exactly, hence
//     Q = r * (-q^-1) mod 2^64 -- an exact division, one multiply.
//
// The host computes the O(1) constants per context (psi^-1 = psi^(q-2) as
// the reference does, N^-1, the final-stage scaled root, Barrett and
// Montgomery constants) and the kernel writes the context header beside the
// tables, so a context is ready after one launch for any number of (N, q).
#include <cuda_runtime.h>

#include <cstdint>

#include "internal.h"
#include "launch.h"
#include "tables.h"

namespace axhel_impl {

namespace {

__device__ __forceinline__ uint64_t redc(uint64_t lo, uint64_t hi, uint64_t q, uint64_t mninv)
{
    const uint64_t m = lo * mninv;  // lo + m q == 0 (mod 2^64)
    const uint64_t t = hi + __umul64hi(m, q) + (lo != 0 ? 1 : 0);
    return t >= q ? t - q : t;
}

__device__ __forceinline__ uint64_t mont_mul(uint64_t a, uint64_t b, uint64_t q, uint64_t mninv)
{
    return redc(a * b, __umul64hi(a, b), q, mninv);
}

__global__ void __launch_bounds__(256) gen_tables_kernel(const __grid_constant__ TableGenArgs a)
{
    const TableGenJob& j = a.job[blockIdx.y];
    const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t n = j.n;
    if (idx == 0) *reinterpret_cast<ModCtx*>(j.base) = j.hdr;
    if (idx >= 2 * n) return;
    ulonglong2* out = reinterpret_cast<ulonglong2*>(j.base + kCtxHeaderBytes) + idx;  // fwd[0..n) then inv[0..n)
    const bool inv = idx >= n;
    const uint32_t i = (uint32_t)(inv ? idx - n : idx);
    if (inv && i == 0) {
        *out = make_ulonglong2(0, 0);
        return;
    }
    const uint32_t sh = 32 - j.logn;
    const uint32_t e = inv ? (__brev(i - 1) >> sh) + 1 : (__brev(i) >> sh);
    const uint64_t base = inv ? j.psiinv_m : j.psi_m;
    uint64_t acc = j.one_m;
    for (int b = 31 - __clz(e | 1); b >= 0; --b) {  // e < 2^17
        acc = mont_mul(acc, acc, j.q, j.mninv);
        if ((e >> b) & 1) acc = mont_mul(acc, base, j.q, j.mninv);
    }
    const uint64_t w = redc(acc, 0, j.q, j.mninv);           // out of Montgomery form: psi^e mod q
    const uint64_t r = mont_mul(w, j.r2m, j.q, j.mninv);     // w 2^64 mod q
    *out = make_ulonglong2(w, r * j.mninv);                  // Q = (w 2^64 - r) / q
}

}  // namespace

cudaError_t launch_gen_tables(const TableGenArgs& a, uint64_t max_n, cudaStream_t s)
{
    if (a.njobs == 0) return cudaSuccess;
    const uint64_t bx = (2 * max_n + 255) / 256;
    count_launch();
    ProfScope prof(s, "gen_tables");
    gen_tables_kernel<<<dim3((unsigned)bx, a.njobs), 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace axhel_impl
