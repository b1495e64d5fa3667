// C-ABI shim over the reference AXHEL native backend, compiled together with
// the reference's own source files by oracle/Makefile into
// oracle/_ref/libaxhel_ref.so.
//
// TEST INFRASTRUCTURE ONLY: used by tests/ and tests/golden/make_golden.py to
// pin the oracle restatement, and by the bench's CPU-baseline / reference arm
// to time the reference's own CPU implementation.  It calls the reference's
// public API (axhel/include/axhel/*.hpp) unmodified; the only private entry
// point used is detail::GenerateNTTTables (axhel/ntt/ntt-tables.hpp:23), to
// read back the tables the autonomous NTT constructor builds.
#include <axhel/axhel.hpp>
#include "ntt/ntt-tables.hpp"

#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

using unipi::axhel::NTT;
using unipi::axhel::NTTMultiplyOperand;

extern "C" {

int ref_ntt_tables(uint64_t n, uint64_t q, uint64_t psi, uint64_t* fwd, uint64_t* inv, uint64_t* ninv)
{
    size_t logn = 0;
    while ((uint64_t{1} << logn) < n) ++logn;
    auto t = unipi::axhel::detail::GenerateNTTTables(n, logn, q, psi);
    for (uint64_t i = 0; i < n; ++i) {
        fwd[2 * i] = t.root_powers[i].operand;
        fwd[2 * i + 1] = t.root_powers[i].quotient;
        inv[2 * i] = t.inv_root_powers[i].operand;
        inv[2 * i + 1] = t.inv_root_powers[i].quotient;
    }
    ninv[0] = t.inv_degree_modulo.operand;
    ninv[1] = t.inv_degree_modulo.quotient;
    return 0;
}

void* ref_ntt_create(uint64_t n, uint64_t q, uint64_t psi) { return new NTT(n, q, psi); }

void* ref_ntt_create_external(uint64_t n, uint64_t q, const uint64_t* fwd, const uint64_t* inv,
                              const uint64_t* ninv)
{
    return new NTT(n, q, reinterpret_cast<const NTTMultiplyOperand*>(fwd),
                   reinterpret_cast<const NTTMultiplyOperand*>(inv), NTTMultiplyOperand{ninv[0], ninv[1]});
}

void ref_ntt_destroy(void* h) { delete static_cast<NTT*>(h); }

void ref_ntt_forward(void* h, uint64_t* res, const uint64_t* op, uint64_t in_f, uint64_t out_f)
{
    static_cast<NTT*>(h)->ComputeForward(res, op, in_f, out_f);
}

void ref_ntt_inverse(void* h, uint64_t* res, const uint64_t* op, uint64_t in_f, uint64_t out_f)
{
    static_cast<NTT*>(h)->ComputeInverse(res, op, in_f, out_f);
}

void ref_add_vv(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q)
{
    unipi::axhel::EltwiseAddMod(r, a, b, n, q);
}
void ref_add_vs(uint64_t* r, const uint64_t* a, uint64_t b, uint64_t n, uint64_t q)
{
    unipi::axhel::EltwiseAddMod(r, a, b, n, q);
}
void ref_sub_vv(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q)
{
    unipi::axhel::EltwiseSubMod(r, a, b, n, q);
}
void ref_sub_vs(uint64_t* r, const uint64_t* a, uint64_t b, uint64_t n, uint64_t q)
{
    unipi::axhel::EltwiseSubMod(r, a, b, n, q);
}
void ref_mul(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q, uint64_t f)
{
    unipi::axhel::EltwiseMulMod(r, a, b, n, q, f);
}
void ref_fma(uint64_t* r, const uint64_t* a, uint64_t s, const uint64_t* c, uint64_t n, uint64_t q, uint64_t f)
{
    unipi::axhel::EltwiseFMAMod(r, a, s, c, n, q, f);
}
void ref_reduce(uint64_t* r, const uint64_t* a, uint64_t n, uint64_t q, uint64_t in_f, uint64_t out_f)
{
    unipi::axhel::EltwiseReduceMod(r, a, n, q, in_f, out_f);
}

// The lazy round trip the reference tests and SEAL use, over `count` limbs
// stored back to back (limb i uses handle i % nh):
//   ComputeForward(1, 4) -> EltwiseReduceMod(4 -> 2) -> ComputeInverse(2, 1)
// Limbs are spread over `threads` std::threads (the library itself is
// single-threaded; each thread calls the shared const NTT objects, as SEAL does).
void ref_roundtrip_batch(void* const* handles, uint64_t nh, uint64_t* data, uint64_t n, uint64_t count,
                         int threads)
{
    if (threads < 1) threads = 1;
    if (static_cast<uint64_t>(threads) > count) threads = static_cast<int>(count ? count : 1);
    auto work = [&](uint64_t begin, uint64_t end) {
        for (uint64_t i = begin; i < end; ++i) {
            const NTT* ntt = static_cast<const NTT*>(handles[i % nh]);
            uint64_t* x = data + i * n;
            ntt->ComputeForward(x, x, 1, 4);
            unipi::axhel::EltwiseReduceMod(x, x, n, ntt->Modulus(), 4, 2);
            ntt->ComputeInverse(x, x, 2, 1);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back(work, count * t / threads, count * (t + 1) / threads);
    for (auto& th : pool) th.join();
}

}  // extern "C"
