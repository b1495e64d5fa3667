// The unipi::axhel C++ drop-in, called the way the reference's own tests and
// SEAL call it: host pointers, one (N, q) limb per call, in place and out of
// place, shared const NTT objects across threads.  Restates cases of the
// reference's tests/public/test_ntt.cpp, test_eltwise.cpp, test_reduce.cpp and
// test_polymul.cpp against the C oracle (oracle/axhel_oracle.c, linked in).
// Built and run by tests/test_dropin_gpu.py; exits non-zero on any mismatch.
#include <axhel/axhel.hpp>
#include <axhel/ntt/ntt-rns.hpp>

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <thread>
#include <vector>

extern "C" {
#include "../../oracle/axhel_oracle.h"
}

using unipi::axhel::NTT;
using unipi::axhel::NTTMultiplyOperand;
using Vec = std::vector<uint64_t>;

static int g_fail = 0;
#define CHECK(cond, ...)                                          \
    do {                                                          \
        if (!(cond)) {                                            \
            std::fprintf(stderr, "FAIL %s:%d ", __FILE__, __LINE__); \
            std::fprintf(stderr, __VA_ARGS__);                     \
            std::fprintf(stderr, "\n");                            \
            ++g_fail;                                              \
        }                                                         \
    } while (0)

static const uint64_t kSeed = 0x415848454cULL;

static Vec rand_vec(uint64_t* st, size_t n, uint64_t bound)
{
    Vec v(n);
    orc_random_vector(v.data(), n, bound, st);
    return v;
}

struct Tables {
    Vec fwd, inv;
    uint64_t ninv[2];
};
static Tables tables(uint64_t n, uint64_t q, uint64_t psi)
{
    Tables t;
    t.fwd.resize(2 * n);
    t.inv.resize(2 * n);
    orc_ntt_tables(n, q, psi, t.fwd.data(), t.inv.data(), t.ninv);
    return t;
}

static void test_known_vector()
{
    NTT ntt(8, 17, 3);
    Vec x{1, 2, 3, 4, 5, 6, 7, 8};
    ntt.ComputeForward(x.data(), x.data(), 1, 1);
    CHECK((x == Vec{5, 0, 13, 8, 9, 11, 5, 8}), "known vector forward");
    ntt.ComputeInverse(x.data(), x.data(), 1, 1);
    CHECK((x == Vec{1, 2, 3, 4, 5, 6, 7, 8}), "known vector inverse");
    CHECK(ntt.Degree() == 8 && ntt.Modulus() == 17, "accessors");
}

static void test_external_tables()
{
    const std::vector<NTTMultiplyOperand> fwd{{1, 1085102592571150095ULL}, {13, 14106333703424951235ULL},
                                              {9, 9765923333140350855ULL}, {15, 16276538888567251425ULL},
                                              {3, 3255307777713450285ULL}, {5, 5425512962855750475ULL},
                                              {10, 10851025925711500950ULL}, {11, 11936128518282651045ULL}};
    const std::vector<NTTMultiplyOperand> inv{{0, 0}, {6, 6510615555426900570ULL},
                                              {7, 7595718147998050665ULL}, {12, 13021231110853801140ULL},
                                              {14, 15191436295996101330ULL}, {2, 2170205185142300190ULL},
                                              {8, 8680820740569200760ULL}, {4, 4340410370284600380ULL}};
    NTT ntt(8, 17, fwd.data(), inv.data(), NTTMultiplyOperand{15, 16276538888567251425ULL});
    Vec x{1, 2, 3, 4, 5, 6, 7, 8}, y(8);
    ntt.ComputeForward(y.data(), x.data(), 1, 1);
    CHECK((y == Vec{5, 0, 13, 8, 9, 11, 5, 8}), "external tables forward");
    NTT copy = ntt;  // shallow copy shares the tables
    copy.ComputeInverse(y.data(), y.data(), 1, 1);
    CHECK(y == x, "external tables inverse via copy");
    NTT moved = std::move(copy);
    CHECK(moved.Degree() == 8 && copy.Degree() == 0, "move leaves an empty object");
}

// The external tables are borrowed (ntt.hpp:34-37): tables the caller
// rewrites in place after construction are the ones the next transform uses.
static void test_external_tables_borrowed()
{
    const uint64_t n = 4096, q = orc_find_ntt_prime(n, 50);
    const uint64_t psi1 = orc_find_primitive_root(n, q);
    const uint64_t psi2 = orc_pow_mod(psi1, 3, q);  // another primitive 2n-th root (3 is odd)
    Tables t1 = tables(n, q, psi1), t2 = tables(n, q, psi2);
    std::vector<uint64_t> fwd = t1.fwd, inv = t1.inv;  // the caller's tables
    NTT ntt(n, q, reinterpret_cast<const NTTMultiplyOperand*>(fwd.data()),
            reinterpret_cast<const NTTMultiplyOperand*>(inv.data()), NTTMultiplyOperand{t1.ninv[0], t1.ninv[1]});
    uint64_t st[313];
    orc_mt64_seed(st, kSeed ^ 0xB0220);
    const Vec x = rand_vec(st, n, q);
    Vec y(n), e(n);
    ntt.ComputeForward(y.data(), x.data(), 1, 4);
    orc_ntt_compute_forward(e.data(), x.data(), n, q, t1.fwd.data(), 1, 4);
    CHECK(y == e, "borrowed tables: forward with the first tables");
    std::copy(t2.fwd.begin(), t2.fwd.end(), fwd.begin());  // rewritten in place, same storage
    std::copy(t2.inv.begin(), t2.inv.end(), inv.begin());
    ntt.ComputeForward(y.data(), x.data(), 1, 4);
    orc_ntt_compute_forward(e.data(), x.data(), n, q, t2.fwd.data(), 1, 4);
    CHECK(y == e, "borrowed tables: forward sees the rewritten table");
    const Vec z = rand_vec(st, n, 2 * q);
    ntt.ComputeInverse(y.data(), z.data(), 2, 2);
    orc_ntt_compute_inverse(e.data(), z.data(), n, q, t2.inv.data(), t1.ninv, 2, 2);
    CHECK(y == e, "borrowed tables: inverse sees the rewritten table");
}

static void test_transforms_vs_oracle()
{
    uint64_t st[313];
    orc_mt64_seed(st, kSeed ^ 0xC0FFEE);
    for (uint64_t n : {8ull, 256ull, 4096ull, 32768ull, 65536ull, 131072ull}) {
        for (unsigned bits : {30u, 50u, 59u, 62u}) {
            const uint64_t q = orc_find_ntt_prime(n, bits);
            const uint64_t psi = orc_find_primitive_root(n, q);
            NTT ntt(n, q, psi);
            Tables t = tables(n, q, psi);
            for (uint64_t of : {4ull, 1ull}) {
                Vec x = rand_vec(st, n, 4 * q), exp = x, got(n);
                orc_ntt_compute_forward(exp.data(), exp.data(), n, q, t.fwd.data(), 4, of);
                ntt.ComputeForward(got.data(), x.data(), 4, of);
                CHECK(got == exp, "forward n=%llu bits=%u out=%llu", (unsigned long long)n, bits,
                      (unsigned long long)of);
            }
            for (uint64_t of : {2ull, 1ull}) {
                Vec y = rand_vec(st, n, 2 * q), exp = y;
                orc_ntt_compute_inverse(exp.data(), exp.data(), n, q, t.inv.data(), t.ninv, 2, of);
                ntt.ComputeInverse(y.data(), y.data(), 2, of);
                CHECK(y == exp, "inverse n=%llu bits=%u out=%llu", (unsigned long long)n, bits,
                      (unsigned long long)of);
            }
        }
    }
}

static void test_lazy_round_trip_seal_style()
{
    // SEAL: ntt_negacyclic_harvey_lazy -> ComputeForward(p, p, 4, 4); the lazy
    // composition of test_ntt.cpp:141-150.
    uint64_t st[313];
    orc_mt64_seed(st, kSeed ^ 0x4e5454);
    for (uint64_t n : {1024ull, 16384ull}) {
        const uint64_t q = orc_find_ntt_prime(n, 60);
        NTT ntt(n, q, orc_find_primitive_root(n, q));
        Vec orig = rand_vec(st, n, q), x = orig;
        ntt.ComputeForward(x.data(), x.data(), 4, 4);
        unipi::axhel::EltwiseReduceMod(x.data(), x.data(), n, q, 4, 2);
        ntt.ComputeInverse(x.data(), x.data(), 2, 1);
        CHECK(x == orig, "lazy round trip n=%llu", (unsigned long long)n);
    }
}

static void test_eltwise_host_pointers()
{
    uint64_t st[313];
    orc_mt64_seed(st, kSeed ^ 0xE17);
    for (unsigned bits : {20u, 40u, 50u, 60u, 62u}) {
        const uint64_t q = orc_find_ntt_prime(1024, bits);
        for (size_t n : {0ul, 1ul, 3ul, 33ul, 1025ul, 65537ul}) {
            Vec a = rand_vec(st, n, q), b = rand_vec(st, n, q), got(n), exp(n);
            unipi::axhel::EltwiseAddMod(got.data(), a.data(), b.data(), n, q);
            orc_add_vv(exp.data(), a.data(), b.data(), n, q);
            CHECK(got == exp, "add n=%zu", n);
            unipi::axhel::EltwiseSubMod(got.data(), a.data(), q - 1, n, q);
            orc_sub_vs(exp.data(), a.data(), q - 1, n, q);
            CHECK(got == exp, "sub-vs n=%zu", n);
            for (uint64_t f : {1ull, 2ull, 4ull}) {
                Vec x = rand_vec(st, n, f * q), y = rand_vec(st, n, f * q);
                unipi::axhel::EltwiseMulMod(got.data(), x.data(), y.data(), n, q, f);
                orc_mul(exp.data(), x.data(), y.data(), n, q, f);
                CHECK(got == exp, "mul n=%zu f=%llu", n, (unsigned long long)f);
            }
            Vec x = rand_vec(st, n, bits >= 61 ? ~0ull : 8 * q), c = rand_vec(st, n, q);
            unipi::axhel::EltwiseFMAMod(got.data(), x.data(), 12345, c.data(), n, q, 8);
            orc_fma(exp.data(), x.data(), 12345, c.data(), n, q, 8);
            CHECK(got == exp, "fma n=%zu", n);
            Vec r = rand_vec(st, n, ~0ull);
            unipi::axhel::EltwiseReduceMod(got.data(), r.data(), n, q, q, 1);
            orc_reduce(exp.data(), r.data(), n, q, q, 1);
            CHECK(got == exp, "barrett reduce n=%zu", n);
            // in place, result aliasing operand1
            Vec al = a;
            unipi::axhel::EltwiseMulMod(al.data(), al.data(), b.data(), n, q, 1);
            orc_mul(exp.data(), a.data(), b.data(), n, q, 1);
            CHECK(al == exp, "mul in place n=%zu", n);
        }
        // unsupported factor leaves the result untouched
        Vec a(16, 1), out(16, 777);
        unipi::axhel::EltwiseMulMod(out.data(), a.data(), a.data(), 16, q, 3);
        CHECK(out == Vec(16, 777), "unsupported factor");
        unipi::axhel::EltwiseReduceMod(out.data(), a.data(), 16, q, 4, 4);
        CHECK(out == Vec(16, 777), "unmatched reduce pair");
    }
}

static void test_polymul()
{
    // test_polymul.cpp:222-234 with host pointers.
    uint64_t st[313];
    orc_mt64_seed(st, kSeed ^ 0x504f4c594d554cULL);
    for (uint64_t n : {8ull, 32ull, 64ull}) {
        const uint64_t q = orc_find_ntt_prime(n, 62);
        NTT ntt(n, q, orc_find_primitive_root(n, q));
        Vec a = rand_vec(st, n, q), b = rand_vec(st, n, q), A = a, B = b, out(n);
        ntt.ComputeForward(A.data(), A.data(), 1, 1);
        ntt.ComputeForward(B.data(), B.data(), 1, 1);
        unipi::axhel::EltwiseMulMod(out.data(), A.data(), B.data(), n, q, 1);
        ntt.ComputeInverse(out.data(), out.data(), 1, 1);
        Vec ref(n, 0);
        for (uint64_t i = 0; i < n; ++i)
            for (uint64_t j = 0; j < n; ++j) {
                const uint64_t p = (uint64_t)(((unsigned __int128)a[i] * b[j]) % q);
                const uint64_t k = i + j;
                if (k < n)
                    ref[k] = (ref[k] + p) % q;
                else
                    ref[k - n] = (ref[k - n] + q - p) % q;
            }
        CHECK(out == ref, "polymul n=%llu", (unsigned long long)n);
    }
}

static void test_device_pointers()
{
    const uint64_t n = 4096, q = orc_find_ntt_prime(n, 55);
    NTT ntt(n, q, orc_find_primitive_root(n, q));
    uint64_t st[313];
    orc_mt64_seed(st, kSeed ^ 0xD);
    Vec x = rand_vec(st, n, q), host = x;
    uint64_t* d = nullptr;
    cudaMalloc(&d, n * 8);
    cudaMemcpy(d, x.data(), n * 8, cudaMemcpyHostToDevice);
    ntt.ComputeForward(d, d, 1, 4);
    ntt.ComputeForward(host.data(), host.data(), 1, 4);
    Vec back(n);
    cudaMemcpy(back.data(), d, n * 8, cudaMemcpyDeviceToHost);
    CHECK(back == host, "device-pointer forward equals host-pointer forward");
    cudaFree(d);
}

static void test_threads_share_one_ntt()
{
    // SEAL shares one cached const NTT across threads.
    const uint64_t n = 8192, q = orc_find_ntt_prime(n, 59);
    const uint64_t psi = orc_find_primitive_root(n, q);
    const NTT ntt(n, q, psi);
    Tables t = tables(n, q, psi);
    std::vector<std::thread> pool;
    std::vector<int> ok(8, 0);
    for (int k = 0; k < 8; ++k)
        pool.emplace_back([&, k] {
            uint64_t st[313];
            orc_mt64_seed(st, kSeed + k);
            int good = 1;
            for (int r = 0; r < 20; ++r) {
                Vec x = rand_vec(st, n, q), exp = x;
                orc_ntt_compute_forward(exp.data(), exp.data(), n, q, t.fwd.data(), 1, 4);
                ntt.ComputeForward(x.data(), x.data(), 1, 4);
                good &= x == exp;
            }
            ok[k] = good;
        });
    for (auto& th : pool) th.join();
    for (int k = 0; k < 8; ++k) CHECK(ok[k], "thread %d", k);
}

static void test_rns_batches(uint64_t n)
{
    // One call per polynomial instead of one per limb (ntt-rns.hpp): equal to
    // the per-limb calls, host and device pointers, in and out of place.
    // 15 limbs of N = 65536 (7.5 MiB) are staged in chunks of 4 limbs.
    const size_t L = 5, count = 3 * L;
    std::vector<NTT> ntts;
    std::vector<uint64_t> qs;
    for (size_t i = 0; i < L; ++i) {
        const uint64_t q = orc_find_ntt_prime_near(n, 40 + 4 * (unsigned)i, 1, 2);
        qs.push_back(q);
        ntts.emplace_back(n, q, orc_find_primitive_root(n, q));
    }
    uint64_t st[313];
    orc_mt64_seed(st, kSeed ^ 0x524E53);
    Vec x(count * n);
    for (size_t i = 0; i < count; ++i) {
        Vec v = rand_vec(st, n, 4 * qs[i % L]);
        std::copy(v.begin(), v.end(), x.begin() + i * n);
    }
    for (uint64_t out_f : {1, 4}) {
        Vec want(count * n), got(count * n), inplace = x;
        for (size_t i = 0; i < count; ++i)
            ntts[i % L].ComputeForward(want.data() + i * n, x.data() + i * n, 4, out_f);
        unipi::axhel::ComputeForwardRNS(ntts.data(), L, got.data(), x.data(), count, 4, out_f);
        CHECK(got == want, "ComputeForwardRNS N=%llu out_f=%llu", (unsigned long long)n, (unsigned long long)out_f);
        unipi::axhel::ComputeForwardRNS(ntts.data(), L, inplace.data(), inplace.data(), count, 4, out_f);
        CHECK(inplace == want, "ComputeForwardRNS in place out_f=%llu", (unsigned long long)out_f);
        for (uint64_t inv_out : {1, 2}) {
            Vec iwant(count * n), igot(count * n);
            Vec lazy2 = want;  // inverse inputs in [0, 2q)
            for (size_t i = 0; i < count; ++i)
                for (size_t k = 0; k < n; ++k) {
                    uint64_t& v = lazy2[i * n + k];
                    if (v >= 2 * qs[i % L]) v -= 2 * qs[i % L];
                }
            for (size_t i = 0; i < count; ++i)
                ntts[i % L].ComputeInverse(iwant.data() + i * n, lazy2.data() + i * n, 2, inv_out);
            unipi::axhel::ComputeInverseRNS(ntts.data(), L, igot.data(), lazy2.data(), count, 2, inv_out);
            CHECK(igot == iwant, "ComputeInverseRNS out_f=%llu", (unsigned long long)inv_out);
        }
    }
    // device pointers: used in place, no staging
    uint64_t* d = nullptr;
    cudaMalloc(&d, count * n * 8);
    cudaMemcpy(d, x.data(), count * n * 8, cudaMemcpyHostToDevice);
    unipi::axhel::ComputeForwardRNS(ntts.data(), L, d, d, count, 4, 4);
    Vec back(count * n), want(count * n);
    cudaMemcpy(back.data(), d, count * n * 8, cudaMemcpyDeviceToHost);
    unipi::axhel::ComputeForwardRNS(ntts.data(), L, want.data(), x.data(), count, 4, 4);
    CHECK(back == want, "ComputeForwardRNS on device pointers");
    cudaFree(d);
}

int main()
{
    test_known_vector();
    test_external_tables();
    test_external_tables_borrowed();
    test_transforms_vs_oracle();
    test_lazy_round_trip_seal_style();
    test_eltwise_host_pointers();
    test_polymul();
    test_device_pointers();
    test_threads_share_one_ntt();
    test_rns_batches(4096);
    test_rns_batches(65536);
    if (g_fail) {
        std::fprintf(stderr, "%d failure(s)\n", g_fail);
        return 1;
    }
    std::printf("drop-in C++ API: all checks passed\n");
    return 0;
}
