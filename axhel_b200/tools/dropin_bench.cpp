// Per-call cost of the unipi::axhel C++ API in the way the Microsoft SEAL
// integration calls it (integration/seal/SEAL-4.4.5-AXHEL.patch:139-160,
// 189, 222): host (pageable) pointers, one RNS limb per call, in place,
// several host threads sharing one cached const NTT object:
//   NTT::ComputeForward(p, p, 4, 4)      (ntt.cpp:173-186)
//   NTT::ComputeInverse(p, p, 2, 1)      (ntt.cpp:192-204)
//   EltwiseMulMod(p, p, b, N, q, 4)      (eltwise-mul-mod.cpp:81-94)
// and the plain single-limb round trip of the N = 4096 configuration:
//   ComputeForward(a,a,1,1), ComputeForward(b,b,1,1), EltwiseMulMod(c,a,b,N,q,1),
//   EltwiseAddMod(c,c,s,N,q), ComputeInverse(c,c,1,1).
//
// The program uses only the public declarations of include/axhel/*.hpp, so
// the same source links against this library (axhel_b200/dropin_bench) or
// against the reference native backend (oracle/_ref/dropin_bench_ref) to
// time both sides of a drop-in.
//
//   dropin_bench <threads> <seconds per case> <logn>:<q>:<psi> ...
//
// One JSON line per (operation, degree): mean microseconds per call seen by
// each thread, and calls per second over all threads.
//
// Built against this library (AXHEL_RNS defined), it also times a whole RNS
// polynomial of L = 24 limbs -- the loop SEAL runs over a ciphertext's moduli
// (ntt_negacyclic_harvey over coeff_modulus) -- as 24 per-limb
// ComputeForward calls and as one ComputeForwardRNS call
// (axhel/ntt/ntt-rns.hpp, not in the reference API), both on host memory.
#include <axhel/axhel.hpp>
#ifdef AXHEL_RNS
#include <axhel/ntt/ntt-rns.hpp>
#endif

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <thread>
#include <vector>

namespace ax = unipi::axhel;
using Clock = std::chrono::steady_clock;

namespace {

struct Case {
    unsigned logn;
    uint64_t q, psi;
};

// Deterministic fill with residues below `bound`.
void fill(std::vector<uint64_t>& v, uint64_t bound, uint64_t seed)
{
    uint64_t x = seed * 0x9E3779B97F4A7C15ull + 1;
    for (auto& w : v) {
        x ^= x >> 12;
        x ^= x << 25;
        x ^= x >> 27;
        w = (x * 0x2545F4914F6CDD1Dull) % bound;
    }
}

struct Result {
    double us_per_call, calls_per_s;
};

// Runs `body(thread, buffers)` on `threads` threads, each for `seconds`
// after 3 untimed calls and a common start.
template <class Setup, class Body>
Result run(int threads, double seconds, Setup setup, Body body)
{
    std::atomic<int> ready{0};
    std::atomic<bool> go{false};
    std::vector<double> per_call(threads, 0.0);
    std::vector<uint64_t> calls(threads, 0);
    std::vector<std::thread> pool;
    Clock::time_point t0;
    for (int t = 0; t < threads; ++t) {
        pool.emplace_back([&, t] {
            auto st = setup(t);
            for (int i = 0; i < 3; ++i) body(st);
            ready.fetch_add(1);
            while (!go.load()) std::this_thread::yield();
            const auto a = Clock::now();
            const auto end = a + std::chrono::duration<double>(seconds);
            uint64_t k = 0;
            Clock::time_point b;
            do {
                body(st);
                ++k;
                b = Clock::now();
            } while (b < end);
            calls[t] = k;
            per_call[t] = std::chrono::duration<double, std::micro>(b - a).count() / k;
        });
    }
    while (ready.load() < threads) std::this_thread::yield();
    t0 = Clock::now();
    go.store(true);
    for (auto& th : pool) th.join();
    const double wall = std::chrono::duration<double>(Clock::now() - t0).count();
    double us = 0;
    uint64_t total = 0;
    for (int t = 0; t < threads; ++t) {
        us += per_call[t];
        total += calls[t];
    }
    return Result{us / threads, total / wall};
}

void emit(const char* op, const Case& c, int threads, const Result& r)
{
    std::printf("{\"op\": \"%s\", \"logn\": %u, \"q\": %llu, \"threads\": %d, \"us_per_call\": %.3f, "
                "\"calls_per_s\": %.1f}\n",
                op, c.logn, (unsigned long long)c.q, threads, r.us_per_call, r.calls_per_s);
    std::fflush(stdout);
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s <threads> <seconds> <logn>:<q>:<psi> ...\n", argv[0]);
        return 2;
    }
    const int threads = std::atoi(argv[1]);
    const double seconds = std::atof(argv[2]);
    if (threads < 1 || threads > 256 || !(seconds > 0)) return 2;
    for (int a = 3; a < argc; ++a) {
        Case c{};
        unsigned long long q = 0, psi = 0;
        if (std::sscanf(argv[a], "%u:%llu:%llu", &c.logn, &q, &psi) != 3) return 2;
        c.q = q;
        c.psi = psi;
        const uint64_t n = 1ull << c.logn;
        const ax::NTT ntt(n, c.q, c.psi);  // one cached object shared by every thread
        struct Bufs {
            std::vector<uint64_t> x, y, a, b, c;
        };
        auto setup = [&](int t) {
            Bufs s;
            s.x.resize(n);
            s.y.resize(n);
            fill(s.x, 2 * c.q, 11 + t);
            fill(s.y, 4 * c.q, 23 + t);
            return s;
        };
        emit("forward_4_4", c, threads,
             run(threads, seconds, setup, [&](Bufs& s) { ntt.ComputeForward(s.x.data(), s.x.data(), 4, 4); }));
        emit("inverse_2_1", c, threads,
             run(threads, seconds, setup, [&](Bufs& s) { ntt.ComputeInverse(s.x.data(), s.x.data(), 2, 1); }));
        emit("mulmod_4", c, threads, run(threads, seconds, setup, [&](Bufs& s) {
                 ax::EltwiseMulMod(s.x.data(), s.x.data(), s.y.data(), n, c.q, 4);
             }));
        auto setup_rt = [&](int t) {
            Bufs s;
            s.x.resize(n);
            s.y.resize(n);
            s.a.resize(n);
            s.b.resize(n);
            s.c.resize(n);
            fill(s.x, c.q, 31 + t);
            fill(s.y, c.q, 37 + t);
            return s;
        };
        const uint64_t scalar = c.q / 3;
        emit("round_trip_c1", c, threads, run(threads, seconds, setup_rt, [&](Bufs& s) {
                 s.a = s.x;
                 s.b = s.y;
                 ntt.ComputeForward(s.a.data(), s.a.data(), 1, 1);
                 ntt.ComputeForward(s.b.data(), s.b.data(), 1, 1);
                 ax::EltwiseMulMod(s.c.data(), s.a.data(), s.b.data(), n, c.q, 1);
                 ax::EltwiseAddMod(s.c.data(), s.c.data(), scalar, n, c.q);
                 ntt.ComputeInverse(s.c.data(), s.c.data(), 1, 1);
             }));
#ifdef AXHEL_RNS
        // an RNS polynomial of 24 limbs (the same modulus stands in for the
        // 24 distinct ones of a ciphertext: the cost does not depend on it)
        constexpr size_t L = 24;
        const std::vector<ax::NTT> limbs(L, ntt);
        auto setup_poly = [&](int t) {
            Bufs s;
            s.x.resize(n * L);
            fill(s.x, 2 * c.q, 41 + t);
            return s;
        };
        emit("rns24_per_limb_calls", c, threads, run(threads, seconds, setup_poly, [&](Bufs& s) {
                 for (size_t i = 0; i < L; ++i) limbs[i].ComputeForward(s.x.data() + i * n, s.x.data() + i * n, 4, 4);
             }));
        emit("rns24_one_call", c, threads, run(threads, seconds, setup_poly, [&](Bufs& s) {
                 ax::ComputeForwardRNS(limbs.data(), L, s.x.data(), s.x.data(), L, 4, 4);
             }));
#endif
    }
    return 0;
}
