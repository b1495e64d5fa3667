// Per-kernel wall-time samples of the REFERENCE native backend, over the
// scenario matrix of the reference's own benchmark
// (benchmark/src/axhel_benchmark.cpp:48-50 degrees x widths, kernel names
// :1047-1166), for the CPU side of the per-kernel comparison table.
//
// TEST/MEASUREMENT INFRASTRUCTURE: compiled by oracle/Makefile against the
// reference compiled from its sources (oracle/_ref/libaxhel_ref.so) and run
// only by bench.py's CPU-baseline leg (--kernel-table).  The reference's
// benchmark counts Arm PMU cycles, which this host cannot read; this program
// uses std::chrono::steady_clock instead and prints nanoseconds.
//
//   kernel_timer_ref <repetitions> <warmup> <batch> <degree>:<bits>:<q>:<root> ...
//
// One JSON line per (scenario, kernel): the modulus and factors of the
// scenario and `repetitions` raw samples, each the time of `batch`
// consecutive calls.  Inputs are uniform in each kernel's input range
// (a fixed xorshift stream per scenario); NTTs run in place, their tables
// built before timing, as the reference benchmark does (:1140-1166).
#include <axhel/axhel.hpp>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <string>
#include <vector>

namespace ax = unipi::axhel;
using Clock = std::chrono::steady_clock;

namespace {

struct Rng {
    uint64_t x;
    uint64_t next()
    {
        x ^= x >> 12;
        x ^= x << 25;
        x ^= x >> 27;
        return x * 0x2545F4914F6CDD1Dull;
    }
    // uniform below bound (bound 0 = any 64-bit value); rejection keeps it exact
    uint64_t below(uint64_t bound)
    {
        if (bound == 0) return next();
        const uint64_t lim = UINT64_MAX - UINT64_MAX % bound;
        uint64_t v;
        do v = next();
        while (v >= lim);
        return v % bound;
    }
};

std::vector<uint64_t> vec(Rng& r, size_t n, uint64_t bound)
{
    std::vector<uint64_t> v(n);
    for (auto& w : v) w = r.below(bound);
    return v;
}

void timed(const char* name, uint64_t degree, unsigned bits, uint64_t q, uint64_t mod_f, uint64_t in_f,
           uint64_t out_f, int reps, int warm, int batch, const std::function<void()>& call)
{
    for (int i = 0; i < warm; ++i) call();
    std::printf("{\"kernel\": \"%s\", \"poly_degree\": %llu, \"qi_bits\": %u, \"modulus\": %llu, \"mod_factor\": %llu, "
                "\"input_mod_factor\": %llu, \"output_mod_factor\": %llu, \"batch\": %d, \"raw_ns\": [",
                name, (unsigned long long)degree, bits, (unsigned long long)q, (unsigned long long)mod_f,
                (unsigned long long)in_f, (unsigned long long)out_f, batch);
    for (int r = 0; r < reps; ++r) {
        const auto a = Clock::now();
        for (int b = 0; b < batch; ++b) call();
        const auto e = Clock::now();
        std::printf("%s%.1f", r ? ", " : "", std::chrono::duration<double, std::nano>(e - a).count());
    }
    std::printf("]}\n");
    std::fflush(stdout);
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s <reps> <warmup> <batch> <degree>:<bits>:<q>:<root> ...\n", argv[0]);
        return 2;
    }
    const int reps = std::atoi(argv[1]), warm = std::atoi(argv[2]), batch = std::atoi(argv[3]);
    if (reps < 1 || warm < 0 || batch < 1) return 2;
    for (int a = 4; a < argc; ++a) {
        unsigned long long degree = 0, q = 0, root = 0;
        unsigned bits = 0;
        if (std::sscanf(argv[a], "%llu:%u:%llu:%llu", &degree, &bits, &q, &root) != 4) return 2;
        const uint64_t n = degree;
        Rng rng{degree * 1000003ull + bits + 0x415848454Cull};
        std::vector<uint64_t> res(n);
        auto a1 = vec(rng, n, q), b1 = vec(rng, n, q);
        const uint64_t sc = rng.below(q);
        uint64_t* r = res.data();
        auto T = [&](const char* name, uint64_t mf, uint64_t fi, uint64_t fo, const std::function<void()>& f) {
            timed(name, n, bits, q, mf, fi, fo, reps, warm, batch, f);
        };
        T("add_vv", 0, 0, 0, [&] { ax::EltwiseAddMod(r, a1.data(), b1.data(), n, q); });
        T("sub_vv", 0, 0, 0, [&] { ax::EltwiseSubMod(r, a1.data(), b1.data(), n, q); });
        T("add_vs", 0, 0, 0, [&] { ax::EltwiseAddMod(r, a1.data(), sc, n, q); });
        T("sub_vs", 0, 0, 0, [&] { ax::EltwiseSubMod(r, a1.data(), sc, n, q); });
        for (uint64_t f : {1ull, 2ull, 4ull}) {
            auto x = vec(rng, n, f * q), y = vec(rng, n, f * q);
            const std::string name = "mul_f" + std::to_string(f);
            T(name.c_str(), f, 0, 0, [&] { ax::EltwiseMulMod(r, x.data(), y.data(), n, q, f); });
        }
        for (uint64_t f : {1ull, 2ull, 4ull, 8ull}) {
            auto x = vec(rng, n, f * q), c = vec(rng, n, f * q);
            const uint64_t s = rng.below(f * q);
            const std::string name = "fma_f" + std::to_string(f);
            T(name.c_str(), f, 0, 0, [&] { ax::EltwiseFMAMod(r, x.data(), s, c.data(), n, q, f); });
        }
        struct Red {
            const char* name;
            uint64_t fi, fo;
            bool arbitrary;
        };
        for (const Red& d : {Red{"reduce_2to1", 2, 1, false}, Red{"reduce_4to1", 4, 1, false},
                             Red{"reduce_4to2", 4, 2, false}, Red{"reduce_barrett", 0, 1, true}}) {
            auto x = vec(rng, n, d.arbitrary ? 0 : d.fi * q);
            const uint64_t fi = d.arbitrary ? q : d.fi;
            T(d.name, 0, fi, d.fo, [&] { ax::EltwiseReduceMod(r, x.data(), n, q, fi, d.fo); });
        }
        const ax::NTT ntt(n, q, root);  // tables outside the timed region
        auto w = vec(rng, n, q);
        uint64_t* pw = w.data();
        T("ntt_forward", 0, 1, 1, [&] { ntt.ComputeForward(pw, pw, 1, 1); });
        T("ntt_forward_lazy", 0, 1, 4, [&] { ntt.ComputeForward(pw, pw, 1, 4); });
        ntt.ComputeForward(pw, pw, 1, 1);  // inverse inputs in [0, q)
        T("ntt_inverse", 0, 1, 1, [&] { ntt.ComputeInverse(pw, pw, 1, 1); });
        T("ntt_inverse_lazy", 0, 1, 2, [&] { ntt.ComputeInverse(pw, pw, 1, 2); });
    }
    return 0;
}
