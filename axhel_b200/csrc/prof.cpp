// Launch accounting, the optional per-kernel event timer and NVTX ranges.
//
// When enabled (axhel_cuda_profile_enable), every kernel launch of this
// library is bracketed by two CUDA events recorded on the launching stream;
// axhel_cuda_profile_report aggregates launches and device time per kernel
// configuration.  Off by default: then a launch costs one relaxed atomic add.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/axhel_cuda.h"
#include "launch.h"

namespace axhel_impl {

namespace {
std::atomic<uint64_t> g_launches{0};
std::atomic<bool> g_prof{false};
std::mutex g_prof_mu;
struct Rec {
    std::string name;
    cudaEvent_t a, b;
};
std::vector<Rec> g_recs;
thread_local Rec t_open;
thread_local bool t_has_open = false;
}  // namespace

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

bool nvtx_enabled()
{
    static const bool on = [] {
        const char* e = std::getenv("AXHEL_NVTX");
        return e && *e && std::strcmp(e, "0") != 0;
    }();
    return on;
}

ProfScope::ProfScope(cudaStream_t s, const char* fmt, ...)
    : s_(s), on_(g_prof.load(std::memory_order_relaxed)), nvtx_(nvtx_enabled())
{
    if (!on_ && !nvtx_) return;
    char name[128];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(name, sizeof name, fmt, ap);
    va_end(ap);
    if (nvtx_) nvtxRangePushA(name);
    if (!on_) return;
    t_open.name = name;
    cudaEventCreate(&t_open.a);
    cudaEventCreate(&t_open.b);
    cudaEventRecord(t_open.a, s_);
    t_has_open = true;
}

ProfScope::~ProfScope()
{
    if (nvtx_) nvtxRangePop();
    if (!on_ || !t_has_open) return;
    cudaEventRecord(t_open.b, s_);
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_recs.push_back(t_open);
    t_has_open = false;
}

}  // namespace axhel_impl

using namespace axhel_impl;

extern "C" {

uint64_t axhel_cuda_launch_count(void) { return g_launches.load(); }

axhel_status_t axhel_cuda_profile_enable(int on)
{
    g_prof.store(on != 0);
    return AXHEL_OK;
}

axhel_status_t axhel_cuda_profile_report(char* buf, uint64_t len, uint64_t* needed)
{
    std::vector<Rec> recs;
    {
        std::lock_guard<std::mutex> lk(g_prof_mu);
        recs.swap(g_recs);
    }
    struct Agg {
        uint64_t n = 0;
        double ms = 0;
    };
    std::map<std::string, Agg> agg;
    for (auto& r : recs) {
        cudaEventSynchronize(r.b);
        float ms = 0;
        if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
            auto& g = agg[r.name];
            g.n += 1;
            g.ms += ms;
        }
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    std::string out;
    char line[256];
    for (auto& kv : agg) {
        std::snprintf(line, sizeof line, "%s %llu %.6f\n", kv.first.c_str(), (unsigned long long)kv.second.n,
                      kv.second.ms);
        out += line;
    }
    if (needed) *needed = out.size() + 1;
    if (buf && len) {
        const size_t m = out.size() < len - 1 ? out.size() : len - 1;
        out.copy(buf, m);
        buf[m] = 0;
    }
    return AXHEL_OK;
}

}  // extern "C"
