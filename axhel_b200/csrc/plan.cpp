// Pass planner: how an N = 2^logn transform is split into passes, and with
// which register depth and tile width each pass runs.
//
// Priority: an explicit override (axhel_cuda_plan_set) > the autotuner table
// (loaded from ntt_plans.txt beside the library, or axhel_cuda_plan_load) >
// the built-in default.  Table lines:
//   <inverse 0|1> <logn> <limb-bucket> <npass> (<lg> <lr> <tg>){npass}
// where limb-bucket = floor(log2(limbs)) clamped to [0, 15].  A lookup takes
// the nearest bucket at or below the requested one, else the nearest above.
// Lines `B <logn> <row stages>` give the uneven-batch engine's split of an
// N = 2^logn job into its strided and contiguous passes.
#include <dlfcn.h>

#include <cstdio>
#include <cstring>
#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "internal.h"
#include "launch.h"

namespace axhel_impl {

namespace {

std::mutex g_mu;
std::map<std::pair<int, uint32_t>, NttPlan> g_override;
std::atomic<size_t> g_override_count{0};  // g_override.size(), read without the lock
std::map<std::tuple<int, uint32_t, int>, NttPlan> g_table;
std::map<uint32_t, int> g_batch_override, g_batch_table;  // logn -> contiguous-pass stages
bool g_table_tried = false;

int bucket_of(uint64_t limbs)
{
    int b = 0;
    while (b < 15 && (2ull << b) <= limbs) ++b;
    return b;
}

// Built-in heuristic.  One pass up to 2^13 (the whole transform in shared
// memory), otherwise two passes of ceil/floor(logn/2) stages.  The forward
// runs the strided column pass first, the inverse last, with identical
// configurations, so a fused INTT -> op -> NTT chain can merge them.
NttPlan default_plan(bool inverse, uint32_t logn, uint64_t limbs)
{
    NttPlan p{};
    const uint64_t want_ctas = 2ull * (uint64_t)sm_count();
    if (logn <= 13) {
        p.npass = 1;
        p.pass[0] = PassCfg{(int)logn, logn <= 3 ? (int)logn : 4, 1};
        return p;
    }
    const int A = (int)(logn + 1) / 2;  // strided column pass
    const int B = (int)logn - A;        // contiguous row pass
    PassCfg col{A, 4, 16};
    PassCfg row{B, 4, 1};
    const int row_tg_log = 8 - (B - 4);  // 256 threads
    row.tg = row_tg_log > 0 ? (1 << row_tg_log) : 1;
    if ((uint64_t)row.tg > (1ull << A)) row.tg = 1 << A;
    // Narrow the tiles when a small batch would leave SMs idle.
    auto ctas = [&](const PassCfg& c) { return limbs * ((1ull << (logn - c.lg)) / (uint64_t)c.tg); };
    while (col.tg > 4 && ctas(col) < want_ctas) col.tg >>= 1;
    while (row.tg > 1 && ctas(row) < want_ctas) row.tg >>= 1;
    p.npass = 2;
    if (inverse) {
        p.pass[0] = row;
        p.pass[1] = col;
    } else {
        p.pass[0] = col;
        p.pass[1] = row;
    }
    return p;
}

std::string lib_dir()
{
    Dl_info info;
    if (dladdr(reinterpret_cast<void*>(&default_plan), &info) && info.dli_fname) {
        std::string f(info.dli_fname);
        auto pos = f.find_last_of('/');
        if (pos != std::string::npos) return f.substr(0, pos);
    }
    return ".";
}

int load_table_locked(const char* path)
{
    std::FILE* fp = std::fopen(path, "r");
    if (!fp) return -1;
    char line[512];
    int n = 0;
    while (std::fgets(line, sizeof line, fp)) {
        if (line[0] == '#' || line[0] == '\n') continue;
        if (line[0] == 'K') {  // cluster form: kind logn lga lr csize max_limbs
            int kind, logn, lga, lr, cs;
            unsigned long long mx;
            if (std::sscanf(line + 1, "%d %d %d %d %d %llu", &kind, &logn, &lga, &lr, &cs, &mx) == 6 && kind >= 0 &&
                kind <= 3 && logn >= 10 && logn <= 17) {
                const ClusterCfg c{lga, lr, cs, (uint64_t)mx};
                if (mx == 0 || cluster_cfg_valid(kind, (uint32_t)logn, c)) {
                    cluster_plan_table_set(kind, (uint32_t)logn, c);
                    ++n;
                }
            }
            continue;
        }
        if (line[0] == 'B') {
            int logn, row;
            if (std::sscanf(line + 1, "%d %d", &logn, &row) == 2 && logn > 0 &&
                batch_row_valid((uint32_t)logn, row)) {
                g_batch_table[(uint32_t)logn] = row;
                ++n;
            }
            continue;
        }
        int inv, logn, bucket, npass, v[9] = {0};
        int got = std::sscanf(line, "%d %d %d %d %d %d %d %d %d %d %d %d %d", &inv, &logn, &bucket, &npass, &v[0],
                              &v[1], &v[2], &v[3], &v[4], &v[5], &v[6], &v[7], &v[8]);
        if (got < 4 || npass < 1 || npass > 3 || got < 4 + 3 * npass) continue;
        NttPlan p{};
        p.npass = npass;
        for (int i = 0; i < npass; ++i) p.pass[i] = PassCfg{v[3 * i], v[3 * i + 1], v[3 * i + 2]};
        if (!plan_valid(p, (uint32_t)logn, inv != 0)) continue;
        g_table[std::make_tuple(inv ? 1 : 0, (uint32_t)logn, bucket)] = p;
        ++n;
    }
    std::fclose(fp);
    return n;
}

void ensure_table_locked()
{
    if (g_table_tried) return;
    g_table_tried = true;
    const std::string path = lib_dir() + "/ntt_plans.txt";
    load_table_locked(path.c_str());
}

}  // namespace

bool plan_valid(const NttPlan& p, uint32_t logn, bool inverse)
{
    if (p.npass < 1 || p.npass > 3) return false;
    uint32_t sum = 0;
    for (int i = 0; i < p.npass; ++i) {
        const PassCfg& c = p.pass[i];
        if (!pass_supported(c)) return false;
        if (c.lr > c.lg || c.tg < 1 || (c.tg & (c.tg - 1))) return false;
        if (((uint64_t)c.tg << (c.lg - c.lr)) > (uint64_t)(c.lr >= 5 ? 256 : 512)) return false;
        sum += (uint32_t)c.lg;
    }
    if (sum != logn) return false;
    // A tile never straddles two blocks: tg <= groups per limb and, for a
    // strided pass, tg <= stride.
    uint32_t s0 = 0;
    for (int i = 0; i < p.npass; ++i) {
        const PassCfg& c = p.pass[i];
        if ((uint64_t)c.tg > (1ull << (logn - c.lg))) return false;
        const uint32_t lgS = inverse ? s0 : logn - s0 - (uint32_t)c.lg;
        if (lgS > 0 && (uint64_t)c.tg > (1ull << lgS)) return false;
        if ((size_t)c.tg * ((size_t(1) << c.lg) + 1) * 8 > 227 * 1024) return false;
        s0 += (uint32_t)c.lg;
    }
    return true;
}

NttPlan plan_for(bool inverse, uint32_t logn, uint64_t limbs)
{
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_override.find({inverse ? 1 : 0, logn});
    if (it != g_override.end()) return it->second;
    ensure_table_locked();
    const int b = bucket_of(limbs);
    for (int d = 0; d <= 15; ++d) {
        for (int cand : {b - d, b + d}) {
            if (cand < 0 || cand > 15) continue;
            auto t = g_table.find(std::make_tuple(inverse ? 1 : 0, logn, cand));
            if (t != g_table.end()) return t->second;
        }
    }
    return default_plan(inverse, logn, limbs);
}

bool plan_overridden(bool inverse, uint32_t logn)
{
    if (g_override_count.load(std::memory_order_acquire) == 0) return false;  // the usual case, no lock
    std::lock_guard<std::mutex> lk(g_mu);
    return g_override.count({inverse ? 1 : 0, logn}) != 0;
}

void plan_override(bool inverse, uint32_t logn, const NttPlan* p)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (p)
        g_override[{inverse ? 1 : 0, logn}] = *p;
    else
        g_override.erase({inverse ? 1 : 0, logn});
    g_override_count.store(g_override.size(), std::memory_order_release);
}

bool batch_row_valid(uint32_t logn, int row)
{
    const int lo = (int)logn - 9 > 5 ? (int)logn - 9 : 5;
    const int hi = (int)logn - 5 < 9 ? (int)logn - 5 : 9;
    return logn >= 10 && logn <= 17 && row >= lo && row <= hi;
}

int batch_row_stages(uint32_t logn)
{
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_batch_override.find(logn);
    if (it != g_batch_override.end()) return it->second;
    ensure_table_locked();
    auto t = g_batch_table.find(logn);
    if (t != g_batch_table.end()) return t->second;
    return (int)logn - 5 < 9 ? (int)logn - 5 : 9;  // the contiguous pass as wide as a tile allows
}

void batch_row_override(uint32_t logn, int row)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (row)
        g_batch_override[logn] = row;
    else
        g_batch_override.erase(logn);
}

void plan_table_ensure()
{
    static std::once_flag once;
    std::call_once(once, [] {
        std::lock_guard<std::mutex> lk(g_mu);
        ensure_table_locked();
    });
}

int plan_load(const char* path)
{
    std::lock_guard<std::mutex> lk(g_mu);
    ensure_table_locked();  // the shipped table first; `path` entries override it
    if (!path) {
        const std::string def = lib_dir() + "/ntt_plans.txt";
        return load_table_locked(def.c_str());
    }
    return load_table_locked(path);
}

}  // namespace axhel_impl
