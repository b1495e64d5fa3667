// Serving loop: continuous batching of transform jobs on one GPU.
//
// Requests (any job kind of the batch engine: forward, inverse, or the fused
// INTT -> MulMod/FMAMod -> NTT chain, each of any degree 2^10..2^17 and limb
// count) are submitted from any host thread and return at once with an id.
// (Batches run as one launch per phase by default, so batches on different
// streams share the SMs tile by tile; AXHEL_SERVER_PERSISTENT selects the
// single persistent launch instead.  max_batch_words caps a batch's size so
// that one large request does not hold small ones back.)
// A scheduler thread admits pending requests in arrival order while their
// device bytes fit the HBM budget, stages host operands into stream-ordered
// pool allocations, and launches every admitted request as ONE persistent
// batch kernel on one of `max_inflight` streams; requests that arrive while
// batches are running are admitted into the next batch as soon as a stream
// and budget free up, so their work overlaps on the device with the batches
// already there.  A completion thread retires batches in order (CUDA event),
// releases their memory from the budget and wakes the waiters.  Twiddle
// tables stay resident in the table cache; the batch descriptors of each
// stream live in a reusable device buffer.
//
// A request's result is computed by the same kernel code whether it runs
// alone or in a mix, so it is bit-identical either way.
#include <cuda_runtime.h>
#include <sys/prctl.h>

#include <algorithm>
#include <cmath>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/axhel_cuda.h"
#include "batch.h"
#include "internal.h"

using Clock = std::chrono::steady_clock;

namespace {

thread_local std::string t_serve_error;

axhel_status_t sfail(axhel_status_t st, const std::string& m)
{
    t_serve_error = m;
    return st;
}

constexpr int kPending = -1, kRunning = -2;

// The server's threads sleep in short waits (the completer's poll); Linux
// stretches every such sleep by the thread's timer slack, 50 us by default,
// which would land in each request's latency.
void tighten_timer_slack() { prctl(PR_SET_TIMERSLACK, 1000UL, 0, 0, 0); }
constexpr size_t kStagingBytes = 1 << 20;  // descriptor buffers per slot at creation (pinned host, device)

bool is_device(const void* p) { return p && axhel_cuda_is_device_pointer(p); }

struct Req {
    uint64_t id = 0;
    axhel_request_t r{};
    std::vector<axhel_ntt_t> ntts;
    std::vector<uint64_t> scalars;
    uint64_t words = 0;  // count * N
    bool in_dev = false, out_dev = false, vec_dev = false;
    size_t need = 0;     // device bytes charged to the budget
    uint64_t* d_in = nullptr;
    uint64_t* d_out = nullptr;
    uint64_t* d_vec = nullptr;
    Clock::time_point t_submit, t_start, t_done;
    int status = kPending;
    uint64_t batch = 0;
    uint32_t batch_size = 0;
};

struct Slot {
    int lane = 0;  // 0: small requests (high-priority stream), 1: the rest
    cudaStream_t stream = nullptr;
    axhel_impl::LaunchLanes lanes;  // a phase's launches side by side (same priority)
    int* err_host = nullptr;        // pinned word the kernel's error status is copied into
    unsigned char* host_img = nullptr;  // pinned staging of the batch descriptors
    size_t host_cap = 0;
    unsigned char* dev_img = nullptr;   // the slot's device descriptor buffer (kStagingBytes, at creation)
    std::vector<unsigned char*> retired;  // outgrown staging, freed with the server
    bool busy = false;
};

// A batch on the GPU: its requests in the order their results land, each
// with the event recorded after its result copy.
struct Inflight {
    std::vector<Req*> reqs;
    std::vector<cudaEvent_t> done;
    int slot = 0;
    uint64_t id = 0;
};

}  // namespace

struct axhel_server {
    axhel_server_config_t cfg{};
    int device = 0;
    cudaMemPool_t pool = nullptr;
    std::mutex mu;
    std::condition_variable cv_sched, cv_done, cv_wait;
    std::deque<Req*> pending[2];  // per lane, arrival order
    std::unordered_map<uint64_t, std::unique_ptr<Req>> reqs;
    std::deque<Inflight> inflight;
    std::vector<Slot> slots;
    size_t in_use = 0, peak_in_use = 0;
    uint64_t next_id = 1, batches = 0, completed = 0, max_batch = 0;
    int lanes = 1;
    bool stop = false, paused = false;
    std::vector<double> lat_ms;  // submit -> done of every completed request
    std::thread sched, comp;
    std::string fatal;
    std::vector<cudaEvent_t> event_pool;  // reused completion events
    std::atomic<int> debug_fail_at{-1};   // failure injection: staging of the next batch fails at this request
    double host_us_total = 0;             // scheduler time spent in launch(), all batches

    cudaEvent_t get_event()
    {
        std::lock_guard<std::mutex> lk(mu);
        if (!event_pool.empty()) {
            cudaEvent_t e = event_pool.back();
            event_pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        return e;
    }

    void scheduler();
    void completer();
    axhel_status_t launch(Slot& s, int slot_index, std::vector<Req*>& take, Inflight& f);
};

// Gives back to the pool, in stream order on `st`, every buffer staged for
// take[0 .. n): after a failure part-way through a batch, nothing it staged
// stays allocated while the scheduler returns its bytes to the budget.
static void unstage(cudaStream_t st, const std::vector<Req*>& take, size_t n)
{
    for (size_t i = 0; i < n && i < take.size(); ++i) {
        Req* q = take[i];
        if (!q->in_dev && q->d_in) cudaFreeAsync(q->d_in, st);
        if (!q->out_dev && q->d_out && q->d_out != q->d_in) cudaFreeAsync(q->d_out, st);
        if (!q->vec_dev && q->d_vec) cudaFreeAsync(q->d_vec, st);
        q->d_in = q->d_out = q->d_vec = nullptr;
    }
}

axhel_status_t axhel_server::launch(Slot& s, int slot_index, std::vector<Req*>& take, Inflight& f)
{
    cudaStream_t st = s.stream;
    std::vector<axhel_job_t> jobs(take.size());
    const int fail_at = debug_fail_at.exchange(-1);  // failure injection (tests): one batch
    for (size_t i = 0; i < take.size(); ++i) {
        Req* q = take[i];
        const size_t bytes = q->words * 8;
        // device operands are used in place; host ones get pool buffers
        q->d_in = q->in_dev ? const_cast<uint64_t*>(q->r.input) : nullptr;
        q->d_out = q->out_dev ? q->r.output : nullptr;
        q->d_vec = (q->r.vector && q->vec_dev) ? const_cast<uint64_t*>(q->r.vector) : nullptr;
        cudaError_t e = cudaSuccess;
        if (!q->in_dev) {
            e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&q->d_in), bytes, pool, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(q->d_in, q->r.input, bytes, cudaMemcpyHostToDevice, st);
            else q->d_in = nullptr;
        }
        if (e == cudaSuccess && !q->out_dev) {
            if (q->in_dev || q->r.output != q->r.input) {
                e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&q->d_out), bytes, pool, st);
                if (e != cudaSuccess) q->d_out = nullptr;
            } else {
                q->d_out = q->d_in;  // in place on the staged copy
            }
        }
        if (e == cudaSuccess && (int)i == fail_at) e = cudaErrorMemoryAllocation;
        if (e == cudaSuccess && q->r.vector && !q->vec_dev) {
            e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&q->d_vec), bytes, pool, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(q->d_vec, q->r.vector, bytes, cudaMemcpyHostToDevice, st);
            else q->d_vec = nullptr;
        }
        if (e != cudaSuccess) {
            unstage(st, take, i + 1);
            return sfail(AXHEL_ERR_NOMEM, std::string("request staging: ") + cudaGetErrorString(e));
        }
        axhel_job_t& j = jobs[i];
        j.kind = q->r.kind;
        j.n_ntts = (uint32_t)q->ntts.size();
        j.ntts = q->ntts.data();
        j.count = q->r.count;
        j.result = q->d_out;
        j.operand = q->d_in;
        j.vector = q->d_vec;
        j.scalars = q->scalars.empty() ? nullptr : q->scalars.data();
        j.input_mod_factor = q->r.input_mod_factor;
        j.output_mod_factor = q->r.output_mod_factor;
    }
    // batch descriptors into this stream's reusable buffer
    std::vector<unsigned char> img;
    size_t zo = 0, zb = 0;
    axhel_impl::BatchArgs args{};
    std::string err;
    const bool per_phase = !(cfg.flags & AXHEL_SERVER_PERSISTENT);
    std::vector<axhel_impl::ClassLaunch> classes;
    // The descriptors go to the slot's own device buffer, laid out for its
    // address in one pass; the slot's previous batch has completed, and the
    // copy is stream-ordered after it anyway.  A batch too large for it gets a
    // buffer from the stream-ordered pool, returned after the batch: no
    // cudaMalloc / cudaFree (which wait for the whole device) while other
    // batches run.
    void* desc = s.dev_img;
    bool own_desc = false;
    axhel_status_t rc = axhel_impl::batch_build(jobs.data(), jobs.size(), s.dev_img, img, &zo, &zb, &args, nullptr,
                                                &err, per_phase ? &classes : nullptr);
    if (rc == AXHEL_OK && img.size() > kStagingBytes) {
        if (cudaMallocFromPoolAsync(&desc, img.size(), pool, st) != cudaSuccess) {
            unstage(st, take, take.size());
            return sfail(AXHEL_ERR_NOMEM, "batch descriptor buffer");
        }
        own_desc = true;
        rc = axhel_impl::batch_build(jobs.data(), jobs.size(), static_cast<unsigned char*>(desc), img, &zo, &zb,
                                     &args, nullptr, &err, per_phase ? &classes : nullptr);
    }
    if (rc) {
        if (own_desc) cudaFreeAsync(desc, st);
        unstage(st, take, take.size());
        return sfail(rc, err);
    }
    if (img.size() > s.host_cap) {
        // The outgrown buffer is kept until the server is destroyed:
        // cudaFreeHost would wait for every stream of the device.
        unsigned char* grown = nullptr;
        const size_t cap = std::max<size_t>(img.size() * 2, s.host_cap * 2);
        if (cudaMallocHost(reinterpret_cast<void**>(&grown), cap) != cudaSuccess) {
            if (own_desc) cudaFreeAsync(desc, st);
            unstage(st, take, take.size());
            return sfail(AXHEL_ERR_NOMEM, "pinned descriptor staging");
        }
        if (s.host_img) s.retired.push_back(s.host_img);
        s.host_img = grown;
        s.host_cap = cap;
    }
    // the slot's previous batch has completed, so its staging copy is done
    std::memcpy(s.host_img, img.data(), img.size());
    cudaError_t e = cudaMemcpyAsync(desc, s.host_img, img.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = per_phase ? axhel_impl::batch_launch_classes(classes, st, &s.lanes) : axhel_impl::batch_launch_args(args, st);
    // only the persistent kernel's dependency waits can set the error word
    if (e == cudaSuccess && !per_phase)
        e = cudaMemcpyAsync(s.err_host, args.error, sizeof(int), cudaMemcpyDeviceToHost, st);
    else if (per_phase)
        *s.err_host = AXHEL_OK;
    // results back smallest first; each request completes at its own event
    std::vector<Req*> order(take);
    std::stable_sort(order.begin(), order.end(), [](const Req* a, const Req* b) { return a->words < b->words; });
    for (Req* q : order) {
        if (e == cudaSuccess && !q->out_dev)
            e = cudaMemcpyAsync(q->r.output, q->d_out, q->words * 8, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) {
            cudaEvent_t ev = get_event();
            if (!ev) e = cudaErrorMemoryAllocation;
            if (e == cudaSuccess) e = cudaEventRecord(ev, st);
            if (ev) f.done.push_back(ev);
        }
    }
    unstage(st, take, take.size());  // in stream order, after the copies back
    if (own_desc) cudaFreeAsync(desc, st);  // after the error word's copy, in stream order
    if (e != cudaSuccess) return sfail(AXHEL_ERR_CUDA, std::string("batch launch: ") + cudaGetErrorString(e));
    f.reqs = order;
    f.slot = slot_index;
    return AXHEL_OK;
}

void axhel_server::scheduler()
{
    cudaSetDevice(device);
    tighten_timer_slack();
    std::unique_lock<std::mutex> lk(mu);
    const bool by_arrival = cfg.flags & AXHEL_SERVER_ARRIVAL_PRIORITY;
    const bool smallest_first = cfg.flags & AXHEL_SERVER_SMALLEST_FIRST;
    auto free_slot = [&](int lane) {
        if (by_arrival) {
            // A lane's slots are in decreasing stream priority: the new batch
            // takes the first free slot below the youngest batch in flight,
            // so every batch in flight outranks the ones launched after it
            // (the highest free one when the lane is idle; the lowest free
            // one when none is left below).
            int youngest = -1, first = -1, last = -1;
            for (size_t i = 0; i < slots.size(); ++i) {
                if (slots[i].lane != lane) continue;
                if (slots[i].busy) {
                    youngest = (int)i;
                } else {
                    if (first < 0) first = (int)i;
                    last = (int)i;
                }
            }
            if (youngest < 0) return first;
            for (size_t i = (size_t)youngest + 1; i < slots.size(); ++i)
                if (slots[i].lane == lane && !slots[i].busy) return (int)i;
            return last;
        }
        for (size_t i = 0; i < slots.size(); ++i)
            if (slots[i].lane == lane && !slots[i].busy) return (int)i;
        return -1;
    };
    auto runnable = [&](int lane) { return !pending[lane].empty() && free_slot(lane) >= 0; };
    // Admission order of a lane's queue: arrival order, or (smallest first)
    // requests pending longer than the aging bound in arrival order, then
    // the rest by size.
    const auto aging = std::chrono::microseconds(cfg.aging_us);
    auto order_queue = [&](std::deque<Req*>& queue) {
        if (!smallest_first || queue.size() < 2) return;
        const auto now = Clock::now();
        std::stable_sort(queue.begin(), queue.end(), [&](const Req* a, const Req* b) {
            const bool ao = now - a->t_submit >= aging, bo = now - b->t_submit >= aging;
            if (ao != bo) return ao;
            if (ao) return a->id < b->id;
            return a->words < b->words;
        });
    };
    for (;;) {
        cv_sched.wait(lk, [&] { return stop || (!paused && (runnable(0) || runnable(1))); });
        if (stop) break;
        // the high-priority lane first, then the other
        const int first = (cfg.flags & AXHEL_SERVER_LARGE_FIRST) ? 1 : 0;
        const int lane = runnable(first) ? first : 1 - first;
        std::deque<Req*>& queue = pending[lane];
        order_queue(queue);
        // admit in queue order while the budget allows
        std::vector<Req*> take;
        size_t bytes = 0;
        uint64_t words = 0;
        while (!queue.empty() && take.size() < cfg.max_batch_requests) {
            Req* q = queue.front();
            if (q->status != kPending) {  // cancelled
                queue.pop_front();
                continue;
            }
            if (in_use + bytes + q->need > cfg.hbm_budget_bytes) break;
            if (cfg.max_batch_words && !take.empty() && words + q->words > cfg.max_batch_words) break;
            if (cfg.batch_size_ratio && !take.empty()) {
                const uint64_t a = take.front()->words, b = q->words;
                if (std::max(a, b) > (uint64_t)cfg.batch_size_ratio * std::min(a, b)) break;
            }
            bytes += q->need;
            words += q->words;
            queue.pop_front();
            take.push_back(q);
        }
        if (take.empty()) {
            // The head does not fit next to the batches in flight: wait until
            // one of them releases its memory (every request fits an empty
            // budget: larger ones are refused at submit), or it is cancelled.
            const size_t held = in_use;
            cv_sched.wait(lk, [&] {
                return stop || paused || in_use < held || queue.empty() || queue.front()->status != kPending;
            });
            continue;
        }
        const int si = free_slot(lane);
        slots[si].busy = true;
        in_use += bytes;
        peak_in_use = std::max(peak_in_use, in_use);
        const uint64_t bid = ++batches;
        const auto now = Clock::now();
        for (Req* q : take) {
            q->status = kRunning;
            q->t_start = now;
            q->batch = bid;
            q->batch_size = (uint32_t)take.size();
        }
        max_batch = std::max<uint64_t>(max_batch, take.size());
        lk.unlock();
        Inflight f;
        f.id = bid;
        const auto h0 = Clock::now();
        const axhel_status_t rc = launch(slots[si], si, take, f);
        const double host_us = std::chrono::duration<double, std::micro>(Clock::now() - h0).count();
        lk.lock();
        host_us_total += host_us;
        if (rc) {
            for (Req* q : take) {
                q->status = rc;
                q->t_done = Clock::now();
            }
            cudaStreamSynchronize(slots[si].stream);
            for (cudaEvent_t ev : f.done) event_pool.push_back(ev);
            slots[si].busy = false;
            in_use -= bytes;
            cv_wait.notify_all();
            continue;
        }
        inflight.push_back(std::move(f));
        cv_done.notify_one();
    }
}

void axhel_server::completer()
{
    cudaSetDevice(device);
    tighten_timer_slack();
    std::vector<std::pair<Inflight*, cudaEvent_t>> heads;
    std::vector<cudaError_t> state;
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        cv_done.wait(lk, [&] { return !inflight.empty() || stop; });
        if (inflight.empty()) {
            if (stop) break;
            continue;
        }
        // Poll the oldest pending result of every batch in flight (batches of
        // the two lanes finish out of launch order, and a request completes
        // as soon as its own result has landed), querying the events without
        // the lock so that the scheduler keeps admitting meanwhile.  Only this
        // thread removes batches, and appending to the deque keeps references
        // to its elements valid.
        heads.clear();
        for (Inflight& f : inflight) heads.emplace_back(&f, f.done.empty() ? nullptr : f.done.front());
        lk.unlock();
        state.assign(heads.size(), cudaErrorNotReady);
        for (size_t i = 0; i < heads.size(); ++i)
            if (heads[i].second) state[i] = cudaEventQuery(heads[i].second);
        lk.lock();
        bool progress = false, emptied = false;
        for (size_t i = 0; i < heads.size(); ++i) {
            cudaError_t e = state[i];
            if (e == cudaErrorNotReady) continue;
            Inflight& f = *heads[i].first;
            Slot& sl = slots[f.slot];
            while (!f.reqs.empty()) {
                cudaEvent_t ev = f.done.front();
                Req* q = f.reqs.front();
                q->status = (e == cudaSuccess) ? *sl.err_host : AXHEL_ERR_CUDA;
                q->t_done = Clock::now();
                lat_ms.push_back(std::chrono::duration<double, std::milli>(q->t_done - q->t_submit).count());
                for (axhel_ntt_t h : q->ntts) axhel_cuda_ntt_release(h);
                q->ntts.clear();
                ++completed;
                in_use -= q->need;
                event_pool.push_back(ev);
                f.done.erase(f.done.begin());
                f.reqs.erase(f.reqs.begin());
                progress = true;
                if (f.reqs.empty()) break;
                e = cudaEventQuery(f.done.front());  // the batch's next result, often landed too
                if (e == cudaErrorNotReady) break;
            }
            if (f.reqs.empty()) {
                for (cudaEvent_t ev : f.done) event_pool.push_back(ev);
                f.done.clear();
                sl.busy = false;
                emptied = true;
            }
        }
        if (emptied)
            for (auto it = inflight.begin(); it != inflight.end();) it = it->reqs.empty() ? inflight.erase(it) : it + 1;
        if (progress) {
            cv_wait.notify_all();
            cv_sched.notify_all();
        } else {
            cv_done.wait_for(lk, std::chrono::microseconds(10));
        }
    }
}

extern "C" {

axhel_status_t axhel_server_create(const axhel_server_config_t* cfg, axhel_server_t* out)
{
    if (!cfg || !out) return sfail(AXHEL_ERR_INVALID, "null argument");
    *out = nullptr;
    if (cfg->hbm_budget_bytes == 0 || cfg->max_inflight == 0 || cfg->max_inflight > 16 ||
        cfg->max_batch_requests == 0)
        return sfail(AXHEL_ERR_INVALID, "budget > 0, 1 <= max_inflight <= 16, max_batch_requests > 0");
    auto s = std::make_unique<axhel_server>();
    s->cfg = *cfg;
    cudaError_t e = cudaGetDevice(&s->device);
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = s->device;
    if (e == cudaSuccess) e = cudaMemPoolCreate(&s->pool, &props);
    if (e == cudaSuccess) {
        uint64_t keep = cfg->hbm_budget_bytes;  // keep freed blocks for reuse up to the budget
        e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    s->lanes = cfg->small_request_words ? 2 : 1;
    int prio_low = 0, prio_high = 0;
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
    s->slots.resize((size_t)cfg->max_inflight * s->lanes);
    for (size_t i = 0; i < s->slots.size(); ++i) {
        Slot& sl = s->slots[i];
        // with two lanes, lane 0 (small requests) gets the highest priority:
        // its CTAs are dispatched ahead of the large lane's as SMs free up
        sl.lane = s->lanes == 2 ? (int)(i / cfg->max_inflight) : 1;
        const bool large_first = cfg->flags & AXHEL_SERVER_LARGE_FIRST;
        int prio = (sl.lane == 0) != large_first ? prio_high : prio_low;
        if (cfg->flags & AXHEL_SERVER_ARRIVAL_PRIORITY) {
            // the lane's k-th slot at the k-th highest priority (the rest at
            // the lowest): the order in which the scheduler fills them
            const int k = (int)(i % cfg->max_inflight);
            prio = std::min(prio_high + k, prio_low);  // greater numbers are lower priorities
        }
        if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&sl.stream, cudaStreamNonBlocking, prio);
        if (e == cudaSuccess) e = axhel_impl::lanes_create(&sl.lanes, prio);
        if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&sl.err_host), sizeof(int));
        // descriptor staging for batches of up to a few hundred requests,
        // allocated now rather than on a slot's first batch
        if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&sl.host_img), kStagingBytes);
        if (e == cudaSuccess) sl.host_cap = kStagingBytes;
        if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&sl.dev_img), kStagingBytes);
    }
    if (e == cudaSuccess && cfg->reserve_bytes) {
        // map the pool's memory now: growing it later takes tens of
        // milliseconds, in the path of whichever request needs it
        void* r = nullptr;
        cudaStream_t st = s->slots[0].stream;
        e = cudaMallocFromPoolAsync(&r, std::min(cfg->reserve_bytes, cfg->hbm_budget_bytes), s->pool, st);
        if (e == cudaSuccess) e = cudaFreeAsync(r, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) {
        for (Slot& sl : s->slots) {
            if (sl.stream) cudaStreamDestroy(sl.stream);
            axhel_impl::lanes_destroy(&sl.lanes);
            if (sl.err_host) cudaFreeHost(sl.err_host);
            if (sl.host_img) cudaFreeHost(sl.host_img);
            if (sl.dev_img) cudaFree(sl.dev_img);
        }
        if (s->pool) cudaMemPoolDestroy(s->pool);
        return sfail(AXHEL_ERR_CUDA, std::string("server setup: ") + cudaGetErrorString(e));
    }
    axhel_server* p = s.get();
    p->sched = std::thread([p] { p->scheduler(); });
    p->comp = std::thread([p] { p->completer(); });
    *out = s.release();
    return AXHEL_OK;
}

axhel_status_t axhel_server_submit(axhel_server_t s, const axhel_request_t* r, uint64_t* id)
{
    if (!s || !r || !id) return sfail(AXHEL_ERR_INVALID, "null argument");
    if (!r->ntts || r->n_ntts == 0 || !r->input || !r->output || r->count == 0)
        return sfail(AXHEL_ERR_INVALID, "request needs handles, input, output and count > 0");
    {
        // the batch engine's contract, checked now so that a bad request
        // fails alone rather than the batch it would join
        const axhel_job_t j{r->kind,  r->n_ntts, r->ntts,    r->count,           r->output,
                            r->input, r->vector, r->scalars, r->input_mod_factor, r->output_mod_factor};
        std::string err;
        const axhel_status_t st = axhel_impl::batch_check_job(j, "request", &err);
        if (st) return sfail(st, err);
    }
    auto q = std::make_unique<Req>();
    q->r = *r;
    const uint64_t n = r->ntts[0] ? axhel_cuda_ntt_degree(r->ntts[0]) : 0;
    if (n < 1024) return sfail(AXHEL_ERR_UNSUPPORTED, "served degrees are 2^10 .. 2^17");
    for (uint32_t i = 0; i < r->n_ntts; ++i) {
        if (!r->ntts[i] || axhel_cuda_ntt_degree(r->ntts[i]) != n)
            return sfail(AXHEL_ERR_INVALID, "handles must share one degree");
        q->ntts.push_back(r->ntts[i]);
    }
    if (r->scalars) q->scalars.assign(r->scalars, r->scalars + r->n_ntts);
    q->words = r->count * n;
    q->in_dev = is_device(r->input);
    q->out_dev = is_device(r->output);
    q->vec_dev = is_device(r->vector);
    const size_t bytes = q->words * 8;
    q->need = (q->in_dev ? 0 : bytes) + (q->out_dev || (!q->in_dev && r->output == r->input) ? 0 : bytes) +
              (r->vector && !q->vec_dev ? bytes : 0);
    if (q->need > s->cfg.hbm_budget_bytes)
        return sfail(AXHEL_ERR_REJECTED, "request needs " + std::to_string(q->need) + " device bytes, over the budget");
    for (axhel_ntt_t h : q->ntts) axhel_cuda_ntt_retain(h);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) {
        for (axhel_ntt_t h : q->ntts) axhel_cuda_ntt_release(h);
        return sfail(AXHEL_ERR_INVALID, "server stopping");
    }
    q->id = s->next_id++;
    q->t_submit = Clock::now();
    *id = q->id;
    const int lane = (s->lanes == 2 && q->words <= s->cfg.small_request_words) ? 0 : 1;
    s->pending[lane].push_back(q.get());
    s->reqs.emplace(q->id, std::move(q));
    s->cv_sched.notify_one();
    return AXHEL_OK;
}

axhel_status_t axhel_server_wait(axhel_server_t s, uint64_t id, uint64_t timeout_us, axhel_request_info_t* info)
{
    if (!s) return sfail(AXHEL_ERR_INVALID, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return sfail(AXHEL_ERR_INVALID, "unknown request id");
    Req* q = it->second.get();
    const bool ok = s->cv_wait.wait_for(lk, std::chrono::microseconds(timeout_us),
                                        [&] { return q->status != kPending && q->status != kRunning; });
    if (!ok) return sfail(AXHEL_ERR_TIMEOUT, "request not finished");
    if (info) {
        info->status = q->status;
        info->queue_ms = std::chrono::duration<double, std::milli>(q->t_start - q->t_submit).count();
        info->latency_ms = std::chrono::duration<double, std::milli>(q->t_done - q->t_submit).count();
        info->batch_id = q->batch;
        info->batch_size = q->batch_size;
    }
    const int st = q->status;
    for (axhel_ntt_t h : q->ntts) axhel_cuda_ntt_release(h);  // cancelled / rejected requests still hold them
    s->reqs.erase(it);
    return st;
}

axhel_status_t axhel_server_cancel(axhel_server_t s, uint64_t id)
{
    if (!s) return sfail(AXHEL_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return sfail(AXHEL_ERR_INVALID, "unknown request id");
    Req* q = it->second.get();
    if (q->status != kPending) return sfail(AXHEL_ERR_BUSY, "request already running or finished");
    q->status = AXHEL_ERR_CANCELLED;
    q->t_start = q->t_done = Clock::now();
    s->cv_wait.notify_all();
    s->cv_sched.notify_all();
    return AXHEL_OK;
}

axhel_status_t axhel_server_pause(axhel_server_t s, int paused)
{
    if (!s) return sfail(AXHEL_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    s->paused = paused != 0;
    s->cv_sched.notify_all();
    return AXHEL_OK;
}

axhel_status_t axhel_server_stats(axhel_server_t s, axhel_server_stats_t* out, int reset_latencies)
{
    if (!s || !out) return sfail(AXHEL_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    std::vector<double> v = s->lat_ms;
    std::sort(v.begin(), v.end());
    auto pct = [&](double p) { return v.empty() ? 0.0 : v[std::min(v.size() - 1, (size_t)(p * (v.size() - 1) + 0.5))]; };
    out->completed = s->completed;
    out->batches = s->batches;
    out->max_batch_requests = s->max_batch;
    out->pending = s->pending[0].size() + s->pending[1].size();
    out->in_use_bytes = s->in_use;
    out->peak_in_use_bytes = s->peak_in_use;
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
    out->samples = v.size();
    uint64_t used = 0;  // a 64-bit attribute value
    out->pool_used_bytes =
        cudaMemPoolGetAttribute(s->pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess ? (uint64_t)used : 0;
    out->host_us_per_batch = s->batches ? s->host_us_total / (double)s->batches : 0.0;
    if (reset_latencies) s->lat_ms.clear();
    return AXHEL_OK;
}

axhel_status_t axhel_server_destroy(axhel_server_t s)
{
    if (!s) return AXHEL_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_sched.notify_all();
        s->cv_done.notify_all();
    }
    s->sched.join();
    s->comp.join();  // drains the batches still in flight
    for (Slot& sl : s->slots) {
        cudaStreamSynchronize(sl.stream);
        cudaStreamDestroy(sl.stream);
        axhel_impl::lanes_destroy(&sl.lanes);
        cudaFreeHost(sl.err_host);
        if (sl.host_img) cudaFreeHost(sl.host_img);
        if (sl.dev_img) cudaFree(sl.dev_img);
        for (unsigned char* r : sl.retired) cudaFreeHost(r);
    }
    for (cudaEvent_t ev : s->event_pool) cudaEventDestroy(ev);
    for (auto& kv : s->reqs)
        for (axhel_ntt_t h : kv.second->ntts) axhel_cuda_ntt_release(h);
    cudaMemPoolDestroy(s->pool);
    delete s;
    return AXHEL_OK;
}

const char* axhel_server_last_error(void) { return t_serve_error.c_str(); }

axhel_status_t axhel_server_debug_fail_staging(axhel_server_t s, uint32_t request)
{
    if (!s) return sfail(AXHEL_ERR_INVALID, "null server");
    s->debug_fail_at.store((int)std::min<uint32_t>(request, 1u << 30));
    return AXHEL_OK;
}

axhel_status_t axhel_server_drive(axhel_server_t server, const axhel_request_t* templates, uint32_t n_templates,
                                  uint64_t* const* outputs, uint32_t copies, const double* isolated_ms,
                                  double rate_per_s, double seconds, uint64_t seed, axhel_drive_result_t* out)
{
    if (!server || !templates || !n_templates || !outputs || !copies || !out || rate_per_s <= 0 || seconds <= 0)
        return sfail(AXHEL_ERR_INVALID, "bad drive arguments");
    std::memset(out, 0, sizeof *out);
    struct Live {
        uint64_t id;
        uint32_t t, c;
    };
    std::vector<std::vector<uint32_t>> free_copies(n_templates);
    for (uint32_t t = 0; t < n_templates; ++t)
        for (uint32_t c = 0; c < copies; ++c) free_copies[t].push_back(copies - 1 - c);
    std::mutex fm;
    std::deque<Live> live;
    std::condition_variable lv;
    bool done = false;
    std::vector<double> lat, slow, iso, queue, lat_large, lat_rest;
    // templates in the top quarter of isolated latency
    std::vector<char> large(n_templates, 0);
    if (isolated_ms) {
        std::vector<double> v(isolated_ms, isolated_ms + n_templates);
        std::sort(v.begin(), v.end());
        const double cut = v[(size_t)(0.75 * (n_templates - 1) + 0.5)];
        for (uint32_t t = 0; t < n_templates; ++t) large[t] = isolated_ms[t] >= cut;
    }
    uint64_t failed = 0;
    // collector: waits for requests in submission order, frees their copies
    std::thread collector([&] {
        for (;;) {
            Live l;
            {
                std::unique_lock<std::mutex> lk(fm);
                lv.wait(lk, [&] { return done || !live.empty(); });
                if (live.empty()) return;
                l = live.front();
                live.pop_front();
            }
            axhel_request_info_t info{};
            const axhel_status_t st = axhel_server_wait(server, l.id, 120000000ull, &info);
            std::lock_guard<std::mutex> lk(fm);
            if (st != AXHEL_OK) {
                ++failed;
            } else {
                lat.push_back(info.latency_ms);
                queue.push_back(info.queue_ms);
                (large[l.t] ? lat_large : lat_rest).push_back(info.latency_ms);
                if (isolated_ms) {
                    slow.push_back(info.latency_ms / isolated_ms[l.t]);
                    iso.push_back(isolated_ms[l.t]);
                }
            }
            free_copies[l.t].push_back(l.c);
        }
    });
    // producer: Poisson arrivals (exponential gaps), uniform template choice
    uint64_t x = seed ? seed : 0x9e3779b97f4a7c15ull;
    auto next_u = [&]() {  // xorshift64*: uniform in (0, 1)
        x ^= x >> 12;
        x ^= x << 25;
        x ^= x >> 27;
        return ((x * 0x2545F4914F6CDD1Dull) >> 11) * (1.0 / 9007199254740992.0) + 1e-18;
    };
    // arrivals on time: this (the caller's) thread sleeps with a 1 us timer
    // slack while it produces them, and gets its own back afterwards
    const int old_slack = prctl(PR_GET_TIMERSLACK, 0, 0, 0, 0);
    tighten_timer_slack();
    const auto t0 = Clock::now();
    const auto end = t0 + std::chrono::duration<double>(seconds);
    auto t = t0;
    axhel_status_t rc = AXHEL_OK;
    while (true) {
        t += std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(-std::log(next_u()) / rate_per_s));
        if (t >= end) break;
        std::this_thread::sleep_until(t);
        const uint32_t k = (uint32_t)(next_u() * n_templates) % n_templates;
        uint32_t c;
        {
            std::lock_guard<std::mutex> lk(fm);
            if (free_copies[k].empty()) {
                ++out->skipped;
                continue;
            }
            c = free_copies[k].back();
            free_copies[k].pop_back();
        }
        axhel_request_t r = templates[k];
        r.output = outputs[(size_t)k * copies + c];
        uint64_t id = 0;
        rc = axhel_server_submit(server, &r, &id);
        if (rc) break;
        ++out->submitted;
        std::lock_guard<std::mutex> lk(fm);
        live.push_back(Live{id, k, c});
        lv.notify_one();
    }
    {
        std::lock_guard<std::mutex> lk(fm);
        done = true;
        lv.notify_all();
    }
    collector.join();
    if (old_slack > 0) prctl(PR_SET_TIMERSLACK, (unsigned long)old_slack, 0, 0, 0);
    const double wall = std::chrono::duration<double>(Clock::now() - t0).count();
    auto pct = [](std::vector<double> v, double p) {
        if (v.empty()) return 0.0;
        std::sort(v.begin(), v.end());
        return v[std::min(v.size() - 1, (size_t)(p * (v.size() - 1) + 0.5))];
    };
    out->completed = lat.size();
    out->failed = failed;
    out->wall_s = wall;
    out->jobs_per_s = lat.size() / wall;
    out->p50_ms = pct(lat, 0.5);
    out->p99_ms = pct(lat, 0.99);
    out->p50_slowdown = pct(slow, 0.5);
    out->p99_slowdown = pct(slow, 0.99);
    out->isolated_p99_ms = pct(iso, 0.99);
    out->p50_queue_ms = pct(queue, 0.5);
    out->p99_queue_ms = pct(queue, 0.99);
    out->p99_large_ms = pct(lat_large, 0.99);
    out->p99_rest_ms = pct(lat_rest, 0.99);
    return rc;
}

}  // extern "C"
