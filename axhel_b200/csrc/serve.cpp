// Serving loop: continuous batching of transform jobs on one GPU.
//
// Requests (any job kind of the batch engine: forward, inverse, or the fused
// INTT -> MulMod/FMAMod -> NTT chain, each of any degree 2^10..2^17 and limb
// count) are submitted from any host thread and return at once with an id.
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

#include <algorithm>
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
    cudaStream_t stream = nullptr;
    void* scratch = nullptr;
    size_t cap = 0;
    int* err_host = nullptr;  // pinned word the kernel's error status is copied into
    bool busy = false;
};

struct Inflight {
    cudaEvent_t done = nullptr;
    std::vector<Req*> reqs;
    size_t bytes = 0;
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
    std::deque<Req*> pending;
    std::unordered_map<uint64_t, std::unique_ptr<Req>> reqs;
    std::deque<Inflight> inflight;
    std::vector<Slot> slots;
    size_t in_use = 0, peak_in_use = 0;
    uint64_t next_id = 1, batches = 0, completed = 0, max_batch = 0;
    bool stop = false, paused = false;
    std::vector<double> lat_ms;  // submit -> done of every completed request
    std::thread sched, comp;
    std::string fatal;

    void scheduler();
    void completer();
    axhel_status_t launch(Slot& s, int slot_index, std::vector<Req*>& take, Inflight& f);
};

axhel_status_t axhel_server::launch(Slot& s, int slot_index, std::vector<Req*>& take, Inflight& f)
{
    cudaStream_t st = s.stream;
    std::vector<axhel_job_t> jobs(take.size());
    for (size_t i = 0; i < take.size(); ++i) {
        Req* q = take[i];
        const size_t bytes = q->words * 8;
        q->d_in = const_cast<uint64_t*>(q->r.input);
        q->d_out = q->r.output;
        q->d_vec = const_cast<uint64_t*>(q->r.vector);
        cudaError_t e = cudaSuccess;
        if (!q->in_dev) {
            e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&q->d_in), bytes, pool, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(q->d_in, q->r.input, bytes, cudaMemcpyHostToDevice, st);
        }
        if (e == cudaSuccess && !q->out_dev) {
            if (q->in_dev || q->r.output != q->r.input)
                e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&q->d_out), bytes, pool, st);
            else
                q->d_out = q->d_in;  // in place on the staged copy
        }
        if (e == cudaSuccess && q->r.vector && !q->vec_dev) {
            e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&q->d_vec), bytes, pool, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(q->d_vec, q->r.vector, bytes, cudaMemcpyHostToDevice, st);
        }
        if (e != cudaSuccess) return sfail(AXHEL_ERR_NOMEM, std::string("request staging: ") + cudaGetErrorString(e));
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
    axhel_status_t rc = axhel_impl::batch_build(jobs.data(), jobs.size(), nullptr, img, &zo, &zb, &args, nullptr, &err);
    if (rc) return sfail(rc, err);
    if (img.size() > s.cap) {
        cudaStreamSynchronize(st);  // the old buffer may still be read by this stream's last batch
        if (s.scratch) cudaFree(s.scratch);
        s.scratch = nullptr;
        s.cap = 0;
        const size_t cap = std::max<size_t>(img.size() * 2, 1 << 20);
        if (cudaMalloc(&s.scratch, cap) != cudaSuccess) return sfail(AXHEL_ERR_NOMEM, "batch descriptor buffer");
        s.cap = cap;
    }
    rc = axhel_impl::batch_build(jobs.data(), jobs.size(), static_cast<unsigned char*>(s.scratch), img, &zo, &zb,
                                 &args, nullptr, &err);
    if (rc) return sfail(rc, err);
    cudaError_t e = cudaMemcpyAsync(s.scratch, img.data(), img.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = axhel_impl::batch_launch_args(args, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s.err_host, args.error, sizeof(int), cudaMemcpyDeviceToHost, st);
    for (Req* q : take) {
        if (e != cudaSuccess) break;
        if (!q->out_dev) e = cudaMemcpyAsync(q->r.output, q->d_out, q->words * 8, cudaMemcpyDeviceToHost, st);
        if (!q->in_dev) cudaFreeAsync(q->d_in, st);
        if (!q->out_dev && q->d_out != q->d_in) cudaFreeAsync(q->d_out, st);
        if (q->r.vector && !q->vec_dev) cudaFreeAsync(q->d_vec, st);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f.done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(f.done, st);
    if (e != cudaSuccess) return sfail(AXHEL_ERR_CUDA, std::string("batch launch: ") + cudaGetErrorString(e));
    f.slot = slot_index;
    return AXHEL_OK;
}

void axhel_server::scheduler()
{
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        cv_sched.wait(lk, [&] {
            if (stop) return true;
            if (paused || pending.empty()) return false;
            return std::any_of(slots.begin(), slots.end(), [](const Slot& s) { return !s.busy; });
        });
        if (stop) break;
        // admit in arrival order while the budget allows
        std::vector<Req*> take;
        size_t bytes = 0;
        while (!pending.empty() && take.size() < cfg.max_batch_requests) {
            Req* q = pending.front();
            if (q->status != kPending) {  // cancelled
                pending.pop_front();
                continue;
            }
            if (in_use + bytes + q->need > cfg.hbm_budget_bytes) break;
            bytes += q->need;
            pending.pop_front();
            take.push_back(q);
        }
        if (take.empty()) {
            // The head does not fit next to the batches in flight: wait until
            // one of them releases its memory (every request fits an empty
            // budget: larger ones are refused at submit), or it is cancelled.
            const size_t held = in_use;
            cv_sched.wait(lk, [&] {
                return stop || paused || in_use < held || pending.empty() || pending.front()->status != kPending;
            });
            continue;
        }
        int si = 0;
        while (slots[si].busy) ++si;
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
        f.reqs = take;
        f.bytes = bytes;
        f.id = bid;
        const axhel_status_t rc = launch(slots[si], si, take, f);
        lk.lock();
        if (rc) {
            for (Req* q : take) {
                q->status = rc;
                q->t_done = Clock::now();
            }
            if (f.done) cudaEventDestroy(f.done);
            cudaStreamSynchronize(slots[si].stream);
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
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        cv_done.wait(lk, [&] { return !inflight.empty() || stop; });
        if (inflight.empty()) {
            if (stop) break;
            continue;
        }
        cudaEvent_t ev = inflight.front().done;
        lk.unlock();
        const cudaError_t e = cudaEventSynchronize(ev);
        lk.lock();
        Inflight f = std::move(inflight.front());
        inflight.pop_front();
        Slot& s = slots[f.slot];
        const int kernel_status = (e == cudaSuccess) ? *s.err_host : AXHEL_ERR_CUDA;
        const auto now = Clock::now();
        for (Req* q : f.reqs) {
            q->status = kernel_status;
            q->t_done = now;
            lat_ms.push_back(std::chrono::duration<double, std::milli>(now - q->t_submit).count());
            for (axhel_ntt_t h : q->ntts) axhel_cuda_ntt_release(h);
            q->ntts.clear();
            ++completed;
        }
        cudaEventDestroy(f.done);
        s.busy = false;
        in_use -= f.bytes;
        cv_sched.notify_all();
        cv_wait.notify_all();
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
    s->slots.resize(cfg->max_inflight);
    for (Slot& sl : s->slots) {
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&sl.err_host), sizeof(int));
    }
    if (e != cudaSuccess) {
        for (Slot& sl : s->slots) {
            if (sl.stream) cudaStreamDestroy(sl.stream);
            if (sl.err_host) cudaFreeHost(sl.err_host);
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
    if (r->kind < AXHEL_JOB_FORWARD || r->kind > AXHEL_JOB_CHAIN_FMA) return sfail(AXHEL_ERR_INVALID, "kind");
    if (!r->ntts || r->n_ntts == 0 || !r->input || !r->output || r->count == 0)
        return sfail(AXHEL_ERR_INVALID, "request needs handles, input, output and count > 0");
    if (r->kind == AXHEL_JOB_CHAIN_MUL && !r->vector) return sfail(AXHEL_ERR_INVALID, "chain multiplicand missing");
    if (r->kind == AXHEL_JOB_CHAIN_FMA && !r->scalars) return sfail(AXHEL_ERR_INVALID, "chain scalars missing");
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
    s->pending.push_back(q.get());
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
    out->pending = s->pending.size();
    out->in_use_bytes = s->in_use;
    out->peak_in_use_bytes = s->peak_in_use;
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
    out->samples = v.size();
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
        if (sl.scratch) cudaFree(sl.scratch);
        cudaStreamDestroy(sl.stream);
        cudaFreeHost(sl.err_host);
    }
    for (auto& kv : s->reqs)
        for (axhel_ntt_t h : kv.second->ntts) axhel_cuda_ntt_release(h);
    cudaMemPoolDestroy(s->pool);
    delete s;
    return AXHEL_OK;
}

const char* axhel_server_last_error(void) { return t_serve_error.c_str(); }

}  // extern "C"
