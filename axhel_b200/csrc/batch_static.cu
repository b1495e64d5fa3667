// Uneven batches without any device allocation.
//
// Some callers cannot allocate device memory when they run a batch: serving
// processes whose HBM is reserved up front by their own caching allocator or
// a fixed memory budget (an extra cudaMalloc would fail or fragment it), and
// latency-critical loops where cudaMalloc / cudaFree would synchronize the
// whole device and stall work on other streams.  For them,
// axhel_cuda_batch_run_static runs the same persistent batch kernel as
// axhel_cuda_batch_run, but keeps the batch's scratch -- job descriptors,
// the tile table, per-limb completion counters, the work counter and the
// error word -- in one file-scope static device array of kStaticScratchBytes
// that every device loading the library holds until the process exits.  The
// caller still passes the inputs and outputs; nothing else is allocated.
//
// The array's name is a host-side stand-in in host code, not a device
// address: the first call on each device resolves the device address with
// cudaGetSymbolAddress while that device is current, and later calls reuse
// it.  Make that first call before any stream capture.  The resolved address
// belongs to the device's context as it was then: after a cudaDeviceReset
// the module may be loaded again elsewhere, so this entry point must not be
// used across a reset of the device.  Every call waits for its batch to
// finish (it reads the error word back) before it returns.
//
// Every call shares the one array and leaves its contents behind; each call
// rewrites the descriptors and clears the counters it uses (they travel in
// the same host-to-device copy), so calls that overlap on the GPU -- from
// several streams or host threads at once -- race and must not be issued.
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "../../include/axhel_cuda.h"
#include "batch.h"
#include "internal.h"

namespace {

// 1 MiB: room for the descriptors of e.g. 512 jobs of up to 48 limbs
// (about 0.5 MiB); larger batches are rejected with AXHEL_ERR_UNSUPPORTED.
constexpr size_t kStaticScratchBytes = size_t(1) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_batch_scratch[kStaticScratchBytes];

std::mutex g_addr_mu;
unsigned char* g_addr[kMaxDevices] = {};

// Device address of g_batch_scratch on the current device (resolved once).
axhel_status_t scratch_address(unsigned char** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        axhel_impl::batch_set_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        return AXHEL_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        axhel_impl::batch_set_error("device index out of range");
        return AXHEL_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_batch_scratch);
        if (e != cudaSuccess || !p) {
            axhel_impl::batch_set_error(std::string("cudaGetSymbolAddress(static batch scratch): ") +
                                        cudaGetErrorString(e));
            return AXHEL_ERR_CUDA;
        }
        g_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_addr[dev];
    return AXHEL_OK;
}

}  // namespace

extern "C" axhel_status_t axhel_cuda_batch_run_static(const axhel_job_t* jobs, uint64_t n_jobs, void* stream)
{
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    std::vector<unsigned char> img;
    size_t zero_off = 0, zero_bytes = 0;
    axhel_impl::BatchArgs args{};
    std::string err;
    // size first, so an oversized batch is refused before any device work
    axhel_status_t st = axhel_impl::batch_build(jobs, n_jobs, nullptr, img, &zero_off, &zero_bytes, &args, nullptr, &err);
    if (st) {
        axhel_impl::batch_set_error(err);
        return st;
    }
    if (img.size() > kStaticScratchBytes) {
        axhel_impl::batch_set_error("batch needs " + std::to_string(img.size()) +
                                    " bytes of descriptors and counters; the static scratch holds " +
                                    std::to_string(kStaticScratchBytes) +
                                    " bytes: split the batch or use axhel_cuda_batch_run");
        return AXHEL_ERR_UNSUPPORTED;
    }
    if (args.total_tiles == 0) return AXHEL_OK;
    unsigned char* base = nullptr;
    st = scratch_address(&base);
    if (st) return st;
    st = axhel_impl::batch_build(jobs, n_jobs, base, img, &zero_off, &zero_bytes, &args, nullptr, &err);
    if (st) {
        axhel_impl::batch_set_error(err);
        return st;
    }
    // descriptors and zeroed counters / work counter / error word, in one copy
    cudaError_t e = cudaMemcpyAsync(base, img.data(), img.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = axhel_impl::batch_launch_args(args, s);
    int word = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&word, args.error, sizeof word, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        axhel_impl::batch_set_error(std::string("static batch: ") + cudaGetErrorString(e));
        return AXHEL_ERR_CUDA;
    }
    if (word) {
        axhel_impl::batch_set_error("a dependency wait in the batch kernel timed out");
        return word;
    }
    return AXHEL_OK;
}
