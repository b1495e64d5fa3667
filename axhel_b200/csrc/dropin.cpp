// The unipi::axhel C++ drop-in (include/axhel/*.hpp), implemented on the
// C-ABI (include/axhel_cuda.h).
//
// Same signatures and semantics as the reference public API: calls are
// synchronous (results are visible on return), result may alias the
// operands, n == 0 is a no-op, and unsupported mod-factors leave the result
// untouched.  Pointers may be host memory (the reference's and SEAL's usage:
// operands are copied into per-thread pinned buffers; small ones are read
// and written there by the kernels themselves through the device's mapping
// of that memory, larger ones go by DMA to per-thread device buffers and
// back) or device memory (used in place, no copies).  Each host thread issues its work on its own
// per-thread default stream, so const NTT objects shared between threads (as
// SEAL's process-wide cache does) are safe to use concurrently.
// CUDA failures throw std::runtime_error: there is no CPU fallback.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/axhel/axhel.hpp"
#include "../../include/axhel/ntt/ntt-rns.hpp"
#include "../../include/axhel/util/debug.hpp"
#include "../../include/axhel_cuda.h"

namespace unipi {
namespace axhel {

namespace {

void check(axhel_status_t st, const char* what)
{
    if (st != AXHEL_OK) throw std::runtime_error(std::string("AXHEL ") + what + ": " + axhel_last_error());
}

void check_cuda(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string("AXHEL ") + what + ": " + cudaGetErrorString(e));
}

inline cudaStream_t stream() { return cudaStreamPerThread; }

// Default bound for staging host operands through pinned buffers.
constexpr size_t kPinnedStagingMax = size_t(1) << 30;
// Default bounds for operands the kernels access in the pinned buffers
// directly (no DMA copy).  Element-wise kernels read and write them once in
// contiguous runs: 512 KiB (MulMod at N = 2^16: 105 against 120 us per call
// by DMA; at 2^17 the mapped route gains 3 % on one thread and loses 20 %
// with eight threads calling).  The inverse transform reads contiguous rows, but from 2^16 words
// it runs as two passes over the buffers: 256 KiB.  The forward transform's
// first pass reads strided columns, short PCIe requests that cost more than
// a DMA copy from 2^15 words up (with eight threads calling, 210 against
// 136 us per call at N = 2^15): 128 KiB.
constexpr size_t kZeroCopyEltwise = size_t(512) << 10;
constexpr size_t kZeroCopyInverse = size_t(256) << 10;
constexpr size_t kZeroCopyForward = size_t(128) << 10;

// Growable per-thread device staging buffers (one per operand slot).
struct Staging {
    uint64_t* buf[4] = {nullptr, nullptr, nullptr, nullptr};
    size_t cap[4] = {0, 0, 0, 0};
    ~Staging()
    {
        for (auto* p : buf)
            if (p) cudaFree(p);
    }
    uint64_t* get(int slot, size_t words)
    {
        if (cap[slot] < words) {
            if (buf[slot]) cudaFree(buf[slot]);
            buf[slot] = nullptr;
            cap[slot] = 0;
            check_cuda(cudaMalloc(&buf[slot], words * sizeof(uint64_t)), "staging allocation");
            cap[slot] = words;
        }
        return buf[slot];
    }
};
thread_local Staging t_staging;

// Growable per-thread pinned host buffers: a host operand is copied into one
// by the CPU and from there to the device by DMA (and results the other way),
// instead of handing pageable memory to cudaMemcpyAsync, which stages it
// through the driver's own buffers and returns only when the copy is done.
// The buffers are mapped into the device's address space (`dev` is the
// device's view of `buf`), so a kernel can also read and write them itself.
struct Bounce {
    uint64_t* buf[4] = {nullptr, nullptr, nullptr, nullptr};
    uint64_t* dev[4] = {nullptr, nullptr, nullptr, nullptr};
    size_t cap[4] = {0, 0, 0, 0};
    ~Bounce()
    {
        for (auto* p : buf)
            if (p) cudaFreeHost(p);
    }
    uint64_t* get(int slot, size_t words)
    {
        if (cap[slot] < words) {
            if (buf[slot]) cudaFreeHost(buf[slot]);
            buf[slot] = dev[slot] = nullptr;
            cap[slot] = 0;
            check_cuda(cudaHostAlloc(reinterpret_cast<void**>(&buf[slot]), words * sizeof(uint64_t),
                                     cudaHostAllocMapped | cudaHostAllocPortable),
                       "pinned staging allocation");
            void* d = nullptr;
            const cudaError_t e = cudaHostGetDevicePointer(&d, buf[slot], 0);
            if (e != cudaSuccess) {
                cudaFreeHost(buf[slot]);
                buf[slot] = nullptr;
                check_cuda(e, "pinned staging mapping");
            }
            dev[slot] = static_cast<uint64_t*>(d);
            cap[slot] = words;
        }
        return buf[slot];
    }
};
thread_local Bounce t_bounce;

// Host operands up to this many bytes go through the pinned buffers; larger
// ones through cudaMemcpyAsync on the pageable memory itself.  Environment
// variable AXHEL_PINNED_STAGING_MAX (bytes; 0 = never), read once.
size_t pinned_max()
{
    static const size_t v = [] {
        const char* e = std::getenv("AXHEL_PINNED_STAGING_MAX");
        return e ? (size_t)std::strtoull(e, nullptr, 10) : kPinnedStagingMax;
    }();
    return v;
}

// Host operands up to this many bytes are not copied to the device at all:
// the kernels read them from, and write results to, the mapped pinned
// buffers over PCIe.  For a small call that saves a DMA copy each way, whose
// set-up costs more than moving the data.  `deflt`: the operation's bound
// (above).  Environment variable AXHEL_ZERO_COPY_MAX (bytes; 0 = never), read
// once, sets all of them.
size_t zero_copy_max(size_t deflt)
{
    static const char* env = std::getenv("AXHEL_ZERO_COPY_MAX");
    static const size_t v = env ? (size_t)std::strtoull(env, nullptr, 10) : 0;
    return std::min(env ? v : deflt, pinned_max());
}

// Whether p is device memory, asked of the driver once per pointer and call:
// the answer cannot change during a synchronous call, and the query takes a
// driver lock that several host threads contend for (0.1 us alone, about
// 3 us each with eight threads calling at once).  An in-place call (SEAL's
// result == operand) asks once instead of twice.
struct PtrMemo {
    const void* p[4];
    bool dev[4];
    int n = 0;
};
thread_local PtrMemo t_memo;

bool is_device(const void* p)
{
    PtrMemo& m = t_memo;
    for (int i = 0; i < m.n; ++i)
        if (m.p[i] == p) return m.dev[i];
    const bool d = axhel_cuda_is_device_pointer(p) != 0;
    if (m.n < 4) {
        m.p[m.n] = p;
        m.dev[m.n] = d;
        ++m.n;
    }
    return d;
}

// Device view of an input operand: the pointer itself if it is device
// memory, else a staged copy.
const uint64_t* input(const uint64_t* p, uint64_t n, int slot, size_t zc = kZeroCopyEltwise)
{
    if (!p || is_device(p)) return p;
    const size_t bytes = n * sizeof(uint64_t);
    if (bytes <= zero_copy_max(zc)) {
        std::memcpy(t_bounce.get(slot, n), p, bytes);
        return t_bounce.dev[slot];
    }
    uint64_t* d = t_staging.get(slot, n);
    const void* src = p;
    if (bytes <= pinned_max()) {
        uint64_t* h = t_bounce.get(slot, n);
        std::memcpy(h, p, bytes);
        src = h;
    }
    check_cuda(cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, stream()), "host to device copy");
    return d;
}

// Device destination for `result`: itself, pinned slot 3 (mapped, written by
// the kernels directly) or device staging slot 3.
struct Output {
    uint64_t* host = nullptr;
    uint64_t* dev = nullptr;
    uint64_t n = 0;
    bool mapped = false;
    // Constructed first in every call: starts the call's pointer memo.
    Output(uint64_t* r, uint64_t count, size_t zc = kZeroCopyEltwise) : n(count)
    {
        t_memo.n = 0;
        if (is_device(r)) {
            dev = r;
        } else if (count * sizeof(uint64_t) <= zero_copy_max(zc)) {
            host = r;
            t_bounce.get(3, count);
            dev = t_bounce.dev[3];
            mapped = true;
        } else {
            host = r;
            dev = t_staging.get(3, count);
        }
    }
    void finish()
    {
        const size_t bytes = n * sizeof(uint64_t);
        uint64_t* bounce = (host && bytes <= pinned_max()) ? t_bounce.get(3, n) : nullptr;
        if (host && !mapped)
            check_cuda(cudaMemcpyAsync(bounce ? bounce : host, dev, bytes, cudaMemcpyDeviceToHost, stream()),
                       "device to host copy");
        check_cuda(cudaStreamSynchronize(stream()), "stream synchronize");
        if (bounce) std::memcpy(host, bounce, bytes);
    }
};

}  // namespace

// --------------------------------------------------------------- eltwise

void EltwiseAddMod(uint64_t* result, const uint64_t* operand1, const uint64_t* operand2, uint64_t n, uint64_t modulus)
{
    if (n == 0) return;
    Output out(result, n);
    const uint64_t* a = input(operand1, n, 0);
    const uint64_t* b = input(operand2, n, 1);
    AXHEL_LOG("EltwiseAddMod vector-vector -> CUDA, n=" << n << (out.host ? ", host result" : ", device result"));
    check(axhel_cuda_eltwise_add_vv(out.dev, a, b, n, modulus, stream()), "EltwiseAddMod");
    out.finish();
}

void EltwiseAddMod(uint64_t* result, const uint64_t* operand1, uint64_t operand2, uint64_t n, uint64_t modulus)
{
    if (n == 0) return;
    Output out(result, n);
    const uint64_t* a = input(operand1, n, 0);
    AXHEL_LOG("EltwiseAddMod vector-scalar -> CUDA, n=" << n << (out.host ? ", host result" : ", device result"));
    check(axhel_cuda_eltwise_add_vs(out.dev, a, operand2, n, modulus, stream()), "EltwiseAddMod");
    out.finish();
}

void EltwiseSubMod(uint64_t* result, const uint64_t* operand1, const uint64_t* operand2, uint64_t n, uint64_t modulus)
{
    if (n == 0) return;
    Output out(result, n);
    const uint64_t* a = input(operand1, n, 0);
    const uint64_t* b = input(operand2, n, 1);
    AXHEL_LOG("EltwiseSubMod vector-vector -> CUDA, n=" << n << (out.host ? ", host result" : ", device result"));
    check(axhel_cuda_eltwise_sub_vv(out.dev, a, b, n, modulus, stream()), "EltwiseSubMod");
    out.finish();
}

void EltwiseSubMod(uint64_t* result, const uint64_t* operand1, uint64_t operand2, uint64_t n, uint64_t modulus)
{
    if (n == 0) return;
    Output out(result, n);
    const uint64_t* a = input(operand1, n, 0);
    AXHEL_LOG("EltwiseSubMod vector-scalar -> CUDA, n=" << n << (out.host ? ", host result" : ", device result"));
    check(axhel_cuda_eltwise_sub_vs(out.dev, a, operand2, n, modulus, stream()), "EltwiseSubMod");
    out.finish();
}

void EltwiseMulMod(uint64_t* result, const uint64_t* operand1, const uint64_t* operand2, uint64_t n, uint64_t modulus,
                   uint64_t mod_factor)
{
    if (n == 0 || (mod_factor != 1 && mod_factor != 2 && mod_factor != 4)) return;  // eltwise-mul-mod.cpp:83-93
    Output out(result, n);
    const uint64_t* a = input(operand1, n, 0);
    const uint64_t* b = input(operand2, n, 1);
    AXHEL_LOG("EltwiseMulMod -> CUDA, mod_factor=" << mod_factor << ", n=" << n);
    check(axhel_cuda_eltwise_mul(out.dev, a, b, n, modulus, mod_factor, stream()), "EltwiseMulMod");
    out.finish();
}

void EltwiseFMAMod(uint64_t* res, const uint64_t* op1, uint64_t op2, const uint64_t* op3, uint64_t n, uint64_t mod,
                   uint64_t mod_factor)
{
    if (n == 0 || (mod_factor != 1 && mod_factor != 2 && mod_factor != 4 && mod_factor != 8)) return;
    Output out(res, n);
    const uint64_t* a = input(op1, n, 0);
    const uint64_t* c = input(op3, n, 1);
    AXHEL_LOG("EltwiseFMAMod -> CUDA, mod_factor=" << mod_factor << ", n=" << n << (c ? ", addend" : ""));
    check(axhel_cuda_eltwise_fma(out.dev, a, op2, c, n, mod, mod_factor, stream()), "EltwiseFMAMod");
    out.finish();
}

void EltwiseReduceMod(uint64_t* res, const uint64_t* op, uint64_t n, uint64_t mod, uint64_t in_mod_factor,
                      uint64_t out_mod_factor)
{
    if (n == 0) return;
    Output out(res, n);
    const bool matched = in_mod_factor == 1 || (out_mod_factor == 2 && in_mod_factor <= 2) ||
                         (in_mod_factor == 2 && out_mod_factor == 1) ||
                         (in_mod_factor == 4 && (out_mod_factor == 1 || out_mod_factor == 2)) ||
                         in_mod_factor == mod;
    if (!matched) return;  // eltwise-reduce-mod.cpp:32-128: an unmatched pair writes nothing
    const uint64_t* a = input(op, n, 0);
    AXHEL_LOG("EltwiseReduceMod -> CUDA, in_factor=" << in_mod_factor << ", out_factor=" << out_mod_factor
                                                      << ", n=" << n);
    check(axhel_cuda_eltwise_reduce(out.dev, a, n, mod, in_mod_factor, out_mod_factor, stream()), "EltwiseReduceMod");
    out.finish();
}

// ------------------------------------------------------------------ NTT

class NTT::Impl {
public:
    uint64_t degree{0};
    uint64_t modulus{0};
    axhel_ntt_t handle{nullptr};
    // External tables, borrowed as the reference does (ntt.hpp:34-37): read
    // again before every transform, so a caller that updates them in place
    // gets the results the reference would give.
    const NTTMultiplyOperand* ext_fwd{nullptr};
    const NTTMultiplyOperand* ext_inv{nullptr};
    NTTMultiplyOperand ext_ninv{0, 0};
    ~Impl() { axhel_cuda_ntt_release(handle); }
};

NTT::NTT(uint64_t degree, uint64_t modulus, uint64_t root_of_unity) : impl_(std::make_shared<Impl>())
{
    impl_->degree = degree;
    impl_->modulus = modulus;
    check(axhel_cuda_ntt_create(degree, modulus, root_of_unity, &impl_->handle), "NTT tables");
}

NTT::NTT(uint64_t degree, uint64_t modulus, const NTTMultiplyOperand* root_powers,
         const NTTMultiplyOperand* inv_root_powers, NTTMultiplyOperand inv_degree_modulo)
    : impl_(std::make_shared<Impl>())
{
    static_assert(sizeof(NTTMultiplyOperand) == 16, "NTTMultiplyOperand layout");
    impl_->degree = degree;
    impl_->modulus = modulus;
    const uint64_t ninv[2] = {inv_degree_modulo.operand, inv_degree_modulo.quotient};
    check(axhel_cuda_ntt_create_external(degree, modulus, reinterpret_cast<const uint64_t*>(root_powers),
                                         reinterpret_cast<const uint64_t*>(inv_root_powers), ninv, &impl_->handle),
          "NTT external tables");
    impl_->ext_fwd = root_powers;
    impl_->ext_inv = inv_root_powers;
    impl_->ext_ninv = inv_degree_modulo;
}

NTT::~NTT() = default;
NTT::NTT(const NTT&) noexcept = default;
NTT& NTT::operator=(const NTT&) noexcept = default;
NTT::NTT(NTT&&) noexcept = default;
NTT& NTT::operator=(NTT&&) noexcept = default;

void NTT::ComputeForward(uint64_t* result, const uint64_t* operand, uint64_t input_mod_factor,
                         uint64_t output_mod_factor) const
{
    const uint64_t n = impl_->degree;
    if (impl_->ext_fwd)
        check(axhel_cuda_ntt_refresh_external(impl_->handle, reinterpret_cast<const uint64_t*>(impl_->ext_fwd),
                                              nullptr, nullptr, stream()),
              "NTT external tables");
    Output out(result, n, kZeroCopyForward);
    const uint64_t* a = input(operand, n, 0, kZeroCopyForward);
    AXHEL_LOG("NTT::ComputeForward -> CUDA, N=" << n << ", out_factor=" << output_mod_factor
                                                 << (out.host ? ", host operands" : ", device operands"));
    check(axhel_cuda_ntt_forward(impl_->handle, out.dev, a, input_mod_factor, output_mod_factor, stream()),
          "ComputeForward");
    out.finish();
}

void NTT::ComputeInverse(uint64_t* result, const uint64_t* operand, uint64_t input_mod_factor,
                         uint64_t output_mod_factor) const
{
    const uint64_t n = impl_->degree;
    if (impl_->ext_inv) {
        const uint64_t ninv[2] = {impl_->ext_ninv.operand, impl_->ext_ninv.quotient};
        check(axhel_cuda_ntt_refresh_external(impl_->handle, nullptr,
                                              reinterpret_cast<const uint64_t*>(impl_->ext_inv), ninv, stream()),
              "NTT external tables");
    }
    Output out(result, n, kZeroCopyInverse);
    const uint64_t* a = input(operand, n, 0, kZeroCopyInverse);
    AXHEL_LOG("NTT::ComputeInverse -> CUDA, N=" << n << ", out_factor=" << output_mod_factor
                                                 << (out.host ? ", host operands" : ", device operands"));
    check(axhel_cuda_ntt_inverse(impl_->handle, out.dev, a, input_mod_factor, output_mod_factor, stream()),
          "ComputeInverse");
    out.finish();
}

uint64_t NTT::Degree() const noexcept { return impl_ ? impl_->degree : 0; }
uint64_t NTT::Modulus() const noexcept { return impl_ ? impl_->modulus : 0; }

// ------------------------------------------------------------- RNS batches

namespace detail {
struct NTTAccess {
    static axhel_ntt_t handle(const NTT& t) { return t.impl_ ? t.impl_->handle : nullptr; }
};
}  // namespace detail

namespace {

std::vector<axhel_ntt_t> rns_handles(const NTT* ntts, size_t n_ntts, uint64_t* degree)
{
    if (!ntts || n_ntts == 0 || n_ntts > 64) throw std::invalid_argument("AXHEL RNS transform: 1..64 NTT objects");
    std::vector<axhel_ntt_t> hs(n_ntts);
    *degree = ntts[0].Degree();
    for (size_t i = 0; i < n_ntts; ++i) {
        hs[i] = detail::NTTAccess::handle(ntts[i]);
        if (!hs[i] || ntts[i].Degree() != *degree)
            throw std::invalid_argument("AXHEL RNS transform: NTT objects of one degree needed");
    }
    return hs;
}

// Per-thread events marking the end of each chunk of a pipelined call.
struct ChunkEvents {
    std::vector<cudaEvent_t> ev;
    ~ChunkEvents()
    {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
    cudaEvent_t get(size_t i)
    {
        while (ev.size() <= i) {
            cudaEvent_t e = nullptr;
            check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
            ev.push_back(e);
        }
        return ev[i];
    }
};
thread_local ChunkEvents t_events;

// A batch of limbs whose operand and result are both host memory, too large
// for the mapped route: staged in chunks of limbs (about 2 MiB each), so that
// the CPU's copies into and out of the pinned buffers overlap the GPU's
// copies and transform of the neighbouring chunks.  `run(handles, n_handles,
// data, limbs)` transforms `limbs` limbs in place on the device, limb i with
// handles[i % n_handles].  Returns false (nothing done) where this does not
// apply.
template <class Run>
bool rns_pipelined(const std::vector<axhel_ntt_t>& hs, uint64_t n, uint64_t* result, const uint64_t* operand,
                   size_t count, size_t zc, Run run)
{
    const size_t words = count * n, bytes_all = words * sizeof(uint64_t);
    const size_t per = std::max<size_t>(1, (size_t(2) << 20) / (n * sizeof(uint64_t)));
    const size_t nch = (count + per - 1) / per;
    t_memo.n = 0;
    if (nch < 2 || bytes_all <= zero_copy_max(zc) || bytes_all > pinned_max() || is_device(result) ||
        is_device(operand))
        return false;
    uint64_t* hin = t_bounce.get(0, words);
    uint64_t* hout = t_bounce.get(3, words);
    uint64_t* d = t_staging.get(0, words);
    std::vector<axhel_ntt_t> rot(hs.size());
    for (size_t c = 0; c <= nch; ++c) {
        if (c < nch) {  // stage chunk c, queue its copies and transform
            const size_t f = c * per, k = std::min(per, count - f), off = f * n, bytes = k * n * sizeof(uint64_t);
            std::memcpy(hin + off, operand + off, bytes);
            check_cuda(cudaMemcpyAsync(d + off, hin + off, bytes, cudaMemcpyHostToDevice, stream()),
                       "host to device copy");
            for (size_t j = 0; j < hs.size(); ++j) rot[j] = hs[(f + j) % hs.size()];
            check(run(rot.data(), rot.size(), d + off, k), "RNS transform");
            check_cuda(cudaMemcpyAsync(hout + off, d + off, bytes, cudaMemcpyDeviceToHost, stream()),
                       "device to host copy");
            check_cuda(cudaEventRecord(t_events.get(c), stream()), "event record");
        }
        if (c >= 1) {  // unstage chunk c-1 once its copy back is done
            const size_t f = (c - 1) * per, k = std::min(per, count - f), off = f * n;
            check_cuda(cudaEventSynchronize(t_events.get(c - 1)), "event synchronize");
            std::memcpy(result + off, hout + off, k * n * sizeof(uint64_t));
        }
    }
    return true;
}

}  // namespace

void ComputeForwardRNS(const NTT* ntts, size_t n_ntts, uint64_t* result, const uint64_t* operand, size_t count,
                       uint64_t /*input_mod_factor*/, uint64_t output_mod_factor)
{
    if (count == 0) return;
    uint64_t n = 0;
    const std::vector<axhel_ntt_t> hs = rns_handles(ntts, n_ntts, &n);
    if (rns_pipelined(hs, n, result, operand, count, kZeroCopyForward,
                      [&](const axhel_ntt_t* h, size_t nh, uint64_t* p, size_t k) {
                          return axhel_cuda_ntt_forward_batch(h, nh, p, p, k, 1, output_mod_factor, stream());
                      }))
        return;
    const uint64_t words = (uint64_t)count * n;
    Output out(result, words, kZeroCopyForward);
    const uint64_t* a = input(operand, words, 0, kZeroCopyForward);
    check(axhel_cuda_ntt_forward_batch(hs.data(), n_ntts, out.dev, a, count, 1, output_mod_factor, stream()),
          "ComputeForwardRNS");
    out.finish();
}

void ComputeInverseRNS(const NTT* ntts, size_t n_ntts, uint64_t* result, const uint64_t* operand, size_t count,
                       uint64_t /*input_mod_factor*/, uint64_t output_mod_factor)
{
    if (count == 0) return;
    uint64_t n = 0;
    const std::vector<axhel_ntt_t> hs = rns_handles(ntts, n_ntts, &n);
    if (rns_pipelined(hs, n, result, operand, count, kZeroCopyInverse,
                      [&](const axhel_ntt_t* h, size_t nh, uint64_t* p, size_t k) {
                          return axhel_cuda_ntt_inverse_batch(h, nh, p, p, k, 2, output_mod_factor, stream());
                      }))
        return;
    const uint64_t words = (uint64_t)count * n;
    Output out(result, words, kZeroCopyInverse);
    const uint64_t* a = input(operand, words, 0, kZeroCopyInverse);
    // input factor 2: the per-limb ComputeInverse's contract (inputs in [0, 2q)), no fused reduction
    check(axhel_cuda_ntt_inverse_batch(hs.data(), n_ntts, out.dev, a, count, 2, output_mod_factor, stream()),
          "ComputeInverseRNS");
    out.finish();
}

}  // namespace axhel
}  // namespace unipi
