/*
 * axhel_cuda.h — C-ABI of the B200 (sm_100a) implementation of AXHEL's hot
 * path: the negacyclic Harvey NTT/INTT and the element-wise modular kernels.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, returns
 * an axhel_status_t, and never allocates on behalf of the caller's data.
 * Data pointers are DEVICE pointers unless stated otherwise; calls are
 * asynchronous on the given CUDA stream (a cudaStream_t passed as void*,
 * NULL = the legacy default stream).  Residues are uint64_t, moduli q < 2^62.
 *
 * Results are bit-identical to the reference native backend (AXHEL,
 * axhel/ntt/ntt-native.cpp and axhel/eltwise/eltwise-*-mod.cpp), including the lazy
 * representatives of forward output factor 4 ([0,4q)) and inverse output
 * factor 2 ([0,2q)).  Each entry point names the reference interface it
 * replaces (paths relative to the AXHEL project root).
 *
 * The C++ drop-in (include/axhel/axhel.hpp, namespace unipi::axhel) is built
 * on these functions.
 */
#ifndef AXHEL_CUDA_H
#define AXHEL_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t axhel_status_t;
#define AXHEL_OK 0
#define AXHEL_ERR_INVALID 1     /* bad argument (size, factor, pointer, modulus) */
#define AXHEL_ERR_CUDA 2        /* a CUDA runtime call failed; see axhel_last_error() */
#define AXHEL_ERR_NOMEM 3       /* device or pinned host allocation failed */
#define AXHEL_ERR_UNSUPPORTED 4 /* degree / configuration outside the supported range */
#define AXHEL_ERR_BUSY 5        /* serving queue full */
#define AXHEL_ERR_TIMEOUT 6     /* a bounded wait expired */
#define AXHEL_ERR_REJECTED 7    /* serving admission refused (over the HBM budget) */
#define AXHEL_ERR_CANCELLED 8   /* serving request cancelled before it ran */

/* Opaque handle to the device-resident tables of one (N, q) transform. */
typedef struct axhel_ntt_ctx* axhel_ntt_t;

/* Smallest and largest supported degree N (powers of two). */
#define AXHEL_MIN_DEGREE 2u
#define AXHEL_MAX_DEGREE 131072u

const char* axhel_status_string(axhel_status_t status);
/* Message of the last failure on the calling thread ("" if none). */
const char* axhel_last_error(void);
int axhel_version(void);

/* ---------------------------------------------------------------------- */
/* NTT tables                                                             */
/* ---------------------------------------------------------------------- */

/* Replaces NTT::NTT(degree, modulus, root_of_unity)
 * (axhel/include/axhel/ntt/ntt.hpp:32, axhel/ntt/ntt.cpp:136-152).
 * Generates the forward/inverse Shoup tables once per (degree, modulus, root)
 * (process-wide cache), on the device, and keeps them resident there.  The
 * returned handle holds one reference; release it with axhel_cuda_ntt_release.
 * The modulus must be odd (NTT moduli are primes q = 1 mod 2N). */
axhel_status_t axhel_cuda_ntt_create(uint64_t degree, uint64_t modulus, uint64_t root_of_unity,
                                     axhel_ntt_t* out);

/* Many NTT::NTT(degree, modulus, root_of_unity) at once (new; the cold start
 * of a parameter set with many RNS moduli): out[i] for (degrees[i],
 * moduli[i], roots[i]), cache hits shared.  The tables of all contexts not
 * yet cached are generated by one kernel launch per 96 contexts -- entry for
 * entry equal to GenerateNTTTables (axhel/ntt/ntt-tables.cpp:81-140) -- and
 * are ready when the call returns.  On failure no handle is returned. */
axhel_status_t axhel_cuda_ntt_create_many(uint64_t count, const uint64_t* degrees, const uint64_t* moduli,
                                          const uint64_t* roots, axhel_ntt_t* out);

/* Replaces NTT::NTT(degree, modulus, root_powers, inv_root_powers, inv_degree_modulo)
 * (ntt.hpp:37, ntt.cpp:124-133).  root_powers / inv_root_powers are HOST
 * arrays of `degree` {operand, quotient} pairs (2*degree words, the layout of
 * NTTMultiplyOperand, ntt.hpp:14-18); inv_degree is one pair.  They are
 * copied to the device at creation; axhel_cuda_ntt_refresh_external re-reads
 * them (the reference borrows them and reads them at every transform). */
axhel_status_t axhel_cuda_ntt_create_external(uint64_t degree, uint64_t modulus, const uint64_t* root_powers,
                                              const uint64_t* inv_root_powers, const uint64_t* inv_degree,
                                              axhel_ntt_t* out);

/* The reference's external-table NTT borrows the caller's tables and reads
 * them at every transform (ntt.hpp:34-37); this re-reads them from the
 * caller's HOST arrays into the handle's device copy, in stream order, so
 * that a transform issued after it sees the tables as they are now.  Either
 * table may be NULL (not re-read); the inverse table needs inv_degree.  Only
 * for handles made by axhel_cuda_ntt_create_external.  The C++ drop-in calls
 * it before every transform of such an NTT. */
axhel_status_t axhel_cuda_ntt_refresh_external(axhel_ntt_t ntt, const uint64_t* root_powers,
                                               const uint64_t* inv_root_powers, const uint64_t* inv_degree,
                                               void* stream);

axhel_status_t axhel_cuda_ntt_retain(axhel_ntt_t ntt);
axhel_status_t axhel_cuda_ntt_release(axhel_ntt_t ntt);
/* NTT::Degree / NTT::Modulus (ntt.hpp:56-59; 0 for a null handle, ntt.cpp:210-216). */
uint64_t axhel_cuda_ntt_degree(axhel_ntt_t ntt);
uint64_t axhel_cuda_ntt_modulus(axhel_ntt_t ntt);
/* Copies the resident tables back to HOST arrays (2*N, 2*N and 2 words). */
axhel_status_t axhel_cuda_ntt_read_tables(axhel_ntt_t ntt, uint64_t* root_powers, uint64_t* inv_root_powers,
                                          uint64_t* inv_degree);

/* ---------------------------------------------------------------------- */
/* NTT transforms (device pointers)                                       */
/* ---------------------------------------------------------------------- */

/* Replaces NTT::ComputeForward(result, operand, input_mod_factor, output_mod_factor)
 * (ntt.hpp:49, ntt.cpp:173-186).  Input in [0, 4q) (the factor is accepted and
 * ignored, as in the reference); output bit-reversed, in [0, 4q) when
 * output_mod_factor == 4, else in [0, q).  result may equal operand. */
axhel_status_t axhel_cuda_ntt_forward(axhel_ntt_t ntt, uint64_t* result, const uint64_t* operand,
                                      uint64_t input_mod_factor, uint64_t output_mod_factor, void* stream);

/* Replaces NTT::ComputeInverse (ntt.hpp:53, ntt.cpp:192-204).  Input in
 * [0, 2q), bit-reversed; output natural order, in [0, 2q) when
 * output_mod_factor == 2, else in [0, q).  input_mod_factor is ignored. */
axhel_status_t axhel_cuda_ntt_inverse(axhel_ntt_t ntt, uint64_t* result, const uint64_t* operand,
                                      uint64_t input_mod_factor, uint64_t output_mod_factor, void* stream);

/* Batched forms (new; the reference has one call per limb).  `count` limbs of
 * one degree N stored back to back (limb stride N words); limb i uses
 * ntts[i % n_ntts] (n_ntts <= 64), e.g. the RNS limbs of many ciphertexts in
 * [ciphertext][polynomial][limb][N] order.  Each limb's result equals the
 * single-call result bit for bit.  One launch per pass covers all limbs. */
axhel_status_t axhel_cuda_ntt_forward_batch(const axhel_ntt_t* ntts, uint64_t n_ntts, uint64_t* result,
                                            const uint64_t* operand, uint64_t count, uint64_t input_mod_factor,
                                            uint64_t output_mod_factor, void* stream);
/* As above for the inverse.  input_mod_factor == 4 additionally fuses
 * EltwiseReduceMod(4 -> 2) in front of the transform (the lazy round trip
 * ComputeForward(1,4) -> EltwiseReduceMod(4,2) -> ComputeInverse(2,·));
 * any other factor is ignored as in the reference. */
axhel_status_t axhel_cuda_ntt_inverse_batch(const axhel_ntt_t* ntts, uint64_t n_ntts, uint64_t* result,
                                            const uint64_t* operand, uint64_t count, uint64_t input_mod_factor,
                                            uint64_t output_mod_factor, void* stream);

/* Fused INTT -> MulMod -> NTT over a batch (new; one kernel chain replaces
 *   ComputeInverse(x, x, in_f, 2); EltwiseMulMod(x, x, m, N, q, 2);
 *   ComputeForward(x, x, 1, out_f)
 * per limb).  `multiplicand` has the same layout as `operand`, values in
 * [0, 2q).  in_f == 4 fuses EltwiseReduceMod(4,2) ahead of the inverse. */
axhel_status_t axhel_cuda_ntt_chain_mul_batch(const axhel_ntt_t* ntts, uint64_t n_ntts, uint64_t* result,
                                              const uint64_t* operand, const uint64_t* multiplicand, uint64_t count,
                                              uint64_t input_mod_factor, uint64_t output_mod_factor, void* stream);

/* Forward transform then dyadic product over a batch (new; SEAL's
 * dyadic_product_coeffmod on a freshly transformed operand, fused into the
 * transform's last pass): replaces, per limb,
 *   ComputeForward(r, x, in_f, 4); EltwiseMulMod(r, r, m, N, q, 4)
 * (ntt.cpp:173-186, eltwise-mul-mod.cpp:18-94).  Inputs in [0, 4q);
 * `multiplicand` (device, the layout of operand, values in [0, 4q), in the
 * forward's bit-reversed order) must not be `result`.  Output [0, q). */
axhel_status_t axhel_cuda_ntt_forward_mul_batch(const axhel_ntt_t* ntts, uint64_t n_ntts, uint64_t* result,
                                                const uint64_t* operand, const uint64_t* multiplicand,
                                                uint64_t count, void* stream);
/* Dyadic product then inverse transform over a batch (new; the product
 * fused into the inverse's first pass): replaces, per limb,
 *   EltwiseMulMod(r, x, m, N, q, 4); ComputeInverse(r, r, 2, out_f)
 * (eltwise-mul-mod.cpp:18-94, ntt.cpp:192-204).  Operand and `multiplicand`
 * in [0, 4q), bit-reversed order; `multiplicand` must not be `result`.
 * Output natural order, [0, 2q) for out_f == 2, else [0, q). */
axhel_status_t axhel_cuda_ntt_mul_inverse_batch(const axhel_ntt_t* ntts, uint64_t n_ntts, uint64_t* result,
                                                const uint64_t* operand, const uint64_t* multiplicand,
                                                uint64_t count, uint64_t output_mod_factor, void* stream);

/* Fused NTT -> MulMod -> INTT over a batch (new; the polynomial product in
 * evaluation form, SEAL's multiply_plain): one kernel chain replaces
 *   ComputeForward(x, x, in_f, 4); EltwiseMulMod(x, x, m, N, q, 4);
 *   ComputeInverse(x, x, 2, out_f)
 * per limb (ntt.cpp:173-204, eltwise-mul-mod.cpp:18-94): the forward's last
 * pass, the dyadic product and the inverse's first pass run as one pass.
 * Inputs in [0, 4q); `multiplicand` (device, the layout of operand, values
 * in [0, 4q), in the forward's bit-reversed order) must not be `result`.
 * Output natural order, [0, 2q) for out_f == 2, else [0, q). */
axhel_status_t axhel_cuda_ntt_product_batch(const axhel_ntt_t* ntts, uint64_t n_ntts, uint64_t* result,
                                            const uint64_t* operand, const uint64_t* multiplicand, uint64_t count,
                                            uint64_t input_mod_factor, uint64_t output_mod_factor, void* stream);

/* Fused INTT -> FMAMod -> NTT (new):
 *   ComputeInverse(x, x, in_f, 2); EltwiseFMAMod(x, x, scalars[i % n_ntts], addend_or_null, N, q, 2);
 *   ComputeForward(x, x, 1, out_f)
 * scalars is a HOST array of n_ntts values in [0, 2q); addend (device, same
 * layout as operand, values in [0, 2q)) may be NULL. */
axhel_status_t axhel_cuda_ntt_chain_fma_batch(const axhel_ntt_t* ntts, uint64_t n_ntts, uint64_t* result,
                                              const uint64_t* operand, const uint64_t* scalars, const uint64_t* addend,
                                              uint64_t count, uint64_t input_mod_factor, uint64_t output_mod_factor,
                                              void* stream);

/* ---------------------------------------------------------------------- */
/* Uneven batches in one persistent launch (new)                          */
/* ---------------------------------------------------------------------- */

#define AXHEL_JOB_FORWARD 1u   /* ComputeForward(in_f, out_f) on every limb */
#define AXHEL_JOB_INVERSE 2u   /* ComputeInverse; in_f == 4 fuses ReduceMod(4,2) on load */
#define AXHEL_JOB_CHAIN_MUL 3u /* ComputeInverse(in_f,2) -> MulMod(., vector, 2) -> ComputeForward(1,out_f) */
#define AXHEL_JOB_CHAIN_FMA 4u /* ComputeInverse(in_f,2) -> FMAMod(., scalars[m], vector|NULL, 2) -> ComputeForward */
/* Element-wise jobs: the reference's eltwise call on every limb, limb i with
 * the modulus of ntts[i % n_ntts].  Replace the per-limb loops over
 * EltwiseAddMod / EltwiseSubMod (eltwise-add-mod.hpp:13,17,
 * eltwise-sub-mod.hpp:13,17), EltwiseMulMod (eltwise-mul-mod.hpp:14),
 * EltwiseFMAMod (eltwise-fma-mod.hpp:15) and EltwiseReduceMod
 * (eltwise-reduce-mod.hpp:14). */
#define AXHEL_JOB_ADD 5u    /* AddMod(result, operand, vector) or, vector NULL, (operand, scalars[m]) */
#define AXHEL_JOB_SUB 6u    /* SubMod, operands as ADD */
#define AXHEL_JOB_MUL 7u    /* MulMod(result, operand, vector, in_f), in_f in {1, 2, 4} */
#define AXHEL_JOB_FMA 8u    /* FMAMod(result, operand, scalars[m], vector | NULL, in_f), in_f in {1, 2, 4, 8} */
#define AXHEL_JOB_REDUCE 9u /* ReduceMod(result, operand, in_f, out_f): the reference's matched pairs */
/* REDUCE input factor meaning "equal to each limb's modulus": the reference's
 * Barrett branch (EltwiseReduceMod with in_f == q) for inputs of any value. */
#define AXHEL_FACTOR_MODULUS 0xFFFFFFFFFFFFFFFFull

/* One job of a batch: `count` limbs of one degree N (2^10 <= N <= 2^17)
 * stored back to back, limb i using ntts[i % n_ntts]; result/operand/vector
 * are DEVICE pointers (result may equal operand), scalars a HOST array of
 * n_ntts values (chain FMA, FMA, and ADD/SUB without a vector).  Factors the
 * reference would silently ignore (a MulMod factor of 3, an unmatched
 * ReduceMod pair) are refused with AXHEL_ERR_INVALID when the batch is
 * built. */
typedef struct axhel_job {
    uint32_t kind;
    uint32_t n_ntts;
    const axhel_ntt_t* ntts;
    uint64_t count;
    uint64_t* result;
    const uint64_t* operand;
    const uint64_t* vector;
    const uint64_t* scalars;
    uint64_t input_mod_factor;
    uint64_t output_mod_factor;
} axhel_job_t;

typedef struct axhel_batch* axhel_batch_t;

/* Builds the device descriptors of a batch of jobs of mixed degree, limb
 * count and kind (owned by the batch; the NTT handles are retained).  Each
 * job's result equals the per-limb reference call sequence bit for bit. */
axhel_status_t axhel_cuda_batch_create(const axhel_job_t* jobs, uint64_t n_jobs, axhel_batch_t* out);
/* Runs the whole batch as ONE persistent kernel launch on `stream` (after
 * clearing its counters); may be captured into a CUDA graph. */
axhel_status_t axhel_cuda_batch_launch(axhel_batch_t batch, void* stream);
/* Same, through a CUDA graph instantiated on first use and replayed after. */
axhel_status_t axhel_cuda_batch_graph_launch(axhel_batch_t batch, void* stream);
/* Runs the batch as ordinary launches, phase after phase: one per (phase,
 * tile class, pass width), each a grid of that class's tiles of all jobs,
 * plus one for each of a phase's largest jobs; one CTA per tile, no waits
 * inside a launch; same results.  A phase's launches run side by side on
 * three streams the batch creates on its first call outside a stream
 * capture, forked from `stream` by an event and joined back into it; may be
 * captured into a CUDA graph on `stream`. */
axhel_status_t axhel_cuda_batch_launch_phased(axhel_batch_t batch, void* stream);
/* Waits for `stream` and returns AXHEL_ERR_TIMEOUT if a dependency wait
 * inside the kernel gave up (bounded at 2 s), else AXHEL_OK. */
axhel_status_t axhel_cuda_batch_status(axhel_batch_t batch, void* stream);
axhel_status_t axhel_cuda_batch_destroy(axhel_batch_t batch);
/* create + launch + status + destroy (synchronous). */
axhel_status_t axhel_cuda_batch_run(const axhel_job_t* jobs, uint64_t n_jobs, void* stream);
/* Message of the last batch failure on the calling thread. */
const char* axhel_cuda_batch_last_error(void);
/* Bound of every dependency wait inside the batch kernel (1 ms .. 10 s;
 * default 2 s). */
axhel_status_t axhel_cuda_batch_set_wait_ns(axhel_batch_t batch, uint64_t ns);
/* No counterpart in the reference.  axhel_cuda_batch_run without any device
 * allocation, for callers that cannot call cudaMalloc while they run (a
 * process whose HBM is reserved up front by its own allocator or a fixed
 * budget; a latency-critical loop where cudaMalloc/cudaFree would
 * synchronize the device).  The batch's descriptors and counters live in a
 * static 1 MiB device array per device; a batch that needs more returns
 * AXHEL_ERR_UNSUPPORTED.  The first call on a device resolves that array's
 * address (make it before any stream capture); the address is kept for the
 * process, so the entry point must not be used across a cudaDeviceReset.
 * All calls share the array: calls that overlap on the GPU race and must not
 * be issued.  Each call waits for its batch to finish before it returns;
 * results equal axhel_cuda_batch_run's bit for bit. */
axhel_status_t axhel_cuda_batch_run_static(const axhel_job_t* jobs, uint64_t n_jobs, void* stream);
/* Failure-detection hook: makes every dependency of job `job` unreachable
 * (its waits run out), so the launch ends with AXHEL_ERR_TIMEOUT while the
 * device stays usable.  For tests. */
axhel_status_t axhel_cuda_batch_debug_unreachable(axhel_batch_t batch, uint64_t job);

/* ---------------------------------------------------------------------- */
/* Serving loop: continuous batching on one GPU (new)                      */
/* ---------------------------------------------------------------------- */

typedef struct axhel_server* axhel_server_t;

#define AXHEL_SERVER_PERSISTENT 1u /* run each batch as one persistent launch (default: one launch per phase) */
/* Batches in flight get stream priorities in launch order (the oldest the
 * highest), so the GPU dispatches their tiles first come first served
 * instead of sharing the SMs between them. */
#define AXHEL_SERVER_ARRIVAL_PRIORITY 2u
/* Admission takes the smallest pending requests first (fewest residues);
 * a request pending longer than aging_us goes ahead of them in arrival
 * order, so large requests are not starved. */
#define AXHEL_SERVER_SMALLEST_FIRST 4u
/* With two lanes (small_request_words > 0), the lane of the LARGER requests
 * gets the high stream priority instead of the small one: the largest
 * requests, which set the latency tail, pass the small ones on the SMs. */
#define AXHEL_SERVER_LARGE_FIRST 8u

typedef struct axhel_server_config {
    uint64_t hbm_budget_bytes;    /* device bytes the server may hold for staged operands */
    uint64_t max_batch_words;     /* residues admitted into one batch (0 = no cap; a larger request runs alone) */
    uint64_t small_request_words; /* requests up to this many residues take the high-priority lane (0 = one lane) */
    uint32_t max_inflight;        /* batches concurrently on the GPU per lane (1..16 streams) */
    uint32_t max_batch_requests;  /* requests admitted into one batch */
    uint32_t flags;               /* AXHEL_SERVER_* */
    uint32_t aging_us;            /* AXHEL_SERVER_SMALLEST_FIRST: pending time after which arrival order wins */
    uint64_t reserve_bytes;       /* device memory mapped for staging at creation (capped at the budget; 0 = on
                                     demand): growing the pool later stalls the request that needs it */
    uint32_t batch_size_ratio;    /* a batch only takes requests within this factor of the size of its first one
                                     (0 = any size): small requests do not wait inside a large one's batch */
    uint32_t reserved;
} axhel_server_config_t;

/* One request: a job of the batch engine (AXHEL_JOB_*).  input / output /
 * vector may be HOST memory (staged by the server; pinned memory keeps the
 * copies asynchronous) or DEVICE memory (used in place).  Buffers must stay
 * valid until axhel_server_wait returns for the request. */
typedef struct axhel_request {
    uint32_t kind;
    uint32_t n_ntts;
    const axhel_ntt_t* ntts;
    uint64_t count;
    const uint64_t* input;
    uint64_t* output;
    const uint64_t* vector;
    const uint64_t* scalars;
    uint64_t input_mod_factor;
    uint64_t output_mod_factor;
} axhel_request_t;

typedef struct axhel_request_info {
    int32_t status;       /* AXHEL_OK, AXHEL_ERR_CANCELLED, AXHEL_ERR_TIMEOUT, ... */
    uint32_t batch_size;  /* requests in the launch that ran it */
    uint64_t batch_id;
    double queue_ms;      /* submit -> admitted */
    double latency_ms;    /* submit -> result available */
} axhel_request_info_t;

typedef struct axhel_server_stats {
    uint64_t completed, batches, max_batch_requests, pending, in_use_bytes, peak_in_use_bytes, samples;
    double p50_ms, p99_ms;    /* submit -> done latency over completed requests */
    uint64_t pool_used_bytes; /* device bytes allocated from the staging pool now (frees land in stream order) */
    double host_us_per_batch; /* mean scheduler time per batch: staging, descriptors, launches */
} axhel_server_stats_t;

/* Starts the scheduler and completion threads on the current device. */
axhel_status_t axhel_server_create(const axhel_server_config_t* config, axhel_server_t* out);
/* Queues a request; returns at once with its id.  AXHEL_ERR_REJECTED if the
 * request alone needs more device memory than the budget. */
axhel_status_t axhel_server_submit(axhel_server_t server, const axhel_request_t* request, uint64_t* id);
/* Waits (at most timeout_us) for a request; on completion returns its status
 * and forgets it.  AXHEL_ERR_TIMEOUT if still pending or running. */
axhel_status_t axhel_server_wait(axhel_server_t server, uint64_t id, uint64_t timeout_us, axhel_request_info_t* info);
/* Cancels a request that has not been admitted yet (AXHEL_ERR_BUSY otherwise). */
axhel_status_t axhel_server_cancel(axhel_server_t server, uint64_t id);
/* Holds (1) or resumes (0) admission; running batches are unaffected. */
axhel_status_t axhel_server_pause(axhel_server_t server, int paused);
axhel_status_t axhel_server_stats(axhel_server_t server, axhel_server_stats_t* out, int reset_latencies);
/* Stops admission, drains the batches in flight, frees everything. */
axhel_status_t axhel_server_destroy(axhel_server_t server);

/* Load driver (new; a measuring tool for the serving loop): submits requests
 * drawn uniformly from `templates` at Poisson arrival times of mean rate
 * `rate_per_s` for `seconds`, from one C++ thread, and waits for all of
 * them.  Template t writes its result to outputs[t * copies + c] for a copy c
 * not in use by another in-flight request of the same template (an arrival
 * finding none free is skipped and counted).  isolated_ms[t] (may be NULL)
 * is the template's latency alone, for the slowdown percentiles. */
typedef struct axhel_drive_result {
    uint64_t submitted, completed, skipped, failed;
    double wall_s, jobs_per_s;
    double p50_ms, p99_ms, p50_slowdown, p99_slowdown, isolated_p99_ms;
    double p50_queue_ms, p99_queue_ms; /* submit -> admitted into a batch */
    double p99_large_ms;               /* p99 latency of the templates in the top quarter of isolated latency */
    double p99_rest_ms;                /* p99 latency of the other templates */
} axhel_drive_result_t;
axhel_status_t axhel_server_drive(axhel_server_t server, const axhel_request_t* templates, uint32_t n_templates,
                                  uint64_t* const* outputs, uint32_t copies, const double* isolated_ms,
                                  double rate_per_s, double seconds, uint64_t seed, axhel_drive_result_t* out);
const char* axhel_server_last_error(void);
/* Failure-injection hook (new; for tests): staging of the next batch fails
 * at its request `request` (0-based, in admission order) as a device
 * allocation failure would, after the requests before it were staged.  The
 * batch's requests end with AXHEL_ERR_NOMEM and every buffer already staged
 * for them goes back to the pool. */
axhel_status_t axhel_server_debug_fail_staging(axhel_server_t server, uint32_t request);

/* ---------------------------------------------------------------------- */
/* Element-wise (device pointers); result may alias any operand.           */
/* ---------------------------------------------------------------------- */

/* EltwiseAddMod vector-vector / vector-scalar (axhel/include/axhel/eltwise/eltwise-add-mod.hpp:13,17). */
axhel_status_t axhel_cuda_eltwise_add_vv(uint64_t* result, const uint64_t* operand1, const uint64_t* operand2,
                                         uint64_t n, uint64_t modulus, void* stream);
axhel_status_t axhel_cuda_eltwise_add_vs(uint64_t* result, const uint64_t* operand1, uint64_t operand2, uint64_t n,
                                         uint64_t modulus, void* stream);
/* EltwiseSubMod (eltwise-sub-mod.hpp:13,17). */
axhel_status_t axhel_cuda_eltwise_sub_vv(uint64_t* result, const uint64_t* operand1, const uint64_t* operand2,
                                         uint64_t n, uint64_t modulus, void* stream);
axhel_status_t axhel_cuda_eltwise_sub_vs(uint64_t* result, const uint64_t* operand1, uint64_t operand2, uint64_t n,
                                         uint64_t modulus, void* stream);
/* EltwiseMulMod (eltwise-mul-mod.hpp:14); mod_factor 1, 2 or 4, any other
 * value writes nothing (eltwise-mul-mod.cpp:83-93) and returns AXHEL_OK. */
axhel_status_t axhel_cuda_eltwise_mul(uint64_t* result, const uint64_t* operand1, const uint64_t* operand2,
                                      uint64_t n, uint64_t modulus, uint64_t mod_factor, void* stream);
/* EltwiseFMAMod (eltwise-fma-mod.hpp:15); op3 may be NULL; mod_factor 1, 2, 4 or 8. */
axhel_status_t axhel_cuda_eltwise_fma(uint64_t* result, const uint64_t* operand1, uint64_t operand2,
                                      const uint64_t* operand3, uint64_t n, uint64_t modulus, uint64_t mod_factor,
                                      void* stream);
/* EltwiseReduceMod (eltwise-reduce-mod.hpp:14); the (in, out) pairs of
 * eltwise-reduce-mod.cpp:32-128, including the Barrett form in_factor == modulus;
 * an unmatched pair writes nothing. */
axhel_status_t axhel_cuda_eltwise_reduce(uint64_t* result, const uint64_t* operand, uint64_t n, uint64_t modulus,
                                         uint64_t input_mod_factor, uint64_t output_mod_factor, void* stream);

/* Fused tensor product of two ciphertexts (new; replaces the per-limb call
 * sequence t0 = MulMod(c0,d0); t1 = MulMod(c0,d1); u = MulMod(c1,d0);
 * t1 = AddMod(t1,u); t2 = MulMod(c1,d1) with factor `mod_factor`, then
 * ReduceMod(·,4,1)).  Inputs: `count` limbs of n words each, stored back to back;
 * limb i uses moduli[i % n_moduli] (HOST array, n_moduli <= 64). */
axhel_status_t axhel_cuda_tensor_product(uint64_t* r0, uint64_t* r1, uint64_t* r2, const uint64_t* c0,
                                         const uint64_t* c1, const uint64_t* d0, const uint64_t* d1, uint64_t n,
                                         uint64_t count, const uint64_t* moduli, uint64_t n_moduli,
                                         uint64_t mod_factor, void* stream);

/* ---------------------------------------------------------------------- */
/* Plans: autotuned pass configuration                                    */
/* ---------------------------------------------------------------------- */

/* Force the pass split for (inverse, log2 N): npass passes of lg[i] stages
 * (sum == log2 N), lr[i] register stages and tg[i] groups per CTA.
 * npass == 0 restores the default.  Used by the autotuner. */
axhel_status_t axhel_cuda_plan_set(int inverse, uint32_t log_degree, uint32_t npass, const uint32_t* lg,
                                   const uint32_t* lr, const uint32_t* tg);
/* Reads the plan used for (inverse, log2 N, count limbs); arrays of >= 3. */
axhel_status_t axhel_cuda_plan_get(int inverse, uint32_t log_degree, uint64_t count, uint32_t* npass, uint32_t* lg,
                                   uint32_t* lr, uint32_t* tg);
/* Single-launch forms of a few limbs (new; no counterpart in the reference,
 * whose transforms run on the host): one thread-block cluster of `csize` CTAs
 * (2..16) per limb, the passes exchanging the limb through the cluster's
 * shared memory instead of HBM.  `kind`: 0 forward and 1 inverse transforms
 * (`lga` first-pass stages), 2 the INTT -> MulMod/FMAMod -> NTT chains and
 * 3 the NTT -> MulMod -> INTT product (`lga` stages in the contiguous
 * groups); `lr` register stages.  Used for 2^10 <= N <= 2^17 and count <=
 * max_limbs; max_limbs == 0 turns it off for (kind, log2 N), lga == 0
 * restores the built-in choice.  A pass plan set by axhel_cuda_plan_set for
 * the same degree (the inverse plan, for kinds 2 and 3) takes precedence.
 * Every choice computes the same bits. */
axhel_status_t axhel_cuda_cluster_plan_set(int kind, uint32_t log_degree, uint32_t lga, uint32_t lr,
                                           uint32_t csize, uint64_t max_limbs);
axhel_status_t axhel_cuda_cluster_plan_get(int kind, uint32_t log_degree, uint32_t* lga, uint32_t* lr,
                                           uint32_t* csize, uint64_t* max_limbs);
/* Loads an autotuner table (text, one plan per line); NULL = the table shipped
 * beside the library.  Returns the number of plans loaded via *loaded. */
axhel_status_t axhel_cuda_plan_load(const char* path, uint32_t* loaded);
/* Uneven-batch engine (new): stages of the contiguous pass of an N = 2^log_degree
 * job (the strided pass takes the rest), in [max(5, log N - 9), min(9, log N - 5)];
 * 0 restores the table / default.  Applies to batches created afterwards.
 * Used by the autotuner; every split computes the same bits. */
axhel_status_t axhel_cuda_batch_split_set(uint32_t log_degree, uint32_t row_stages);
axhel_status_t axhel_cuda_batch_split_get(uint32_t log_degree, uint32_t* row_stages);

/* ---------------------------------------------------------------------- */
/* Host-pointer helpers used by the C++ drop-in                           */
/* ---------------------------------------------------------------------- */

/* 1 if p is device (or managed) memory visible to the current device. */
int axhel_cuda_is_device_pointer(const void* p);
/* Number of kernel launches issued by this library since load (all threads). */
uint64_t axhel_cuda_launch_count(void);

/* Per-kernel device timing: while enabled, each launch of this library is
 * bracketed by CUDA events on its own stream.  The report (one line per
 * kernel configuration: "<name...> <launches> <total_ms>") drains the
 * records; *needed receives the buffer size required. */
axhel_status_t axhel_cuda_profile_enable(int on);

/* Compute-roofline probe (new): the reference's forward (inverse = 0) or
 * inverse butterfly, on values held in registers with the twiddles of `ntt`,
 * over a full-device grid; returns the measured butterflies per second.  An
 * N-point transform needs (N/2) log2 N butterflies. */
axhel_status_t axhel_cuda_butterfly_peak(axhel_ntt_t ntt, int inverse, double* butterflies_per_s, void* stream);
axhel_status_t axhel_cuda_profile_report(char* buf, uint64_t len, uint64_t* needed);

#ifdef __cplusplus
}
#endif

#endif /* AXHEL_CUDA_H */
