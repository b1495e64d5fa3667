/*
 * CPU oracle for the AXHEL hot path (plain C restatement).
 *
 * TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the
 * bench's CPU-baseline leg as the checker; never linked into or called by the
 * shipped CUDA library.  Each function cites the reference file:line whose
 * algorithm it restates (paths relative to the AXHEL project root).
 *
 * Parity pin: the restatement is checked against (1) the reference's own
 * known-answer vectors (tests/public/test_ntt.cpp:32-46, the explicit N=8
 * tables of example/example.cpp:314-345) and (2) the reference native backend
 * compiled from its sources into oracle/_ref (see oracle/Makefile), on seeded
 * inputs, by tests/test_oracle.py and tests/golden/make_golden.py.
 */
#include "axhel_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

typedef unsigned __int128 u128;

/* ---------------------------------------------------------------------- */
/* number theory                                                          */
/* ---------------------------------------------------------------------- */

/* BitWidth: axhel/include/axhel/number-theory/uint-arith.hpp:25-27 */
uint64_t orc_bit_width(uint64_t x) { return x ? 64u - (uint64_t)__builtin_clzll(x) : 0; }

/* MulHighU64: uint-arith.hpp:40-44 */
uint64_t orc_mul_hi(uint64_t a, uint64_t b) { return (uint64_t)(((u128)a * b) >> 64); }

/* MultiplyUIntModLazy: uint-arith.hpp:48-52.  Result in [0, 2q). */
uint64_t orc_shoup_lazy(uint64_t value, uint64_t w, uint64_t w_quot, uint64_t q)
{
    uint64_t est = orc_mul_hi(value, w_quot);
    return value * w - est * q;
}

/* ComputeShoupQuotient: uint-arith.hpp:56-60, floor(w * 2^64 / q). */
uint64_t orc_shoup_quotient(uint64_t w, uint64_t q) { return (uint64_t)(((u128)w << 64) / q); }

/* ConditionalSubtractNative: modular-reduction.hpp:22-25 */
static inline uint64_t csub(uint64_t x, uint64_t bound) { return x >= bound ? x - bound : x; }

/* ReduceInputNative<F>: modular-reduction.hpp:48-67 (cascade 8->4->2->1). */
uint64_t orc_reduce_input(uint64_t x, uint64_t q, uint64_t factor)
{
    if (factor == 8) x = csub(x, 4 * q);
    if (factor >= 4) x = csub(x, 2 * q);
    if (factor >= 2) x = csub(x, q);
    return x;
}

/* Barrett factor: multiply-factor.cpp:11-19 called as in eltwise-mul-mod.cpp:25-30
 * (alpha = 62, beta = -2): mu = floor(2^(k-2) * 2^64 / q), k = BitWidth(q). */
uint64_t orc_barrett_factor(uint64_t q)
{
    uint64_t k = orc_bit_width(q);
    return (uint64_t)(((u128)((uint64_t)1 << (k - 2)) << 64) / q);
}

/* floor(hi:lo / 2^shift) truncated to 64 bits (eltwise-mul-mod.cpp:48). */
static inline uint64_t shift_right_128(uint64_t hi, uint64_t lo, uint64_t shift)
{
    return shift ? (lo >> shift) | (hi << (64 - shift)) : lo;
}

/* One Barrett product as in eltwise-mul-mod.cpp:40-60; x, y already in [0,q). */
static inline uint64_t barrett_mul(uint64_t x, uint64_t y, uint64_t q, uint64_t mu, uint64_t shift)
{
    u128 prod = (u128)x * y;
    uint64_t lo = (uint64_t)prod, hi = (uint64_t)(prod >> 64);
    uint64_t c1 = shift_right_128(hi, lo, shift);
    uint64_t qhat = orc_mul_hi(c1, mu);
    uint64_t z = lo - qhat * q;
    return orc_reduce_input(z, q, 4);
}

/* ---------------------------------------------------------------------- */
/* tables                                                                 */
/* ---------------------------------------------------------------------- */

/* PowMod: axhel/ntt/ntt-tables.cpp:24-41 */
static uint64_t table_pow_mod(uint64_t base, uint64_t e, uint64_t q)
{
    uint64_t r = 1;
    base %= q;
    while (e) {
        if (e & 1) r = (uint64_t)(((u128)r * base) % q);
        e >>= 1;
        if (e) base = (uint64_t)(((u128)base * base) % q);
    }
    return r;
}

/* NextBitReversedIndex: ntt-tables.cpp:54-65 (bit-reversed increment). */
static uint64_t next_bitrev(uint64_t cur, uint64_t n)
{
    uint64_t bit = n >> 1;
    while (cur & bit) { cur ^= bit; bit >>= 1; }
    return cur ^ bit;
}

/* GenerateNTTTables: ntt-tables.cpp:81-140.
 *   fwd[i]  = psi^bitrev(i)                         (i = 0..N-1)
 *   inv[0]  = {0, 0};  inv[i] = psi^-(bitrev(i-1)+1) (i = 1..N-1)
 *   ninv    = N^-1 mod q
 * each stored as {operand, Shoup quotient}. */
int orc_ntt_tables(uint64_t n, uint64_t q, uint64_t psi, uint64_t* fwd, uint64_t* inv, uint64_t* ninv)
{
    uint64_t* seq = (uint64_t*)malloc(n * sizeof(uint64_t));
    if (!seq) return -1;
    seq[0] = 1;
    for (uint64_t i = 1; i < n; ++i) seq[i] = (uint64_t)(((u128)seq[i - 1] * psi) % q);
    uint64_t rev = 0;
    for (uint64_t i = 0; i < n; ++i) {
        fwd[2 * i] = seq[rev];
        fwd[2 * i + 1] = orc_shoup_quotient(seq[rev], q);
        if (i + 1 < n) rev = next_bitrev(rev, n);
    }
    uint64_t psi_inv = table_pow_mod(psi, q - 2, q);
    seq[0] = 1;
    for (uint64_t i = 1; i < n; ++i) seq[i] = (uint64_t)(((u128)seq[i - 1] * psi_inv) % q);
    inv[0] = 0;
    inv[1] = 0;
    rev = 0;
    for (uint64_t i = 1; i < n; ++i) {
        uint64_t w = seq[rev + 1];
        inv[2 * i] = w;
        inv[2 * i + 1] = orc_shoup_quotient(w, q);
        if (i + 1 < n) rev = next_bitrev(rev, n);
    }
    uint64_t d = table_pow_mod(n % q, q - 2, q);
    ninv[0] = d;
    ninv[1] = orc_shoup_quotient(d, q);
    free(seq);
    return 0;
}

/* ---------------------------------------------------------------------- */
/* NTT                                                                    */
/* ---------------------------------------------------------------------- */

/* NTTNegacyclicHarveyLazyNative: axhel/ntt/ntt-native.cpp:19-55 with the
 * butterfly ForwardButterflyNative of axhel/ntt/ntt-internal.hpp:20-31. */
void orc_ntt_forward_lazy(uint64_t* x, uint64_t n, uint64_t q, const uint64_t* fwd)
{
    const uint64_t q2 = q << 1;
    for (uint64_t m = 1, gap = n >> 1; m < n; m <<= 1, gap >>= 1) {
        for (uint64_t i = 0; i < m; ++i) {
            const uint64_t w = fwd[2 * (m + i)], wq = fwd[2 * (m + i) + 1];
            uint64_t* xp = x + i * 2 * gap;
            uint64_t* yp = xp + gap;
            for (uint64_t j = 0; j < gap; ++j) {
                uint64_t gx = csub(xp[j], q2);
                uint64_t t = orc_shoup_lazy(yp[j], w, wq, q);
                xp[j] = gx + t;
                yp[j] = gx + q2 - t;
            }
        }
    }
}

/* InverseNTTNegacyclicHarveyLazyNative: ntt-native.cpp:61-142 with the
 * butterfly InverseButterflyNative of ntt-internal.hpp:37-49 and the final
 * stage that folds in N^-1 (ntt-native.cpp:101-141). */
void orc_ntt_inverse_lazy(uint64_t* x, uint64_t n, uint64_t q, const uint64_t* inv, const uint64_t* ninv)
{
    const uint64_t q2 = q << 1;
    uint64_t root = 1, m = n >> 1, gap = 1;
    for (; m > 1; m >>= 1, gap <<= 1) {
        for (uint64_t i = 0; i < m; ++i, ++root) {
            const uint64_t w = inv[2 * root], wq = inv[2 * root + 1];
            uint64_t* xp = x + i * 2 * gap;
            uint64_t* yp = xp + gap;
            for (uint64_t j = 0; j < gap; ++j) {
                uint64_t u = xp[j], v = yp[j];
                xp[j] = csub(u + v, q2);
                yp[j] = orc_shoup_lazy(u + q2 - v, w, wq, q);
            }
        }
    }
    /* scaled root = reduce2->1(Shoup(w_last, N^-1)) with a fresh quotient */
    uint64_t sr = orc_shoup_lazy(inv[2 * root], ninv[0], ninv[1], q);
    sr = csub(sr, q);
    const uint64_t srq = orc_shoup_quotient(sr, q);
    uint64_t* xp = x;
    uint64_t* yp = x + gap;
    for (uint64_t j = 0; j < gap; ++j) {
        uint64_t gx = csub(xp[j], q2);
        uint64_t y = yp[j];
        xp[j] = orc_shoup_lazy(gx + y, ninv[0], ninv[1], q);
        yp[j] = orc_shoup_lazy(gx + q2 - y, sr, srq, q);
    }
}

/* NTT::ComputeForward: axhel/ntt/ntt.cpp:173-186 (input factor unused; any
 * output factor other than 4 normalizes with ReduceMod 4->1, ntt.cpp:79-91). */
void orc_ntt_compute_forward(uint64_t* res, const uint64_t* op, uint64_t n, uint64_t q,
                             const uint64_t* fwd, uint64_t in_f, uint64_t out_f)
{
    (void)in_f;
    if (res != op) memmove(res, op, n * sizeof(uint64_t));
    orc_ntt_forward_lazy(res, n, q, fwd);
    if (out_f != 4) orc_reduce(res, res, n, q, 4, 1);
}

/* NTT::ComputeInverse: ntt.cpp:192-204 (output factor 2 = lazy, otherwise
 * ReduceMod 2->1, ntt.cpp:106-118). */
void orc_ntt_compute_inverse(uint64_t* res, const uint64_t* op, uint64_t n, uint64_t q,
                             const uint64_t* inv, const uint64_t* ninv, uint64_t in_f, uint64_t out_f)
{
    (void)in_f;
    if (res != op) memmove(res, op, n * sizeof(uint64_t));
    orc_ntt_inverse_lazy(res, n, q, inv, ninv);
    if (out_f != 2) orc_reduce(res, res, n, q, 2, 1);
}

typedef struct {
    uint64_t *res;
    const uint64_t* op;
    uint64_t n, begin, end, nq, in_f, out_f;
    const uint64_t* qs;
    const uint64_t* const* fwds;
} fwd_batch_arg;

static void* fwd_batch_worker(void* p)
{
    fwd_batch_arg* a = (fwd_batch_arg*)p;
    for (uint64_t i = a->begin; i < a->end; ++i) {
        uint64_t k = i % a->nq;
        orc_ntt_compute_forward(a->res + i * a->n, a->op + i * a->n, a->n, a->qs[k], a->fwds[k],
                                a->in_f, a->out_f);
    }
    return NULL;
}

void orc_ntt_forward_batch(uint64_t* res, const uint64_t* op, uint64_t n, uint64_t count,
                           const uint64_t* qs, const uint64_t* const* fwds, uint64_t nq,
                           uint64_t in_f, uint64_t out_f, int threads)
{
    if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (threads < 1) threads = 1;
    if ((uint64_t)threads > count) threads = (int)(count ? count : 1);
    pthread_t tid[256];
    fwd_batch_arg args[256];
    if (threads > 256) threads = 256;
    for (int t = 0; t < threads; ++t) {
        fwd_batch_arg a = {res, op, n, count * t / threads, count * (t + 1) / threads, nq, in_f, out_f, qs, fwds};
        args[t] = a;
        pthread_create(&tid[t], NULL, fwd_batch_worker, &args[t]);
    }
    for (int t = 0; t < threads; ++t) pthread_join(tid[t], NULL);
}

/* ---------------------------------------------------------------------- */
/* element-wise                                                           */
/* ---------------------------------------------------------------------- */

/* EltwiseAddModNative (vector-vector / vector-scalar): eltwise-add-mod.cpp:15-47 */
void orc_add_vv(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q)
{
    for (uint64_t i = 0; i < n; ++i) { uint64_t s = a[i] + b[i]; r[i] = s - (uint64_t)(s >= q) * q; }
}
void orc_add_vs(uint64_t* r, const uint64_t* a, uint64_t b, uint64_t n, uint64_t q)
{
    for (uint64_t i = 0; i < n; ++i) { uint64_t s = a[i] + b; r[i] = s - (uint64_t)(s >= q) * q; }
}

/* EltwiseSubModNative: eltwise-sub-mod.cpp:15-47 */
void orc_sub_vv(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q)
{
    for (uint64_t i = 0; i < n; ++i) { uint64_t x = a[i], y = b[i]; r[i] = x - y + (uint64_t)(x < y) * q; }
}
void orc_sub_vs(uint64_t* r, const uint64_t* a, uint64_t b, uint64_t n, uint64_t q)
{
    for (uint64_t i = 0; i < n; ++i) { uint64_t x = a[i]; r[i] = x - b + (uint64_t)(x < b) * q; }
}

/* EltwiseMulMod: dispatch eltwise-mul-mod.cpp:81-94 (factors 1, 2, 4; any
 * other factor writes nothing), kernel EltwiseMulModNative eltwise-mul-mod.cpp:18-63. */
void orc_mul(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q, uint64_t factor)
{
    if (factor != 1 && factor != 2 && factor != 4) return;
    const uint64_t mu = orc_barrett_factor(q), shift = orc_bit_width(q) - 2;
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t x = orc_reduce_input(a[i], q, factor);
        uint64_t y = orc_reduce_input(b[i], q, factor);
        r[i] = barrett_mul(x, y, q, mu, shift);
    }
}

/* EltwiseFMAMod: dispatch eltwise-fma-mod.cpp:96-112 (factors 1, 2, 4, 8),
 * kernel EltwiseFMAModNative eltwise-fma-mod.cpp:18-78. */
void orc_fma(uint64_t* r, const uint64_t* a, uint64_t s, const uint64_t* c, uint64_t n, uint64_t q,
             uint64_t factor)
{
    if (factor != 1 && factor != 2 && factor != 4 && factor != 8) return;
    const uint64_t mu = orc_barrett_factor(q), shift = orc_bit_width(q) - 2;
    const uint64_t sr = orc_reduce_input(s, q, factor);
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t v = barrett_mul(orc_reduce_input(a[i], q, factor), sr, q, mu, shift);
        if (c) {
            v += orc_reduce_input(c[i], q, factor);
            if (v >= q) v -= q;
        }
        r[i] = v;
    }
}

/* EltwiseReduceModNative: eltwise-reduce-mod.cpp:32-128.  The branches are
 * tried in the reference's order; an unmatched (in, out) pair writes nothing. */
void orc_reduce(uint64_t* r, const uint64_t* a, uint64_t n, uint64_t q, uint64_t in_f, uint64_t out_f)
{
    if (in_f == 1 || (out_f == 2 && in_f <= 2)) {
        if (r != a) memmove(r, a, n * sizeof(uint64_t));
        return;
    }
    if (in_f == 2 && out_f == 1) {
        for (uint64_t i = 0; i < n; ++i) r[i] = csub(a[i], q);
        return;
    }
    if (in_f == 4 && out_f == 1) {
        for (uint64_t i = 0; i < n; ++i) r[i] = csub(csub(a[i], 2 * q), q);
        return;
    }
    if (in_f == 4 && out_f == 2) {
        for (uint64_t i = 0; i < n; ++i) r[i] = csub(a[i], 2 * q);
        return;
    }
    if (in_f == q) {
        /* BarrettReduceUInt64Native: eltwise-reduce-mod.cpp:19-29 */
        const uint64_t mu = orc_barrett_factor(q), shift = orc_bit_width(q) - 2;
        for (uint64_t i = 0; i < n; ++i) {
            uint64_t x = a[i];
            uint64_t z = x - orc_mul_hi(x >> shift, mu) * q;
            r[i] = orc_reduce_input(z, q, 4);
        }
    }
}

/* ---------------------------------------------------------------------- */
/* multi-limb call sequences (checkers for full-size batches)             */
/* ---------------------------------------------------------------------- */

/* One limb of a batch job: the reference's per-limb call sequence.
 *   kind 1: ComputeForward(in_f, out_f)                       ntt.cpp:173-186
 *   kind 2: [ReduceMod(4,2) if in_f == 4] ComputeInverse(2, out_f)  ntt.cpp:192-204
 *   kind 3: [ReduceMod(4,2)] ComputeInverse(2,2) -> MulMod(., vec, 2) -> ComputeForward(1, out_f)
 *   kind 4: [ReduceMod(4,2)] ComputeInverse(2,2) -> FMAMod(., s, vec|NULL, 2) -> ComputeForward(1, out_f)
 * The ReduceMod(4,2) ahead of the inverse is eltwise-reduce-mod.cpp:110-118. */
static void job_limb(uint32_t kind, uint64_t* res, const uint64_t* op, const uint64_t* vec, uint64_t s,
                     uint64_t n, uint64_t q, const uint64_t* fwd, const uint64_t* inv, const uint64_t* ninv,
                     uint64_t in_f, uint64_t out_f)
{
    if (kind == 1) {
        orc_ntt_compute_forward(res, op, n, q, fwd, in_f, out_f);
        return;
    }
    const uint64_t* src = op;
    if (in_f == 4) {
        orc_reduce(res, op, n, q, 4, 2);
        src = res;
    }
    if (kind == 2) {
        orc_ntt_compute_inverse(res, src, n, q, inv, ninv, 2, out_f);
        return;
    }
    orc_ntt_compute_inverse(res, src, n, q, inv, ninv, 2, 2);
    if (kind == 3)
        orc_mul(res, res, vec, n, q, 2);
    else
        orc_fma(res, res, s, vec, n, q, 2);
    orc_ntt_compute_forward(res, res, n, q, fwd, 1, out_f);
}

typedef struct {
    uint32_t kind;
    uint64_t* res;
    const uint64_t *op, *vec, *scalars, *qs;
    const uint64_t* const* fwds;
    const uint64_t* const* invs;
    const uint64_t* const* ninvs;
    uint64_t n, nq, in_f, out_f, begin, end;
} job_arg;

static void* job_worker(void* p)
{
    job_arg* a = (job_arg*)p;
    for (uint64_t i = a->begin; i < a->end; ++i) {
        const uint64_t k = i % a->nq;
        job_limb(a->kind, a->res + i * a->n, a->op + i * a->n, a->vec ? a->vec + i * a->n : NULL,
                 a->scalars ? a->scalars[k] : 0, a->n, a->qs[k], a->fwds ? a->fwds[k] : NULL,
                 a->invs ? a->invs[k] : NULL, a->ninvs ? a->ninvs[k] : NULL, a->in_f, a->out_f);
    }
    return NULL;
}

static int clamp_threads(int threads, uint64_t count)
{
    if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    if ((uint64_t)threads > count) threads = (int)(count ? count : 1);
    return threads;
}

void orc_job_batch(uint32_t kind, uint64_t* res, const uint64_t* op, const uint64_t* vec,
                   const uint64_t* scalars, uint64_t n, uint64_t count, const uint64_t* qs,
                   const uint64_t* const* fwds, const uint64_t* const* invs, const uint64_t* const* ninvs,
                   uint64_t nq, uint64_t in_f, uint64_t out_f, int threads)
{
    threads = clamp_threads(threads, count);
    pthread_t tid[256];
    job_arg args[256];
    for (int t = 0; t < threads; ++t) {
        job_arg a = {kind, res, op, vec, scalars, qs, fwds, invs, ninvs, n, nq, in_f, out_f,
                     count * t / threads, count * (t + 1) / threads};
        args[t] = a;
        pthread_create(&tid[t], NULL, job_worker, &args[t]);
    }
    for (int t = 0; t < threads; ++t) pthread_join(tid[t], NULL);
}

typedef struct {
    uint64_t *r0, *r1, *r2;
    const uint64_t *c0, *c1, *d0, *d1, *qs;
    uint64_t n, nq, factor, begin, end;
} tensor_arg;

static void* tensor_worker(void* p)
{
    tensor_arg* a = (tensor_arg*)p;
    const uint64_t n = a->n;
    uint64_t* u = (uint64_t*)malloc(n * sizeof(uint64_t));
    for (uint64_t i = a->begin; i < a->end && u; ++i) {
        const uint64_t q = a->qs[i % a->nq], o = i * n;
        orc_mul(a->r0 + o, a->c0 + o, a->d0 + o, n, q, a->factor);
        orc_mul(a->r1 + o, a->c0 + o, a->d1 + o, n, q, a->factor);
        orc_mul(u, a->c1 + o, a->d0 + o, n, q, a->factor);
        orc_add_vv(a->r1 + o, a->r1 + o, u, n, q);
        orc_mul(a->r2 + o, a->c1 + o, a->d1 + o, n, q, a->factor);
        orc_reduce(a->r0 + o, a->r0 + o, n, q, 4, 1);
        orc_reduce(a->r1 + o, a->r1 + o, n, q, 4, 1);
        orc_reduce(a->r2 + o, a->r2 + o, n, q, 4, 1);
    }
    free(u);
    return NULL;
}

void orc_tensor_batch(uint64_t* r0, uint64_t* r1, uint64_t* r2, const uint64_t* c0, const uint64_t* c1,
                      const uint64_t* d0, const uint64_t* d1, uint64_t n, uint64_t count, const uint64_t* qs,
                      uint64_t nq, uint64_t factor, int threads)
{
    threads = clamp_threads(threads, count);
    pthread_t tid[256];
    tensor_arg args[256];
    for (int t = 0; t < threads; ++t) {
        tensor_arg a = {r0, r1, r2, c0, c1, d0, d1, qs, n, nq, factor, count * t / threads,
                        count * (t + 1) / threads};
        args[t] = a;
        pthread_create(&tid[t], NULL, tensor_worker, &args[t]);
    }
    for (int t = 0; t < threads; ++t) pthread_join(tid[t], NULL);
}

/* ---------------------------------------------------------------------- */
/* reference test-suite generators: tests/common/{reference,parameters}.hpp */
/* ---------------------------------------------------------------------- */

/* pow_mod: tests/common/reference.hpp:28-36 */
uint64_t orc_pow_mod(uint64_t a, uint64_t e, uint64_t q)
{
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = (uint64_t)(((u128)r * a) % q);
        a = (uint64_t)(((u128)a * a) % q);
        e >>= 1;
    }
    return r;
}

/* is_prime64: tests/common/parameters.hpp:29-51 (deterministic Miller-Rabin). */
int orc_is_prime(uint64_t n)
{
    static const uint64_t small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    static const uint64_t bases[] = {2, 325, 9375, 28178, 450775, 9780504, 1795265022};
    if (n < 2) return 0;
    for (unsigned i = 0; i < sizeof small / sizeof small[0]; ++i)
        if (n % small[i] == 0) return n == small[i];
    uint64_t d = n - 1;
    unsigned s = 0;
    while ((d & 1) == 0) { d >>= 1; ++s; }
    for (unsigned i = 0; i < sizeof bases / sizeof bases[0]; ++i) {
        uint64_t a = bases[i];
        if (a % n == 0) continue;
        uint64_t x = orc_pow_mod(a % n, d, n);
        if (x == 1 || x == n - 1) continue;
        int composite = 1;
        for (unsigned r = 1; r < s; ++r) {
            x = (uint64_t)(((u128)x * x) % n);
            if (x == n - 1) { composite = 0; break; }
        }
        if (composite) return 0;
    }
    return 1;
}

/* find_ntt_prime: parameters.hpp:53-70 — largest prime q = 1 mod 2N below 2^bits
 * (0 when none / arguments unsupported). */
uint64_t orc_find_ntt_prime(uint64_t degree, unsigned bits)
{
    if (bits < 2 || bits >= 63) return 0;
    const uint64_t step = 2 * degree;
    const uint64_t hi = ((uint64_t)1 << bits) - 1, lo = (uint64_t)1 << (bits - 1);
    uint64_t q = hi - ((hi - 1) % step);
    while (q >= lo && q > step) {
        if (orc_is_prime(q)) return q;
        if (q < step) break;
        q -= step;
    }
    return 0;
}

/* find_ntt_prime_near: parameters.hpp:74-108 — deterministic search down from
 * lo + (hi-lo)*num/den, then upward. */
uint64_t orc_find_ntt_prime_near(uint64_t degree, unsigned bits, uint64_t num, uint64_t den)
{
    if (bits < 2 || bits >= 63 || den == 0 || num > den) return 0;
    const uint64_t step = 2 * degree;
    const uint64_t lo = (uint64_t)1 << (bits - 1), hi = ((uint64_t)1 << bits) - 1;
    const uint64_t target = lo + (uint64_t)(((u128)(hi - lo)) * num / den);
    uint64_t q = target - ((target - 1) % step);
    while (q >= lo && q > step) {
        if (orc_is_prime(q)) return q;
        if (q < lo + step) break;
        q -= step;
    }
    q = target - ((target - 1) % step);
    if (q < target) q += step;
    while (q <= hi && orc_bit_width(q) == bits) {
        if (orc_is_prime(q)) return q;
        if (q > hi - step) break;
        q += step;
    }
    return 0;
}

/* find_primitive_2n_root: parameters.hpp:110-122 — smallest generator a >= 2
 * whose power a^((q-1)/2N) has order exactly 2N. */
uint64_t orc_find_primitive_root(uint64_t degree, uint64_t q)
{
    const uint64_t order = 2 * degree, e = (q - 1) / order;
    for (uint64_t a = 2; a < 100000; ++a) {
        uint64_t psi = orc_pow_mod(a, e, q);
        if (psi != 1 && orc_pow_mod(psi, degree, q) == q - 1 && orc_pow_mod(psi, order, q) == 1) return psi;
    }
    return 0;
}

/* mt19937_64 (Matsumoto & Nishimura, 64-bit Mersenne Twister; the engine the
 * reference tests seed with test_seed(), parameters.hpp:142-146). */
#define MT_N 312
#define MT_M 156
void orc_mt64_seed(uint64_t* st, uint64_t seed)
{
    st[0] = seed;
    for (uint64_t i = 1; i < MT_N; ++i) st[i] = 6364136223846793005ULL * (st[i - 1] ^ (st[i - 1] >> 62)) + i;
    st[MT_N] = MT_N;
}

uint64_t orc_mt64_next(uint64_t* st)
{
    const uint64_t upper = 0xFFFFFFFF80000000ULL, lower = 0x7FFFFFFFULL, matrix = 0xB5026F5AA96619E9ULL;
    if (st[MT_N] >= MT_N) {
        for (int i = 0; i < MT_N; ++i) {
            uint64_t x = (st[i] & upper) | (st[(i + 1) % MT_N] & lower);
            uint64_t xa = x >> 1;
            if (x & 1) xa ^= matrix;
            st[i] = st[(i + MT_M) % MT_N] ^ xa;
        }
        st[MT_N] = 0;
    }
    uint64_t y = st[st[MT_N]++];
    y ^= (y >> 29) & 0x5555555555555555ULL;
    y ^= (y << 17) & 0x71D67FFFEDA60000ULL;
    y ^= (y << 37) & 0xFFF7EEE000000000ULL;
    y ^= y >> 43;
    return y;
}

/* bounded_random: parameters.hpp:253-263 (rejection sampling). */
uint64_t orc_bounded_random(uint64_t* st, uint64_t bound)
{
    const uint64_t threshold = (uint64_t)(-bound) % bound;
    for (;;) {
        uint64_t x = orc_mt64_next(st);
        if (x >= threshold) return x % bound;
    }
}

/* random_vector: parameters.hpp:265-270 */
void orc_random_vector(uint64_t* out, uint64_t n, uint64_t bound, uint64_t* st)
{
    for (uint64_t i = 0; i < n; ++i) out[i] = orc_bounded_random(st, bound);
}
