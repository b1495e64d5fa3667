/*
 * CPU oracle for the AXHEL hot path: a plain-C restatement of the reference's
 * native backend (negacyclic Harvey NTT/INTT, twiddle tables, element-wise
 * modular kernels) plus the reference test suite's deterministic parameter
 * and input generators.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library links, loads or
 * calls this code; it is the checker that tests, the smoke check and the
 * bench's CPU-baseline leg compare the CUDA path against.  Every function
 * names the reference file:line it restates (paths relative to the AXHEL
 * project root).  Parity pin: tests/test_oracle.py checks this restatement
 * against the reference's own known-answer vectors and against the reference
 * native backend compiled from source (oracle/_ref, built by oracle/Makefile).
 */
#ifndef AXHEL_ORACLE_H
#define AXHEL_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- number theory (axhel/include/axhel/number-theory/uint-arith.hpp) ---- */
uint64_t orc_bit_width(uint64_t x);
uint64_t orc_mul_hi(uint64_t a, uint64_t b);
uint64_t orc_shoup_lazy(uint64_t value, uint64_t w, uint64_t w_quot, uint64_t q);
uint64_t orc_shoup_quotient(uint64_t w, uint64_t q);
uint64_t orc_reduce_input(uint64_t x, uint64_t q, uint64_t factor);
uint64_t orc_barrett_factor(uint64_t q);

/* ---- tables (axhel/ntt/ntt-tables.cpp) ---- */
/* fwd/inv: 2*N words each, interleaved {operand, quotient}; ninv: 2 words. */
int orc_ntt_tables(uint64_t n, uint64_t q, uint64_t psi,
                   uint64_t* fwd, uint64_t* inv, uint64_t* ninv);

/* ---- NTT kernels (axhel/ntt/ntt-native.cpp, axhel/ntt/ntt.cpp) ---- */
void orc_ntt_forward_lazy(uint64_t* x, uint64_t n, uint64_t q, const uint64_t* fwd);
void orc_ntt_inverse_lazy(uint64_t* x, uint64_t n, uint64_t q, const uint64_t* inv,
                          const uint64_t* ninv);
void orc_ntt_compute_forward(uint64_t* res, const uint64_t* op, uint64_t n, uint64_t q,
                             const uint64_t* fwd, uint64_t in_f, uint64_t out_f);
void orc_ntt_compute_inverse(uint64_t* res, const uint64_t* op, uint64_t n, uint64_t q,
                             const uint64_t* inv, const uint64_t* ninv,
                             uint64_t in_f, uint64_t out_f);
/* Same as above over `count` independent limbs laid out back to back; limb i
 * uses modulus qs[i % nq] and tables fwds/invs/ninvs at index (i % nq).  Runs
 * on up to `threads` host threads (0 = one per online core). */
void orc_ntt_forward_batch(uint64_t* res, const uint64_t* op, uint64_t n, uint64_t count,
                           const uint64_t* qs, const uint64_t* const* fwds, uint64_t nq,
                           uint64_t in_f, uint64_t out_f, int threads);

/* ---- element-wise kernels (axhel/eltwise/eltwise-*-mod.cpp) ---- */
void orc_add_vv(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q);
void orc_add_vs(uint64_t* r, const uint64_t* a, uint64_t b, uint64_t n, uint64_t q);
void orc_sub_vv(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q);
void orc_sub_vs(uint64_t* r, const uint64_t* a, uint64_t b, uint64_t n, uint64_t q);
void orc_mul(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q,
             uint64_t factor);
void orc_fma(uint64_t* r, const uint64_t* a, uint64_t s, const uint64_t* c, uint64_t n,
             uint64_t q, uint64_t factor);
void orc_reduce(uint64_t* r, const uint64_t* a, uint64_t n, uint64_t q, uint64_t in_f,
                uint64_t out_f);

/* ---- multi-limb call sequences (full-size batch checkers) ---- */
/* One job of `count` limbs stored back to back, limb i with modulus
 * qs[i % nq] and its tables; kind as AXHEL_JOB_FORWARD/INVERSE/CHAIN_MUL/
 * CHAIN_FMA (1..4): the reference's per-limb call sequence for that kind
 * (forward; [ReduceMod 4->2] inverse; [ReduceMod 4->2] inverse(2,2) ->
 * MulMod/FMAMod(., 2) -> forward(1, out_f)).  vec / scalars may be NULL
 * where the kind does not use them.  Limbs run on up to `threads` threads. */
void orc_job_batch(uint32_t kind, uint64_t* res, const uint64_t* op, const uint64_t* vec,
                   const uint64_t* scalars, uint64_t n, uint64_t count, const uint64_t* qs,
                   const uint64_t* const* fwds, const uint64_t* const* invs, const uint64_t* const* ninvs,
                   uint64_t nq, uint64_t in_f, uint64_t out_f, int threads);
/* The tensor-product call sequence per limb: t0 = MulMod(c0,d0), t1 = MulMod(c0,d1),
 * u = MulMod(c1,d0), t1 = AddMod(t1,u), t2 = MulMod(c1,d1) (factor `factor`),
 * then ReduceMod(., 4, 1) on each result. */
void orc_tensor_batch(uint64_t* r0, uint64_t* r1, uint64_t* r2, const uint64_t* c0, const uint64_t* c1,
                      const uint64_t* d0, const uint64_t* d1, uint64_t n, uint64_t count, const uint64_t* qs,
                      uint64_t nq, uint64_t factor, int threads);

/* ---- reference test-suite generators (tests/common/parameters.hpp) ---- */
uint64_t orc_pow_mod(uint64_t a, uint64_t e, uint64_t q);
int orc_is_prime(uint64_t n);
uint64_t orc_find_ntt_prime(uint64_t degree, unsigned bits);
uint64_t orc_find_ntt_prime_near(uint64_t degree, unsigned bits, uint64_t num, uint64_t den);
uint64_t orc_find_primitive_root(uint64_t degree, uint64_t q);

/* mt19937_64 (the standard 64-bit Mersenne Twister) and the reference's
 * rejection-sampled bounded draw; state is 313 words (312 + index). */
void orc_mt64_seed(uint64_t* state, uint64_t seed);
uint64_t orc_mt64_next(uint64_t* state);
uint64_t orc_bounded_random(uint64_t* state, uint64_t bound);
void orc_random_vector(uint64_t* out, uint64_t n, uint64_t bound, uint64_t* state);

#ifdef __cplusplus
}
#endif
#endif
