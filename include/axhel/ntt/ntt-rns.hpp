// Batched RNS transforms for C++ callers (new; no counterpart in the
// reference API).  One call replaces the per-limb loop a caller such as SEAL
// runs over a polynomial's RNS components (integration/seal/
// SEAL-4.4.5-AXHEL.patch:189-222 calls ComputeForward / ComputeInverse once
// per limb): `count` limbs of Degree() words stored back to back, limb i
// transformed by ntts[i % n_ntts], exactly as
//
//     for (size_t i = 0; i < count; ++i)
//         ntts[i % n_ntts].ComputeForward(result + i * N, operand + i * N, in_f, out_f);
//
// bit for bit, in one batched launch.  Host or device pointers (host data is
// staged in one copy each way); result may equal operand; synchronous.  As
// in the per-limb calls, the input factor is not used (forward inputs in
// [0, 4q), inverse inputs in [0, 2q)).  At most 64 NTT objects of one degree.
#pragma once

#include <stddef.h>
#include <stdint.h>

#include "axhel/ntt/ntt.hpp"

namespace unipi {
namespace axhel {

    void ComputeForwardRNS(const NTT *ntts, size_t n_ntts, uint64_t *result, const uint64_t *operand, size_t count,
                           uint64_t input_mod_factor = 1, uint64_t output_mod_factor = 1);

    void ComputeInverseRNS(const NTT *ntts, size_t n_ntts, uint64_t *result, const uint64_t *operand, size_t count,
                           uint64_t input_mod_factor = 1, uint64_t output_mod_factor = 1);

} // namespace axhel
} // namespace unipi
