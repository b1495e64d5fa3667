// EltwiseMulMod: same declaration as the reference
// (axhel/include/axhel/eltwise/eltwise-mul-mod.hpp:14).
#pragma once

#include <stdint.h>

namespace unipi {
namespace axhel {

    /// @brief result[i] = operand1[i] * operand2[i] mod modulus, in [0, modulus).
    /// @pre inputs in [0, mod_factor * modulus); mod_factor 1, 2 or 4 (any other
    /// value leaves result untouched, as in the reference).
    void EltwiseMulMod(uint64_t* result, const uint64_t* operand1, const uint64_t* operand2, uint64_t n, uint64_t modulus, uint64_t mod_factor);

}
}
