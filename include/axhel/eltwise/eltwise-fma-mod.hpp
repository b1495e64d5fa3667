// EltwiseFMAMod: same declaration as the reference
// (axhel/include/axhel/eltwise/eltwise-fma-mod.hpp:15).
#pragma once

#include <stdint.h>

namespace unipi {
namespace axhel {

    /// @brief res[i] = (op1[i] * op2 + op3[i]) mod mod; op3 may be null (no addend).
    /// @pre op1[i], op2 and op3[i] in [0, mod_factor * mod); mod_factor 1, 2, 4 or 8.
    void EltwiseFMAMod(uint64_t* res, const uint64_t* op1, uint64_t op2, const uint64_t* op3, uint64_t n, uint64_t mod, uint64_t mod_factor);

}
}
