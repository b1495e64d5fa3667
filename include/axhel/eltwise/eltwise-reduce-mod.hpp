// EltwiseReduceMod: same declaration as the reference
// (axhel/include/axhel/eltwise/eltwise-reduce-mod.hpp:14).
#pragma once

#include <stdint.h>

namespace unipi {
namespace axhel {

    /// @brief Maps [0, in_mod_factor * mod) to [0, out_mod_factor * mod).
    /// Supported pairs as in the reference: (1, *), (2, 2), (2, 1), (4, 1),
    /// (4, 2) and the Barrett form in_mod_factor == mod (any uint64 input).
    void EltwiseReduceMod(uint64_t* res, const uint64_t* op, uint64_t n, uint64_t mod, uint64_t in_mod_factor, uint64_t out_mod_factor);

}
}
