// EltwiseSubMod: same declarations as the reference
// (axhel/include/axhel/eltwise/eltwise-sub-mod.hpp:13,17).
#pragma once

#include <stdint.h>

namespace unipi {
namespace axhel {

    /// @brief result[i] = (operand1[i] - operand2[i]) mod modulus.
    /// @pre operand1[i], operand2[i] in [0, modulus).  Host or device pointers.
    void EltwiseSubMod(uint64_t* result, const uint64_t* operand1, const uint64_t* operand2, uint64_t n, uint64_t modulus);

    /// @brief result[i] = (operand1[i] - operand2) mod modulus.
    void EltwiseSubMod(uint64_t* result, const uint64_t* operand1, uint64_t operand2, uint64_t n, uint64_t modulus);

}
}
