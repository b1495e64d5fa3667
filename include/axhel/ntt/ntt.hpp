// Negacyclic NTT object: same declarations as the reference
// (axhel/include/axhel/ntt/ntt.hpp:14-65).  The tables live on the GPU.
#pragma once

#include <stddef.h>
#include <stdint.h>
#include <memory>

namespace unipi {
namespace axhel {

    namespace detail { struct NTTAccess; }  // the batched functions of ntt-rns.hpp reach the device tables

    /// @brief A twiddle factor with its Shoup quotient floor(operand * 2^64 / q).
    struct NTTMultiplyOperand
    {
        uint64_t operand;
        uint64_t quotient;
    };


    /// @brief Negacyclic Number Theoretic Transform of one (degree, modulus).
    /// Copies share the same device-resident tables.  const methods may be
    /// called from several host threads at once.
    class NTT {

        public:
        /// @brief Generates the tables (once per (degree, modulus, root) per
        /// process) and keeps them resident on the current CUDA device.
        /// @param degree power of two in [2, 131072].
        /// @param modulus NTT-friendly prime, modulus = 1 mod 2*degree, < 2^62.
        /// @param root_of_unity primitive 2*degree-th root of unity mod modulus.
        NTT(uint64_t degree, uint64_t modulus, uint64_t root_of_unity);

        /// @brief Uses caller-supplied tables (degree entries each, in the
        /// reference's order).  They are copied to the device here.
        NTT(uint64_t degree, uint64_t modulus, const NTTMultiplyOperand *root_powers, const NTTMultiplyOperand *inv_root_powers, NTTMultiplyOperand inv_degree_modulo);

        ~NTT();

        NTT(const NTT &) noexcept;
        NTT &operator=(const NTT &) noexcept;

        NTT(NTT &&) noexcept;
        NTT &operator=(NTT &&) noexcept;

        /// @brief Forward negacyclic NTT (bit-reversed output).  Output in
        /// [0, 4q) when output_mod_factor == 4, else [0, q).  Input in [0, 4q).
        /// Host or device pointers; result may equal operand.  Synchronous.
        void ComputeForward(uint64_t *result, const uint64_t *operand, uint64_t input_mod_factor = 1, uint64_t output_mod_factor = 1) const;

        /// @brief Inverse negacyclic NTT (natural-order output).  Output in
        /// [0, 2q) when output_mod_factor == 2, else [0, q).  Input in [0, 2q).
        void ComputeInverse(uint64_t *result, const uint64_t *operand, uint64_t input_mod_factor = 1, uint64_t output_mod_factor = 1) const;

        /// @brief Polynomial degree (0 for a moved-from object).
        uint64_t Degree() const noexcept;

        /// @brief Modulus (0 for a moved-from object).
        uint64_t Modulus() const noexcept;

    private:
        friend struct detail::NTTAccess;
        class Impl;

        std::shared_ptr<Impl> impl_;
    };

} // namespace axhel
} // namespace unipi
