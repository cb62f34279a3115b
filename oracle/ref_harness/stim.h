// Declaration-only stand-in for the handful of Stim type names that the
// reference's executor headers mention (src/clifft/backend/backend.h:258,
// src/clifft/frontend/hir.h:355, src/clifft/util/stim_mask.h:26).
//
// The executor (src/clifft/svm/*) and the bytecode passes never call Stim on
// the sampling path; Stim is only reached through the compiler and through
// `get_statevector` (src/clifft/svm/svm.cc:770-783). Stim v1.15.0 is not
// available offline, so the harness supplies just enough of the type surface
// for those translation units to compile. `to_flat_unitary_matrix` is defined
// by the harness to throw, so a call through get_statevector fails loudly.
// Test infrastructure only; nothing here is shipped.
#pragma once

#include <complex>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace stim {

template <size_t W>
struct simd_bits_range_ref {
    uint64_t* u64;
};

template <size_t W>
struct PauliString {
    bool sign = false;
    simd_bits_range_ref<W> xs{nullptr};
    simd_bits_range_ref<W> zs{nullptr};
};

template <size_t W>
struct Tableau {
    size_t num_qubits = 0;
    std::vector<std::complex<float>> to_flat_unitary_matrix(bool little_endian) const;
    bool operator==(const Tableau& other) const;
};

}  // namespace stim
