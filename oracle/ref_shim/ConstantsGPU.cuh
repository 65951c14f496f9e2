// Stand-in for the reference's src/ConstantsGPU.cuh (see README): the names
// the *_forPrime wrappers of test/cpuNTT*.cpp mention, with no behaviour.
#pragma once
#include <cstdint>

namespace FIDESlib {
struct Constants {
    uint64_t primes[64];
};
struct Global {
    void* psi[64];
    void* inv_psi[64];
    void* psi_middle_scale[64];
    void* inv_psi_middle_scale[64];
};
}  // namespace FIDESlib

#define hC_ (host_constants)
#define hG_ (host_global)
