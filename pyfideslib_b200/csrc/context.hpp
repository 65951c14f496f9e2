// context.hpp -- host-side state behind the C ABI: moduli, CRT/twiddle tables
// in HBM, key store, ciphertext objects and the key-switch workspace.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/fides_b200.h"
#include "common.cuh"
#include "kernels.hpp"

struct fides_ct {
    int level = -1;
    double scale = 1.0;
    int noise_deg = 1;
    int slots = 0;
    uint64_t* buf = nullptr;  // c0 at buf, c1 at buf + cap*N
    int cap = 0;              // limbs per component
    int ring = 0;             // N
    uint64_t* c0() const { return buf; }
    uint64_t* c1(size_t N) const { return buf + (size_t)cap * N; }
};

struct fides_pt {
    int level = -1;
    double scale = 1.0;
    int noise_deg = 1;
    int slots = 0;
    uint64_t* m = nullptr;
    int cap = 0;
};

struct fides_sk {
    std::vector<int8_t> coeff;  // ternary coefficients
    uint64_t* s = nullptr;       // device, evaluation form over all L+K primes
};

struct fides_pk {
    uint64_t* b = nullptr;  // device, evaluation form over the L ciphertext moduli
    uint64_t* a = nullptr;
};

namespace fides {

struct SwitchKey {
    uint64_t* b = nullptr;  // [dnum][L+K][N]
    uint64_t* a = nullptr;
};

// Moduli and host copies of the per-prime constants.
struct HostTables {
    std::vector<uint64_t> prime;  // L+K
    std::vector<PrimeConst> pc;
    std::vector<uint64_t> root;
};

std::vector<uint64_t> find_ntt_primes(int logN, int bits, int count, uint64_t upper_exclusive);
uint64_t smallest_generator(uint64_t p);
uint64_t powmod(uint64_t a, uint64_t e, uint64_t p);
uint64_t mulmod(uint64_t a, uint64_t b, uint64_t p);
uint64_t invmod(uint64_t a, uint64_t p);
bool is_prime(uint64_t n);

}  // namespace fides

struct fides_ctx {
    int device = 0;
    cudaStream_t st = nullptr;
    int logN = 0, N = 0, L = 0, K = 0, dnum = 0, alpha = 0;
    double default_scale = 0;
    fides::HostTables host;
    fides::DevCtx dev{};
    void* table_mem = nullptr;
    size_t table_bytes = 0;

    // key-switch workspace (per context, sized for the top level)
    uint64_t* ws = nullptr;
    size_t ws_limbs = 0;
    uint64_t *E0 = nullptr, *E1 = nullptr, *E2 = nullptr, *XT = nullptr, *DIG = nullptr, *XB = nullptr,
             *XA = nullptr, *W = nullptr, *T = nullptr;
    size_t dig_stride = 0;  // limbs per digit in DIG

    fides::SwitchKey relin;
    bool has_relin = false;
    std::map<uint32_t, fides::SwitchKey> galois_keys;
    std::map<uint32_t, fides::SwitchKey> host_generated;  // galois 0 = relin (for export)

    int tuned_variant = 0;
    std::vector<float> tune_ms;
    std::string last_error;
    std::recursive_mutex mu;

    size_t limb_bytes() const { return sizeof(uint64_t) * (size_t)N; }
};

namespace fides {
// helpers shared by api.cpp / client.cpp
fides_status set_err(fides_ctx* c, fides_status s, const std::string& msg);
fides_status check_cuda(fides_ctx* c, const char* where);
fides_status ct_reserve(fides_ctx* c, fides_ct* ct, int level);
fides_status build_context(fides_ctx* c, const fides_params* p);
bool select_moduli(const fides_params* prm, std::vector<uint64_t>& q, std::vector<uint64_t>& p);
void free_context(fides_ctx* c);
LimbMap map_single(const uint64_t* in, uint64_t* out, int count, int nq, int q0, int level = -1,
                   const uint64_t* in2 = nullptr, const uint64_t* in3 = nullptr);
void keyswitch_core(fides_ctx* c, int level, const uint64_t* e2, const SwitchKey& k, const uint64_t* c0_for_rot,
                    uint32_t galois);
}  // namespace fides
