// context.hpp -- host-side state behind the C ABI: moduli, CRT/twiddle tables
// in HBM, key store, ciphertext objects and the key-switch workspace.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
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
    // completion of the last asynchronous download of this buffer: the buffer
    // is released or overwritten only after it
    mutable cudaEvent_t d2h_ev = nullptr;
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
    uint64_t* a = nullptr;  // null for a seeded key: digit d's a half is uniform_mod(uniform_stream(a_seed, d + 1), prime, j)
    uint64_t a_seed = 0;
    bool seeded = false;
};

// Key-switch workspace for `cap` batch elements; element b's buffers sit at
// the element-0 pointers + b*stride words.  Sized for the top level.
struct Workspace {
    cudaStream_t st = nullptr;  // stream the engine queues this workspace's work on
    uint64_t* base = nullptr;
    size_t stride = 0;  // words per element
    int cap = 0;
    size_t dig_stride = 0;  // limbs per digit in DIG
    uint64_t *E0 = nullptr, *E1 = nullptr, *E2 = nullptr, *XT = nullptr, *DIG = nullptr, *XB = nullptr,
             *XA = nullptr, *W = nullptr, *T = nullptr;
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

struct BootPrecomp;  // bootstrap.cpp

}  // namespace fides

struct fides_ctx {
    int device = 0;
    cudaStream_t st = nullptr;
    // copy streams: uploads and asynchronous downloads run on the copy
    // engines beside the kernels queued on `st`, ordered by events
    cudaStream_t h2d = nullptr, d2h = nullptr;
    int logN = 0, N = 0, L = 0, K = 0, dnum = 0, alpha = 0;
    double default_scale = 0;
    fides::HostTables host;
    fides::DevCtx dev{};
    void* table_mem = nullptr;
    void* tc_mem = nullptr;  // tensor-core conversion tables
    size_t table_bytes = 0;

    // key-switch workspaces: one element for single operations, a larger one
    // (allocated on first use) for batches
    fides::Workspace ws1;
    fides::Workspace wsb;

    fides::SwitchKey relin;
    bool has_relin = false;
    std::map<uint32_t, fides::SwitchKey> galois_keys;
    std::map<uint32_t, fides::SwitchKey> host_generated;  // galois 0 = relin (for export)

    // bootstrapping precomputation (diagonal plaintexts, series), by slot count
    std::map<int, std::shared_ptr<fides::BootPrecomp>> boot;

    int tuned_variant = 0;   // forward NTT variant
    int tuned_inverse = 0;   // inverse NTT configuration
    std::vector<float> tune_ms;
    int tuned_conv = 0;  // base-conversion accumulator: 0 128-bit, 1 split 32-bit products
    std::vector<float> conv_ms;
    // giant steps of linear transforms summed in the extended basis before one
    // ModDown per input: 0 never, 1 in the bootstrap's transforms, 2 in every
    // linear transform
    int giant_moddown = 1;
    int compress_keys = 1;  // keys generated here that store b and a seed for a: bit 0 Galois, bit 1 relinearisation
    std::string last_error;
    std::recursive_mutex mu;

    size_t limb_bytes() const { return sizeof(uint64_t) * (size_t)N; }
};

namespace fides {
// helpers shared by api.cpp / client.cpp
fides_status set_err(fides_ctx* c, fides_status s, const std::string& msg);
fides_status check_cuda(fides_ctx* c, const char* where);
// The context's device error word (kDevErr* bits), read after the work queued
// on `st` (default: the context stream); cleared when `clear`.
uint32_t read_device_error(fides_ctx* c, cudaStream_t st = nullptr, bool clear = false);
// FIDES_TIMEOUT with a message when the word is set (and clears it), else OK.
fides_status consume_device_error(fides_ctx* c, cudaStream_t st = nullptr);
// Canonical-embedding encode of `slots` complex values (interleaved re, im)
// at `scale` into level+1 evaluation limbs at dm (device), on the context stream.
fides_status encode_dev(fides_ctx* c, const double* values, int slots, int level, double scale, uint64_t* dm);
// In-place rescale of n ciphertexts at one level, batched over launches;
// results equal one fides_rescale each
fides_status rescale_batch(fides_ctx* c, int n, fides_ct* const* cts);
// fides_linear_transform_batch with `boot` marking the bootstrap's own
// transforms (the context's giant_moddown decides per caller)
fides_status linear_transform_batch(fides_ctx* c, int nx, const fides_ct* const* xs, int n, const int32_t* offsets,
                                    const fides_pt* const* pts, int bstep, int rescale, fides_ct* const* outs,
                                    bool boot);
// Encoding of slot values already in HBM (z: `slots` complex), slot j taking
// factor * z[(j - shift) mod slots]: queued on the context stream, no
// synchronisation; a coefficient at or above 2^63 sets the device word *bad.
fides_status encode_dev_z(fides_ctx* c, const double2* z, int slots, int shift, double factor, int level,
                          double scale, uint64_t* dm, int* bad);
// Per-limb integer constant z mod q_j with its Shoup companion, z of any sign.
void int_const_limbs(const fides_ctx* c, int64_t z, int nlimbs, uint64_t (*out)[2]);
// Output buffer of `level`+1 limbs per component, stream-ordered on `st`
// (default: the context stream).
fides_status ct_reserve(fides_ctx* c, fides_ct* ct, int level, cudaStream_t st = nullptr);
// `st` (default: the context stream) waits for a pending asynchronous
// download of the ciphertext's buffer.
void ct_quiesce(fides_ctx* c, const fides_ct* ct, cudaStream_t st = nullptr);
fides_status build_context(fides_ctx* c, const fides_params* p);
bool select_moduli(const fides_params* prm, std::vector<uint64_t>& q, std::vector<uint64_t>& p);
void free_context(fides_ctx* c);
LimbMap map_single(const uint64_t* in, uint64_t* out, int count, int nq, int q0, int level = -1,
                   const uint64_t* in2 = nullptr, const uint64_t* in3 = nullptr);
fides_status ws_reserve(fides_ctx* c, Workspace& w, int cap);
// (Re)allocate a switching key's storage: b only when seeded, b and a otherwise.
fides_status key_alloc(fides_ctx* c, SwitchKey& k, bool seeded);
void ws_free(Workspace& w);

// ---- engine (engine.cpp): batched evaluation steps over nb <= kMaxBatch elements ----
// ModUp of x[b] (level+1 evaluation limbs each) into w.XT / w.DIG.
void eng_modup(fides_ctx* c, Workspace& w, int level, int nb, const uint64_t* const* x);
// HMult + relinearisation (+ rescale) of pairs (a0,a1)x(b0,b1) into (out0,out1).
void eng_hmult(fides_ctx* c, Workspace& w, int level, int nb, const uint64_t* const* a0, const uint64_t* const* a1,
               const uint64_t* const* b0, const uint64_t* const* b1, uint64_t* const* out0, uint64_t* const* out1,
               bool rescale, const SwitchKey& key);
// Hoisted rotations of ngroups ciphertexts (c0[g], c1[g]) by nper Galois
// elements each: element b = g * nper + r rotates ciphertext g by galois[b]
// with keys[b]; the ModUps of the ngroups inputs run as one batch and every
// element's inner product reads its group's digits.  ngroups * nper <= w.cap.
void eng_rotate_groups(fides_ctx* c, Workspace& w, int level, int ngroups, int nper, const uint64_t* const* c0,
                       const uint64_t* const* c1, const SwitchKey* const* keys, const uint32_t* galois,
                       uint64_t* const* out0, uint64_t* const* out1);
// Rotations of nb ciphertexts (element b: (c0[b], c1[b]) by galois[b] with
// keys[b]) summed per output before ModDown: output u is the sum of elements
// start[u] .. start[u+1]-1, brought down from the extended basis once
// instead of once per rotation (ModDown is linear; the two differ only in
// the rounding of the division by P, each within its usual bound).
void eng_rotate_sum(fides_ctx* c, Workspace& w, int level, int nb, const uint64_t* const* c0,
                    const uint64_t* const* c1, const SwitchKey* const* keys, const uint32_t* galois, int nout,
                    const int* start, uint64_t* const* out0, uint64_t* const* out1);
// Rotation of element b by galois[b] with keys[b]; hoisted=true: all elements
// rotate the same ciphertext (c0[0], c1[0]) and share one ModUp.
void eng_rotate(fides_ctx* c, Workspace& w, int level, int nb, const uint64_t* const* c0, const uint64_t* const* c1,
                const SwitchKey* const* keys, const uint32_t* galois, uint64_t* const* out0, uint64_t* const* out1,
                bool hoisted);
}  // namespace fides
