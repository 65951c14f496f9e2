// kernels.hpp -- host-side launchers of the sm_100a kernels.
#pragma once
#include <vector>

#include "common.cuh"

namespace fides {

// forward-NTT prologues (pass 1 loads)
enum { FL_PLAIN = 0, FL_SWITCHMOD = 1 };
// forward-NTT epilogues (pass 2 stores); v = NTT value, j = prime, l = level
enum {
    FS_PLAIN = 0,    // out = v
    FS_MODDOWN = 1,  // out = (in2 - v) * P^-1 (+ in3)
    FS_RESCALE = 2,  // out = (in2 - v) * q_l^-1
    FS_MDRS = 3,     // out = (in3 + in2 * P^-1 - v) * q_l^-1
};
// inverse-NTT prologues (pass A loads)
enum { IL_PLAIN = 0, IL_MUL = 1, IL_AXPY_PINV = 2 };
// inverse-NTT epilogues (pass B scale): N^-1 times 1 / ModUp hat-inverse / ModDown hat-inverse
enum { IS_PLAIN = 0, IS_MODUP = 1, IS_MODDOWN = 2 };

// process-wide count of kernels launched by this library
uint64_t launch_count();
void count_launches(int n);

bool ntt_supported(int logN);
int ntt_num_variants();
int ntt_num_inverse_variants();
int ntt_inverse_of(int forward_variant);
// Forward NTT of every limb in `map`: pass 1 reads seg.in (writes seg.out),
// pass 2 transforms seg.out in place and applies the epilogue.  load / store
// >= 0 override the per-segment modes.
void ntt_forward(const DevCtx& ctx, const LimbMap& map, int load, int store, cudaStream_t st);
// Per-device set-up of this ring dimension's kernels (the fused kernel's
// shared-memory opt-in), before any launch or stream capture.
void ntt_prepare(const DevCtx& ctx);
// Forward NTT column pass alone (seg.in -> seg.out), for the fused key switch.
void ntt_forward_cols(const DevCtx& ctx, const LimbMap& map, int load, cudaStream_t st);
// Row pass of the ModUp digits fused with the key-switch inner product:
//   XB[m] = sum_d D_d[t] kb[d][t],  XA[m] = sum_d D_d[t] ka[d][t]
// over the extended basis m in [0, level+1+K) (prime t = m, or L + m - n for
// the special limbs), for nb batch elements (blockIdx.y).  D_d[t] is the
// column-pass output of digit d's limb in DIG, finished by the row stages
// here, or the original evaluation limb `own` when t lies in digit d.
struct KsFuseArgs {
    const uint64_t* dig;  // ModUp digits of element 0 after the column pass
    const uint64_t* own;  // key-switched polynomial in evaluation form, element 0
    const uint64_t* kb;   // switching key halves [dnum][L+K][N] (one key for the batch)
    const uint64_t* ka;
    uint64_t* xb;         // outputs of element 0 [level+1+K][N]
    uint64_t* xa;
    size_t dig_stride;    // limbs per digit in dig
    size_t bstride;       // words between consecutive elements of dig, own, xb, xa
    int level;
    int fp_sums;          // 1: exact FP64 sums for primes below 2^50
    int m0;               // first output limb of a launch (set by the launcher)
};
void ntt_rows_keyswitch(const DevCtx& ctx, const KsFuseArgs& a, int nb, cudaStream_t st);
// the fused row pass keeps one transformed tile per digit in shared memory
bool ntt_rows_keyswitch_supported(const DevCtx& ctx);
// Inverse NTT: pass A reads seg.in (+in2 for the prologue), writes seg.out;
// pass B finishes seg.out in place.
void ntt_inverse(const DevCtx& ctx, const LimbMap& map, int load, int store, cudaStream_t st);

// ---- element-wise and base-conversion kernels (ks.cu) ----
// Batched kernels take per-element pointers in kernel parameters (up to
// kMaxBatch elements); workspace buffers of element b sit at ptr + b*bstride.
struct TensorArgs {
    const uint64_t* a0[kMaxBatch];
    const uint64_t* a1[kMaxBatch];
    const uint64_t* b0[kMaxBatch];
    const uint64_t* b1[kMaxBatch];
    uint64_t* e0;
    uint64_t* e1;
    uint64_t* e2;
    size_t bstride;
};
void launch_tensor(const DevCtx& ctx, int n, int nb, const TensorArgs& args, cudaStream_t st);
void launch_modup_conv(const DevCtx& ctx, int level, int nb, const uint64_t* xt, uint64_t* dig, size_t dig_stride,
                       size_t bstride, cudaStream_t st);
struct KsArgs {
    const uint64_t* own[kMaxBatch];  // evaluation values of the key-switched polynomial (own-digit limbs)
    const uint64_t* kb[kMaxBatch];   // switching key halves of each element
    const uint64_t* ka[kMaxBatch];   // null: a seeded key, a half regenerated from a_seed
    uint64_t a_seed[kMaxBatch];      // seeded keys: uniform_stream(key seed, 0); digit d's stream is this ^ (d+1) << 48
    const uint64_t* c0[kMaxBatch];   // rotations: c0 of the input (P*c0 added), else null
    uint32_t galois[kMaxBatch];      // rotations: automorphism X -> X^g applied as a gather, else 0
    const uint64_t* dig;             // ModUp digits of element 0
    uint64_t* xb;                    // outputs of element 0 (extended basis)
    uint64_t* xa;
    size_t dig_stride;               // limbs per digit in dig
    size_t bstride;                  // words between consecutive elements' xb / xa
    size_t dig_bstride;              // words between consecutive elements' dig (0: shared ModUp)
    int dig_group;                   // > 0: element b reads the ModUp of element dig_elem[b] (grouped hoisting)
    uint8_t dig_elem[kMaxBatch];
};
// plain: no rotation in any element (vectorised variant)
void launch_ks_inner(const DevCtx& ctx, int level, int nb, const KsArgs& args, bool plain, cudaStream_t st);
struct MdArgs {
    const uint64_t* y[2];     // scaled special limbs of the two halves (element 0)
    uint64_t* w[2];           // conversion outputs
    const uint64_t* ttop[2];  // fused rescale: INTT(e_l + P^-1 x_l) of each half, else null
    size_t bstride;
};
void launch_moddown_conv(const DevCtx& ctx, int level, int nb, const MdArgs& args, cudaStream_t st);
// the conversion kernels keep up to 16 inputs (digit moduli / special moduli) in registers
bool conv_supported(const DevCtx& ctx);
constexpr int kConvVariants = 5;  // see DevCtx::conv_variant
// ModUp and ModDown conversions as exact int8-split tcgen05 contractions
// (conv_tc.cu); chunk = targets per MMA (32 or 16)
bool conv_tc_eligible(const DevCtx& ctx);   // shapes the kernels handle
bool conv_tc_supported(const DevCtx& ctx);  // eligible and the B tables built
// byte offsets of the per-(level, digit) and per-(level, fused) B matrices
size_t conv_tc_table_layout(const DevCtx& ctx, std::vector<uint64_t>& offs);
void conv_tc_build_tables(const DevCtx& ctx, cudaStream_t st);
void launch_modup_conv_tc(const DevCtx& ctx, int level, int nb, const uint64_t* xt, uint64_t* dig, size_t dig_stride,
                          size_t bstride, cudaStream_t st, int chunk);
void launch_moddown_conv_tc(const DevCtx& ctx, int level, int nb, const MdArgs& md, cudaStream_t st, int chunk);
// override every segment's prologue / epilogue mode (-1 keeps the segment's own)
void set_modes(LimbMap& map, int lmode, int smode);

// Sums of key-switch results in the extended basis before one ModDown: for
// output u < nout, elements start[u] .. start[u+1]-1 of x[0] (XB) and x[1]
// (XA) -- n ciphertext limbs then K special limbs each, element b at
// x + b*bstride -- are added into element start[u].
struct ExtSumArgs {
    int start[kMaxBatch + 1];
    int nout, n;
    uint64_t* x[2];
    size_t bstride;
};
void launch_ext_sum(const DevCtx& ctx, const ExtSumArgs& args, cudaStream_t st);

// element-wise helpers; limbs 0..n-1 use primes q0..q0+n-1
enum { EW_ADD = 0, EW_SUB = 1, EW_NEG = 2, EW_MUL = 3, EW_COPY = 4 };
void launch_elementwise(const DevCtx& ctx, int op, int n, int q0, const uint64_t* a, const uint64_t* b,
                        uint64_t* out, cudaStream_t st);
// out = a * c_j (+ b) with one constant per limb from a device table [n][2] (value, Shoup)
void launch_scalar_mac(const DevCtx& ctx, int n, const uint64_t* a, const uint64_t* cj, const uint64_t* b,
                       uint64_t* out, cudaStream_t st);
// out = a + c_j with one constant per limb (device table [n])
void launch_scalar_add(const DevCtx& ctx, int n, const uint64_t* a, const uint64_t* cj, uint64_t* out,
                       cudaStream_t st);
// Plaintext dot product of ciphertexts (BSGS inner sums):
//   o0 = sum_k c0[k] * p[k],  o1 = sum_k c1[k] * p[k]   (+ o0 / o1 when accumulate)
// over limbs 0..nlimbs-1 with one 128-bit accumulator per output, n <= kMaxBatch.
struct DotArgs {
    const uint64_t* c0[kMaxBatch];
    const uint64_t* c1[kMaxBatch];
    const uint64_t* p[kMaxBatch];
    int n;
    int accumulate;
    uint64_t* o0;
    uint64_t* o1;
};
void launch_dot_pt(const DevCtx& ctx, int nlimbs, const DotArgs& args, cudaStream_t st);
// Integer linear combination over ciphertext components, with per-limb
// integer constants z[k][j] (value, Shoup companion) and an optional constant
// added to component 0:
//   out0 = sum_k z_k in0_k + add0_j,   out1 = sum_k z_k in1_k   over limbs 0..nlimbs-1.
constexpr int kMaxLin = 8;
constexpr int kMaxLinLimbs = 64;
struct LinArgs {
    const uint64_t* in0[kMaxLin];
    const uint64_t* in1[kMaxLin];
    int n;
    int has_add;
    int q0;  // prime of limb 0
    uint64_t* out0;
    uint64_t* out1;
    uint64_t z[kMaxLin][kMaxLinLimbs][2];
    uint64_t add0[kMaxLinLimbs];
};
void launch_lincomb(const DevCtx& ctx, int nlimbs, const LinArgs& args, cudaStream_t st);
// Multiplication by the monomial X^k (0 <= k < 2N) of both components of a
// ciphertext in evaluation form: slot i scales by psi^((2 brev(i) + 1) k).
void launch_mult_monomial(const DevCtx& ctx, int nlimbs, const uint64_t* in0, const uint64_t* in1, uint64_t* out0,
                          uint64_t* out1, uint32_t k, cudaStream_t st);
// automorphism gather over nlimbs limbs (any primes): out[j] = in[slot(galois_inv, j)]
void launch_automorph(const DevCtx& ctx, int nlimbs, const uint64_t* in, uint64_t* out, uint32_t galois_inv,
                      cudaStream_t st);

}  // namespace fides
