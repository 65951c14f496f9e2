/*
 * fides_b200.h -- C ABI of the B200 CKKS evaluation core.
 *
 * Plain pointers and sizes only.  Every call returns a fides_status and never
 * throws or exits.  Residue arrays are uint64, limb-major ([limb][N]), in the
 * evaluation (NTT, bit-reversed) representation that OpenFHE calls
 * EVALUATION and FIDESlib exchanges through RawCipherText
 * (src/CKKS/openfhe-interface/RawCiphertext.cuh:19-93).
 *
 * Prime indices: 0..L-1 are the ciphertext moduli q_0..q_{L-1}, L..L+K-1 the
 * special (key-switching) moduli p_0..p_{K-1}.  A ciphertext at level l has
 * l+1 limbs (q_0..q_l).  Switching keys are dnum polynomials over all L+K
 * primes: arrays of dnum*(L+K)*N words.  Digits are contiguous groups of
 * alpha = ceil(L/dnum) moduli (OpenFHE's HYBRID key-switching partition).
 *
 * Each function names the FIDESlib interface it replaces.
 */
#ifndef FIDES_B200_H
#define FIDES_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    FIDES_OK = 0,
    FIDES_BAD_ARG = 1,
    FIDES_OOM = 2,
    FIDES_LEVEL_MISMATCH = 3,
    FIDES_KEY_MISSING = 4,
    FIDES_TIMEOUT = 5,
    FIDES_CUDA_ERR = 6,
    FIDES_UNSUPPORTED = 7,
    FIDES_BUSY = 8
} fides_status;

typedef struct fides_ctx fides_ctx;
typedef struct fides_ct fides_ct; /* device-resident ciphertext */
typedef struct fides_pt fides_pt; /* device-resident plaintext  */
typedef struct fides_sk fides_sk; /* secret key (client side)   */
typedef struct fides_pk fides_pk; /* public key (client side)   */
typedef struct fides_plan fides_plan; /* captured CUDA graph of a batched evaluation */
typedef struct fides_server fides_server; /* continuous-batching request loop */

typedef struct {
    int log_n;            /* ring dimension N = 2^log_n, 8 <= log_n <= 16 */
    int num_q;            /* L: number of ciphertext moduli (levels 0..L-1) */
    int num_p;            /* K: number of special moduli (0 = derive from the digit size) */
    int dnum;             /* number of key-switching digits */
    const uint64_t* q;    /* optional explicit moduli (num_q entries), NULL to generate */
    const uint64_t* p;    /* optional explicit special moduli (num_p entries) */
    int q0_bits;          /* generated moduli sizes (defaults 60 / 50 / 60 when 0) */
    int qi_bits;
    int p_bits;
    int device;           /* CUDA device ordinal */
    double default_scale; /* encoding scale, default 2^qi_bits */
    /* optional primitive 2N-th roots of unity psi, one per modulus (num_q and
     * num_p entries), that fix the evaluation representation: OpenFHE's own
     * roots, as RawParams carries them (root_of_unity / SPECIALroot_of_unity,
     * src/CKKS/openfhe-interface/RawCiphertext.cu:235,306) and SetupConstants
     * takes them (src/ConstantsGPU.cu:195-199).  NULL: psi = g^((p-1)/2N) with
     * g the smallest generator, FIDESlib's rule without OpenFHE
     * (unity_root, src/ConstantsGPU.cu:61).  A value with psi^N != -1 mod p
     * is refused. */
    const uint64_t* q_root;
    const uint64_t* p_root;
} fides_params;

/* ---- context (replaces CKKS::GenCryptoContextGPU / ContextData ctor,
 *      src/CKKS/Context.cu:37-98, and SetupConstants, src/ConstantsGPU.cu:127-708) ---- */
fides_status fides_ctx_create(const fides_params* params, fides_ctx** out);
fides_status fides_ctx_destroy(fides_ctx* ctx);
/* Host-only: the moduli fides_ctx_create would generate for these parameters
 * (descending search for primes = 1 mod 2N; Parameters / computeK,
 * src/CKKS/Context.cu:275-295).  q gets num_q entries, p up to 64; *num_p_out
 * receives K. */
fides_status fides_generate_moduli(const fides_params* params, uint64_t* q, uint64_t* p, int* num_p_out);
/* moduli actually used: q[0..L-1], p[0..K-1]; any pointer may be NULL */
fides_status fides_ctx_info(const fides_ctx* ctx, int* log_n, int* num_q, int* num_p, int* dnum, uint64_t* q,
                            uint64_t* p);
/* wait for all queued work of this context (CryptoContextImpl::Synchronize, api/CryptoContext.hpp:242) */
fides_status fides_ctx_synchronize(fides_ctx* ctx);
/* last error message of this context (static storage owned by the context) */
const char* fides_ctx_last_error(const fides_ctx* ctx);
/* The CUDA stream (cudaStream_t) all work of this context is queued on, for
 * callers that time or order work around it (FIDESlib keeps per-partition
 * streams in ContextData, src/CKKS/Context.cuh:85-98). */
fides_status fides_ctx_stream(const fides_ctx* ctx, void** stream);
/* Autotuner: time every forward NTT variant (occupancy, twiddle-fetch
 * policy, integer or double-precision butterflies, row twiddles staged or
 * formed in the kernel) and every inverse configuration on one element's
 * ModUp digits and on the same shape batched over four elements, and keep
 * the fastest of each (sum of the two times).
 * Runs once in fides_ctx_create; call again to re-tune.  *variant receives
 * the forward variant, times_ms[v] (num_variants entries, at most 16) the
 * forward time of variant v plus that of its paired inverse configuration;
 * any pointer may be NULL.  Results never depend on the variant. */
fides_status fides_autotune(fides_ctx* ctx, int* variant, float* times_ms, int* num_variants);
/* The base-conversion variant the autotuner chose (0: two coefficients per
 * thread with 128-bit sums, 1: the same with split 32-bit partial products,
 * for moduli below 2^60, 2: one coefficient per thread, 3 and 4: ModUp on
 * the tensor cores as an exact int8-split contraction with 32 or 16 targets
 * per matrix product) and the time of each on the ModUp conversion of four
 * top-level elements (times_ms: 5 entries, 0 when not eligible). */
fides_status fides_autotune_conv_info(const fides_ctx* ctx, int* accumulator, float* times_ms);
/* Force the conversion variant (0..4, for measurements and tests; 3 and 4
 * run the ModUp conversion on the tensor cores as an exact int8-split
 * contraction with 32 or 16 targets per matrix product, digits of at most 16
 * moduli); -1 restores the tuned choice. */
fides_status fides_set_conv_accumulator(fides_ctx* ctx, int accumulator);
/* Key-switch inner product (identical results in every form; for
 * measurements and tests).  Bit 0: the digit products of primes below 2^50
 * are summed exactly on the FP64 pipes (else 128-bit integer sums).  Bit 1:
 * HMult's inner product runs in the epilogue of the ModUp digits' NTT row
 * pass (else in its own kernel).  Bit 2: the same for HMult batches of eight
 * or more elements only.  Bit 3: that fused row pass in two launches, the
 * ciphertext-prime outputs (one digit tile less in shared memory) at 3 CTAs
 * per SM and the special-prime outputs at 2 (forward NTT variant 9 only).
 * Default 13 (FP64 sums, fused for batches of 8+, split launch). */
fides_status fides_set_keyswitch_variant(fides_ctx* ctx, int variant);
/* Giant steps of the baby-step giant-step linear transforms: each input's
 * giant-step rotations are added in the extended basis (Q and the special
 * moduli) and brought down by one ModDown, instead of one ModDown per
 * rotation.  The two agree up to the rounding of the division by P.  scope 0:
 * never; 1 (default): in the bootstrap's CoeffsToSlots / SlotsToCoeffs;
 * 2: also in fides_linear_transform(_batch), whose default results are bit
 * for bit those of composing rotations, products and additions.  The
 * reference hoists the ModDown of its baby steps instead (MODDOWN_HOIST,
 * src/CKKS/LinearTransform.cu:111-190). */
fides_status fides_set_giant_step_moddown(fides_ctx* ctx, int scope);
/* Device error word of this context, read after the work queued so far
 * without clearing it: bit 0 is set once a tensor-core conversion gave up its
 * bounded wait for its matrix products (its outputs are then invalid).  The
 * next synchronising call (fides_ctx_synchronize, fides_ct_download, a
 * serving completion) reports a set word as FIDES_TIMEOUT with a message and
 * clears it.  No counterpart in the reference, whose kernels do not wait. */
fides_status fides_ctx_device_status(fides_ctx* ctx, uint32_t* flags);
/* Write `flags` into the device error word from the host (ordered after the
 * queued work): exercises the reporting path without any kernel failing. */
fides_status fides_ctx_inject_device_error(fides_ctx* ctx, uint32_t flags);
/* Force forward NTT variant `variant` with its paired inverse configuration
 * (for measurements and tests); -1 restores the tuned choices. */
fides_status fides_set_ntt_variant(fides_ctx* ctx, int variant);
/* Number of kernels this library has launched so far (process-wide). */
uint64_t fides_kernel_launches(void);

/* ---- keys (replaces KeySwitchingKey::Initialize, src/CKKS/KeySwitchingKey.cu:20-35,
 *      and the GetEvalKeySwitchKey / GetRotationKeySwitchKey imports,
 *      RawCiphertext.cu:468-602) ---- */
/* Relinearisation key: b, a are dnum*(L+K)*N words each (host memory),
 * canonical residues like every uploaded operand. */
fides_status fides_key_upload_relin(fides_ctx* ctx, const uint64_t* b, const uint64_t* a);
/* Rotation / conjugation key for the automorphism X -> X^galois (galois odd, < 2N). */
fides_status fides_key_upload_galois(fides_ctx* ctx, uint32_t galois, const uint64_t* b, const uint64_t* a);
/* Galois element of a slot rotation by `index` with `slots` slots
 * (Ciphertext::normalyzeIndex, Ciphertext.cpp:157; RNSPoly.cpp:559 gives the
 * inverse element used by the permutation). */
uint32_t fides_rotation_galois(const fides_ctx* ctx, int32_t index, int slots);

/* ---- ciphertexts (replaces Ciphertext::load / store, Ciphertext.cpp:270-309) ----
 * Residues are limb-major, (level+1)*N words per component, each one
 * canonical (below its modulus), as OpenFHE's raw ciphertexts hold them; the
 * exact double-precision kernels rely on that and the upload does not scan
 * for it.  Uploads run on a copy stream beside the kernels already queued
 * (the host buffers must stay unchanged until fides_ctx_synchronize; pinned
 * memory lets the copy overlap); later operations on the ciphertext wait for
 * them. */
fides_status fides_ct_upload(fides_ctx* ctx, const uint64_t* c0, const uint64_t* c1, int level, double scale,
                             int noise_deg, int slots, fides_ct** out);
fides_status fides_ct_download(fides_ctx* ctx, const fides_ct* ct, uint64_t* c0, uint64_t* c1);
/* Queue the download without waiting, on the download stream after the
 * kernels queued so far; the host buffers (pinned for overlap) are valid after
 * fides_ctx_synchronize.  Freeing or overwriting the ciphertext waits for it. */
fides_status fides_ct_download_async(fides_ctx* ctx, const fides_ct* ct, uint64_t* c0, uint64_t* c1);
fides_status fides_ct_info(const fides_ct* ct, int* level, double* scale, int* noise_deg, int* slots);
fides_status fides_ct_create(fides_ctx* ctx, fides_ct** out); /* empty, filled by an operation */
/* Overwrite the residues of an existing ciphertext (same level, buffer kept):
 * refreshes the inputs of a captured plan without re-capturing it. */
fides_status fides_ct_write(fides_ctx* ctx, fides_ct* ct, const uint64_t* c0, const uint64_t* c1);
fides_status fides_ct_copy(fides_ctx* ctx, const fides_ct* src, fides_ct* dst);
fides_status fides_ct_free(fides_ctx* ctx, fides_ct* ct);
/* Device residues of a ciphertext: (l+1)*N words each, valid until the next
 * operation that writes this ciphertext. */
fides_status fides_ct_device_ptrs(const fides_ct* ct, uint64_t** c0, uint64_t** c1);
/* Drop to a lower level by discarding limbs (CryptoContextImpl::SetLevel). */
fides_status fides_ct_set_level(fides_ctx* ctx, fides_ct* ct, int level);

fides_status fides_pt_upload(fides_ctx* ctx, const uint64_t* m, int level, double scale, int noise_deg, int slots,
                             fides_pt** out);
fides_status fides_pt_free(fides_ctx* ctx, fides_pt* pt);

/* ---- raw-residue interop: the shapes FIDESlib exchanges with OpenFHE,
 *      RawCipherText / RawPlainText / RawKeySwitchKey
 *      (src/CKKS/openfhe-interface/RawCiphertext.cuh:19-93), filled by
 *      GetRawCipherText / GetRawPlainText / GetKeySwitchKey (RawCiphertext.cu:48-75,
 *      172-220, 468-602) and loaded by Ciphertext / Plaintext / KeySwitchingKey
 *      ::Initialize (KeySwitchingKey.cu:20-35).  One array of N words per limb,
 *      with the limb's modulus beside it.  Imports check every residue is
 *      canonical and every modulus belongs to the context. ---- */
typedef enum { FIDES_FORMAT_EVALUATION = 0, FIDES_FORMAT_COEFFICIENT = 1 } fides_format;
typedef struct {
    uint64_t** sub_0;  /* numRes limbs of N words: component 0 */
    uint64_t** sub_1;  /* numRes limbs of N words: component 1 */
    uint64_t* moduli;  /* numRes moduli: limb i is mod q_i of the context */
    int numRes;        /* limbs (level + 1); on export: capacity in, limbs out */
    int N;
    int format;        /* fides_format: EVALUATION is bit-reversed NTT order, as OpenFHE holds it */
    double Noise;      /* scaling factor */
    int NoiseLevel;    /* noise scale degree */
    int slots;
} fides_raw_ct;
typedef struct {
    uint64_t** sub_0;
    uint64_t* moduli;
    int numRes;
    int N;
    int format;
    double Noise;
    int NoiseLevel;
    int slots;
} fides_raw_pt;
typedef struct {
    /* r_key[(h * dnum + d) * nlimbs + i]: half h (0 = a, 1 = b, RawKeySwitchKey's
     * order), digit d, limb i of N words; r_key_moduli the same indexing.  Each
     * digit polynomial covers the L + K primes of the context once, in any order. */
    uint64_t** r_key;
    uint64_t* r_key_moduli;
    int dnum;
    int nlimbs;  /* L + K */
    int N;
} fides_raw_key;
/* Device ciphertext from a RawCipherText (COEFFICIENT input is transformed on the device). */
fides_status fides_ct_import_raw(fides_ctx* ctx, const fides_raw_ct* raw, fides_ct** out);
/* RawCipherText of a device ciphertext into caller buffers (raw->numRes >= level + 1
 * limb buffers per component; raw->format selects the output format). */
fides_status fides_ct_export_raw(fides_ctx* ctx, const fides_ct* ct, fides_raw_ct* raw);
/* Device plaintext from a RawPlainText (LoadPlaintext, api/CryptoContext.cpp:230-246). */
fides_status fides_pt_import_raw(fides_ctx* ctx, const fides_raw_pt* raw, fides_pt** out);
/* Switching key from a RawKeySwitchKey: galois 0 = relinearisation key, else the
 * automorphism X -> X^galois (LoadContext's key loading, api/CryptoContext.cpp:199-213). */
fides_status fides_key_import_raw(fides_ctx* ctx, uint32_t galois, const fides_raw_key* raw);
/* RawKeySwitchKey of a resident key into caller buffers (limbs in context order). */
fides_status fides_key_export_raw(fides_ctx* ctx, uint32_t galois, fides_raw_key* raw);

/* ---- evaluation (api/CryptoContext.hpp:110-181 -> CKKS::Ciphertext, Ciphertext.cuh:34-500) ---- */
/* EvalMult + relinearisation (+ Rescale when `rescale` != 0): Ciphertext::mult, Ciphertext.cpp:409-622 */
fides_status fides_hmult(fides_ctx* ctx, const fides_ct* a, const fides_ct* b, fides_ct* out, int rescale);
/* EvalSquare: Ciphertext::square, Ciphertext.cpp:624 */
fides_status fides_square(fides_ctx* ctx, const fides_ct* a, fides_ct* out, int rescale);
/* Rescale: Ciphertext::rescale, Ciphertext.cpp:379-398 */
fides_status fides_rescale(fides_ctx* ctx, const fides_ct* a, fides_ct* out);
/* EvalRotate: Ciphertext::rotate, Ciphertext.cpp:756-926 */
fides_status fides_rotate(fides_ctx* ctx, const fides_ct* a, int32_t index, fides_ct* out);
/* EvalFastRotation (hoisted, one shared ModUp): Ciphertext::rotate_hoisted, Ciphertext.cpp:1053-1226 */
fides_status fides_rotate_hoisted(fides_ctx* ctx, const fides_ct* a, int n, const int32_t* indices, fides_ct** outs);
/* Batched EvalMult (+ Rescale) of n independent pairs (a[i], b[i]) -> out[i],
 * levels may differ between pairs.  Pairs at one level share every launch,
 * up to 32 per launch, so the relinearisation key is read once per batch
 * from HBM (the reference's batched path is LimbPartitionBatch.cu:21-604).
 * Results are identical to n calls of fides_hmult. */
fides_status fides_hmult_batch(fides_ctx* ctx, int n, const fides_ct* const* a, const fides_ct* const* b,
                               fides_ct* const* out, int rescale);
/* Batched EvalRotate: out[i] = rotation of a[i] by indices[i] (own keys). */
fides_status fides_rotate_batch(fides_ctx* ctx, int n, const fides_ct* const* a, const int32_t* indices,
                                fides_ct* const* out);
/* Plan of a batched evaluation captured into one CUDA graph: n independent
 * pairs (levels may differ) go through HMult + relinearisation (+ rescale)
 * and then, if `indices` is not NULL, a rotation of each product by
 * indices[i]; results land in out[i].  Creating the plan allocates every
 * output and intermediate buffer and captures the kernel sequence once;
 * fides_plan_launch replays it (a single graph launch) on the context
 * stream, reading the inputs' current residues (fides_ct_write refreshes
 * them).  a, b and out must outlive the plan.  No counterpart in the
 * reference, which captures per-level graphs of one key switch
 * (LimbPartitionMGPU.cu:581-640, FIDESLIB_USE_GRAPH_CAPTURE). */
fides_status fides_plan_hmult_rotate(fides_ctx* ctx, int n, const fides_ct* const* a, const fides_ct* const* b,
                                     const int32_t* indices, int rescale, fides_ct* const* out, fides_plan** plan);
fides_status fides_plan_launch(fides_ctx* ctx, fides_plan* plan);
fides_status fides_plan_free(fides_ctx* ctx, fides_plan* plan);
/* Diagonal-form plaintext matrix times ciphertext, baby-step giant-step:
 *   out = sum_k pt_k' (.) Rot(x, offsets[k])
 * computed as  sum_g Rot( sum_{b} pts[k] (.) Rot(x, b), g*bstep )  with
 * offsets[k] = g*bstep + b, g = floor(offsets[k] / bstep), 0 <= b < bstep.
 * pts[k] must hold diagonal k pre-rotated by g*bstep slots (slot j holds
 * diag_k[j - g*bstep]), encoded at x's level or above.  Baby steps share one
 * hoisted ModUp, each giant's inner sum is one fused dot-product launch, the
 * giant rotations are one batched key switch.  Rescales when `rescale` != 0.
 * Rotation keys: every nonzero b and every nonzero g*bstep.
 * Reference: LinearTransform (CKKS/LinearTransform.cu:67-258) with
 * dotProductPt_ (CKKS/ElemenwiseBatchKernels.cu:651). */
fides_status fides_linear_transform(fides_ctx* ctx, const fides_ct* x, int n, const int32_t* offsets,
                                    const fides_pt* const* pts, int bstep, int rescale, fides_ct* out);
/* The same transform applied to nx ciphertexts at one level (outs[u] for
 * xs[u]): each input's baby steps share its own hoisted ModUp, the giant
 * rotations of all inputs run as one batched key switch.  Results equal nx
 * calls of fides_linear_transform. */
fides_status fides_linear_transform_batch(fides_ctx* ctx, int nx, const fides_ct* const* xs, int n,
                                          const int32_t* offsets, const fides_pt* const* pts, int bstep, int rescale,
                                          fides_ct* const* outs);
/* EvalConjugate: Ciphertext::conjugate, Ciphertext.cpp:933 */
fides_status fides_conjugate(fides_ctx* ctx, const fides_ct* a, fides_ct* out);
/* Apply an automorphism whose key was uploaded with fides_key_upload_galois */
fides_status fides_automorphism(fides_ctx* ctx, const fides_ct* a, uint32_t galois, fides_ct* out);
/* EvalAdd / EvalSub / EvalNegate: Ciphertext::add/sub, Ciphertext.cpp:177-230 */
fides_status fides_add(fides_ctx* ctx, const fides_ct* a, const fides_ct* b, fides_ct* out);
fides_status fides_sub(fides_ctx* ctx, const fides_ct* a, const fides_ct* b, fides_ct* out);
fides_status fides_negate(fides_ctx* ctx, const fides_ct* a, fides_ct* out);
/* EvalAdd(ct, pt) / EvalMult(ct, pt): Ciphertext::addPt / multPt, Ciphertext.cpp:232,329 */
fides_status fides_add_pt(fides_ctx* ctx, const fides_ct* a, const fides_pt* p, fides_ct* out);
fides_status fides_mult_pt(fides_ctx* ctx, const fides_ct* a, const fides_pt* p, fides_ct* out, int rescale);
/* EvalAdd(ct, double) / EvalMult(ct, double): Ciphertext::addScalar / multScalar */
fides_status fides_add_scalar(fides_ctx* ctx, const fides_ct* a, double v, fides_ct* out);
fides_status fides_mult_scalar(fides_ctx* ctx, const fides_ct* a, double v, fides_ct* out, int rescale);

/* Integer scalar product out = z * a (value times z, scale kept): multIntScalar,
 * src/CKKS/ApproxModEval.cu (multIntScalar). */
fides_status fides_mult_int(fides_ctx* ctx, const fides_ct* a, int64_t z, fides_ct* out);
/* Multiplication by the monomial X^power (0 <= power < 2N): Ciphertext::multMonomial,
 * used by src/CKKS/Bootstrap.cu:268 and ApproxModEval.cu.  X^(N/2) multiplies every
 * slot by i. */
fides_status fides_mult_monomial(fides_ctx* ctx, const fides_ct* a, uint32_t power, fides_ct* out);
/* ModRaise: limb 0 of a (mod q_0), lifted to (-q_0/2, q_0/2] and re-expressed
 * over all L ciphertext moduli (level L-1): src/CKKS/Bootstrap.cu:380. */
fides_status fides_mod_raise(fides_ctx* ctx, const fides_ct* a, fides_ct* out);
/* EvalChebyshevSeries (api/CryptoContext.hpp:171-173, src/CKKS/ApproxModEval.cu:370):
 * sum_k coeffs[k] T_k(y), y = (2x - (lo + hi)) / (hi - lo), degree <= 2047.
 * Consumes ceil(log2(degree + 1)) + 1 levels (+1 when [lo, hi] != [-1, 1]). */
fides_status fides_chebyshev_series(fides_ctx* ctx, const fides_ct* a, const double* coeffs, int degree, double lo,
                                    double hi, fides_ct* out);

/* ---- bootstrapping (api/CryptoContext.hpp:80-82,180-181 EvalBootstrapSetup /
 *      EvalBootstrapKeyGen / EvalBootstrap; src/CKKS/Bootstrap.cu:169-320) ---- */
typedef struct {
    int slots;           /* slots of the ciphertexts bootstrapped: a power of two up to N/2
                            (0 means N/2, full packing); below N/2 (sparse packing) the
                            raised polynomial is first projected onto the n-slot subring
                            by log2(N/2n) rotate-and-add steps */
    int level_budget[2]; /* levels of CoeffsToSlots and SlotsToCoeffs (0 means 3) */
    int cheb_degree;     /* degree of the EvalMod Chebyshev series (0 means 119) */
    double K;            /* EvalMod input range [-K, K] in units of q_0 (0 means 16) */
    int double_angle;    /* double-angle iterations (0 means 3) */
    int correction;      /* the input is multiplied by 2^correction before ModRaise and the
                            result's scale corrected after (exact): EvalMod's noise then
                            weighs 2^correction times less against the message, valid while
                            every message coefficient times D 2^correction stays below
                            2^-8 q_0 (0: none) */
} fides_boot_params;
/* Precompute the CoeffsToSlots / SlotsToCoeffs diagonals (device-resident)
 * and the EvalMod series.  The keys it needs: relinearisation, conjugation
 * and the rotations listed by fides_bootstrap_info. */
fides_status fides_bootstrap_setup(fides_ctx* ctx, const fides_boot_params* params);
/* Output level of a bootstrapped ciphertext and the rotation indices the
 * bootstrap needs keys for (rotations may be NULL to query the count): first
 * the CoeffsToSlots / SlotsToCoeffs rotations over `slots` slots (|index| <=
 * slots / 2), then, for sparse packing, the indices slots, 2 slots, ..., N/4
 * over the full N/2 slots (the subring projection).  fides_bootstrap_keygen
 * generates them with the right slot counts. */
fides_status fides_bootstrap_info(fides_ctx* ctx, int slots, int* output_level, int* num_rotations,
                                  int32_t* rotations);
/* EvalBootstrapKeyGen (api/CryptoContext.hpp:181): the rotation keys
 * fides_bootstrap_info lists and the conjugation key, for a bootstrap set up
 * for `slots` (0: N/2). */
fides_status fides_bootstrap_keygen(fides_ctx* ctx, const fides_sk* sk, int slots, uint64_t seed);
/* EvalBootstrap: refresh a ciphertext (only its limb 0 is read) to the
 * output level, same slots and message. */
fides_status fides_bootstrap(fides_ctx* ctx, const fides_ct* in, fides_ct* out);
/* EvalBootstrap with numIterations (api/CryptoContext.hpp:180-181): 1 is
 * fides_bootstrap; 2 bootstraps again the first result's error, scaled by
 * 2^precision (0: 12), and subtracts it (about precision more bits).  For 2
 * the input must be at or above the bootstrap's output level; the result is
 * one level below that output level. */
fides_status fides_bootstrap_iter(fides_ctx* ctx, const fides_ct* in, int iterations, int precision,
                                  fides_ct* out);
/* EvalBootstrap of n ciphertexts of the same slot count together: the linear
 * transforms batch their giant-step rotations over the inputs, and EvalMod
 * runs the 2n real / imaginary lanes through one batched HMult per step.
 * out[i] equals fides_bootstrap(in[i]) bit for bit.  No counterpart in the
 * reference, which bootstraps one ciphertext per call (Bootstrap.cu:169-320). */
fides_status fides_bootstrap_batch(fides_ctx* ctx, int n, const fides_ct* const* in, fides_ct* const* out);

/* ---- serving: continuous batching over one context (no counterpart in the
 *      reference, which has no serving layer) ---- */
typedef enum { FIDES_OP_HMULT = 0, FIDES_OP_ROTATE = 1, FIDES_OP_BOOTSTRAP = 2 } fides_op;
typedef struct {
    uint64_t completed;    /* requests finished since the last reset */
    uint64_t batches;      /* batches launched */
    double p50_ms;         /* latency submit -> completion, median */
    double p99_ms;         /* 99th percentile */
    double mean_queue_ms;  /* submit -> batch launch */
    double throughput;     /* completed requests per second (first submit -> last completion) */
    size_t reserved_bytes; /* HBM currently charged against the budget */
} fides_srv_stats_t;
/* Start the loop: `num_streams` streams, each with a workspace for
 * `max_batch` requests, and a fixed HBM budget (bytes) that the workspaces
 * and the outputs of admitted requests are charged against. */
fides_status fides_srv_create(fides_ctx* ctx, size_t hbm_budget, int max_batch, int num_streams,
                              fides_server** out);
/* Queue a request: FIDES_OP_HMULT (a*b, relinearised and rescaled) or
 * FIDES_OP_ROTATE (a rotated by index).  a, b and out must stay alive until
 * the request completes; the result lands in out. */
fides_status fides_srv_submit(fides_server* srv, int op, const fides_ct* a, const fides_ct* b, int32_t index,
                              fides_ct* out, uint64_t* request_id);
/* Wait for a request (FIDES_TIMEOUT after timeout_s); returns its status. */
fides_status fides_srv_wait(fides_server* srv, uint64_t request_id, double timeout_s);
fides_status fides_srv_stats(fides_server* srv, fides_srv_stats_t* out);
fides_status fides_srv_reset_stats(fides_server* srv);
/* Drain the queue, stop the loop, release its streams and workspaces. */
fides_status fides_srv_destroy(fides_server* srv);

/* ---- raw limb kernels on device memory (LimbPartition NTT/INTT entry points,
 *      src/CKKS/LimbPartition.cu; used for the plain RNS polynomial multiply) ---- */
/* In-place forward / inverse NTT of `nlimbs` limbs at `data` (device pointer),
 * limb i using prime index prime0 + i. */
fides_status fides_ntt(fides_ctx* ctx, uint64_t* data, int prime0, int nlimbs, int inverse);
/* The same transform over npoly polynomials of nlimbs limbs each, polynomial k
 * at data + k * poly_stride words, in one launch pair (the batched form the
 * key-switch pipeline uses; LimbPartitionBatch.cu runs NTT_ per partition). */
fides_status fides_ntt_batch(fides_ctx* ctx, uint64_t* data, size_t poly_stride, int npoly, int prime0, int nlimbs,
                             int inverse);
/* c = a * b in R_q for nlimbs limbs of coefficient-form inputs (device
 * pointers): NTT of a and b into a_ntt / b_ntt (caller-provided device
 * scratch), then one INTT with the product fused into its load.  `c` may
 * alias a or b. */
fides_status fides_polymul(fides_ctx* ctx, const uint64_t* a, const uint64_t* b, uint64_t* c, uint64_t* a_ntt,
                           uint64_t* b_ntt, int prime0, int nlimbs);

/* Same product as fides_polymul, but allocating nothing and asking for no
 * scratch: for callers that cannot obtain device memory when they multiply
 * (hosts whose own allocator owns the whole device, loops that must not call
 * cudaMalloc/cudaFree because those synchronise the device).  No counterpart in the
 * reference.  The scratch is a fixed 8 MiB device array inside the library
 * (2^19 words per operand): nlimbs * N must not exceed 2^19, larger calls
 * return FIDES_BAD_ARG.  The first call on a device looks the array up
 * (cudaGetSymbolAddress) and should precede any stream capture.  All calls
 * share the array; calls that overlap on the GPU race and must be serialised
 * by the caller.  `c` may alias a or b. */
fides_status fides_polymul_noalloc(fides_ctx* ctx, const uint64_t* a, const uint64_t* b, uint64_t* c, int prime0,
                                   int nlimbs);

/* ---- client side (OpenFHE's role in FIDESlib: KeyGen, Encrypt, Decrypt,
 *      MakeCKKSPackedPlaintext; api/CryptoContext.hpp:71-106) ---- */
/* Secret key with `hamming_weight` nonzero ternary coefficients (0 = uniform ternary). */
fides_status fides_keygen(fides_ctx* ctx, uint64_t seed, int hamming_weight, fides_sk** out);
fides_status fides_sk_free(fides_ctx* ctx, fides_sk* sk);
/* Public key (b = -a s + e, a) over the ciphertext moduli (KeyGen's publicKey). */
fides_status fides_keygen_public(fides_ctx* ctx, const fides_sk* sk, uint64_t seed, fides_pk** out);
fides_status fides_pk_free(fides_ctx* ctx, fides_pk* pk);
/* Public-key encryption: c = (v b + e0 + m, v a + e1), v uniform ternary. */
fides_status fides_encrypt_pk(fides_ctx* ctx, const fides_pk* pk, const double* values, int slots, int level,
                              double scale, uint64_t seed, fides_ct** out);
/* Generate and upload the relinearisation key (EvalMultKeyGen). */
fides_status fides_keygen_relin(fides_ctx* ctx, const fides_sk* sk, uint64_t seed);
/* Generate and upload rotation keys for the given slot indices (EvalRotateKeyGen). */
fides_status fides_keygen_rotations(fides_ctx* ctx, const fides_sk* sk, int n, const int32_t* indices, int slots,
                                    uint64_t seed);
fides_status fides_keygen_conjugate(fides_ctx* ctx, const fides_sk* sk, uint64_t seed);
/* Key compression for the switching keys generated from here on, a bit
 * mask: bit 0 the rotation and conjugation keys (the default, 1), bit 1 the
 * relinearisation key.  A compressed key stores its b half and the seed of
 * its uniform a half, which the key-switch kernels regenerate (one
 * counter-based hash per coefficient) instead of reading it: half the HBM per
 * key and half the key bytes read per key switch.  A compressed
 * relinearisation key turns off the key switch fused into the digits' NTT
 * row pass (batched HMults read an explicit a half once per batch).
 * Uploaded or imported keys keep both halves.  The key layout this replaces:
 * KeySwitchingKey a / b (src/CKKS/KeySwitchingKey.cu:20-35); the reference
 * has no compressed form. */
fides_status fides_set_key_compression(fides_ctx* ctx, int mask);
/* Export generated switching keys (dnum*(L+K)*N words each) for interop tests. */
fides_status fides_key_export(fides_ctx* ctx, uint32_t galois, uint64_t* b, uint64_t* a);
/* Encode `slots` complex values (re, im interleaved) at `level` and `scale`
 * into evaluation-form residues m[(level+1)*N] (host memory).  The FFT,
 * rounding and NTT run on the device.  Replaces OpenFHE's
 * MakeCKKSPackedPlaintext, which the reference calls on the CPU
 * (api/CryptoContext.cpp:475-514). */
fides_status fides_encode(fides_ctx* ctx, const double* values, int slots, int level, double scale, uint64_t* m);
/* Encrypt with the secret key (symmetric CKKS encryption); the error and
 * uniform polynomials are drawn on the device from `seed`. */
fides_status fides_encrypt(fides_ctx* ctx, const fides_sk* sk, const double* values, int slots, int level,
                           double scale, uint64_t seed, fides_ct** out);
/* Synthetic ciphertext with residues drawn uniformly on the device (seeded):
 * benchmark and test input without a host round trip. */
fides_status fides_ct_random(fides_ctx* ctx, int level, uint64_t seed, fides_ct** out);
/* Decrypt and decode into `slots` complex values (re, im interleaved): the
 * CRT of the first three moduli and the decoding FFT run on the device, only
 * the slots are copied back.  Replaces OpenFHE's Decrypt
 * (api/CryptoContext.cpp:560-626). */
fides_status fides_decrypt(fides_ctx* ctx, const fides_sk* sk, const fides_ct* ct, double* values, int slots);

#ifdef __cplusplus
}
#endif
#endif
