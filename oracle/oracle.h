/*
 * oracle.h -- CPU restatement of the CKKS-RNS evaluation path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg (and
 * the `--impl reference` arm, which times it as the CPU implementation of the
 * path) may load it.  The product library never links or calls it.
 *
 * Every routine cites the FIDESlib file:line whose behaviour it restates.  The
 * arithmetic is exact modular arithmetic on canonical residues in [0, p); the
 * formulas (bit-reversed evaluation order, partial-digit ModUp constants,
 * ModDown, OpenFHE-style rescale with the centred SwitchModulus, the
 * automorphism scatter rule) follow the reference so that residues agree bit
 * for bit.
 *
 * Conventions (shared with the CUDA path):
 *   - A polynomial is limb-major: limb i occupies a[i*N .. i*N+N-1].
 *   - Prime indices: 0..L-1 are the Q primes q_0..q_{L-1}; L..L+K-1 are the
 *     special primes p_0..p_{K-1}.
 *   - A ciphertext at level l has n = l+1 Q limbs (primes 0..l).
 *   - An extended-basis polynomial at level l has n+K limbs: Q primes 0..l
 *     followed by the K special primes.
 *   - Digits are contiguous blocks of alpha = ceil(L/dnum) Q primes (the
 *     OpenFHE HYBRID partition).  At level l digit d holds the primes
 *     d*alpha .. min(d*alpha+alpha-1, l); digits with no prime <= l are idle.
 *   - Switching keys are [dnum][L+K][N] arrays (one RNS polynomial per digit)
 *     in evaluation (NTT, bit-reversed) form.
 */
#ifndef FIDES_ORACLE_H
#define FIDES_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_MAXP 128

typedef struct or_ctx {
    int logN, N;
    int L;  /* number of Q primes */
    int K;  /* number of special primes */
    int dnum, alpha;
    uint64_t prime[OR_MAXP];
    uint64_t root[OR_MAXP];     /* primitive 2N-th root psi per prime */
    uint64_t n_inv[OR_MAXP];
    uint64_t *psi, *psi_sh;     /* [L+K][N] psi^{bitrev(j)} and Shoup companions */
    uint64_t *ipsi, *ipsi_sh;   /* [L+K][N] psi^{-bitrev(j)} and Shoup companions */
} or_ctx;

/* ---- scalar arithmetic (reference src/Math.cu:20-37, test/MathTest.cu) ---- */
uint64_t or_mulmod(uint64_t a, uint64_t b, uint64_t p);
uint64_t or_powmod(uint64_t a, uint64_t e, uint64_t p);
uint64_t or_invmod(uint64_t a, uint64_t p);
int or_is_prime(uint64_t n);
uint32_t or_bitrev(uint32_t x, int bits);
uint64_t or_generator(uint64_t p);
uint64_t or_unity_root(uint64_t p, uint64_t order);
int or_find_primes(int logN, int bits, int count, uint64_t upper_exclusive, uint64_t* out);

/* ---- context ---- */
or_ctx* or_ctx_new(int logN, int L, int K, int dnum, const uint64_t* primes);
void or_ctx_free(or_ctx* c);
int or_num_digits(const or_ctx* c, int level);
void or_get_psi_tables(const or_ctx* c, int pidx, uint64_t* psi_br, uint64_t* ipsi_br);

/* ---- CRT constants (restated from the definitions OpenFHE exports and the
 *      reference uploads, src/ConstantsGPU.cu:439-645) ---- */
void or_modup_consts(const or_ctx* c, int level, int d, uint64_t* hat_inv /* [alpha] */,
                     uint64_t* hat_mod /* [alpha][L+K] */);
void or_moddown_consts(const or_ctx* c, uint64_t* phat_inv /* [K] */, uint64_t* phat_mod /* [K][L] */,
                       uint64_t* p_inv /* [L] */);

/* ---- limb transforms (src/NTT.cu, test/cpuNTT_nega.cpp:24-95) ---- */
void or_ntt(const or_ctx* c, uint64_t* a, int pidx);
void or_intt(const or_ctx* c, uint64_t* a, int pidx);
void or_ntt_limbs(const or_ctx* c, uint64_t* a, const int* pidx, int nlimbs, int inverse);
/* Independent check: twist by psi^i then cyclic FFT with psi^2, natural order
 * output (test/cpuNTT_nega.cpp:140-160 nega_fft2 + test/cpuNTT.cpp:14-47). */
void or_nega_fft2(uint64_t* a, int logN, uint64_t p, uint64_t psi, int invert);

/* ---- element-wise (src/ModMult.cu, src/AddSub.cu, ElemenwiseBatchKernels.cu) ---- */
void or_polymul(const or_ctx* c, int nlimbs, const int* pidx, const uint64_t* a, const uint64_t* b, uint64_t* out);
void or_tensor(const or_ctx* c, int level, const uint64_t* c0, const uint64_t* c1, const uint64_t* d0,
               const uint64_t* d1, uint64_t* e0, uint64_t* e1, uint64_t* e2);
void or_automorph(const or_ctx* c, int nlimbs, const uint64_t* in, uint64_t* out, uint32_t k);
uint32_t or_rotation_galois(const or_ctx* c, int index, int slots);

/* ---- key switching pipeline ---- */
void or_modup(const or_ctx* c, int level, const uint64_t* in_eval, uint64_t* digits /* [num_d][n+K][N] */);
void or_ks_inner(const or_ctx* c, int level, const uint64_t* digits, const uint64_t* ksk_b, const uint64_t* ksk_a,
                 uint64_t* out_b, uint64_t* out_a);
void or_moddown(const or_ctx* c, int level, const uint64_t* in_ext, uint64_t* out);
void or_rescale(const or_ctx* c, int level, const uint64_t* in, uint64_t* out);

/* ---- composite operations ---- */
void or_hmult(const or_ctx* c, int level, const uint64_t* a0, const uint64_t* a1, const uint64_t* b0,
              const uint64_t* b1, const uint64_t* ksk_b, const uint64_t* ksk_a, int rescale, uint64_t* out0,
              uint64_t* out1);
void or_rotate_hoisted(const or_ctx* c, int level, const uint64_t* c0, const uint64_t* c1, int nrot,
                       const uint32_t* galois, const uint64_t* const* ksk_b, const uint64_t* const* ksk_a,
                       uint64_t* const* out0, uint64_t* const* out1);
void or_rotate(const or_ctx* c, int level, const uint64_t* c0, const uint64_t* c1, uint32_t galois,
               const uint64_t* ksk_b, const uint64_t* ksk_a, uint64_t* out0, uint64_t* out1);

/* ---- misc ---- */
void or_set_threads(int n);
int or_get_threads(void);
void or_random_residues(const or_ctx* c, int nlimbs, const int* pidx, uint64_t seed, uint64_t* out);

#ifdef __cplusplus
}
#endif
#endif
