/*
 * oracle.c -- CPU restatement of the CKKS-RNS evaluation path.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Plain C, exact modular arithmetic
 * through unsigned __int128, OpenMP over limbs so that the same code doubles
 * as the timed CPU baseline.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;

static int g_threads = 0;

void or_set_threads(int n) { g_threads = n; }
int or_get_threads(void) {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* scalar arithmetic                                                        */
/* ------------------------------------------------------------------------ */

uint64_t or_mulmod(uint64_t a, uint64_t b, uint64_t p) { return (uint64_t)(((u128)a * b) % p); }

static inline uint64_t addmod(uint64_t a, uint64_t b, uint64_t p) {
    uint64_t s = a + b;
    return s >= p ? s - p : s;
}
static inline uint64_t submod(uint64_t a, uint64_t b, uint64_t p) { return a >= b ? a - b : a + p - b; }

/* Shoup multiplication by a precomputed constant: w_sh = floor(w * 2^64 / p).
 * Exact for any a < 2^64 and w < p < 2^63 (Shoup; Harvey 2014).  Used only
 * inside the transforms to keep the CPU baseline from being dominated by
 * 128-bit division; every other product uses the plain % path. */
static inline uint64_t shoup_pre(uint64_t w, uint64_t p) { return (uint64_t)(((u128)w << 64) / p); }
static inline uint64_t mulmod_shoup(uint64_t a, uint64_t w, uint64_t w_sh, uint64_t p) {
    uint64_t q = (uint64_t)(((u128)a * w_sh) >> 64);
    uint64_t r = a * w - q * p;
    return r >= p ? r - p : r;
}

/* src/Math.cu:20-37: modpow by square-and-multiply, modinv by Fermat. */
uint64_t or_powmod(uint64_t a, uint64_t e, uint64_t p) {
    uint64_t r = 1 % p;
    a %= p;
    while (e) {
        if (e & 1) r = or_mulmod(r, a, p);
        a = or_mulmod(a, a, p);
        e >>= 1;
    }
    return r;
}

uint64_t or_invmod(uint64_t a, uint64_t p) { return or_powmod(a, p - 2, p); }

int or_is_prime(uint64_t n) {
    static const uint64_t bases[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    if (n < 2) return 0;
    for (int i = 0; i < 12; ++i) {
        if (n == bases[i]) return 1;
        if (n % bases[i] == 0) return 0;
    }
    uint64_t d = n - 1;
    int s = 0;
    while ((d & 1) == 0) {
        d >>= 1;
        ++s;
    }
    for (int i = 0; i < 12; ++i) {
        uint64_t x = or_powmod(bases[i], d, n);
        if (x == 1 || x == n - 1) continue;
        int comp = 1;
        for (int r = 1; r < s; ++r) {
            x = or_mulmod(x, x, n);
            if (x == n - 1) {
                comp = 0;
                break;
            }
        }
        if (comp) return 0;
    }
    return 1;
}

uint32_t or_bitrev(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; ++i) {
        r = (r << 1) | (x & 1);
        x >>= 1;
    }
    return r;
}

/* src/ConstantsGPU.cu:40-62 generator(): the smallest g whose powers g^(phi/f)
 * differ from 1 for every prime factor f of phi = p-1. */
uint64_t or_generator(uint64_t p) {
    uint64_t fact[64];
    int nf = 0;
    uint64_t phi = p - 1, n = phi;
    for (uint64_t i = 2; i * i <= n; ++i) {
        if (n % i == 0) {
            fact[nf++] = i;
            while (n % i == 0) n /= i;
        }
    }
    if (n > 1) fact[nf++] = n;
    for (uint64_t g = 2; g <= p; ++g) {
        int ok = 1;
        for (int i = 0; i < nf && ok; ++i) ok = or_powmod(g, phi / fact[i], p) != 1;
        if (ok) return g;
    }
    return 0;
}

/* src/ConstantsGPU.cu:64-72 unity_root(): g^((q-1)/order). */
uint64_t or_unity_root(uint64_t p, uint64_t order) {
    if ((p - 1) % order != 0) return 0;
    uint64_t g = or_generator(p);
    return or_powmod(g, (p - 1) / order, p);
}

/* Deterministic descending search for NTT-friendly primes p = 1 (mod 2N),
 * p < upper_exclusive, p >= 2^(bits-1).  Returns how many were found. */
int or_find_primes(int logN, int bits, int count, uint64_t upper_exclusive, uint64_t* out) {
    const uint64_t step = 2ull << logN;
    uint64_t lim = upper_exclusive;
    if (bits < 64 && ((1ull << bits) < lim || lim == 0)) lim = 1ull << bits;
    uint64_t lo = 1ull << (bits - 1);
    /* largest candidate < lim with candidate = 1 mod step */
    uint64_t cand = ((lim - 2) / step) * step + 1;
    int found = 0;
    while (found < count && cand > lo) {
        if (or_is_prime(cand)) out[found++] = cand;
        cand -= step;
    }
    return found;
}

/* ------------------------------------------------------------------------ */
/* context                                                                  */
/* ------------------------------------------------------------------------ */

or_ctx* or_ctx_new(int logN, int L, int K, int dnum, const uint64_t* primes) {
    if (L + K > OR_MAXP || logN < 1 || logN > 20 || dnum < 1) return NULL;
    or_ctx* c = (or_ctx*)calloc(1, sizeof(or_ctx));
    c->logN = logN;
    c->N = 1 << logN;
    c->L = L;
    c->K = K;
    c->dnum = dnum;
    c->alpha = (L + dnum - 1) / dnum;
    const int np = L + K, N = c->N;
    c->psi = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)np * N);
    c->psi_sh = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)np * N);
    c->ipsi = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)np * N);
    c->ipsi_sh = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)np * N);
    for (int i = 0; i < np; ++i) c->prime[i] = primes[i];
    int bad = 0;
#pragma omp parallel for schedule(dynamic) num_threads(or_get_threads())
    for (int i = 0; i < np; ++i) {
        uint64_t p = c->prime[i];
        uint64_t psi = or_unity_root(p, 2ull * N);
        if (psi == 0) {
            bad = 1;
            continue;
        }
        c->root[i] = psi;
        c->n_inv[i] = or_invmod((uint64_t)N % p, p);
        uint64_t ipsi = or_invmod(psi, p);
        uint64_t *t = c->psi + (size_t)i * N, *it = c->ipsi + (size_t)i * N;
        /* natural-order powers first, then bit-reverse (ConstantsGPU.cu:226-271) */
        uint64_t* nat = (uint64_t*)malloc(sizeof(uint64_t) * N);
        uint64_t* inat = (uint64_t*)malloc(sizeof(uint64_t) * N);
        nat[0] = 1;
        inat[0] = 1;
        for (int j = 1; j < N; ++j) {
            nat[j] = or_mulmod(nat[j - 1], psi, p);
            inat[j] = or_mulmod(inat[j - 1], ipsi, p);
        }
        for (int j = 0; j < N; ++j) {
            uint32_t r = or_bitrev((uint32_t)j, logN);
            t[j] = nat[r];
            it[j] = inat[r];
            c->psi_sh[(size_t)i * N + j] = shoup_pre(t[j], p);
            c->ipsi_sh[(size_t)i * N + j] = shoup_pre(it[j], p);
        }
        free(nat);
        free(inat);
    }
    if (bad) {
        or_ctx_free(c);
        return NULL;
    }
    return c;
}

void or_ctx_free(or_ctx* c) {
    if (!c) return;
    free(c->psi);
    free(c->psi_sh);
    free(c->ipsi);
    free(c->ipsi_sh);
    free(c);
}

int or_num_digits(const or_ctx* c, int level) { return level / c->alpha + 1; }

void or_get_psi_tables(const or_ctx* c, int pidx, uint64_t* psi_br, uint64_t* ipsi_br) {
    memcpy(psi_br, c->psi + (size_t)pidx * c->N, sizeof(uint64_t) * c->N);
    memcpy(ipsi_br, c->ipsi + (size_t)pidx * c->N, sizeof(uint64_t) * c->N);
}

/* ------------------------------------------------------------------------ */
/* transforms                                                               */
/* ------------------------------------------------------------------------ */

/* Forward negacyclic NTT, Cooley-Tukey over the bit-reversed psi table,
 * natural-order coefficients in, bit-reversed evaluations out:
 *   out[i] = sum_j a_j psi^{(2*bitrev(i)+1) j}.
 * This is the loop of test/cpuNTT_nega.cpp:24-78 without its final bit
 * reversal; the GPU order is that bit-reversed order (NTTtests.cu:933-1040). */
void or_ntt(const or_ctx* c, uint64_t* a, int pidx) {
    const int N = c->N;
    const uint64_t p = c->prime[pidx];
    const uint64_t* w = c->psi + (size_t)pidx * N;
    const uint64_t* wsh = c->psi_sh + (size_t)pidx * N;
    int t = N >> 1;
    for (int m = 1; m < N; m <<= 1, t >>= 1) {
        for (int i = 0; i < m; ++i) {
            const int j1 = 2 * i * t;
            const uint64_t W = w[m + i], Wsh = wsh[m + i];
            for (int j = j1; j < j1 + t; ++j) {
                uint64_t u = a[j];
                uint64_t v = mulmod_shoup(a[j + t], W, Wsh, p);
                a[j] = addmod(u, v, p);
                a[j + t] = submod(u, v, p);
            }
        }
    }
}

/* Inverse: Gentleman-Sande over the bit-reversed inverse table, then N^-1
 * (src/NTT.cu INTT_ with the N^-1 fold of NTTfusions.cuh:432-517). */
void or_intt(const or_ctx* c, uint64_t* a, int pidx) {
    const int N = c->N;
    const uint64_t p = c->prime[pidx];
    const uint64_t* w = c->ipsi + (size_t)pidx * N;
    const uint64_t* wsh = c->ipsi_sh + (size_t)pidx * N;
    int t = 1;
    for (int m = N >> 1; m >= 1; m >>= 1, t <<= 1) {
        for (int i = 0; i < m; ++i) {
            const int j1 = 2 * i * t;
            const uint64_t W = w[m + i], Wsh = wsh[m + i];
            for (int j = j1; j < j1 + t; ++j) {
                uint64_t u = a[j], v = a[j + t];
                a[j] = addmod(u, v, p);
                a[j + t] = mulmod_shoup(submod(u, v, p), W, Wsh, p);
            }
        }
    }
    const uint64_t ni = c->n_inv[pidx], nish = shoup_pre(ni, p);
    for (int j = 0; j < N; ++j) a[j] = mulmod_shoup(a[j], ni, nish, p);
}

void or_ntt_limbs(const or_ctx* c, uint64_t* a, const int* pidx, int nlimbs, int inverse) {
#pragma omp parallel for schedule(static) num_threads(or_get_threads())
    for (int i = 0; i < nlimbs; ++i) {
        if (inverse)
            or_intt(c, a + (size_t)i * c->N, pidx[i]);
        else
            or_ntt(c, a + (size_t)i * c->N, pidx[i]);
    }
}

/* test/cpuNTT_nega.cpp:140-160 + test/cpuNTT.cpp:14-47: an independent
 * formulation (twist by psi^i, cyclic radix-2 FFT with psi^2, natural-order
 * output) used only to pin or_ntt's ordering convention. */
void or_nega_fft2(uint64_t* a, int logN, uint64_t p, uint64_t psi, int invert) {
    const int n = 1 << logN;
    const uint64_t ipsi = or_invmod(psi, p);
    if (!invert)
        for (int i = 0; i < n; ++i) a[i] = or_mulmod(a[i], or_powmod(psi, (uint64_t)i, p), p);
    for (int i = 0; i < n; ++i) {
        int r = (int)or_bitrev((uint32_t)i, logN);
        if (i < r) {
            uint64_t t = a[i];
            a[i] = a[r];
            a[r] = t;
        }
    }
    const uint64_t root = or_mulmod(psi, psi, p), root_1 = or_mulmod(ipsi, ipsi, p);
    for (int len = 2; len <= n; len <<= 1) {
        uint64_t wlen = invert ? root_1 : root;
        for (int i = len; i < n; i <<= 1) wlen = or_mulmod(wlen, wlen, p);
        for (int i = 0; i < n; i += len) {
            uint64_t w = 1;
            for (int j = 0; j < len / 2; ++j) {
                uint64_t u = a[i + j], v = or_mulmod(a[i + j + len / 2], w, p);
                a[i + j] = addmod(u, v, p);
                a[i + j + len / 2] = submod(u, v, p);
                w = or_mulmod(w, wlen, p);
            }
        }
    }
    if (invert) {
        uint64_t ni = or_invmod((uint64_t)n % p, p);
        for (int i = 0; i < n; ++i) a[i] = or_mulmod(a[i], ni, p);
        for (int i = 0; i < n; ++i) a[i] = or_mulmod(a[i], or_powmod(ipsi, (uint64_t)i, p), p);
    }
}

/* ------------------------------------------------------------------------ */
/* element-wise                                                             */
/* ------------------------------------------------------------------------ */

void or_polymul(const or_ctx* c, int nlimbs, const int* pidx, const uint64_t* a, const uint64_t* b, uint64_t* out) {
    const size_t N = c->N;
#pragma omp parallel for schedule(static) num_threads(or_get_threads())
    for (int i = 0; i < nlimbs; ++i) {
        const uint64_t p = c->prime[pidx[i]];
        for (size_t j = 0; j < N; ++j) out[i * N + j] = or_mulmod(a[i * N + j], b[i * N + j], p);
    }
}

/* ElemenwiseBatchKernels.cu:1398 binomialMult_: c0*d0, c0*d1 + c1*d0, c1*d1. */
void or_tensor(const or_ctx* c, int level, const uint64_t* c0, const uint64_t* c1, const uint64_t* d0,
               const uint64_t* d1, uint64_t* e0, uint64_t* e1, uint64_t* e2) {
    const size_t N = c->N;
    const int n = level + 1;
#pragma omp parallel for schedule(static) num_threads(or_get_threads())
    for (int i = 0; i < n; ++i) {
        const uint64_t p = c->prime[i];
        for (size_t j = 0; j < N; ++j) {
            const size_t k = i * N + j;
            uint64_t x0 = c0[k], x1 = c1[k], y0 = d0[k], y1 = d1[k];
            e0[k] = or_mulmod(x0, y0, p);
            e1[k] = addmod(or_mulmod(x0, y1, p), or_mulmod(x1, y0, p), p);
            e2[k] = or_mulmod(x1, y1, p);
        }
    }
}

/* src/Rotation.cuh:14-26 automorph_slot + Rotation.cu:20-27: the value at
 * evaluation slot j moves to slot bitrev(((2*bitrev(j)+1)*k mod 2N) >> 1). */
void or_automorph(const or_ctx* c, int nlimbs, const uint64_t* in, uint64_t* out, uint32_t k) {
    const int N = c->N, logN = c->logN;
    const uint32_t mask = (uint32_t)(2 * N - 1);
#pragma omp parallel for schedule(static) num_threads(or_get_threads())
    for (int i = 0; i < nlimbs; ++i) {
        for (int j = 0; j < N; ++j) {
            uint32_t e = 2 * or_bitrev((uint32_t)j, logN) + 1;
            uint32_t r = (uint32_t)(((uint64_t)e * k) & mask) >> 1;
            out[(size_t)i * N + or_bitrev(r, logN)] = in[(size_t)i * N + j];
        }
    }
}

/* Ciphertext.cpp:157-165 normalyzeIndex + RNSPoly.cpp:559-561
 * automorph_index_precomp: k = 5^(2N - idx) mod 2N. */
uint32_t or_rotation_galois(const or_ctx* c, int index, int slots) {
    const int N = c->N;
    int idx = index % slots;
    if (idx < 0) idx += slots;
    if (idx > slots / 2) idx += N / 2 - slots;
    return (uint32_t)or_powmod(5, (uint64_t)(2 * N - idx), (uint64_t)(2 * N));
}

/* ------------------------------------------------------------------------ */
/* CRT constants                                                            */
/* ------------------------------------------------------------------------ */

static void digit_range(const or_ctx* c, int level, int d, int* lo, int* hi) {
    *lo = d * c->alpha;
    int h = d * c->alpha + c->alpha - 1;
    if (h > level) h = level;
    if (h > c->L - 1) h = c->L - 1;
    *hi = h;
}

/* PartQlHatInvModq / PartQlHatModp for the partial digit at `level`
 * (ConstantsGPU.cu:545-645, Conv.cu:144-287): with D' the primes of digit d
 * that are <= level and Q' their product,
 *   hat_inv[i]    = (Q'/q_i)^-1 mod q_i
 *   hat_mod[i][t] = (Q'/q_i) mod prime t   for every prime index t. */
void or_modup_consts(const or_ctx* c, int level, int d, uint64_t* hat_inv, uint64_t* hat_mod) {
    int lo, hi;
    digit_range(c, level, d, &lo, &hi);
    const int np = c->L + c->K;
    for (int i = lo; i <= hi; ++i) {
        uint64_t qi = c->prime[i], acc = 1;
        for (int k = lo; k <= hi; ++k)
            if (k != i) acc = or_mulmod(acc, c->prime[k] % qi, qi);
        hat_inv[i - lo] = or_invmod(acc, qi);
        for (int t = 0; t < np; ++t) {
            uint64_t pt = c->prime[t], a2 = 1;
            for (int k = lo; k <= hi; ++k)
                if (k != i) a2 = or_mulmod(a2, c->prime[k] % pt, pt);
            hat_mod[(size_t)(i - lo) * np + t] = a2;
        }
    }
}

/* PHatInvModp, PHatModq, PInvModq (ConstantsGPU.cu:482-543, Conv.cu:26-131). */
void or_moddown_consts(const or_ctx* c, uint64_t* phat_inv, uint64_t* phat_mod, uint64_t* p_inv) {
    const int L = c->L, K = c->K;
    for (int k = 0; k < K; ++k) {
        uint64_t pk = c->prime[L + k], acc = 1;
        for (int m = 0; m < K; ++m)
            if (m != k) acc = or_mulmod(acc, c->prime[L + m] % pk, pk);
        phat_inv[k] = or_invmod(acc, pk);
        for (int j = 0; j < L; ++j) {
            uint64_t qj = c->prime[j], a2 = 1;
            for (int m = 0; m < K; ++m)
                if (m != k) a2 = or_mulmod(a2, c->prime[L + m] % qj, qj);
            phat_mod[(size_t)k * L + j] = a2;
        }
    }
    for (int j = 0; j < L; ++j) {
        uint64_t qj = c->prime[j], acc = 1;
        for (int m = 0; m < K; ++m) acc = or_mulmod(acc, c->prime[L + m] % qj, qj);
        p_inv[j] = or_invmod(acc, qj);
    }
}

/* ------------------------------------------------------------------------ */
/* key switching                                                            */
/* ------------------------------------------------------------------------ */

static inline int ext_prime(const or_ctx* c, int level, int m) {
    const int n = level + 1;
    return m < n ? m : c->L + (m - n);
}

/* ModUp (LimbPartitionMGPU.cu:840-848,1124-1151; Conv.cu:144-287):
 * for each active digit d, the primes of the digit keep the input evaluation
 * values; every other prime t of Q_level u P receives
 *   NTT_t( sum_i [INTT_i(x_i) * hat_inv_i]_{q_i} * [Q'/q_i]_t  mod t ). */
void or_modup(const or_ctx* c, int level, const uint64_t* in_eval, uint64_t* digits) {
    const int n = level + 1, K = c->K, N = c->N, np = c->L + c->K;
    const int nd = or_num_digits(c, level);
    const int ext = n + K;
    uint64_t* coef = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n * N);
    memcpy(coef, in_eval, sizeof(uint64_t) * (size_t)n * N);
    {
        int* pid = (int*)malloc(sizeof(int) * n);
        for (int i = 0; i < n; ++i) pid[i] = i;
        or_ntt_limbs(c, coef, pid, n, 1);
        free(pid);
    }
    uint64_t* hat_inv = (uint64_t*)malloc(sizeof(uint64_t) * c->alpha);
    uint64_t* hat_mod = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)c->alpha * np);
    for (int d = 0; d < nd; ++d) {
        int lo, hi;
        digit_range(c, level, d, &lo, &hi);
        or_modup_consts(c, level, d, hat_inv, hat_mod);
        const int nin = hi - lo + 1;
        uint64_t* xt = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)nin * N);
        for (int i = 0; i < nin; ++i) {
            const uint64_t qi = c->prime[lo + i];
            for (int j = 0; j < N; ++j)
                xt[(size_t)i * N + j] = or_mulmod(coef[(size_t)(lo + i) * N + j], hat_inv[i], qi);
        }
        uint64_t* out = digits + (size_t)d * ext * N;
#pragma omp parallel for schedule(dynamic) num_threads(or_get_threads())
        for (int m = 0; m < ext; ++m) {
            const int t = ext_prime(c, level, m);
            uint64_t* o = out + (size_t)m * N;
            if (t >= lo && t <= hi) {
                memcpy(o, in_eval + (size_t)t * N, sizeof(uint64_t) * N);
                continue;
            }
            const uint64_t pt = c->prime[t];
            for (int j = 0; j < N; ++j) {
                u128 acc = 0;
                for (int i = 0; i < nin; ++i) acc += (u128)xt[(size_t)i * N + j] * hat_mod[(size_t)i * np + t];
                o[j] = (uint64_t)(acc % pt);
            }
            or_ntt(c, o, t);
        }
        free(xt);
    }
    free(hat_inv);
    free(hat_mod);
    free(coef);
}

/* Key-switch inner product (ElemenwiseBatchKernels.cu:221-296 fusedDotKSK_2_):
 *   out_b = sum_d D_d * ksk_b[d],  out_a = sum_d D_d * ksk_a[d]  over Q_level u P. */
void or_ks_inner(const or_ctx* c, int level, const uint64_t* digits, const uint64_t* ksk_b, const uint64_t* ksk_a,
                 uint64_t* out_b, uint64_t* out_a) {
    const int n = level + 1, K = c->K, N = c->N, np = c->L + c->K;
    const int nd = or_num_digits(c, level), ext = n + K;
#pragma omp parallel for schedule(static) num_threads(or_get_threads())
    for (int m = 0; m < ext; ++m) {
        const int t = ext_prime(c, level, m);
        const uint64_t pt = c->prime[t];
        for (int j = 0; j < N; ++j) {
            uint64_t sb = 0, sa = 0;
            for (int d = 0; d < nd; ++d) {
                uint64_t x = digits[((size_t)d * ext + m) * N + j];
                sb = addmod(sb, or_mulmod(x, ksk_b[((size_t)d * np + t) * N + j], pt), pt);
                sa = addmod(sa, or_mulmod(x, ksk_a[((size_t)d * np + t) * N + j], pt), pt);
            }
            out_b[(size_t)m * N + j] = sb;
            out_a[(size_t)m * N + j] = sa;
        }
    }
}

/* ModDown (LimbPartition.cu:1911-1993; Conv.cu:26-131 ModDown2;
 * NTTfusions.cuh:245-262 moddown_fusion):
 *   y_k = [INTT_k(x_k) * PHatInv_k]_{p_k}
 *   out_j = (x_j - NTT_j(sum_k y_k * [P/p_k]_{q_j})) * P^-1  mod q_j. */
void or_moddown(const or_ctx* c, int level, const uint64_t* in_ext, uint64_t* out) {
    const int n = level + 1, K = c->K, N = c->N, L = c->L;
    uint64_t* phat_inv = (uint64_t*)malloc(sizeof(uint64_t) * K);
    uint64_t* phat_mod = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)K * L);
    uint64_t* p_inv = (uint64_t*)malloc(sizeof(uint64_t) * L);
    or_moddown_consts(c, phat_inv, phat_mod, p_inv);
    uint64_t* y = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)K * N);
    memcpy(y, in_ext + (size_t)n * N, sizeof(uint64_t) * (size_t)K * N);
#pragma omp parallel for schedule(static) num_threads(or_get_threads())
    for (int k = 0; k < K; ++k) {
        const uint64_t pk = c->prime[L + k];
        uint64_t* yk = y + (size_t)k * N;
        or_intt(c, yk, L + k);
        for (int j = 0; j < N; ++j) yk[j] = or_mulmod(yk[j], phat_inv[k], pk);
    }
#pragma omp parallel for schedule(static) num_threads(or_get_threads())
    for (int i = 0; i < n; ++i) {
        const uint64_t qi = c->prime[i];
        uint64_t* o = out + (size_t)i * N;
        for (int j = 0; j < N; ++j) {
            u128 acc = 0;
            for (int k = 0; k < K; ++k) acc += (u128)y[(size_t)k * N + j] * phat_mod[(size_t)k * L + i];
            o[j] = (uint64_t)(acc % qi);
        }
        or_ntt(c, o, i);
        for (int j = 0; j < N; ++j) o[j] = or_mulmod(submod(in_ext[(size_t)i * N + j], o[j], qi), p_inv[i], qi);
    }
    free(y);
    free(phat_inv);
    free(phat_mod);
    free(p_inv);
}

/* src/CKKS/Rescale.cuh:45-62 SwitchModulus: the centred lift of a value mod om
 * into nm: subtract om when a > floor(om/2), then reduce. */
static inline uint64_t switch_modulus(uint64_t a, uint64_t om, uint64_t nm) {
    if (nm > om) return a > (om >> 1) ? a + (nm - om) : a;
    uint64_t diff = nm - (om % nm);
    u128 v = a;
    if (a > (om >> 1)) v += diff;
    return (uint64_t)(v % nm);
}

/* Rescale (LimbPartitionMGPU.cu:214-394 doubleRescaleMGPU;
 * NTTfusions.cuh:219-242 rescale_fusion, "OpenFHE style"):
 *   T = INTT_l(x_l);  out_j = q_l^-1 * x_j + QlQlInvModqlDivqlModq_j * NTT_j(SwitchModulus(T))
 * with QlQlInvModqlDivqlModq_j = -q_l^-1 mod q_j (a fixed-point identity that
 * tests/test_oracle_pins.py checks against the big-integer definition). */
void or_rescale(const or_ctx* c, int level, const uint64_t* in, uint64_t* out) {
    const int N = c->N;
    const uint64_t ql = c->prime[level];
    uint64_t* top = (uint64_t*)malloc(sizeof(uint64_t) * N);
    memcpy(top, in + (size_t)level * N, sizeof(uint64_t) * N);
    or_intt(c, top, level);
#pragma omp parallel for schedule(static) num_threads(or_get_threads())
    for (int j = 0; j < level; ++j) {
        const uint64_t qj = c->prime[j];
        const uint64_t qinv = or_invmod(ql % qj, qj);
        const uint64_t x = (qj - qinv) % qj;
        uint64_t* o = out + (size_t)j * N;
        for (int i = 0; i < N; ++i) o[i] = switch_modulus(top[i], ql, qj);
        or_ntt(c, o, j);
        for (int i = 0; i < N; ++i)
            o[i] = addmod(or_mulmod(qinv, in[(size_t)j * N + i], qj), or_mulmod(x, o[i], qj), qj);
    }
    free(top);
}

/* ------------------------------------------------------------------------ */
/* composite operations                                                     */
/* ------------------------------------------------------------------------ */

/* Ciphertext.cpp:597-619 (mult, live branch) + :379-398 (rescale):
 * tensor product, key switch of the c1*d1 term with the relinearisation
 * key, add, optional rescale. */
void or_hmult(const or_ctx* c, int level, const uint64_t* a0, const uint64_t* a1, const uint64_t* b0,
              const uint64_t* b1, const uint64_t* ksk_b, const uint64_t* ksk_a, int rescale, uint64_t* out0,
              uint64_t* out1) {
    const int n = level + 1, K = c->K, N = c->N;
    const size_t ln = (size_t)n * N, le = (size_t)(n + K) * N;
    const int nd = or_num_digits(c, level);
    uint64_t* e0 = (uint64_t*)malloc(sizeof(uint64_t) * ln);
    uint64_t* e1 = (uint64_t*)malloc(sizeof(uint64_t) * ln);
    uint64_t* e2 = (uint64_t*)malloc(sizeof(uint64_t) * ln);
    or_tensor(c, level, a0, a1, b0, b1, e0, e1, e2);
    uint64_t* dg = (uint64_t*)malloc(sizeof(uint64_t) * le * nd);
    or_modup(c, level, e2, dg);
    uint64_t* xb = (uint64_t*)malloc(sizeof(uint64_t) * le);
    uint64_t* xa = (uint64_t*)malloc(sizeof(uint64_t) * le);
    or_ks_inner(c, level, dg, ksk_b, ksk_a, xb, xa);
    or_moddown(c, level, xb, e2); /* reuse e2 as scratch for ModDown(b) */
    for (int i = 0; i < n; ++i) {
        const uint64_t p = c->prime[i];
        for (int j = 0; j < N; ++j) e0[(size_t)i * N + j] = addmod(e0[(size_t)i * N + j], e2[(size_t)i * N + j], p);
    }
    or_moddown(c, level, xa, e2);
    for (int i = 0; i < n; ++i) {
        const uint64_t p = c->prime[i];
        for (int j = 0; j < N; ++j) e1[(size_t)i * N + j] = addmod(e1[(size_t)i * N + j], e2[(size_t)i * N + j], p);
    }
    if (rescale) {
        or_rescale(c, level, e0, out0);
        or_rescale(c, level, e1, out1);
    } else {
        memcpy(out0, e0, sizeof(uint64_t) * ln);
        memcpy(out1, e1, sizeof(uint64_t) * ln);
    }
    free(e0);
    free(e1);
    free(e2);
    free(dg);
    free(xb);
    free(xa);
}

/* Ciphertext.cpp:1053-1226 rotate_hoisted (fused branch) and :871-925 rotate:
 * one ModUp of c1; per index, the inner product with that rotation key plus
 * P*c0 in the Q limbs (ElemenwiseBatchKernels.cu:299-396), permuted by the
 * automorphism in the extended basis, then ModDown of both halves. */
void or_rotate_hoisted(const or_ctx* c, int level, const uint64_t* c0, const uint64_t* c1, int nrot,
                       const uint32_t* galois, const uint64_t* const* ksk_b, const uint64_t* const* ksk_a,
                       uint64_t* const* out0, uint64_t* const* out1) {
    const int n = level + 1, K = c->K, N = c->N, L = c->L;
    const size_t le = (size_t)(n + K) * N;
    const int nd = or_num_digits(c, level);
    uint64_t* dg = (uint64_t*)malloc(sizeof(uint64_t) * le * nd);
    or_modup(c, level, c1, dg);
    uint64_t* p_mod = (uint64_t*)malloc(sizeof(uint64_t) * n);
    for (int i = 0; i < n; ++i) {
        uint64_t acc = 1, qi = c->prime[i];
        for (int k = 0; k < K; ++k) acc = or_mulmod(acc, c->prime[L + k] % qi, qi);
        p_mod[i] = acc;
    }
    uint64_t* xb = (uint64_t*)malloc(sizeof(uint64_t) * le);
    uint64_t* xa = (uint64_t*)malloc(sizeof(uint64_t) * le);
    uint64_t* pb = (uint64_t*)malloc(sizeof(uint64_t) * le);
    uint64_t* pa = (uint64_t*)malloc(sizeof(uint64_t) * le);
    for (int r = 0; r < nrot; ++r) {
        or_ks_inner(c, level, dg, ksk_b[r], ksk_a[r], xb, xa);
        for (int i = 0; i < n; ++i) {
            const uint64_t qi = c->prime[i];
            for (int j = 0; j < N; ++j) {
                const size_t k = (size_t)i * N + j;
                xb[k] = addmod(xb[k], or_mulmod(c0[k], p_mod[i], qi), qi);
            }
        }
        or_automorph(c, n + K, xb, pb, galois[r]);
        or_automorph(c, n + K, xa, pa, galois[r]);
        or_moddown(c, level, pb, out0[r]);
        or_moddown(c, level, pa, out1[r]);
    }
    free(dg);
    free(p_mod);
    free(xb);
    free(xa);
    free(pb);
    free(pa);
}

void or_rotate(const or_ctx* c, int level, const uint64_t* c0, const uint64_t* c1, uint32_t galois,
               const uint64_t* ksk_b, const uint64_t* ksk_a, uint64_t* out0, uint64_t* out1) {
    const uint64_t* kb[1] = {ksk_b};
    const uint64_t* ka[1] = {ksk_a};
    uint64_t* o0[1] = {out0};
    uint64_t* o1[1] = {out1};
    or_rotate_hoisted(c, level, c0, c1, 1, &galois, kb, ka, o0, o1);
}

/* splitmix64 stream, reduced per limb; used for seeded synthetic residues. */
static inline uint64_t splitmix64(uint64_t* s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

void or_random_residues(const or_ctx* c, int nlimbs, const int* pidx, uint64_t seed, uint64_t* out) {
    const size_t N = c->N;
    for (int i = 0; i < nlimbs; ++i) {
        uint64_t s = seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(i + 1));
        const uint64_t p = c->prime[pidx[i]];
        for (size_t j = 0; j < N; ++j) out[i * N + j] = (uint64_t)(((u128)splitmix64(&s) * p) >> 64);
    }
}
