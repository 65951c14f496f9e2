/* Host emulation of the exact double-precision arithmetic of the CUDA kernels
 * (pyfideslib_b200/csrc/fp64.cuh) -- test infrastructure only.
 *
 * The device routines are restated with C99 fma() (exactly rounded, like the
 * GPU's __fma_rn) and, for the one round-down FMA, fesetround(FE_DOWNWARD).
 * Built by tests/test_exact_arith.py with -ffp-contract=off so that no other
 * operation is fused.  The drivers run the forward and inverse transforms
 * with the kernels' stage schedule (N = 2^16 as two passes of two radix-16
 * groups) and the key-switch sums against exact 128-bit integer arithmetic.
 */
#include <fenv.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

static const double kRint = 6755399441055744.0; /* 1.5 * 2^52 */
static const double kTwo52 = 4503599627370496.0;
static const uint64_t kMant52 = (1ull << 52) - 1;

static double fp_mulw(double y, double w, double wq, double p) {
    const double h = y * w;
    const double l = fma(y, w, -h);
    const double q = fma(y, wq, kRint) - kRint;
    return fma(-q, p, h) + l;
}

static double fp_center(double x, double p, double pinv) {
    const double q = fma(x, pinv, kRint) - kRint;
    return fma(-q, p, x);
}

static double fma_rd(double a, double b, double c) {
    fesetround(FE_DOWNWARD);
    volatile double r = fma(a, b, c);
    fesetround(FE_TONEAREST);
    return r;
}

static uint64_t fp_to_u(double v, double p, double pinv_up) {
    const double two_p = p + p;
    const double a = v + two_p;
    const double b = v + (two_p + kTwo52);
    const double q = fma_rd(a, pinv_up, kRint) - kRint;
    const double r = fma(-q, p, b);
    uint64_t u;
    memcpy(&u, &r, 8);
    return u & kMant52;
}

static double fp_mulmod(double x, double y, double p, double pinv) {
    const double h = x * y;
    const double l = fma(x, y, -h);
    const double q = fma(h, pinv, kRint) - kRint;
    return fma(-q, p, h) + l;
}

/* the double nearest above 1/p (context.cpp recip_up) */
static double recip_up(uint64_t p) {
    double x = 1.0 / (double)p;
    int e = 0;
    const double f = frexp(x, &e);
    const uint64_t m = (uint64_t)ldexp(f, 53);
    const int sh = 53 - e;
    if (sh < 128 && (u128)m * p < ((u128)1 << sh)) x = nextafter(x, 1.0);
    return x;
}

static uint64_t mulmod(uint64_t a, uint64_t b, uint64_t p) { return (uint64_t)((u128)a * b % p); }

static uint64_t powmod(uint64_t a, uint64_t e, uint64_t p) {
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = mulmod(r, a, p);
        a = mulmod(a, a, p);
        e >>= 1;
    }
    return r;
}

static uint32_t bitrev(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int b = 0; b < bits; ++b)
        if (x >> b & 1) r |= 1u << (bits - 1 - b);
    return r;
}

static uint64_t splitmix(uint64_t* s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* Forward transform with the kernels' schedule: the column pass (stages
 * 0..7) centres X first when s % 4 is odd, the row pass (stages 8..15) when
 * s % 4 is even (its inputs are the column pass's doubles, below 1.7p), and
 * only the row pass ends with fp_to_u; then the inverse (Gentleman-Sande, sum
 * centred every stage, N^-1 folded into the last stage, doubles passed
 * between its two passes).  psi: primitive 2N-th root mod p < 2^50.  pattern 0: random
 * residues, 1: p - 1 everywhere, 2: alternating 0 / p - 1.  Returns the number
 * of coefficients that differ from exact arithmetic (forward) plus those
 * that do not come back (inverse), or -1 if a value left its proven range. */
static int ntt_check_impl(uint64_t p, uint64_t psi, uint64_t seed, int pattern, int gen);

/* Forward variant 9 and its inverse: the row pass's first four stages (8..11) take their
 * twiddles exactly from the table (staged in shared memory) and centre X on
 * even positions as before; its last four (12..15) centre X at every stage
 * and form the twiddle of group offset g > 0 as fp_mulmod(D, psi_br[g])
 * (|w| <= 0.875p, not reduced) with the quotient companion fl(w * pinv_up),
 * D = psi_br[index - g] exact from the table; g = 0 uses D itself.  The
 * inverse's row pass (its first eight stages) forms its per-thread
 * twiddles the same way from the inverse table; its sums are centred at
 * every stage already. */
int emu_ntt_sg_check(uint64_t p, uint64_t psi, uint64_t seed, int pattern) {
    return ntt_check_impl(p, psi, seed, pattern, 2);
}

int emu_ntt_check(uint64_t p, uint64_t psi, uint64_t seed, int pattern) {
    return ntt_check_impl(p, psi, seed, pattern, 0);
}

/* The row pass with generated twiddles (forward variant 9): stages 8..15
 * centre X first at every stage and take the twiddle's quotient companion as
 * fl(w * pinv_up) instead of the correctly rounded w / p (the twiddle itself,
 * psi_br[a 2^k] psi_br[h] mod p, is formed exactly on the integer pipes).
 * The looser companion widens the quotient error to 1/2 + |y| 1.5 2^-52, so
 * |t| <= 1.14p; centring every stage keeps every value below 1.65p. */
int emu_ntt_gen_check(uint64_t p, uint64_t psi, uint64_t seed, int pattern) {
    return ntt_check_impl(p, psi, seed, pattern, 1);
}

static int ntt_check_impl(uint64_t p, uint64_t psi, uint64_t seed, int pattern, int gen) {
    const int logN = 16, N = 1 << logN;
    uint64_t *a = malloc(8 * N), *e = malloc(8 * N), *tw = malloc(8 * N), *itw = malloc(8 * N);
    double *d = malloc(8 * (size_t)N), *W = malloc(8 * (size_t)N), *WQ = malloc(8 * (size_t)N);
    double *IW = malloc(8 * (size_t)N), *IWQ = malloc(8 * (size_t)N);
    const uint64_t ipsi = powmod(psi, 2 * (uint64_t)N - 1, p);
    uint64_t pw = 1, ipw = 1;
    uint64_t *pows = malloc(8 * N), *ipows = malloc(8 * N);
    for (int j = 0; j < N; ++j) {
        pows[j] = pw;
        ipows[j] = ipw;
        pw = mulmod(pw, psi, p);
        ipw = mulmod(ipw, ipsi, p);
    }
    for (int j = 0; j < N; ++j) {
        tw[j] = pows[bitrev(j, logN)];
        itw[j] = ipows[bitrev(j, logN)];
        W[j] = (double)tw[j];
        WQ[j] = W[j] / (double)p;
        IW[j] = (double)itw[j];
        IWQ[j] = IW[j] / (double)p;
    }
    uint64_t s = seed;
    for (int j = 0; j < N; ++j)
        a[j] = pattern == 1 ? p - 1 : pattern == 2 ? ((j & 1) ? p - 1 : 0) : splitmix(&s) % p;
    /* exact forward */
    memcpy(e, a, 8 * N);
    for (int m = 1, t = N / 2; m < N; m <<= 1, t >>= 1)
        for (int i = 0; i < m; ++i)
            for (int j = 2 * i * t; j < 2 * i * t + t; ++j) {
                const uint64_t X = e[j], Y = mulmod(e[j + t], tw[m + i], p);
                e[j] = (X + Y) % p;
                e[j + t] = (X + p - Y) % p;
            }
    const double pd = (double)p, pinv = recip_up(p);
    int bad = 0;
    for (int j = 0; j < N; ++j) d[j] = (double)a[j];
    int st = 0;
    for (int m = 1, t = N / 2; m < N; m <<= 1, t >>= 1, ++st) {
        const int red = st < 8 ? (st % 4) & 1
                        : (gen == 1 ? 1 : (gen == 2 && st >= 12) ? 1 : !((st % 4) & 1));
        for (int i = 0; i < m; ++i) {
            double w = W[m + i], wq = WQ[m + i];
            if (gen == 1 && st >= 8) wq = W[m + i] * pinv;
            if (gen == 2 && st >= 12) {
                /* row-stage index s' = st - 8; the thread's offset h has its
                 * low s' - 4 bits as the group offset g */
                const int g = i & ((1 << (st - 12)) - 1);
                if (g) {
                    w = fp_mulmod(W[m + i - g], W[g], pd, pinv);
                    if (fabs(w) > 0.875 * pd) bad = -1;
                    wq = w * pinv;
                }
            }
            for (int j = 2 * i * t; j < 2 * i * t + t; ++j) {
                double x = d[j];
                const double y = d[j + t];
                if (fabs(y) >= 2251799813685248.0) bad = -1; /* |y| < 2^51 */
                if (gen && st >= 8 && fabs(y) >= 1.7 * pd) bad = -1; /* the stated bound */
                if (red) x = fp_center(x, pd, pinv);
                const double tt = fp_mulw(y, w, wq, pd);
                d[j] = x + tt;
                d[j + t] = x - tt;
            }
        }
        if (st == 15)
            for (int j = 0; j < N; ++j) d[j] = (double)fp_to_u(d[j], pd, pinv);
    }
    if (bad < 0) goto done;
    for (int j = 0; j < N; ++j) bad += (uint64_t)d[j] != e[j];
    /* inverse from the exact forward values */
    {
        const uint64_t ninv = powmod(N, p - 2, p), w1 = itw[1], s1 = mulmod(ninv, w1, p);
        for (int j = 0; j < N; ++j) d[j] = (double)e[j];
        int stg = 0;
        for (int m = N / 2, t = 1; m > 1; m >>= 1, t <<= 1, ++stg) {
            for (int i = 0; i < m; ++i) {
                /* variant 10's inverse row pass (m >= 2^12): the twiddles of
                 * group offset g > 0 are fp_mulmod(D, psi^-1_br[g]) with the
                 * companion fl(w * pinv_up), as in the forward row pass */
                double w = IW[m + i], wq = IWQ[m + i];
                if (gen == 2 && m >= (1 << 12)) {
                    const int g = i & ((m >> 12) - 1);
                    if (g) {
                        w = fp_mulmod(IW[m + i - g], IW[g], pd, pinv);
                        wq = w * pinv;
                    }
                }
                for (int j = 2 * i * t; j < 2 * i * t + t; ++j) {
                    const double x = d[j], y = d[j + t];
                    if (fabs(x - y) >= 2251799813685248.0) { bad = -1; goto done; }
                    if (gen == 2 && fabs(x - y) >= 1.6 * pd) { bad = -1; goto done; }
                    d[j] = fp_center(x + y, pd, pinv);
                    d[j + t] = fp_mulw(x - y, w, wq, pd);
                }
            }
        }
        const double a0 = (double)ninv, a1 = (double)s1, a0q = a0 / pd, a1q = a1 / pd;
        for (int j = 0; j < N / 2; ++j) {
            const double x = d[j], y = d[j + N / 2];
            d[j] = (double)fp_to_u(fp_mulw(x + y, a0, a0q, pd), pd, pinv);
            d[j + N / 2] = (double)fp_to_u(fp_mulw(x - y, a1, a1q, pd), pd, pinv);
        }
        for (int j = 0; j < N; ++j) bad += (uint64_t)d[j] != a[j];
    }
done:
    free(a); free(e); free(tw); free(itw); free(d); free(W); free(WQ); free(IW); free(IWQ); free(pows); free(ipows);
    return bad;
}

/* Key-switch sums: sum of nd products x k reduced by fp_mulmod, centred and
 * floor-reduced, against exact arithmetic, for `trials` random (or, with
 * extreme != 0, maximal) operands.  Returns the number of mismatches. */
int emu_ks_check(uint64_t p, int nd, uint64_t seed, int trials, int extreme) {
    const double pd = (double)p, pinv = recip_up(p);
    uint64_t s = seed;
    int bad = 0;
    for (int t = 0; t < trials; ++t) {
        double acc = 0;
        u128 exact = 0;
        for (int dd = 0; dd < nd; ++dd) {
            const uint64_t x = extreme ? p - 1 : splitmix(&s) % p;
            const uint64_t k = extreme ? p - 1 - (uint64_t)(t & 1) : splitmix(&s) % p;
            acc += fp_mulmod((double)x, (double)k, pd, pinv);
            exact += (u128)x * k;
        }
        bad += fp_to_u(fp_center(acc, pd, pinv), pd, pinv) != (uint64_t)(exact % p);
    }
    return bad;
}

/* Tensor product (k_tensor, double-precision branch): one product (e0, e2)
 * or the sum of two (e1) reduced by fp_mulmod and floor-reduced directly, no
 * centring (|value| < 1.75p lies inside fp_to_u's exact range (-2p, 2p)),
 * against exact arithmetic; extreme != 0 uses p - 1 and p - 2 operands.
 * Returns the number of mismatches. */
int emu_tensor_check(uint64_t p, uint64_t seed, int trials, int extreme) {
    const double pd = (double)p, pinv = recip_up(p);
    uint64_t s = seed;
    int bad = 0;
    for (int t = 0; t < trials; ++t) {
        const uint64_t a0 = extreme ? p - 1 : splitmix(&s) % p, a1 = extreme ? p - 1 - (t & 1) : splitmix(&s) % p;
        const uint64_t b0 = extreme ? p - 1 - (t >> 1 & 1) : splitmix(&s) % p, b1 = extreme ? p - 1 : splitmix(&s) % p;
        const double e0 = fp_mulmod((double)a0, (double)b0, pd, pinv);
        const double e1 = fp_mulmod((double)a0, (double)b1, pd, pinv) + fp_mulmod((double)a1, (double)b0, pd, pinv);
        bad += fp_to_u(e0, pd, pinv) != (uint64_t)((u128)a0 * b0 % p);
        bad += fp_to_u(e1, pd, pinv) != (uint64_t)(((u128)a0 * b1 + (u128)a1 * b0) % p);
    }
    return bad;
}
