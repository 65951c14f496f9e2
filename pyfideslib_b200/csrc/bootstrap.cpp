// bootstrap.cpp -- CKKS bootstrapping and Chebyshev series evaluation over the
// evaluation core.
//
// Reference flow (src/CKKS/Bootstrap.cu:169-320 Bootstrap, :380 ModRaise;
// src/CKKS/CoeffsToSlots.cu:26,161 EvalCoeffsToSlots / EvalLinearTransform;
// src/CKKS/ApproxModEval.cu:24-93 approxModReduction, :370 evalChebyshevSeries,
// :747 applyDoubleAngleIterations):
//   ModRaise -> CoeffsToSlots -> split into real and imaginary parts with the
//   conjugation -> approximate modular reduction (Chebyshev series of a scaled
//   cosine, then double-angle iterations) on both parts -> recombine ->
//   SlotsToCoeffs.
//
// Formulation used here (own derivation, checked numerically in the tests):
//   * After ModRaise the polynomial is p = D*mu + q0*I with small integers I.
//     Declaring its scale K*q0 makes the slot values of CoeffsToSlots
//     t = (D*mu/q0 + I)/K in [-1, 1]; CoeffsToSlots runs at that scale (about
//     2^64, so its noise is small against t), then one integer multiply +
//     rescale brings the scale near the 2^50 moduli without touching t
//     (exact: the multiplier is an integer and the scale is tracked).
//   * Decoding of n = N/2 slots is the special FFT  z = A_logn ... A_1 P_br w
//     (w_k = p_k + i p_{k+n}, P_br the bit reversal, A_s a butterfly stage with
//     diagonals 0, +-2^(s-1) and twiddles zeta^(5^j mod 2^(s+2))).
//     CoeffsToSlots applies A_1^-1 ... A_logn^-1 (output in bit-reversed
//     order), SlotsToCoeffs applies A_logn ... A_1 to that order, so the bit
//     reversal never has to be applied.  Stages are merged into `level
//     budget` groups; each group is one diagonal-form matrix applied by
//     baby-step giant-step (fides_linear_transform), one level each.
//   * EvalMod evaluates g(t) = cos(2 pi (K t - 1/4) / 2^r) by its Chebyshev
//     interpolant on [-1, 1], then r double-angle steps c <- 2c^2 - 1 give
//     sin(2 pi K t) = sin(2 pi D mu / q0) ~ 2 pi D mu / q0; the factor
//     q0 / (2 pi D) is folded into the first SlotsToCoeffs group.
//   * The Chebyshev series is evaluated by recursive splitting
//     p = T_n Q + R (T_{n+k} = 2 T_n T_k - T_{n-k}) down to leaves of degree
//     < 8, which are integer linear combinations of T_1..T_7 computed in one
//     launch and one rescale.  Every product lands on a target level and
//     scale chosen top-down, so no operand ever needs a scale correction
//     beyond the integer rounding of its multiplier (relative 2^-50).
// Real and imaginary parts run in lockstep: every HMult of the series is one
// batched call over both.
#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <new>

#include "context.hpp"

using namespace fides;

namespace fides {

struct BootStage {
    int level = 0;
    int bstep = 1;
    std::vector<int32_t> offsets;
    std::vector<fides_pt*> pts;
};

struct BootPrecomp {
    fides_ctx* c = nullptr;
    int slots = 0;
    double K = 16.0;
    int double_angle = 3;
    int degree = 119;
    int correction = 0;
    std::vector<double> cheb;
    std::vector<BootStage> cts, stc;
    int level_after_cts = 0, level_after_mod = 0, level_out = 0;
    std::vector<int32_t> rotations;  // CoeffsToSlots / SlotsToCoeffs, indices over `slots` slots
    std::vector<int32_t> subsum;     // sparse packing: n, 2n, ..., N/4 over the full N/2 slots
    ~BootPrecomp() {
        for (auto* v : {&cts, &stc})
            for (auto& s : *v)
                for (fides_pt* p : s.pts) {
                    if (p && p->m) cudaFree(p->m);
                    delete p;
                }
    }
};

}  // namespace fides

namespace {

struct Guard {
    std::lock_guard<std::recursive_mutex> lk;
    explicit Guard(fides_ctx* c) : lk(c->mu) { cudaSetDevice(c->device); }
};

int floor_div(int a, int b) {
    int q = a / b;
    if ((a % b) != 0 && ((a < 0) != (b < 0))) --q;
    return q;
}

// (x mod p) of a real value rounded to the nearest integer, |x| < 2^126.
uint64_t real_mod(long double x, uint64_t p) {
    const bool neg = x < 0;
    long double a = floorl((neg ? -x : x) + 0.5L);
    const unsigned __int128 big = (unsigned __int128)a;
    const uint64_t r = (uint64_t)(big % p);
    return neg ? (r ? p - r : 0) : r;
}

// ---------------------------------------------------------------------------
// Diagonal-form slot matrices, built on the device: (M x)[i] =
// sum_o d_o[i] x[(i + o) mod n], the live diagonals of a group held as rows
// of an [rows][n] complex array in HBM.
// ---------------------------------------------------------------------------

// Entry i of diagonal `type` of butterfly stage s (block length 2^s,
// h = 2^(s-1); type 0 at offset 0, 1 at +h, 2 at -h).  With jj = i mod 2^s,
// j = jj mod h and t = exp(2 pi i (5^j mod 2^(s+2)) / 2^(s+2)), written as
// (jj < h | jj >= h):
//   SlotsToCoeffs A_s:     d0 = 1 | -t,           d+ = t | 0,    d- = 0 | 1
//   CoeffsToSlots A_s^-1:  d0 = 1/2 | -conj(t)/2, d+ = 1/2 | 0,  d- = 0 | conj(t)/2
__device__ double2 stage_entry(int type, int s, int i, bool inverse) {
    const int len = 1 << s, h = len >> 1;
    const int jj = i & (len - 1);
    const bool lo = jj < h;
    if (type == 1 && !lo) return make_double2(0, 0);
    if (type == 2 && lo) return make_double2(0, 0);
    if (lo && (type == 0 || inverse)) return make_double2(inverse ? 0.5 : 1.0, 0);
    if (!lo && type == 2 && !inverse) return make_double2(1.0, 0);
    // the twiddle t of j = jj mod h: 5^j mod 4 len, by squaring
    const uint32_t mask = (uint32_t)(len << 2) - 1;
    uint32_t g = 1, b = 5;
    for (uint32_t e = (uint32_t)(jj & (h - 1)); e; e >>= 1) {
        if (e & 1) g = (uint32_t)(((uint64_t)g * b) & mask);
        b = (uint32_t)(((uint64_t)b * b) & mask);
    }
    double sn, cs;
    sincospi((double)g / (double)(len << 1), &sn, &cs);  // angle 2 pi g / (4 len)
    if (!inverse) return type == 0 ? make_double2(-cs, -sn) : make_double2(cs, sn);  // -t (jj >= h) or t
    return type == 0 ? make_double2(-0.5 * cs, 0.5 * sn) : make_double2(0.5 * cs, -0.5 * sn);
}

// C_c = A_s B: C_c[i] = sum_type d_type[i] B_b[(i + o_type) mod n], b the row
// of offset o_c - o_type (src[3 c + type], -1 when absent)
__global__ void k_diag_stage(const double2* __restrict__ B, double2* __restrict__ Cm, const int* __restrict__ src,
                             int n, int s, int inverse) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (i >= n) return;
    const int h = 1 << (s - 1);
    const int off[3] = {0, h, n - h};
    double2 acc = make_double2(0, 0);
#pragma unroll
    for (int type = 0; type < 3; ++type) {
        const int b = src[3 * c + type];
        if (b < 0) continue;
        const double2 d = stage_entry(type, s, i, inverse != 0);
        const double2 x = B[(size_t)b * n + ((i + off[type]) & (n - 1))];
        acc.x += d.x * x.x - d.y * x.y;
        acc.y += d.x * x.y + d.y * x.x;
    }
    Cm[(size_t)c * n + i] = acc;
}

__global__ void k_diag_fill(double2* __restrict__ M, int n, double v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) M[i] = make_double2(v, 0);
}

// largest |entry| of each row (one CTA per row)
__global__ void k_diag_absmax(const double2* __restrict__ M, int n, double* __restrict__ out) {
    __shared__ double red[256];
    double m = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double2 v = M[(size_t)blockIdx.x * n + i];
        m = fmax(m, hypot(v.x, v.y));
    }
    red[threadIdx.x] = m;
    __syncthreads();
    for (int k = blockDim.x / 2; k; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + k]);
        __syncthreads();
    }
    if (!threadIdx.x) out[blockIdx.x] = red[0];
}

// The product of butterfly stages `stages` (the first applied first) in
// diagonal form: offsets in [0, n), increasing, with row[k] the row of
// offs[k] in buf.  Diagonals that come out exactly zero are dropped after
// every stage.
struct DevDiag {
    fides_ctx* c = nullptr;
    int n = 0;
    std::vector<int> offs, row;
    double2* buf = nullptr;
    ~DevDiag() {
        if (buf) cudaFreeAsync(buf, c->st);
    }
};

fides_status diag_group(fides_ctx* c, int n, const std::vector<int>& stages, bool inverse, DevDiag& M) {
    M.c = c;
    M.n = n;
    M.offs = {0};
    M.row = {0};
    if (cudaMallocAsync((void**)&M.buf, (size_t)n * 16, c->st) != cudaSuccess) {
        cudaGetLastError();
        return set_err(c, FIDES_OOM, "bootstrap diagonals");
    }
    count_launches(1);
    k_diag_fill<<<(n + 255) / 256, 256, 0, c->st>>>(M.buf, n, 1.0);
    for (int s : stages) {
        const int h = 1 << (s - 1);
        std::map<int, int> live;  // offset -> row of the current product
        for (size_t k = 0; k < M.offs.size(); ++k) live[M.offs[k]] = M.row[k];
        std::map<int, int> out;  // offset of the new product -> its row
        for (const auto& kv : live)
            for (int oa : {0, h, n - h}) out.emplace((kv.first + oa) % n, 0);
        std::vector<int> src(3 * out.size(), -1), offs;
        int r = 0;
        for (auto& kv : out) {
            kv.second = r;
            const int oa[3] = {0, h, n - h};
            for (int t = 0; t < 3; ++t) {
                auto it = live.find(((kv.first - oa[t]) % n + n) % n);
                if (it != live.end()) src[3 * r + t] = it->second;
            }
            offs.push_back(kv.first);
            ++r;
        }
        // one allocation: the new rows, the source table, the row maxima
        const size_t b_rows = (size_t)r * n * 16, b_src = ((size_t)3 * r * 4 + 15) / 16 * 16;
        char* nb = nullptr;
        if (cudaMallocAsync((void**)&nb, b_rows + b_src + (size_t)r * 8, c->st) != cudaSuccess) {
            cudaGetLastError();
            return set_err(c, FIDES_OOM, "bootstrap diagonals");
        }
        int* dsrc = (int*)(nb + b_rows);
        double* dmax = (double*)(nb + b_rows + b_src);
        cudaMemcpyAsync(dsrc, src.data(), src.size() * 4, cudaMemcpyHostToDevice, c->st);
        count_launches(2);
        k_diag_stage<<<dim3((n + 255) / 256, r), 256, 0, c->st>>>(M.buf, (double2*)nb, dsrc, n, s, inverse ? 1 : 0);
        k_diag_absmax<<<r, 256, 0, c->st>>>((double2*)nb, n, dmax);
        std::vector<double> mx(r);
        cudaMemcpyAsync(mx.data(), dmax, (size_t)r * 8, cudaMemcpyDeviceToHost, c->st);
        cudaFreeAsync(M.buf, c->st);
        M.buf = (double2*)nb;
        cudaStreamSynchronize(c->st);
        fides_status e = check_cuda(c, "bootstrap diagonals");
        if (e != FIDES_OK) return e;
        M.offs.clear();
        M.row.clear();
        for (int k = 0; k < r; ++k)
            if (mx[k] >= 1e-300) {
                M.offs.push_back(offs[k]);
                M.row.push_back(k);
            }
    }
    return FIDES_OK;
}

// Stage groups: `budget` contiguous groups of the logn butterfly stages,
// sizes as equal as possible.
std::vector<std::vector<int>> stage_groups(int logn, int budget, bool descending) {
    budget = std::max(1, std::min(budget, logn));
    std::vector<std::vector<int>> g(budget);
    int s = descending ? logn : 1;
    for (int b = 0; b < budget; ++b) {
        const int cnt = logn / budget + (b < logn % budget ? 1 : 0);
        for (int k = 0; k < cnt; ++k) {
            g[b].push_back(s);
            s += descending ? -1 : 1;
        }
    }
    return g;
}

// scale 0: the modulus of `level`, so the transform keeps the ciphertext's
// scale.  Queued on the context stream; *bad (device) flags a coefficient at
// or above 2^63.
fides_status encode_stage(fides_ctx* c, int n, const DevDiag& M, int level, double factor, double enc_scale,
                          BootStage& st, int* bad) {
    st.level = level;
    // offsets centred in (-n/2, n/2]; baby step ~ sqrt(#diagonals) in units of
    // the smallest offset step
    std::vector<int> offs;
    int unit = n;
    for (int raw : M.offs) {
        int o = raw > n / 2 ? raw - n : raw;
        offs.push_back(o);
        if (o) unit = std::min(unit, std::abs(o) & -std::abs(o));
    }
    if (unit == n) unit = 1;
    const int nd = (int)offs.size();
    int bk = 1;
    while (bk * bk < nd) bk <<= 1;
    st.bstep = bk * unit;
    const double scale = enc_scale > 0 ? enc_scale : (double)c->host.prime[level];
    for (size_t k = 0; k < offs.size(); ++k) {
        const int o = offs[k];
        const int G = floor_div(o, st.bstep) * st.bstep;
        fides_pt* pt = new (std::nothrow) fides_pt();
        if (!pt) return FIDES_OOM;
        pt->cap = level + 1;
        if (cudaMalloc((void**)&pt->m, (size_t)pt->cap * c->limb_bytes()) != cudaSuccess) {
            cudaGetLastError();
            delete pt;
            return set_err(c, FIDES_OOM, "bootstrap plaintext");
        }
        st.pts.push_back(pt);
        st.offsets.push_back(o);
        // slot j of the plaintext holds d_o[(j - G) mod n] * factor
        fides_status s = encode_dev_z(c, M.buf + (size_t)M.row[k] * n, n, G, factor, level, scale, pt->m, bad);
        if (s != FIDES_OK) return s;
        pt->level = level;
        pt->scale = scale;
        pt->noise_deg = 1;
        pt->slots = n;
    }
    return FIDES_OK;
}

// ---------------------------------------------------------------------------
// Lockstep ciphertext arithmetic with exact (level, scale) bookkeeping.
// ---------------------------------------------------------------------------
constexpr int kBaby = 8;
// CoeffsToSlots diagonals are encoded at 2^58: they multiply slot values of
// magnitude ~sqrt(N) |t|, so their rounding error (about sqrt(N) / scale per
// entry) is what bounds the precision of t; each of the three transforms
// grows the ciphertext's scale by 2^8, undone by the normalisation after.
constexpr double kCtsDiagScale = 288230376151711744.0;  // 2^58

using Lanes = std::vector<fides_ct*>;

class Arith {
   public:
    fides_ctx* c;
    fides_status st = FIDES_OK;
    explicit Arith(fides_ctx* cc) : c(cc) {}
    ~Arith() {
        for (fides_ct* t : owned) {
            if (t->buf) cudaFreeAsync(t->buf, c->st);
            delete t;
        }
    }
    Arith(const Arith&) = delete;
    Arith& operator=(const Arith&) = delete;

    Lanes fresh(size_t nl) {
        Lanes v;
        for (size_t i = 0; i < nl; ++i) {
            owned.push_back(new fides_ct());
            v.push_back(owned.back());
        }
        return v;
    }
    bool ok() const { return st == FIDES_OK; }

    // HMult + relinearisation + rescale, all lanes in one batched call
    Lanes mul(const Lanes& a, const Lanes& b) {
        Lanes o = fresh(a.size());
        if (ok()) st = fides_hmult_batch(c, (int)a.size(), a.data(), b.data(), o.data(), 1);
        return o;
    }

    // sum_k z_k x_k + cst (at the result's scale) on limbs 0..level, integer
    // z_k, no rescale; the x_k carry the result's scale (that of the first)
    Lanes ilin(const std::vector<std::pair<const Lanes*, int64_t>>& terms, double cst, int level) {
        const size_t nl = terms[0].first->size();
        Lanes o = fresh(nl);
        for (size_t l = 0; l < nl && ok(); ++l) {
            const double sc = (*terms[0].first)[l]->scale;
            std::vector<const fides_ct*> xs;
            for (size_t k = 0; k < terms.size(); ++k) {
                int_const_limbs(c, terms[k].second, level + 1, zbuf[k]);
                xs.push_back((*terms[k].first)[l]);
            }
            if ((st = ct_reserve(c, o[l], level)) != FIDES_OK) break;
            launch(xs, level, (long double)cst * sc, o[l]);
            meta(o[l], level, sc, xs[0]->slots);
        }
        return o;
    }

    // sum_k c_k x_k + cst with real c_k, landing on (level - 1, target) after
    // one rescale: x_k of any scale s_k is multiplied by the integer
    // round(c_k * target * q_level / s_k), the constant enters as
    // round(cst * target * q_level).  `like` gives the lanes and slots.
    Lanes lin(const std::vector<std::pair<const Lanes*, double>>& terms, double cst, int level, double target,
              const Lanes& like) {
        Lanes o = fresh(like.size());
        const long double tq = (long double)target * (long double)c->host.prime[level];
        for (size_t l = 0; l < like.size() && ok(); ++l) {
            std::vector<const fides_ct*> xs;
            for (size_t k = 0; k < terms.size(); ++k) {
                const fides_ct* x = (*terms[k].first)[l];
                const long double z = (long double)terms[k].second * tq / (long double)x->scale;
                if (!(fabsl(z) < 4.0e18L)) {
                    st = set_err(c, FIDES_BAD_ARG, "coefficient too large for the ciphertext scale");
                    return o;
                }
                int_const_limbs(c, (int64_t)llroundl(z), level + 1, zbuf[k]);
                xs.push_back(x);
            }
            if ((st = ct_reserve(c, o[l], level)) != FIDES_OK) break;
            launch(xs, level, (long double)cst * tq, o[l]);
            meta(o[l], level, (double)tq, like[l]->slots);
        }
        // the lanes' rescales as one batch
        if (ok() && (st = rescale_batch(c, (int)o.size(), o.data())) == FIDES_OK)
            for (fides_ct* x : o) x->scale = target;
        return o;
    }

    // x times the integer z = round(target q / s) and rescaled: level - 1,
    // scale s z / q (exact, within a factor 1 +- 1/(2z) of target)
    Lanes normalize(const Lanes& x, double target) {
        const int level = x[0]->level;
        const long double q = (long double)c->host.prime[level];
        Lanes o = fresh(x.size());
        for (size_t l = 0; l < x.size() && ok(); ++l) {
            const long double zr = (long double)target * q / (long double)x[l]->scale;
            if (!(zr >= 1.0L && zr < 4.0e18L)) {
                st = set_err(c, FIDES_BAD_ARG, "scale out of range for normalisation");
                break;
            }
            const int64_t z = (int64_t)llroundl(zr);
            int_const_limbs(c, z, level + 1, zbuf[0]);
            if ((st = ct_reserve(c, o[l], level)) != FIDES_OK) break;
            launch({x[l]}, level, 0.0L, o[l]);
            meta(o[l], level, (double)((long double)x[l]->scale * (long double)z), x[l]->slots);
        }
        if (ok()) st = rescale_batch(c, (int)o.size(), o.data());
        return o;
    }

    Lanes monomial(const Lanes& a, uint32_t k) {
        Lanes o = fresh(a.size());
        for (size_t l = 0; l < a.size() && ok(); ++l) st = fides_mult_monomial(c, a[l], k, o[l]);
        return o;
    }

   private:
    std::vector<fides_ct*> owned;
    uint64_t zbuf[kMaxLin][kMaxPrimes][2];

    static void meta(fides_ct* o, int level, double scale, int slots) {
        o->level = level;
        o->scale = scale;
        o->noise_deg = 1;
        o->slots = slots;
    }
    // one lincomb launch per chunk of kMaxLinLimbs limbs, constants from zbuf
    void launch(const std::vector<const fides_ct*>& xs, int level, long double add_value, fides_ct* out) {
        const int N = c->N, n = level + 1;
        for (int j0 = 0; j0 < n; j0 += kMaxLinLimbs) {
            const int nlb = std::min(kMaxLinLimbs, n - j0);
            LinArgs la{};
            la.n = (int)xs.size();
            la.q0 = j0;
            for (size_t k = 0; k < xs.size(); ++k) {
                la.in0[k] = xs[k]->c0() + (size_t)j0 * N;
                la.in1[k] = xs[k]->c1(N) + (size_t)j0 * N;
                for (int j = 0; j < nlb; ++j) {
                    la.z[k][j][0] = zbuf[k][j0 + j][0];
                    la.z[k][j][1] = zbuf[k][j0 + j][1];
                }
            }
            la.has_add = add_value != 0;
            for (int j = 0; j < nlb && la.has_add; ++j) la.add0[j] = real_mod(add_value, c->host.prime[j0 + j]);
            la.out0 = out->c0() + (size_t)j0 * N;
            la.out1 = out->c1(N) + (size_t)j0 * N;
            launch_lincomb(c->dev, nlb, la, c->st);
        }
    }
};

// ---------------------------------------------------------------------------
// Chebyshev series  sum_k c_k T_k(x),  x in [-1, 1]
// ---------------------------------------------------------------------------
class Chebyshev {
   public:
    Chebyshev(Arith& a, const Lanes& x, int degree) : A(a), deg(degree) {
        T[1] = x;
        lvl[1] = x[0]->level;
        lvl[0] = 1 << 30;
    }

    // levels of T_k if built (dry run: no GPU work)
    static std::map<int, int> plan_levels(int top, int degree) {
        std::map<int, int> L;
        L[1] = top;
        auto need = [&](auto&& self, int k) -> int {
            auto it = L.find(k);
            if (it != L.end()) return it->second;
            int v = (k % 2 == 0) ? self(self, k / 2) - 1 : std::min(self(self, k / 2), self(self, k / 2 + 1)) - 1;
            L[k] = v;
            return v;
        };
        for (int k = 1; k < std::min(kBaby, degree + 1); ++k) need(need, k);
        for (int n = kBaby; n <= degree; n <<= 1) need(need, n);
        return L;
    }
    // highest level at which the series of degree d can be delivered
    static int feasible(const std::map<int, int>& L, int d) {
        if (d < kBaby) {
            int m = 1 << 30;
            for (int k = 1; k <= d; ++k) m = std::min(m, L.at(k));
            return m - 1;
        }
        int n = kBaby;
        while (2 * n <= d) n <<= 1;
        return std::min({L.at(n) - 1, feasible(L, d - n) - 1, feasible(L, n - 1)});
    }

    Lanes eval(const std::vector<double>& coeffs, int level, double scale) {
        powers((int)coeffs.size() - 1);
        return rec(coeffs, level, scale);
    }

   private:
    Arith& A;
    int deg;
    std::map<int, Lanes> T;
    std::map<int, int> lvl;

    // T_k for k < kBaby and the giant steps kBaby 2^j up to the degree,
    // computed in rounds of equal dependency depth: every round's products
    // go out as one batched HMult (T_2; T_3, T_4; T_5..T_8; T_16; ...)
    void powers(int d) {
        std::vector<int> ks;
        for (int k = 2; k < std::min(kBaby, d + 1); ++k) ks.push_back(k);
        for (int n = kBaby; n <= d; n <<= 1) ks.push_back(n);
        std::map<int, int> depth;
        depth[1] = 0;
        auto dep = [&](auto&& self, int k) -> int {
            auto it = depth.find(k);
            if (it != depth.end()) return it->second;
            const int v = k % 2 == 0 ? self(self, k / 2) + 1 : std::max(self(self, k / 2), self(self, k / 2 + 1)) + 1;
            depth[k] = v;
            return v;
        };
        std::map<int, std::vector<int>> rounds;
        for (int k : ks) {
            // odd k needs T_{k/2} and T_{k/2+1}, even k needs T_{k/2}: both in ks or 1
            rounds[dep(dep, k)].push_back(k);
        }
        for (auto& kv : rounds) {
            std::vector<int> todo;
            for (int k : kv.second)
                if (!T.count(k)) todo.push_back(k);
            // operands of lower depth may not be in ks (a leaf-only power): build them lazily
            for (int k : todo) {
                get(k / 2);
                if (k % 2) get(k / 2 + 1);
            }
            products(todo);
        }
    }

    // T_k for every k in ks (operands present), one batched HMult for all
    void products(const std::vector<int>& ks) {
        if (ks.empty()) return;
        Lanes xa, xb;
        for (int k : ks) {
            const Lanes& a = T.at(k / 2);
            const Lanes& b = k % 2 == 0 ? a : T.at(k / 2 + 1);
            xa.insert(xa.end(), a.begin(), a.end());
            xb.insert(xb.end(), b.begin(), b.end());
        }
        const Lanes all = A.mul(xa, xb);
        const size_t nl = T.at(1).size();
        for (size_t i = 0; i < ks.size(); ++i) T[ks[i]] = finish(ks[i], Lanes(all.begin() + i * nl, all.begin() + (i + 1) * nl));
    }

    // 2 T_{k/2}^2 - 1 (even k) or 2 T_{k/2} T_{k/2+1} - T_1 (odd k) from the product p
    Lanes finish(int k, const Lanes& p) {
        if (k % 2 == 0) return A.ilin({{&p, 2}}, -1.0, p[0]->level);
        // T_1 brought to the product's (level, scale)
        Lanes t1 = A.lin({{&T[1], 1.0}}, 0.0, p[0]->level + 1, p[0]->scale, p);
        return A.ilin({{&p, 2}, {&t1, -1}}, 0.0, p[0]->level);
    }

    const Lanes& get(int k) {
        auto it = T.find(k);
        if (it != T.end()) return it->second;
        get(k / 2);
        if (k % 2) get(k / 2 + 1);
        products({k});
        return T.at(k);
    }

    // The recursion p = T_n Q + R as a tree: leaves (degree < kBaby) are
    // linear combinations of T_1..T_7, every inner node one product T_n Q.
    // Nodes of equal depth are independent, so their products go out as one
    // batched HMult, deepest level first.
    struct Node {
        Lanes val;
        int n = 0, q = -1, r = -1, level = 0, depth = 0;
    };
    std::vector<Node> nodes;

    int build(const std::vector<double>& c, int level, double scale, int depth) {
        const int d = (int)c.size() - 1;
        Node nd;
        nd.level = level;
        nd.depth = depth;
        if (d < kBaby) {
            std::vector<std::pair<const Lanes*, double>> terms;
            for (int k = 1; k <= d; ++k)
                if (c[k] != 0.0) terms.push_back({&get(k), c[k]});
            nd.val = A.lin(terms, c[0], level + 1, scale, T[1]);
            nodes.push_back(nd);
            return (int)nodes.size() - 1;
        }
        int n = kBaby;
        while (2 * n <= d) n <<= 1;
        std::vector<double> q(d - n + 1), r(c.begin(), c.begin() + n);
        q[0] = c[n];
        for (int k = 1; k <= d - n; ++k) {
            q[k] = 2.0 * c[n + k];
            r[n - k] -= c[n + k];
        }
        const Lanes& Tn = get(n);
        const double sq = scale * (double)A.c->host.prime[level + 1] / Tn[0]->scale;
        nd.n = n;
        nd.q = build(q, level + 1, sq, depth + 1);
        nd.r = build(r, level, scale, depth + 1);
        nodes.push_back(nd);
        return (int)nodes.size() - 1;
    }

    Lanes rec(const std::vector<double>& c, int level, double scale) {
        nodes.clear();
        const int root = build(c, level, scale, 0);
        int maxd = 0;
        for (const Node& nd : nodes) maxd = std::max(maxd, nd.depth);
        const size_t nl = T.at(1).size();
        for (int dd = maxd; dd >= 0; --dd) {
            std::vector<int> idx;
            Lanes xa, xb;
            for (int i = 0; i < (int)nodes.size(); ++i)
                if (nodes[i].depth == dd && nodes[i].q >= 0) {
                    idx.push_back(i);
                    const Lanes& tn = T.at(nodes[i].n);
                    const Lanes& qv = nodes[nodes[i].q].val;
                    xa.insert(xa.end(), tn.begin(), tn.end());
                    xb.insert(xb.end(), qv.begin(), qv.end());
                }
            if (idx.empty()) continue;
            const Lanes all = A.mul(xa, xb);
            for (size_t j = 0; j < idx.size(); ++j) {
                Node& nd = nodes[idx[j]];
                const Lanes p(all.begin() + j * nl, all.begin() + (j + 1) * nl);
                nd.val = A.ilin({{&p, 1}, {&nodes[nd.r].val, 1}}, 0.0, nd.level);
            }
        }
        return nodes[root].val;
    }
};

std::vector<double> cheb_coeffs(int degree, double K, int r) {
    const int m = degree + 1;
    std::vector<double> fx(m), c(m, 0.0);
    for (int j = 0; j < m; ++j) {
        const double x = cos(M_PI * (j + 0.5) / m);
        fx[j] = cos(2.0 * M_PI * (K * x - 0.25) / (double)(1 << r));
    }
    for (int k = 0; k < m; ++k) {
        double s = 0;
        for (int j = 0; j < m; ++j) s += fx[j] * cos(M_PI * k * (j + 0.5) / m);
        c[k] = 2.0 * s / m;
    }
    c[0] *= 0.5;
    return c;
}

}  // namespace

extern "C" {

fides_status fides_chebyshev_series(fides_ctx* c, const fides_ct* a, const double* coeffs, int degree, double lo,
                                    double hi, fides_ct* out) {
    if (!c || !a || !a->buf || !coeffs || degree < 0 || degree > 2047 || !(hi > lo) || !out) return FIDES_BAD_ARG;
    Guard g(c);
    if (!c->has_relin) return set_err(c, FIDES_KEY_MISSING, "no relinearisation key");
    Arith A(c);
    Lanes x = {const_cast<fides_ct*>(a)};
    std::vector<double> cf(coeffs, coeffs + degree + 1);
    int top = a->level;
    // The squarings T_2k = 2 T_k^2 - 1 map a scale s to s^2 / q: unless the
    // input's scale sits at its level's modulus the scales run away (doubly
    // exponentially in the depth).  An input off by more than 2^-20 is first
    // brought there, together with the affine map to [-1, 1] (one rescale).
    const double rel = a->scale / (double)c->host.prime[top];
    if (lo != -1.0 || hi != 1.0 || std::fabs(rel - 1.0) > 1.0 / (1 << 20)) {
        if (top < 1) return FIDES_BAD_ARG;
        x = A.lin({{&x, 2.0 / (hi - lo)}}, -(lo + hi) / (hi - lo), top, (double)c->host.prime[top - 1], x);
        top -= 1;
    }
    if (!A.ok()) return A.st;
    const auto L = Chebyshev::plan_levels(top, degree);
    const int lv = Chebyshev::feasible(L, degree);
    if (lv < 0) return set_err(c, FIDES_BAD_ARG, "not enough levels for the Chebyshev series");
    Chebyshev ch(A, x, degree);
    Lanes y = ch.eval(cf, lv, a->scale);
    if (!A.ok()) return A.st;
    fides_status s = fides_ct_copy(c, y[0], out);
    if (s == FIDES_OK) out->slots = a->slots;
    return s;
}

fides_status fides_bootstrap_setup(fides_ctx* c, const fides_boot_params* prm) {
    if (!c || !prm) return FIDES_BAD_ARG;
    Guard g(c);
    const int n = prm->slots > 0 ? prm->slots : c->N / 2;
    if (n < 2 || n > c->N / 2 || (n & (n - 1)))
        return set_err(c, FIDES_BAD_ARG, "bootstrap slots must be a power of two in [2, N/2]");
    int logn = 0;
    while ((1 << logn) < n) ++logn;
    auto bp = std::make_shared<BootPrecomp>();
    bp->c = c;
    bp->slots = n;
    bp->K = prm->K > 0 ? prm->K : 16.0;
    bp->double_angle = prm->double_angle > 0 ? prm->double_angle : 3;
    bp->degree = prm->cheb_degree > 0 ? prm->cheb_degree : 119;
    if (prm->correction < 0 || prm->correction > 20) return FIDES_BAD_ARG;
    bp->correction = prm->correction;
    bp->cheb = cheb_coeffs(bp->degree, bp->K, bp->double_angle);
    const int bc = prm->level_budget[0] > 0 ? prm->level_budget[0] : 3;
    const int bs = prm->level_budget[1] > 0 ? prm->level_budget[1] : 3;
    const int top = c->L - 1;
    // levels: ModRaise at top, CoeffsToSlots, scale normalisation, EvalMod, SlotsToCoeffs
    const auto gc = stage_groups(logn, bc, true);
    const auto gs = stage_groups(logn, bs, false);
    bp->level_after_cts = top - 1 - (int)gc.size();
    const auto Lv = Chebyshev::plan_levels(bp->level_after_cts, bp->degree);
    const int after_cheb = Chebyshev::feasible(Lv, bp->degree);
    bp->level_after_mod = after_cheb - bp->double_angle;
    bp->level_out = bp->level_after_mod - (int)gs.size();
    if (bp->level_out < 0)
        return set_err(c, FIDES_BAD_ARG, "not enough levels for bootstrapping (need " +
                                             std::to_string(top - bp->level_out) + " of " + std::to_string(top) + ")");
    // the diagonals are generated and encoded on the device; one flag for
    // every encoding, read once at the end
    int* bad = nullptr;
    if (cudaMallocAsync((void**)&bad, sizeof(int), c->st) != cudaSuccess) {
        cudaGetLastError();
        return set_err(c, FIDES_OOM, "bootstrap setup");
    }
    cudaMemsetAsync(bad, 0, sizeof(int), c->st);
    struct FlagFree {
        fides_ctx* c;
        int* p;
        ~FlagFree() { cudaFreeAsync(p, c->st); }
    } flag_free{c, bad};
    // CoeffsToSlots: A_1^-1 ... A_logn^-1, highest stages applied first
    for (size_t b = 0; b < gc.size(); ++b) {
        DevDiag M;
        fides_status e = diag_group(c, n, gc[b], true, M);
        if (e != FIDES_OK) return e;
        BootStage st;
        e = encode_stage(c, n, M, top - (int)b, 1.0, kCtsDiagScale, st, bad);
        bp->cts.push_back(std::move(st));
        if (e != FIDES_OK) return e;
    }
    // SlotsToCoeffs: A_logn ... A_1, with q0 / (2 pi D) in the first group
    const double fac = (double)c->host.prime[0] / (2.0 * M_PI * c->default_scale);
    for (size_t b = 0; b < gs.size(); ++b) {
        DevDiag M;
        fides_status e = diag_group(c, n, gs[b], false, M);
        if (e != FIDES_OK) return e;
        BootStage st;
        e = encode_stage(c, n, M, bp->level_after_mod - (int)b, b == 0 ? fac : 1.0, 0.0, st, bad);
        bp->stc.push_back(std::move(st));
        if (e != FIDES_OK) return e;
    }
    int hbad = 0;
    cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, c->st);
    cudaStreamSynchronize(c->st);
    if (hbad) return set_err(c, FIDES_BAD_ARG, "bootstrap diagonal coefficient exceeds 2^63");
    std::vector<int32_t> rot;
    for (auto* v : {&bp->cts, &bp->stc})
        for (auto& st : *v)
            for (int o : st.offsets) {
                const int G = floor_div(o, st.bstep) * st.bstep, b = o - G;
                for (int r : {b, G})
                    if (r && std::find(rot.begin(), rot.end(), r) == rot.end()) rot.push_back(r);
            }
    std::sort(rot.begin(), rot.end());
    bp->rotations = rot;
    for (int r = n; r < c->N / 2; r <<= 1) bp->subsum.push_back(r);
    c->boot[n] = bp;
    return check_cuda(c, "bootstrap setup");
}

fides_status fides_bootstrap_info(fides_ctx* c, int slots, int* output_level, int* num_rotations, int32_t* rotations) {
    if (!c) return FIDES_BAD_ARG;
    Guard g(c);
    auto it = c->boot.find(slots > 0 ? slots : c->N / 2);
    if (it == c->boot.end()) return set_err(c, FIDES_BAD_ARG, "bootstrapping not set up for these slots");
    const BootPrecomp& b = *it->second;
    if (output_level) *output_level = b.level_out;
    if (num_rotations) *num_rotations = (int)(b.rotations.size() + b.subsum.size());
    if (rotations) {
        std::copy(b.rotations.begin(), b.rotations.end(), rotations);
        std::copy(b.subsum.begin(), b.subsum.end(), rotations + b.rotations.size());
    }
    return FIDES_OK;
}

fides_status fides_bootstrap_keygen(fides_ctx* c, const fides_sk* sk, int slots, uint64_t seed) {
    if (!c || !sk) return FIDES_BAD_ARG;
    std::shared_ptr<BootPrecomp> bp;
    {
        Guard g(c);
        auto it = c->boot.find(slots > 0 ? slots : c->N / 2);
        if (it == c->boot.end()) return set_err(c, FIDES_BAD_ARG, "bootstrapping not set up for these slots");
        bp = it->second;
    }
    fides_status s = fides_keygen_rotations(c, sk, (int)bp->rotations.size(), bp->rotations.data(), bp->slots, seed);
    if (s == FIDES_OK && !bp->subsum.empty())
        s = fides_keygen_rotations(c, sk, (int)bp->subsum.size(), bp->subsum.data(), c->N / 2, seed + 7777);
    if (s == FIDES_OK) s = fides_keygen_conjugate(c, sk, seed + 1);
    return s;
}

fides_status fides_bootstrap(fides_ctx* c, const fides_ct* in, fides_ct* out) {
    return fides_bootstrap_batch(c, 1, &in, &out);
}

// Two iterations (the reference's EvalBootstrap(ct, numIterations = 2,
// precision), api/CryptoContext.hpp:180-181, which OpenFHE implements): y =
// the first bootstrap brought to the input's scale, r = in - y carries minus
// the first bootstrap's error e1; r times 2^p is bootstrapped again (its
// message 2^p e1 is of size about 1), the result's scale is taken 2^p times
// larger (its message becomes -e1 + e2 / 2^p) and brought to y's scale, and
// the sum leaves m + e2 / 2^p.  The input must still hold the levels of a
// bootstrap's output; the result is one level below it.
fides_status fides_bootstrap_iter(fides_ctx* c, const fides_ct* in, int iterations, int precision, fides_ct* out) {
    if (!c || !in || !in->buf || !out || iterations < 1 || iterations > 2 || precision < 0 || precision > 30)
        return FIDES_BAD_ARG;
    if (iterations == 1) return fides_bootstrap(c, in, out);
    Guard g(c);
    const int n = in->slots > 0 ? in->slots : c->N / 2;
    auto it = c->boot.find(n);
    if (it == c->boot.end()) return set_err(c, FIDES_BAD_ARG, "bootstrapping not set up for these slots");
    const BootPrecomp& B = *it->second;
    if (in->level < B.level_out || B.level_out < 1)
        return set_err(c, FIDES_BAD_ARG, "a second bootstrap iteration needs the input at the bootstrap's output level");
    const int p = precision > 0 ? precision : 12;
    Arith A(c);
    Lanes bt = A.fresh(1);
    fides_status s = fides_bootstrap(c, in, bt[0]);
    if (s != FIDES_OK) return s;
    Lanes y = A.normalize(bt, in->scale);  // level_out - 1, scale within 2^-50 of the input's
    if (!A.ok()) return A.st;
    Lanes r = A.fresh(3);
    if ((s = fides_sub(c, in, y[0], r[0])) != FIDES_OK) return s;  // -e1 at the input's scale
    if ((s = fides_mult_int(c, r[0], (int64_t)1 << p, r[1])) != FIDES_OK) return s;
    r[1]->scale = in->scale;  // the message is 2^p (-e1)
    r[1]->slots = in->slots;
    if ((s = fides_bootstrap(c, r[1], r[2])) != FIDES_OK) return s;
    r[2]->scale *= (double)(1ll << p);  // message -e1 + e2 / 2^p
    Lanes rr{r[2]};
    Lanes r4 = A.normalize(rr, y[0]->scale);
    if (!A.ok()) return A.st;
    const double sc = y[0]->scale;
    if ((s = fides_add(c, y[0], r4[0], out)) != FIDES_OK) return s;
    out->scale = sc;
    out->slots = in->slots;
    out->noise_deg = 1;
    return check_cuda(c, "bootstrap iterations");
}

fides_status fides_bootstrap_batch(fides_ctx* c, int nin, const fides_ct* const* in, fides_ct* const* out) {
    if (!c || nin < 1 || !in || !out) return FIDES_BAD_ARG;
    for (int u = 0; u < nin; ++u)
        if (!in[u] || !in[u]->buf || !out[u]) return FIDES_BAD_ARG;
    Guard g(c);
    const int n = in[0]->slots > 0 ? in[0]->slots : c->N / 2;
    for (int u = 1; u < nin; ++u)
        if ((in[u]->slots > 0 ? in[u]->slots : c->N / 2) != n)
            return set_err(c, FIDES_BAD_ARG, "batched bootstrap: inputs with different slot counts");
    auto it = c->boot.find(n);
    if (it == c->boot.end()) return set_err(c, FIDES_BAD_ARG, "bootstrapping not set up for these slots");
    const BootPrecomp& B = *it->second;
    if (!c->has_relin) return set_err(c, FIDES_KEY_MISSING, "no relinearisation key");
    const int N = c->N;
    const size_t k = (size_t)nin;
    Arith A(c);
    Lanes x = A.fresh(k);
    fides_status s = FIDES_OK;
    for (size_t u = 0; u < k; ++u) {
        if (B.correction > 0) {
            // message times 2^correction (exact integer product of limb 0 and up)
            Lanes pre = A.fresh(1);
            if ((s = fides_mult_int(c, in[u], (int64_t)1 << B.correction, pre[0])) != FIDES_OK) return s;
            s = fides_mod_raise(c, pre[0], x[u]);
        } else {
            s = fides_mod_raise(c, in[u], x[u]);
        }
        if (s != FIDES_OK) return s;
        x[u]->scale = B.K * (double)c->host.prime[0];
        x[u]->slots = n;
    }
    // sparse packing: the raised polynomial has coefficients everywhere (the
    // overflow q0 I); the trace over the automorphisms X -> X^(5^(n t)),
    // t < N / 2n (the rotations by multiples of n, which fix the subring
    // Z[X^(N/2n)]), is N/2n times its projection onto that subring, the
    // ring of n-slot plaintexts: log2(N/2n) rotate-and-add steps, the factor
    // taken into the declared scale
    for (int32_t r : B.subsum) {
        const uint32_t gal = fides_rotation_galois(c, r, N / 2);
        for (size_t u = 0; u < k; ++u) {
            Lanes rt = A.fresh(2);
            if ((s = fides_automorphism(c, x[u], gal, rt[0])) != FIDES_OK) return s;
            if ((s = fides_add(c, x[u], rt[0], rt[1])) != FIDES_OK) return s;
            rt[1]->scale = 2.0 * x[u]->scale;
            rt[1]->slots = n;
            x[u] = rt[1];
        }
    }
    // CoeffsToSlots from the scale K q0 (about 2^64, growing by 2^8 per
    // transform): its rescaling and key-switching noise and the rounding of
    // its diagonals stay small against t, whose error EvalMod multiplies by
    // 2 pi K and SlotsToCoeffs by about sqrt(n) q0 / (2 pi D)
    for (const BootStage& st : B.cts) {
        Lanes y = A.fresh(k);
        s = linear_transform_batch(c, nin, (const fides_ct* const*)x.data(), (int)st.offsets.size(),
                                   st.offsets.data(), (const fides_pt* const*)st.pts.data(), st.bstep, 1, y.data(),
                                   true);
        if (s != FIDES_OK) return s;
        x = y;
    }
    // integer multiply + rescale: scale -> about half the modulus EvalMod
    // starts at (exactly tracked), values unchanged; the real / imaginary split
    // doubles it, so the Chebyshev input's scale sits at its own level's
    // modulus and the squarings of the series keep their scales next to the
    // moduli they are divided by
    x = A.normalize(x, 0.5 * (double)c->host.prime[B.level_after_cts]);
    if (!A.ok()) return A.st;
    // real and imaginary parts: (x + conj x), -i (x - conj x), each twice the part
    Lanes cj = A.fresh(k);
    for (size_t u = 0; u < k; ++u)
        if ((s = fides_conjugate(c, x[u], cj[u])) != FIDES_OK) return s;
    Lanes re = A.ilin({{&x, 1}, {&cj, 1}}, 0.0, x[0]->level);
    Lanes df = A.ilin({{&x, 1}, {&cj, -1}}, 0.0, x[0]->level);
    Lanes im = A.monomial(df, 3u * (uint32_t)N / 2u);
    if (!A.ok()) return A.st;
    for (size_t u = 0; u < k; ++u) {
        re[u]->scale *= 2.0;
        im[u]->scale *= 2.0;
    }
    // 2k lanes in lockstep: real parts, then imaginary parts
    Lanes v(re);
    v.insert(v.end(), im.begin(), im.end());
    {
        const auto Lv = Chebyshev::plan_levels(v[0]->level, B.degree);
        const int lv = Chebyshev::feasible(Lv, B.degree);
        Chebyshev ch(A, v, B.degree);
        v = ch.eval(B.cheb, lv, v[0]->scale);
        for (int r = 0; r < B.double_angle && A.ok(); ++r) {
            Lanes sq = A.mul(v, v);
            v = A.ilin({{&sq, 2}}, -1.0, sq[0]->level);
        }
    }
    if (!A.ok()) return A.st;
    if (v[0]->level != B.level_after_mod) return set_err(c, FIDES_CUDA_ERR, "bootstrap level plan mismatch");
    Lanes y0(v.begin(), v.begin() + k), y1(v.begin() + k, v.end());
    Lanes iy = A.monomial(y1, (uint32_t)N / 2u);
    Lanes w = A.ilin({{&y0, 1}, {&iy, 1}}, 0.0, v[0]->level);
    if (!A.ok()) return A.st;
    for (const BootStage& st : B.stc) {
        Lanes y = A.fresh(k);
        s = linear_transform_batch(c, nin, (const fides_ct* const*)w.data(), (int)st.offsets.size(),
                                   st.offsets.data(), (const fides_pt* const*)st.pts.data(), st.bstep, 1, y.data(),
                                   true);
        if (s != FIDES_OK) return s;
        w = y;
    }
    // outputs last: an output may alias an input
    std::vector<double> sc(k);
    std::vector<int> slots(k);
    for (size_t u = 0; u < k; ++u) {
        sc[u] = w[u]->scale * in[u]->scale / c->default_scale * (double)(1ll << B.correction);
        slots[u] = in[u]->slots;
    }
    for (size_t u = 0; u < k; ++u) {
        s = fides_ct_copy(c, w[u], out[u]);
        if (s != FIDES_OK) return s;
        out[u]->scale = sc[u];
        out[u]->slots = slots[u];
        out[u]->noise_deg = 1;
    }
    return check_cuda(c, "bootstrap");
}

}  // extern "C"
