// ref_gpu_ntt.cu -- a harness that runs the reference's own GPU forward NTT
// (NTT_<second, ALGO_SHOUP, NTT_NONE> of src/NTT.cu, the multi-limb kernel
// the reference's LimbPartition::ApplyNTT launches, src/CKKS/LimbPartition.cu:364-395)
// on this machine's GPU, for the per-kernel comparison of the forward NTT.
// TEST INFRASTRUCTURE ONLY: built by `make -C oracle ref-gpu` from the
// reference tree (src/NTT.cu compiled unmodified) into oracle/_ref/, loaded
// only by tests/test_gpu_ref_ntt.py.
//
// The reference reads its tables from a __constant__ Constants block and a
// device Global::Globals block that SetupConstants fills from OpenFHE
// (src/ConstantsGPU.cu:127-708).  Here both are allocated at their full
// declared sizes and the fields the forward NTT reads are filled with the
// same definitions SetupConstants uses (src/ConstantsGPU.cu:32-35 mu_new,
// :71-74 shoup_precomp, :188-320 the psi tables): primes, Barrett mu and bit
// widths, the root psi and its Shoup companion, psi_no[j] = psi^j for
// j < 2N, psi[j] = psi_no[bitrev(j)], psi_shoup; every other field is zero.
// Every index the kernel forms from these stays inside the tables by the
// launch geometry of ApplyNTT, which refntt_forward repeats; the limb-to-
// prime map primeid_flattened[k] = k mod nprimes covers the whole launch.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "ConstantsGPU.cuh"
#include "NTT.cuh"

namespace FIDESlib {
__constant__ Constants constants;
}

using namespace FIDESlib;

namespace {

typedef unsigned __int128 u128;

uint64_t mulmod(uint64_t a, uint64_t b, uint64_t p) { return (uint64_t)((u128)a * b % p); }
uint64_t powmod(uint64_t a, uint64_t e, uint64_t p) {
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = mulmod(r, a, p);
        a = mulmod(a, a, p);
        e >>= 1;
    }
    return r;
}
uint32_t bitrev(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int b = 0; b < bits; ++b)
        if (x >> b & 1) r |= 1u << (bits - 1 - b);
    return r;
}
int bit_width(uint64_t x) {
    int b = 0;
    while (x) {
        ++b;
        x >>= 1;
    }
    return b;
}
uint64_t shoup(uint64_t v, uint64_t p) { return (uint64_t)(((u128)(v << 1) << 63) / p); }

struct State {
    int logN = 0, N = 0, np = 0;
    Global::Globals* dglob = nullptr;        // device copy of the table block
    std::vector<void*> tables;               // device tables owned here
} g;

void release() {
    for (void* t : g.tables) cudaFree(t);
    g.tables.clear();
    if (g.dglob) cudaFree(g.dglob);
    g.dglob = nullptr;
}

}  // namespace

extern "C" {

// Tables for nprimes primes (p_i = 1 mod 2N, below 2^62) with the primitive
// 2N-th roots psi[i], ring dimension 2^logN, 12 <= logN <= 16.  0 on success.
int refntt_init(int logN, int nprimes, const uint64_t* primes, const uint64_t* psi) {
    if (logN < 12 || logN > 16 || nprimes < 1 || nprimes > MAXP || !primes || !psi) return 1;
    release();
    const int N = 1 << logN;
    for (int i = 0; i < nprimes; ++i) {
        const uint64_t p = primes[i];
        if (p >= (1ull << 62) || (p - 1) % (2ull * N) != 0) return 2;
        if (powmod(psi[i], N, p) != p - 1) return 3;  // not a primitive 2N-th root
    }
    static Constants hc;
    memset(&hc, 0, sizeof(hc));
    hc.N = N;
    hc.L = nprimes;
    hc.K = 0;
    hc.logN = logN;
    hc.dnum = 1;
    hc.type = 0;
    static Global::Globals hg;
    memset(&hg, 0, sizeof(hg));
    for (int i = 0; i < nprimes; ++i) {
        const uint64_t p = primes[i];
        const int bits = bit_width(p);
        hc.type |= (uint64_t)1 << i;  // 64-bit limbs
        hc.primes[i] = p;
        hc.prime_bits[i] = (uint32_t)bits;
        hc.prime_better_barret_mu[i] = (uint64_t)(((u128)1 << (2 * bits + 1)) / p);  // mu_new, NEIL
        const uint64_t ninv = powmod(N, p - 2, p), iroot = powmod(psi[i], p - 2, p);
        hc.N_shoup[i] = shoup(N % p, p);
        hc.N_inv[i] = ninv;
        hc.N_inv_shoup[i] = shoup(ninv, p);
        hc.root[i] = psi[i];
        hc.root_shoup[i] = shoup(psi[i], p);
        hc.inv_root[i] = iroot;
        hc.inv_root_shoup[i] = shoup(iroot, p);
        std::vector<uint64_t> no(2 * (size_t)N), ino(2 * (size_t)N), br(N), ibr(N), sh(N), ish(N), ms(N), ims(N);
        no[0] = ino[0] = 1;
        for (int j = 1; j < 2 * N; ++j) {
            no[j] = mulmod(no[j - 1], psi[i], p);
            ino[j] = mulmod(ino[j - 1], iroot, p);
        }
        for (int j = 0; j < N; ++j) {
            br[j] = no[bitrev(j, logN)];
            ibr[j] = ino[bitrev(j, logN)];
        }
        const int aw = (logN + 1) / 2;
        for (int j = 0; j < N / (1 << aw); ++j)
            for (int k = 0; k < (1 << aw); ++k) {
                ms[(size_t)j * (1 << aw) + k] = no[(size_t)j * bitrev(k, aw)];
                ims[(size_t)j * (1 << aw) + k] = mulmod(ino[(size_t)j * bitrev(k, aw)], ninv, p);
            }
        for (int j = 0; j < 2 * N; ++j) ino[j] = mulmod(ino[j], ninv, p);
        for (int j = 0; j < N; ++j) {
            sh[j] = shoup(br[j], p);
            ish[j] = shoup(ibr[j], p);
        }
        auto up = [&](const std::vector<uint64_t>& v) -> void* {
            void* d = nullptr;
            if (cudaMalloc(&d, v.size() * 8) != cudaSuccess) return nullptr;
            g.tables.push_back(d);
            cudaMemcpy(d, v.data(), v.size() * 8, cudaMemcpyHostToDevice);
            return d;
        };
        hg.psi[i] = up(br);
        hg.inv_psi[i] = up(ibr);
        hg.psi_no[i] = up(no);
        hg.inv_psi_no[i] = up(ino);
        hg.psi_middle_scale[i] = up(ms);
        hg.inv_psi_middle_scale[i] = up(ims);
        hg.psi_shoup[i] = up(sh);
        hg.inv_psi_shoup[i] = up(ish);
        if (!hg.psi[i] || !hg.inv_psi[i] || !hg.psi_no[i] || !hg.inv_psi_no[i] || !hg.psi_middle_scale[i] ||
            !hg.inv_psi_middle_scale[i] || !hg.psi_shoup[i] || !hg.inv_psi_shoup[i]) {
            release();
            return 4;
        }
    }
    // the limb-to-prime map read by the multi-limb kernel: entry k is prime k mod nprimes
    for (int k = 0; k < (MAXD * 3 + 1) * MAXP; ++k) hc.primeid_flattened[k] = k % nprimes;
    if (cudaMalloc((void**)&g.dglob, sizeof(Global::Globals)) != cudaSuccess) {
        release();
        return 4;
    }
    if (cudaMemcpy(g.dglob, &hg, sizeof(hg), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpyToSymbol(constants, &hc, sizeof(hc)) != cudaSuccess) {
        release();
        return 5;
    }
    g.logN = logN;
    g.N = N;
    g.np = nprimes;
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 5;
}

// Forward NTT of nlimbs limbs in place: limb k at data + k*N uses prime
// (prime0 + k) mod nprimes; aux (nlimbs*N words) holds the pass-1 output;
// limb_ptrs is device scratch for 2*nlimbs pointers.  The two launches of
// LimbPartition::ApplyNTT with their geometry.  0 on success.
int refntt_forward(uint64_t* data, uint64_t* aux, void** limb_ptrs, int prime0, int nlimbs, void* stream) {
    if (!g.dglob || !data || !aux || !limb_ptrs || nlimbs < 1 || prime0 < 0 ||
        prime0 + nlimbs > (MAXD * 3 + 1) * MAXP || nlimbs > 65535)
        return 1;
    const int N = g.N, logN = g.logN;
    std::vector<void*> h(2 * (size_t)nlimbs);
    for (int k = 0; k < nlimbs; ++k) {
        h[k] = data + (size_t)k * N;
        h[nlimbs + k] = aux + (size_t)k * N;
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemcpyAsync(limb_ptrs, h.data(), h.size() * sizeof(void*), cudaMemcpyHostToDevice, st) != cudaSuccess)
        return 2;
    cudaStreamSynchronize(st);  // the host array is released on return
    constexpr int M = 4;
    constexpr ALGO algo = ALGO_SHOUP;
    const dim3 b1{(uint32_t)(1 << ((logN + 1) / 2 - 1))};
    const dim3 b2{(uint32_t)(1 << (logN / 2 - 1))};
    const int bytes1 = 8 * b1.x * (2 * M + 1 + (algo == 2 || algo == ALGO_SHOUP ? 1 : 0));
    const int bytes2 = 8 * b2.x * (2 * M + 1 + (algo == 2 || algo == ALGO_SHOUP ? 1 : 0));
    void** dptr = limb_ptrs;
    void** aptr = limb_ptrs + nlimbs;
    NTT_<false, algo, NTT_NONE><<<dim3{(uint32_t)N / (b1.x * M * 2), (uint32_t)nlimbs}, b1, bytes1, st>>>(
        g.dglob, dptr, prime0, aptr, nullptr, 0, nullptr, nullptr);
    NTT_<true, algo, NTT_NONE><<<dim3{(uint32_t)N / (b2.x * M * 2), (uint32_t)nlimbs}, b2, bytes2, st>>>(
        g.dglob, aptr, prime0, dptr, nullptr, 0, nullptr, nullptr);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

void refntt_release(void) { release(); }

}  // extern "C"
