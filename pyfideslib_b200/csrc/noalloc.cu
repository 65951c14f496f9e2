// noalloc.cu -- polynomial multiply that allocates nothing.
//
// fides_polymul needs two scratch buffers for the forward transforms of its
// operands and asks the caller for them.  Some callers cannot obtain device
// memory at the point where they multiply:
//   * hosts that hand the whole device to their own allocator at start-up and
//     forbid later allocations (fixed-budget serving processes);
//   * latency-critical loops that must not call cudaMalloc / cudaFree, which
//     synchronise the device.
// fides_polymul_noalloc serves them: its scratch is a file-scope __device__
// array of fixed size, allocated when the library is loaded and held by
// every GPU that loads it until the process exits.
//
// Host code may not take the array's address directly (the host-side symbol
// is only a stand-in for the device object), so the device address is looked
// up once per device with cudaGetSymbolAddress, with that device current, the
// first time the entry point runs on it.  That first call should therefore
// come before any stream capture.  All calls share the one array and it keeps
// the last call's contents; nothing in it needs to start at zero, because the
// forward transforms overwrite every word a call reads.  Calls whose work
// overlaps on the GPU (different streams or contexts on one device) race on
// the array and must be serialised by the caller.
#include <mutex>

#include "context.hpp"

namespace {

// 2 operands x 2^19 words = 8 MiB: e.g. 8 limbs at N = 2^16, 32 at N = 2^14.
constexpr size_t kNoAllocWordsPerOperand = size_t(1) << 19;
constexpr int kNoAllocMaxDevices = 64;

__device__ __align__(256) uint64_t g_polymul_scratch[2 * kNoAllocWordsPerOperand];

std::mutex g_setup_mu;
uint64_t* g_scratch_addr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on `device` (current device).
fides_status scratch_for(fides_ctx* c, int device, uint64_t** out) {
    if (device < 0 || device >= kNoAllocMaxDevices)
        return fides::set_err(c, FIDES_UNSUPPORTED, "device ordinal beyond the no-alloc set-up table");
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_polymul_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return fides::set_err(c, FIDES_CUDA_ERR,
                                  std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e));
        }
        g_scratch_addr[device] = static_cast<uint64_t*>(p);
    }
    *out = g_scratch_addr[device];
    return FIDES_OK;
}

}  // namespace

extern "C" fides_status fides_polymul_noalloc(fides_ctx* ctx, const uint64_t* a, const uint64_t* b, uint64_t* c,
                                              int prime0, int nlimbs) {
    using namespace fides;
    if (!ctx || !a || !b || !c || prime0 < 0 || nlimbs < 1 || prime0 + nlimbs > ctx->L + ctx->K)
        return FIDES_BAD_ARG;
    if ((size_t)nlimbs * (size_t)ctx->N > kNoAllocWordsPerOperand)
        return set_err(ctx, FIDES_BAD_ARG,
                       "fides_polymul_noalloc: nlimbs * N = " + std::to_string((size_t)nlimbs * ctx->N) +
                           " words exceeds the fixed scratch of " + std::to_string(kNoAllocWordsPerOperand) +
                           " words per operand");
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    if (cudaSetDevice(ctx->device) != cudaSuccess) return check_cuda(ctx, "polymul_noalloc");
    uint64_t* scratch = nullptr;
    fides_status s = scratch_for(ctx, ctx->device, &scratch);
    if (s != FIDES_OK) return s;
    uint64_t* a_ntt = scratch;
    uint64_t* b_ntt = scratch + kNoAllocWordsPerOperand;
    LimbMap m{};
    m.nseg = 2;
    const uint64_t* ins[2] = {a, b};
    uint64_t* outs[2] = {a_ntt, b_ntt};
    for (int i = 0; i < 2; ++i) {
        LimbSeg& g = m.seg[i];
        g.in = ins[i];
        g.out = outs[i];
        g.count = nlimbs;
        g.skip_lo = nlimbs;
        g.nq = nlimbs;
        g.q0 = prime0;
        m.total += nlimbs;
    }
    ntt_forward(ctx->dev, m, FL_PLAIN, FS_PLAIN, ctx->st);
    ntt_inverse(ctx->dev, map_single(a_ntt, c, nlimbs, nlimbs, prime0, -1, b_ntt), IL_MUL, IS_PLAIN, ctx->st);
    return check_cuda(ctx, "polymul_noalloc");
}
