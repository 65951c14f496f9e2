// Stand-in for the reference's src/CKKS/Context.cuh (see README): a context
// accessor for the never-called *_forPrime wrappers of test/cpuNTT*.cpp.
#pragma once
#include "../ConstantsGPU.cuh"

namespace FIDESlib::CKKS {
struct ShimPrecom {
    Constants constants[1];
    Global* globals;
};
struct ShimContext {
    ShimPrecom precom;
};
inline ShimContext* GetCurrentContext() {
    static Global g{};
    static ShimContext c{{{}, &g}};
    return &c;
}
}  // namespace FIDESlib::CKKS
