// Device helpers shared by the rh3t kernels: padded-node indexing, state
// loads, stage buffer selection and the device error record.
#pragma once
#include "rh3t_dev.h"

namespace rh3t {

__device__ __forceinline__ long long node_of(const Inst& I, int i, int j) {
    return (long long)(i + RH3T_PAD) * I.nyp + (j + RH3T_PAD);
}

__device__ __forceinline__ void load6(const double* __restrict__ buf, long long plane, long long n, double s[6]) {
#pragma unroll
    for (int c = 0; c < 6; ++c) s[c] = buf[c * plane + n];
}

__device__ __forceinline__ bool has_error(const Inst& I) { return I.err->key != ~0ull; }

__device__ __forceinline__ void report(const Inst& I, int phase, int code, unsigned int index) {
    unsigned long long step = (unsigned long long)I.sc->step;
    unsigned long long key = (step << 40) | ((unsigned long long)phase << 37) | ((unsigned long long)code << 32) |
                             (unsigned long long)index;
    atomicMin(&I.err->key, key);
}

__device__ __forceinline__ const double* stage_src(const Inst& I, int stage) {
    return stage == 0 ? I.U : (stage == 1 ? I.A : I.B);
}

} // namespace rh3t
