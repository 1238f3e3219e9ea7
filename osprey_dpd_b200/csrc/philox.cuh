// philox.cuh -- counter-based pair noise for the DPD random force.
//
// The reference draws one uniform number per interacting pair from a single
// serial 64-bit LCG in cell-list order (CCNTCell::Randf, CNTCell.cpp:2454-2465),
// which no parallel evaluation can reproduce.  The engine instead draws the
// same distribution (uniform on [0,1), one number per pair per step) from
// Philox2x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11): counter = (min id, max id) of the pair, key = a mix of
// the run seed and the step.  Both beads of a pair therefore see the same
// number regardless of evaluation order, so F_R stays exactly antisymmetric.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define DPD_HD __host__ __device__ __forceinline__
#else
#define DPD_HD inline
#endif

namespace dpd {

DPD_HD uint32_t philox_step_key(uint64_t seed, int64_t step)
{
    uint32_t s = (uint32_t)seed ^ (uint32_t)(seed >> 32) * 0x85EBCA6Bu;
    s ^= s >> 16;
    s *= 0x7FEB352Du;
    s ^= s >> 15;
    return s + (uint32_t)step * 0xC2B2AE35u;
}

DPD_HD uint32_t philox2x32_10(uint32_t c0, uint32_t c1, uint32_t k)
{
    const uint32_t M = 0xD256D193u, W = 0x9E3779B9u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
        const uint32_t hi = __umulhi(M, c0);
        const uint32_t lo = M * c0;
#else
        const uint64_t prod = (uint64_t)M * (uint64_t)c0;
        const uint32_t hi = (uint32_t)(prod >> 32), lo = (uint32_t)prod;
#endif
        c0 = hi ^ k ^ c1;
        c1 = lo;
        k += W;
    }
    return c0;
}

}  // namespace dpd
