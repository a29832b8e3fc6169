// Device scrambled-Sobol points, bit-exact to torch.quasirandom.SobolEngine.
//
// SobolEngine(d, scramble=True, seed) stores scrambled direction numbers
// sobolstate[d][30] and a shift[d]; its point i (counted from the engine's start)
// is shift ^ (xor of sobolstate[:, j] over the set bits j of gray(i) = i ^ (i >> 1)),
// times 2^-30.  A float32 draw rounds the 30-bit integer to float32 first and then
// scales by 2^-30; a float64 draw is exact except for point 0, which torch computes
// in float32 and casts (torch/quasirandom.py, _first_point).
#pragma once

#include <stdint.h>

namespace nlo {

__device__ __forceinline__ uint32_t sobol_bits(const uint32_t* state /*[30] of one dimension*/,
                                               uint32_t shift, uint64_t index)
{
    uint32_t g = (uint32_t)(index ^ (index >> 1));
    uint32_t v = shift;
    while (g) {
        const int j = __ffs(g) - 1;
        v ^= state[j];
        g &= g - 1;
    }
    return v;
}

template <typename T>
__device__ __forceinline__ T sobol_unit(uint32_t bits, uint64_t index);

template <>
__device__ __forceinline__ float sobol_unit<float>(uint32_t bits, uint64_t)
{
    return __fmul_rn(__uint2float_rn(bits), 9.313225746154785e-10f);  // 2^-30
}

template <>
__device__ __forceinline__ double sobol_unit<double>(uint32_t bits, uint64_t index)
{
    if (index == 0) return (double)__fmul_rn(__uint2float_rn(bits), 9.313225746154785e-10f);
    return (double)bits * 9.313225746154785e-10;
}

}  // namespace nlo
