// Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel Random Numbers: As Easy as 1, 2, 3", SC 2011): ten rounds of
// two 32x32->64 multiplies and a Feistel-like mix, keyed by the seed. The kernels' counter is (pixel, pass in the
// round, depth << 4 | block, job): every number a sample draws is a pure function of the seed and where it is used, so
// a seed fixes every image, whatever thread, launch or batch renders it.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace rtb
{
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k)
{
#pragma unroll
    for (int round = 0; round < 10; ++round)
    {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z);
        const uint32_t lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}
} // namespace rtb
