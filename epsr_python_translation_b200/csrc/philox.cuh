// philox.cuh -- Philox4x32 with ten rounds (Salmon, Moraes, Dror, Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC 2011), the counter-based generator of the batched
// checkerboard Monte Carlo.  Every random number of a move is a pure function of (box key,
// sweep, step, slot, purpose), so the moves of all boxes and slots draw in parallel, a CUDA
// graph can replay a sweep, and the NumPy restatement in the tests reproduces every draw.
#pragma once

#include <stdint.h>

namespace epsr {

struct U4 {
    uint32_t x, y, z, w;
};

__host__ __device__ __forceinline__ void philox_mulhilo(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo) {
    const uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
}

// counter c, key (k0, k1): ten rounds with the published multipliers and Weyl key increments
__host__ __device__ __forceinline__ U4 philox4x32(U4 c, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t h0, l0, h1, l1;
        philox_mulhilo(M0, c.x, h0, l0);
        philox_mulhilo(M1, c.z, h1, l1);
        c = U4{h1 ^ c.y ^ k0, l1, h0 ^ c.w ^ k1, l0};
        k0 += W0;
        k1 += W1;
    }
    return c;
}

// uniform float in [0, 1) from the top 24 bits
__host__ __device__ __forceinline__ float u01(uint32_t v) { return (float)(v >> 8) * (1.0f / 16777216.0f); }

}  // namespace epsr
