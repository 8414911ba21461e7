// ran1.cu -- device ran1 stream (auxiliary_routines.py:324-391), bit-identical.
//
// One warp produces the sequence.  The Park-Miller part is jumped ahead so that lane l
// holds idum after l+1 more steps (Schrage's method computes IA*idum mod IM exactly, so a
// 64-bit modular product with IA^k gives the same value).  The Bays-Durham shuffle is an
// inherently sequential pointer chase; its 32-entry table lives one entry per lane and
// each step is a shift plus a warp shuffle.
#include "common.cuh"

namespace epsr {

__device__ __forceinline__ uint32_t mulmod_im(uint32_t a, uint32_t b) {
    return (uint32_t)(((uint64_t)a * (uint64_t)b) % 2147483647ull);
}

__global__ void ran1_fill_kernel(int32_t *state, float *out, int64_t n) {
    const int lane = threadIdx.x & 31;
    __shared__ int32_t st[35];
    __shared__ Ran1 init;
    int32_t idum = state[0], iy = state[1], mcall = state[2];
    int32_t iv;
    if (idum <= 0 || iy == 0) {
        if (lane == 0) {
            int64_t neg = -(int64_t)idum;
            int32_t w = (int32_t)(uint32_t)(uint64_t)neg;
            int32_t d = w > 1 ? w : 1;
            for (int j = 40; j >= 1; --j) {
                d = ran1_lcg(d);
                if (j <= 32) init.iv[j - 1] = d;
            }
            init.idum = d;
            init.iy = init.iv[0];
        }
        __syncwarp();
        idum = init.idum;
        iy = init.iy;
        iv = init.iv[lane];
    } else {
        iv = state[3 + lane];
    }
    uint32_t mul = 16807u;
    for (int k = 0; k < lane; ++k) mul = mulmod_im(mul, 16807u);
    int64_t done = 0;
    while (done < n) {
        const int cnt = (n - done) >= 32 ? 32 : (int)(n - done);
        const int32_t idl = (int32_t)mulmod_im(mul, (uint32_t)idum);
        int32_t mine = 0;
        for (int s = 0; s < cnt; ++s) {
            const int32_t id = __shfl_sync(0xffffffffu, idl, s);
            const int j = iy >> 26;
            const int32_t nxt = __shfl_sync(0xffffffffu, iv, j);
            if (lane == j) iv = id;
            iy = nxt;
            if (lane == s) mine = iy;
        }
        idum = __shfl_sync(0xffffffffu, idl, cnt - 1);
        if (lane < cnt) out[done + lane] = ran1_out(mine);
        done += cnt;
    }
    st[3 + lane] = iv;
    __syncwarp();
    if (lane == 0) {
        state[0] = idum;
        state[1] = iy;
        state[2] = (int32_t)((uint32_t)mcall + (uint32_t)n);
    }
    state[3 + lane] = st[3 + lane];
}

}  // namespace epsr

extern "C" int epsr_ran1_fill(int32_t *state, float *out, int64_t n, void *stream) {
    if (!state || (n > 0 && !out) || n < 0) {
        epsr_set_error("epsr_ran1_fill: null pointer or negative n");
        return EPSR_ERR_ARG;
    }
    if (n == 0) return EPSR_OK;
    epsr::ran1_fill_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(state, out, n);
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}
