// ran1.cu -- device ran1 stream (auxiliary_routines.py:324-391), bit-identical.
//
// One warp produces the sequence.  The Park-Miller part is jumped ahead so that lane l
// holds idum after l+1 more steps (Schrage's method computes IA*idum mod IM exactly, so a
// 64-bit modular product with IA^k gives the same value).  The Bays-Durham shuffle is an
// inherently sequential pointer chase; its 32-entry table lives one entry per lane and
// each step is a warp shuffle (Ran1Warp in common.cuh).
//
// The reference re-initialises on any call that finds idum <= 0 or iy == 0 (:346).  That
// happens at the first call of a stream and, for the degenerate seed -(2^31-1), again after
// a step that produced idum == 0; a batch therefore ends after such a step and the next
// batch starts with the initialisation.
#include "common.cuh"

namespace epsr {

__global__ void ran1_fill_kernel(int32_t *state, float *out, int64_t n_host, const int32_t *n_dev) {
    const int lane = threadIdx.x & 31;
    const int64_t n = n_dev ? (int64_t)*n_dev : n_host;
    __shared__ int32_t tab[34];
    Ran1Warp g;
    g.load(state);
    const int32_t mcall = state[2];
    __syncwarp();
    int64_t done = 0;
    while (done < n) {
        const int64_t left = n - done;
        int32_t mine;
        const int cnt = g.next(left > 32 ? 32 : (int)left, mine, tab);
        if (lane < cnt) out[done + lane] = ran1_out(mine);
        done += cnt;
    }
    state[3 + lane] = g.iv;
    if (lane == 0) {
        state[0] = g.idum;
        state[1] = g.iy;
        state[2] = (int32_t)((uint32_t)mcall + (uint32_t)n);
    }
}

}  // namespace epsr

extern "C" int epsr_ran1_fill(int32_t *state, float *out, int64_t n, void *stream) {
    if (!state || (n > 0 && !out) || n < 0) {
        epsr_set_error("epsr_ran1_fill: null pointer or negative n");
        return EPSR_ERR_ARG;
    }
    if (n == 0) return EPSR_OK;
    epsr::ran1_fill_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(state, out, n, nullptr);
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}
