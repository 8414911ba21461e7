// abi.cu -- error plumbing and library information of the C ABI (include/epsr_gpu.h).
#include <stdarg.h>
#include <stdio.h>

#include "common.cuh"

static thread_local char g_err[512] = "";

void epsr_set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int epsr_cuda_check(cudaError_t e, const char *what) {
    epsr_set_error("CUDA error %d (%s) in %s", (int)e, cudaGetErrorString(e), what);
    return EPSR_ERR_CUDA;
}

// Copies between device memory and pageable host memory, made only once the stream has
// drained.  A pageable copy that has to wait for earlier work on its stream holds the
// driver's staging path meanwhile, which holds up the pageable copies of every other host
// thread; with the wait taken first, boxes driven from several host threads on their own
// streams do not serialise on each other's kernels.
int epsr_d2h(void *dst, const void *src, size_t bytes, cudaStream_t s) {
    EPSR_CUDA(cudaStreamSynchronize(s));
    EPSR_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
    EPSR_CUDA(cudaStreamSynchronize(s));
    return EPSR_OK;
}

int epsr_h2d(void *dst, const void *src, size_t bytes, cudaStream_t s) {
    EPSR_CUDA(cudaStreamSynchronize(s));
    EPSR_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    EPSR_CUDA(cudaStreamSynchronize(s));
    return EPSR_OK;
}

extern "C" const char *epsr_last_error(void) { return g_err; }

extern "C" const char *epsr_version(void) { return "epsr-b200 0.1 (sm_100a)"; }

extern "C" int epsr_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return -1;
    int k = 0;
    for (int d = 0; d < n; ++d) {
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, d) == cudaSuccess && p.major == 10) ++k;
    }
    return k;
}
