// abi.cu -- error plumbing and library information of the C ABI (include/epsr_gpu.h).
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

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

// ----------------------------------------------------------------- kernel timing
// One record per bracketed launch: the two events, kept until the next enable.  Events come
// from a pool that is reused across enables, so a long run creates no more events than the
// launches of one measurement.
int g_epsr_timing_on = 0;
namespace {
std::mutex g_tm_mu;
std::map<std::string, std::vector<std::pair<cudaEvent_t, cudaEvent_t>>> g_tm;
std::map<std::string, cudaEvent_t> g_tm_open;   // name + stream -> start event
std::vector<cudaEvent_t> g_tm_pool;
size_t g_tm_used = 0;

cudaEvent_t tm_event() {
    if (g_tm_used == g_tm_pool.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        g_tm_pool.push_back(e);
    }
    return g_tm_pool[g_tm_used++];
}
}  // namespace

void epsr_timing_mark(const char *name, cudaStream_t s, int end) {
    std::lock_guard<std::mutex> lk(g_tm_mu);
    char key[160];
    snprintf(key, sizeof(key), "%s@%p", name, (void *)s);
    if (!end) {
        cudaEvent_t e = tm_event();
        if (!e) return;
        cudaEventRecord(e, s);
        g_tm_open[key] = e;
        return;
    }
    auto it = g_tm_open.find(key);
    if (it == g_tm_open.end()) return;
    cudaEvent_t e1 = tm_event();
    if (!e1) return;
    cudaEventRecord(e1, s);
    g_tm[name].push_back({it->second, e1});
    g_tm_open.erase(it);
}

extern "C" int epsr_timing_enable(int32_t on) {
    std::lock_guard<std::mutex> lk(g_tm_mu);
    if (on) {   // a new measurement: earlier records go (disabling keeps them for reading)
        g_tm.clear();
        g_tm_open.clear();
        g_tm_used = 0;
    }
    g_epsr_timing_on = on ? 1 : 0;
    return EPSR_OK;
}

extern "C" int epsr_timing_read(const char *kernel, double *total_ms, int64_t *launches) {
    if (!kernel || !total_ms || !launches) {
        epsr_set_error("epsr_timing_read: null pointer");
        return EPSR_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(g_tm_mu);
    double t = 0.0;
    int64_t n = 0;
    auto it = g_tm.find(kernel);
    if (it != g_tm.end()) {
        for (auto &pr : it->second) {
            EPSR_CUDA(cudaEventSynchronize(pr.second));
            float ms = 0.0f;
            EPSR_CUDA(cudaEventElapsedTime(&ms, pr.first, pr.second));
            t += ms;
            ++n;
        }
    }
    *total_ms = t;
    *launches = n;
    return EPSR_OK;
}
