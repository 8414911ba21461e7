// mlp.cu -- the surrogate network of the delayed-acceptance Monte Carlo: a 1280 -> 128 -> 128
// -> 1 perceptron with SiLU activations, BF16 weights and activations, FP32 accumulation,
// evaluated and trained by one hand-written tcgen05 GEMM kernel with per-layer epilogues.
//
// The GEMM.  One CTA of 128 threads computes a 128 x 128 tile D = A_tile . B_tile^T over a
// K range (split-K over blockIdx.z): thread 0 streams 128 x 64 BF16 tiles of A and B into a
// four-stage shared-memory ring with TMA (SWIZZLE_128B, K-major) and issues four
// tcgen05.mma (M = 128, N = 128, K = 16) per stage, committing each stage back to its ring
// slot; the FP32 accumulator lives in 128 columns of tensor memory.  The four warps then read
// their 32 accumulator rows (tcgen05.ld 32x32b) and run the epilogue of the layer:
//   STORE      D as FP32 (the raw product, for tests);
//   ATOMIC     D added into an FP32 matrix (the weight gradients, split over K = samples);
//   BIAS_SILU  z = D + b, h = silu(z): h in BF16 (row-major, and transposed for the weight
//              gradient), z in FP32 when training;
//   HEAD       z = D + b, h = silu(z), y = h . w3 + b3 per row; when training, rows come in
//              pairs (features before/after, after/before) whose antisymmetric part
//              s = (y0 - y1)/2 is fitted to the target: the loss, dL/dy, dz = dL/dy w3 silu'(z)
//              in BF16 (row-major and transposed) and the w3, b3, b2 gradients;
//   SILU_BWD   dz = D silu'(z_saved) (D = dz2 . W2), BF16 transposed, and the b1 gradient.
// Every mbarrier wait is bounded (2 s): on timeout the kernel records status 1 and returns
// after releasing its tensor memory.
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "common.cuh"
#include "umma.cuh"

namespace epsr {

using bf16 = __nv_bfloat16;
constexpr int MLP_IN = 1280, MLP_H = 128;
constexpr int G_STAGES = 4;
constexpr int G_THREADS = 128;
constexpr size_t G_SMEM = 1024 + 2 * G_STAGES * umma::TILE_BYTES;   // + alignment slack

enum Epi : int { EPI_STORE = 0, EPI_ATOMIC = 1, EPI_BIAS_SILU = 2, EPI_HEAD = 3, EPI_SILU_BWD = 4 };

struct GemmArgs {
    int M, N, K, kslices, epi;
    float *out;
    int ldo;
    const float *bias;
    float *z_out;           // [M][N] FP32 pre-activation (BIAS_SILU, training)
    bf16 *h_out;            // [M][N] BF16 activation (BIAS_SILU)
    bf16 *ht_out;           // [N][ldt] BF16 transposed activation (BIAS_SILU, training)
    int ldt;                // leading dimension of the transposed outputs (>= M)
    const float *w3;        // [N] (HEAD)
    const float *b3;        // [1] (HEAD)
    float *y;               // [M] (HEAD)
    const float *target;    // [M/2] antisymmetric targets (HEAD, training), or null
    float gscale;           // dL/dy scale (1 / number of pairs)
    float *loss;            // [1] sum of squared pair errors (HEAD, training)
    float *dw3, *db3, *db;  // gradients (HEAD: w3, b3, b2; SILU_BWD: b1 in db)
    bf16 *dz_out;           // [M][N] BF16 (HEAD, training)
    bf16 *dzt_out;          // [N][ldt] BF16 transposed (HEAD and SILU_BWD, training)
    const float *z_in;      // [M][N] saved pre-activation (SILU_BWD)
    int *status;
};

__device__ __forceinline__ float sigm(float z) { return 1.0f / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu(float z) { return z * sigm(z); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = sigm(z);
    return s * (1.0f + z * (1.0f - s));
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(G_THREADS) umma_gemm_kernel(const __grid_constant__ CUtensorMap ta,
                                                              const __grid_constant__ CUtensorMap tb, GemmArgs g) {
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full[G_STAGES], empty[G_STAGES], done;
    __shared__ uint32_t tmem_base;
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * umma::TILE_M, n0 = blockIdx.y * umma::TILE_N;
    const int nkb = g.K / umma::TILE_K;
    const int kb0 = (int)((long long)blockIdx.z * nkb / g.kslices);
    const int kb1 = (int)((long long)(blockIdx.z + 1) * nkb / g.kslices);
    const int nk = kb1 - kb0;
    if (warp == 0) {
        umma::tmem_alloc(&tmem_base, 128);
        umma::tmem_relinquish();
    }
    if (tid == 0) {
        for (int s = 0; s < G_STAGES; ++s) {
            umma::mbar_init(&full[s], 1);
            umma::mbar_init(&empty[s], 1);
        }
        umma::mbar_init(&done, 1);
        umma::fence_mbar_init();
        umma::prefetch_tmap(&ta);
        umma::prefetch_tmap(&tb);
    }
    umma::tc_fence_before();
    __syncthreads();
    umma::tc_fence_after();
    const uint32_t tmem = tmem_base;
    auto stage_a = [&](int s) { return smem + (size_t)s * umma::TILE_BYTES; };
    auto stage_b = [&](int s) { return smem + (size_t)(G_STAGES + s) * umma::TILE_BYTES; };
    if (tid == 0) {
        constexpr uint32_t idesc = umma::idesc_bf16_f32(umma::TILE_M, umma::TILE_N);
        const int pro = nk < G_STAGES ? nk : G_STAGES;
        for (int i = 0; i < pro; ++i) {
            umma::mbar_expect_tx(&full[i], 2 * umma::TILE_BYTES);
            umma::tma_load_2d(stage_a(i), &ta, (kb0 + i) * umma::TILE_K, m0, &full[i]);
            umma::tma_load_2d(stage_b(i), &tb, (kb0 + i) * umma::TILE_K, n0, &full[i]);
        }
        for (int i = 0; i < nk; ++i) {
            const int s = i % G_STAGES;
            const uint32_t ph = (uint32_t)(i / G_STAGES) & 1u;
            if (!umma::mbar_wait(&full[s], ph, g.status)) break;
            umma::tc_fence_after();
            const uint64_t ad = umma::sdesc_sw128(stage_a(s)), bd = umma::sdesc_sw128(stage_b(s));
#pragma unroll
            for (int kk = 0; kk < umma::TILE_K / 16; ++kk)   // 32 bytes (16 BF16) further per K-slice
                umma::mma_bf16(tmem, ad + 2 * kk, bd + 2 * kk, idesc, (i > 0 || kk > 0) ? 1u : 0u);
            umma::mma_commit(&empty[s]);
            const int j = i + G_STAGES;
            if (j < nk) {
                if (!umma::mbar_wait(&empty[s], ph, g.status)) break;
                umma::mbar_expect_tx(&full[s], 2 * umma::TILE_BYTES);
                umma::tma_load_2d(stage_a(s), &ta, (kb0 + j) * umma::TILE_K, m0, &full[s]);
                umma::tma_load_2d(stage_b(s), &tb, (kb0 + j) * umma::TILE_K, n0, &full[s]);
            }
        }
        umma::mma_commit(&done);
    }
    __syncwarp();
    const bool ok = umma::mbar_wait(&done, 0, g.status) && nk > 0;
    umma::tc_fence_after();
    const int row = m0 + warp * 32 + lane;
    const bool rv = row < g.M;
    const uint32_t tbase = tmem + ((uint32_t)(warp * 32) << 16);
    float v[16];
    if (ok) {
        if (g.epi == EPI_STORE || g.epi == EPI_ATOMIC) {
            for (int c = 0; c < umma::TILE_N; c += 16) {
                umma::tmem_ld16(tbase + c, v);
                if (rv) {
                    float *o = g.out + (size_t)row * g.ldo + n0 + c;
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        if (n0 + c + i < g.N) {
                            if (g.epi == EPI_STORE) o[i] = v[i];
                            else atomicAdd(o + i, v[i]);
                        }
                    }
                }
            }
        } else if (g.epi == EPI_BIAS_SILU) {
            for (int c = 0; c < umma::TILE_N; c += 16) {
                umma::tmem_ld16(tbase + c, v);
                if (rv) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        const int n = n0 + c + i;
                        const float z = v[i] + g.bias[n];
                        const bf16 h = __float2bfloat16_rn(silu(z));
                        if (g.z_out) g.z_out[(size_t)row * g.N + n] = z;
                        g.h_out[(size_t)row * g.N + n] = h;
                        if (g.ht_out) g.ht_out[(size_t)n * g.ldt + row] = h;
                    }
                }
            }
        } else if (g.epi == EPI_HEAD) {
            float acc = 0.0f;
            for (int c = 0; c < umma::TILE_N; c += 16) {
                umma::tmem_ld16(tbase + c, v);
#pragma unroll
                for (int i = 0; i < 16; ++i) acc += silu(v[i] + g.bias[c + i]) * g.w3[c + i];
            }
            const float y = acc + *g.b3;
            if (rv) g.y[row] = y;
            if (g.target) {
                // rows 2p, 2p+1 are the two orders of pair p (adjacent lanes of one warp)
                const float yo = __shfl_xor_sync(0xffffffffu, y, 1);
                const bool even = (lane & 1) == 0;
                const float s = even ? 0.5f * (y - yo) : 0.5f * (yo - y);
                const float diff = rv ? s - g.target[row >> 1] : 0.0f;
                const float gy = rv ? (even ? diff : -diff) * g.gscale : 0.0f;
                float l = (even && rv) ? diff * diff : 0.0f;
                l = warp_sum(l);
                if (lane == 0) atomicAdd(g.loss, l);
                const float gb3 = warp_sum(gy);
                if (lane == 0) atomicAdd(g.db3, gb3);
                for (int c = 0; c < umma::TILE_N; c += 16) {
                    umma::tmem_ld16(tbase + c, v);
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        const int n = c + i;
                        const float z = v[i] + g.bias[n];
                        const float h = silu(z);
                        const float dz = gy * g.w3[n] * dsilu(z);
                        const bf16 dzb = __float2bfloat16_rn(dz);
                        if (rv) {
                            g.dz_out[(size_t)row * g.N + n] = dzb;
                            g.dzt_out[(size_t)n * g.ldt + row] = dzb;
                        }
                        const float a = warp_sum(gy * h), b = warp_sum(dz);
                        if (lane == 0) {
                            atomicAdd(g.dw3 + n, a);
                            atomicAdd(g.db + n, b);
                        }
                    }
                }
            }
        } else if (g.epi == EPI_SILU_BWD) {
            for (int c = 0; c < umma::TILE_N; c += 16) {
                umma::tmem_ld16(tbase + c, v);
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int n = n0 + c + i;
                    const float dz = rv ? v[i] * dsilu(g.z_in[(size_t)row * g.N + n]) : 0.0f;
                    if (rv) g.dzt_out[(size_t)n * g.ldt + row] = __float2bfloat16_rn(dz);
                    const float b = warp_sum(dz);
                    if (lane == 0) atomicAdd(g.db + n, b);
                }
            }
        }
    }
    umma::tc_fence_before();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tmem, 128);
}

// ----------------------------------------------------------------- Adam
struct AdamArgs {
    float *w, *grad, *m, *v;
    bf16 *wh;      // BF16 copy [n] (or null)
    bf16 *wht;     // BF16 transposed copy of a rows x cols matrix (or null)
    int n, rows, cols;
    float lr, b1, b2, eps, c1, c2, wd;
};

__global__ void adam_kernel(AdamArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const float gr = a.grad[i];
    const float m = a.b1 * a.m[i] + (1.0f - a.b1) * gr;
    const float v = a.b2 * a.v[i] + (1.0f - a.b2) * gr * gr;
    a.m[i] = m;
    a.v[i] = v;
    float w = a.w[i];
    w -= a.lr * ((m * a.c1) / (sqrtf(v * a.c2) + a.eps) + a.wd * w);
    a.w[i] = w;
    a.grad[i] = 0.0f;
    if (a.wh) a.wh[i] = __float2bfloat16_rn(w);
    if (a.wht) {
        const int r = i / a.cols, c = i % a.cols;
        a.wht[(size_t)c * a.rows + r] = __float2bfloat16_rn(w);
    }
}

__global__ void to_bf16_kernel(const float *w, bf16 *wh, bf16 *wht, int rows, int cols) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows * cols) return;
    const bf16 h = __float2bfloat16_rn(w[i]);
    if (wh) wh[i] = h;
    if (wht) wht[(size_t)(i % cols) * rows + i / cols] = h;
}

// ----------------------------------------------------------------- host side
namespace {
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::mutex g_encode_mu;

int get_encode() {
    std::lock_guard<std::mutex> lk(g_encode_mu);
    if (g_encode) return EPSR_OK;
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || !fn || q != cudaDriverEntryPointSuccess) {
        epsr_set_error("cuTensorMapEncodeTiled is not available from the driver");
        return EPSR_ERR_CUDA;
    }
    g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    return EPSR_OK;
}

// Tensor map of a row-major BF16 matrix [rows][cols] (cols contiguous, ld elements between
// rows) read in 128 x 64 boxes with the 128-byte swizzle.  cols and ld must be multiples of 64
// and the base 16-byte aligned, so every box starts on a 16-byte boundary (x = 64 k); rows
// beyond the matrix read as zero.
int make_map(CUtensorMap *m, const void *base, int64_t rows, int64_t cols, int64_t ld) {
    int rc = get_encode();
    if (rc) return rc;
    if (((uintptr_t)base & 15) || cols % umma::TILE_K || ld % umma::TILE_K || ld < cols || rows <= 0) {
        epsr_set_error("tensor map: base %p must be 16-byte aligned, cols %lld and ld %lld multiples of 64", base,
                       (long long)cols, (long long)ld);
        return EPSR_ERR_ARG;
    }
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    cuuint32_t box[2] = {(cuuint32_t)umma::TILE_K, (cuuint32_t)umma::TILE_M};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        epsr_set_error("cuTensorMapEncodeTiled failed (%d) for a %lld x %lld matrix", (int)r, (long long)rows,
                       (long long)cols);
        return EPSR_ERR_CUDA;
    }
    return EPSR_OK;
}

// D[M x N] over K: A [M][lda] and B [N][ldb] row-major BF16 (K contiguous).  The grid covers
// M and N in tiles of 128 (rows past M of A and past N of B read as zero); K is a multiple of
// 64 and is split into kslices ranges (one CTA each, at least one 64-wide block apiece).
int gemm(const void *A, int M, int64_t lda, const void *B, int N, int64_t ldb, int K, int kslices, GemmArgs g,
         cudaStream_t s) {
    if (M <= 0 || N <= 0 || K <= 0 || K % umma::TILE_K || kslices < 1 || kslices > K / umma::TILE_K) {
        epsr_set_error("umma gemm: bad shape M %d N %d K %d kslices %d", M, N, K, kslices);
        return EPSR_ERR_ARG;
    }
    CUtensorMap ta, tb;
    int rc = make_map(&ta, A, M, K, lda);
    if (rc) return rc;
    rc = make_map(&tb, B, N, K, ldb);
    if (rc) return rc;
    g.M = M;
    g.N = N;
    g.K = K;
    g.kslices = kslices;
    EPSR_SMEM_OPTIN(umma_gemm_kernel);
    dim3 grid((M + 127) / 128, (N + 127) / 128, kslices);
    EPSR_TIMED("umma_gemm_kernel", s, umma_gemm_kernel<<<grid, G_THREADS, G_SMEM, s>>>(ta, tb, g));
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}
}  // namespace
}  // namespace epsr

using namespace epsr;

extern "C" int epsr_umma_gemm_f32(const void *a, int32_t m, const void *b, int32_t n, int32_t k, int32_t kslices,
                                  float *out, int32_t ldo, int32_t accumulate, int32_t *status, void *stream) {
    if (!a || !b || !out || !status || ldo < n) {
        epsr_set_error("epsr_umma_gemm_f32: null pointer or ldo < n");
        return EPSR_ERR_ARG;
    }
    GemmArgs g = {};
    g.epi = accumulate ? EPI_ATOMIC : EPI_STORE;
    g.out = out;
    g.ldo = ldo;
    g.status = status;
    return gemm(a, m, k, b, n, k, k, kslices, g, (cudaStream_t)stream);
}

extern "C" int64_t epsr_mlp_work_bytes(int32_t rows) {
    const int64_t R = ((int64_t)rows + 127) / 128 * 128;
    return 256 * 8 + R * MLP_H * (2 + 4 + 2 + 2 + 2 + 2) + R * 4 * 2 + 4096;
}

namespace {
struct MlpWork {
    bf16 *h1, *h1t, *dz2, *dz2t, *dz1t;
    float *z1, *y, *loss;
};
MlpWork carve(void *work, int R) {
    char *p = (char *)work;
    auto take = [&](size_t b) {
        char *r = p;
        p += (b + 255) & ~(size_t)255;
        return (void *)r;
    };
    MlpWork w;
    w.h1 = (bf16 *)take(sizeof(bf16) * (size_t)R * MLP_H);
    w.h1t = (bf16 *)take(sizeof(bf16) * (size_t)R * MLP_H);
    w.dz2 = (bf16 *)take(sizeof(bf16) * (size_t)R * MLP_H);
    w.dz2t = (bf16 *)take(sizeof(bf16) * (size_t)R * MLP_H);
    w.dz1t = (bf16 *)take(sizeof(bf16) * (size_t)R * MLP_H);
    w.z1 = (float *)take(sizeof(float) * (size_t)R * MLP_H);
    w.y = (float *)take(sizeof(float) * (size_t)R);
    w.loss = (float *)take(sizeof(float) * 8);
    return w;
}

int check_net(const epsr_mlp_t *net, const char *who) {
    if (!net || !net->w1 || !net->b1 || !net->w2 || !net->b2 || !net->w3 || !net->b3 || !net->w1h || !net->w2h ||
        !net->w2th || !net->status) {
        epsr_set_error("%s: null network pointer", who);
        return EPSR_ERR_ARG;
    }
    return EPSR_OK;
}
}  // namespace

extern "C" int epsr_mlp_sync_weights(const epsr_mlp_t *net, void *stream) {
    int rc = check_net(net, "epsr_mlp_sync_weights");
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    to_bf16_kernel<<<(MLP_H * MLP_IN + 255) / 256, 256, 0, s>>>(net->w1, (bf16 *)net->w1h, nullptr, MLP_H, MLP_IN);
    to_bf16_kernel<<<(MLP_H * MLP_H + 255) / 256, 256, 0, s>>>(net->w2, (bf16 *)net->w2h, (bf16 *)net->w2th, MLP_H,
                                                                MLP_H);
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}

extern "C" int epsr_mlp_forward(const epsr_mlp_t *net, const void *x, int32_t rows, float *y, void *work,
                                int64_t work_bytes, void *stream) {
    int rc = check_net(net, "epsr_mlp_forward");
    if (rc) return rc;
    if (!x || !y || !work || rows <= 0) {
        epsr_set_error("epsr_mlp_forward: null pointer or no rows");
        return EPSR_ERR_ARG;
    }
    if (work_bytes < epsr_mlp_work_bytes(rows)) {
        epsr_set_error("epsr_mlp_forward: work needs %lld bytes", (long long)epsr_mlp_work_bytes(rows));
        return EPSR_ERR_CAPACITY;
    }
    cudaStream_t s = (cudaStream_t)stream;
    MlpWork w = carve(work, (rows + 127) / 128 * 128);
    GemmArgs g1 = {};
    g1.epi = EPI_BIAS_SILU;
    g1.bias = net->b1;
    g1.h_out = w.h1;
    g1.status = net->status;
    rc = gemm(x, rows, MLP_IN, net->w1h, MLP_H, MLP_IN, MLP_IN, 1, g1, s);
    if (rc) return rc;
    GemmArgs g2 = {};
    g2.epi = EPI_HEAD;
    g2.bias = net->b2;
    g2.w3 = net->w3;
    g2.b3 = net->b3;
    g2.y = y;
    g2.status = net->status;
    return gemm(w.h1, rows, MLP_H, net->w2h, MLP_H, MLP_H, MLP_H, 1, g2, s);
}

extern "C" int epsr_mlp_train_step(const epsr_mlp_t *net, const void *x, const void *xt, int64_t ldxt, int32_t row0,
                                   int32_t rows, const float *target, float lr, int32_t step, float *loss_out,
                                   void *work, int64_t work_bytes, void *stream) {
    int rc = check_net(net, "epsr_mlp_train_step");
    if (rc) return rc;
    if (!x || !xt || !target || !work || rows <= 0 || rows % 128 || row0 % 128 || ldxt < row0 + rows || step < 1 ||
        !net->dw1 || !net->m1 || !net->v1) {
        epsr_set_error("epsr_mlp_train_step: null pointer, or rows/row0 not multiples of 128, or ldxt too small");
        return EPSR_ERR_ARG;
    }
    if (work_bytes < epsr_mlp_work_bytes(rows)) {
        epsr_set_error("epsr_mlp_train_step: work needs %lld bytes", (long long)epsr_mlp_work_bytes(rows));
        return EPSR_ERR_CAPACITY;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int R = rows;
    MlpWork w = carve(work, R);
    const bf16 *xr = (const bf16 *)x + (size_t)row0 * MLP_IN;
    EPSR_CUDA(cudaMemsetAsync(w.loss, 0, sizeof(float), s));
    // forward, layer 1: z1 and h1 (row-major for layer 2, transposed for dW2)
    GemmArgs g1 = {};
    g1.epi = EPI_BIAS_SILU;
    g1.bias = net->b1;
    g1.z_out = w.z1;
    g1.h_out = w.h1;
    g1.ht_out = w.h1t;
    g1.ldt = R;
    g1.status = net->status;
    rc = gemm(xr, R, MLP_IN, net->w1h, MLP_H, MLP_IN, MLP_IN, 1, g1, s);
    if (rc) return rc;
    // forward, layer 2 + head + loss gradient: dz2 (row-major and transposed), dw3, db3, db2
    GemmArgs g2 = {};
    g2.epi = EPI_HEAD;
    g2.bias = net->b2;
    g2.w3 = net->w3;
    g2.b3 = net->b3;
    g2.y = w.y;
    g2.target = target + row0 / 2;
    g2.gscale = 1.0f / (float)(R / 2);
    g2.loss = w.loss;
    g2.dw3 = net->dw3;
    g2.db3 = net->db3;
    g2.db = net->db2;
    g2.dz_out = w.dz2;
    g2.dzt_out = w.dz2t;
    g2.ldt = R;
    g2.status = net->status;
    rc = gemm(w.h1, R, MLP_H, net->w2h, MLP_H, MLP_H, MLP_H, 1, g2, s);
    if (rc) return rc;
    // backward through layer 2: dh1 = dz2 . W2 (B = W2^T rows), dz1 = dh1 silu'(z1) transposed, db1
    GemmArgs g3 = {};
    g3.epi = EPI_SILU_BWD;
    g3.z_in = w.z1;
    g3.dzt_out = w.dz1t;
    g3.ldt = R;
    g3.db = net->db1;
    g3.status = net->status;
    rc = gemm(w.dz2, R, MLP_H, net->w2th, MLP_H, MLP_H, MLP_H, 1, g3, s);
    if (rc) return rc;
    // weight gradients over the R samples: dW1 = dz1^T x (x^T rows are features), dW2 = dz2^T h1
    const int ks = R / 128 < 8 ? R / 128 : 8;
    GemmArgs g4 = {};
    g4.epi = EPI_ATOMIC;
    g4.out = net->dw1;
    g4.ldo = MLP_IN;
    g4.status = net->status;
    // B = x^T restricted to the batch's columns: rows = features, K = samples from row0
    rc = gemm(w.dz1t, MLP_H, R, (const bf16 *)xt + row0, MLP_IN, ldxt, R, ks, g4, s);
    if (rc) return rc;
    GemmArgs g5 = {};
    g5.epi = EPI_ATOMIC;
    g5.out = net->dw2;
    g5.ldo = MLP_H;
    g5.status = net->status;
    rc = gemm(w.dz2t, MLP_H, R, w.h1t, MLP_H, R, R, ks, g5, s);
    if (rc) return rc;
    // Adam (bias-corrected), then the BF16 copies the next forward reads
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f / (1.0f - powf(b1, (float)step)), c2 = 1.0f / (1.0f - powf(b2, (float)step));
    struct P {
        float *w, *gr, *m, *v;
        bf16 *wh, *wht;
        int n, rows, cols;
    } ps[6] = {
        {net->w1, net->dw1, net->m1, net->v1, (bf16 *)net->w1h, nullptr, MLP_H * MLP_IN, MLP_H, MLP_IN},
        {net->b1, net->db1, net->m1 + MLP_H * MLP_IN, net->v1 + MLP_H * MLP_IN, nullptr, nullptr, MLP_H, 1, MLP_H},
        {net->w2, net->dw2, net->m1 + MLP_H * MLP_IN + MLP_H, net->v1 + MLP_H * MLP_IN + MLP_H, (bf16 *)net->w2h,
         (bf16 *)net->w2th,
         MLP_H * MLP_H, MLP_H, MLP_H},
        {net->b2, net->db2, net->m1 + MLP_H * MLP_IN + MLP_H + MLP_H * MLP_H,
         net->v1 + MLP_H * MLP_IN + MLP_H + MLP_H * MLP_H, nullptr, nullptr, MLP_H, 1, MLP_H},
        {net->w3, net->dw3, net->m1 + MLP_H * MLP_IN + 2 * MLP_H + MLP_H * MLP_H,
         net->v1 + MLP_H * MLP_IN + 2 * MLP_H + MLP_H * MLP_H, nullptr, nullptr, MLP_H, 1, MLP_H},
        {net->b3, net->db3, net->m1 + MLP_H * MLP_IN + 3 * MLP_H + MLP_H * MLP_H,
         net->v1 + MLP_H * MLP_IN + 3 * MLP_H + MLP_H * MLP_H, nullptr, nullptr, 1, 1, 1},
    };
    for (auto &p : ps) {
        AdamArgs a = {p.w, p.gr, p.m, p.v, p.wh, p.wht, p.n, p.rows, p.cols, lr, b1, b2, 1e-8f, c1, c2, 0.0f};
        adam_kernel<<<(p.n + 255) / 256, 256, 0, s>>>(a);
    }
    EPSR_CUDA(cudaGetLastError());
    if (loss_out) EPSR_CUDA(cudaMemcpyAsync(loss_out, w.loss, sizeof(float), cudaMemcpyDeviceToDevice, s));
    return EPSR_OK;
}
