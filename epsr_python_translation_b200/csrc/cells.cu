// cells.cu -- cell neighbour list (cellneighbourlist.py:23-233) as a counting sort.
//
// Kernels: (1) cell number of every molecule centre (atomcellno :305) with per-cell counts
// by atomics; (2) exclusive scan of the counts; (3) scatter into cell segments; (4) each
// cell's segment sorted by molecule index, which restores the reference's order (molecules
// are appended in index order, :70-74); (5) neighbour-cell offsets (:97-183) tested in the
// reference's float32 order and compacted in its enumeration order.
#include <math.h>

#include <algorithm>

#include "common.cuh"

namespace epsr {

struct LatHost {
    float l6[6];
    float l9[9];
};

__device__ __forceinline__ int cellcoord(float x, int ncelldiv) {
    float x1 = __fsub_rn(x, nint_f(x));
    int ix = ifix(__fmul_rn(__fadd_rn(x1, 0.5f), (float)ncelldiv));
    while (ix < 0) ix += ncelldiv;
    while (ix >= ncelldiv) ix -= ncelldiv;
    return ix;
}

__global__ void cell_assign_kernel(const float *xadd, const float *yadd, const float *zadd, int nmol, LatHost L,
                                   int na, int nb, int nc, int32_t *molcellno, int32_t *count) {
    int im = blockIdx.x * blockDim.x + threadIdx.x;
    if (im >= nmol) return;
    const float alatx = L.l6[0], blatx = L.l6[1], clatx = L.l6[2], blaty = L.l6[3], claty = L.l6[4],
                clatz = L.l6[5];
    float fc = __fdiv_rn(zadd[im], clatz);
    float fb = __fdiv_rn(__fsub_rn(yadd[im], __fmul_rn(fc, claty)), blaty);
    float fa = __fdiv_rn(__fsub_rn(__fsub_rn(xadd[im], __fmul_rn(fb, blatx)), __fmul_rn(fc, clatx)), alatx);
    int ia = cellcoord(fa, na), ib = cellcoord(fb, nb), ic = cellcoord(fc, nc);
    int cell = ia + na * (ib + nb * ic);
    molcellno[im] = cell + 1;
    atomicAdd(count + cell, 1);
}

// Exclusive scan of one value per thread across the block; returns the prefix and writes
// the block total to *total (all threads).  Uses at most 32 warps.
__device__ __forceinline__ int block_exclusive_scan(int v, int *total) {
    __shared__ int wsum[32];
    __shared__ int wpre[33];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int w = 0; w < nw; ++w) {
            wpre[w] = acc;
            acc += wsum[w];
        }
        wpre[32] = acc;
    }
    __syncthreads();
    int r = wpre[wid] + incl - v;
    *total = wpre[32];
    __syncthreads();
    return r;
}

// single-block exclusive scan of count[0..n) into start[0..n], and the maximum count
__global__ void scan_kernel(const int32_t *count, int n, int32_t *start, int32_t *maxc) {
    int carry = 0, mx = 0;
    for (int base = 0; base < n; base += blockDim.x) {
        int i = base + threadIdx.x;
        int v = i < n ? count[i] : 0;
        mx = max(mx, v);
        int tot;
        int pre = block_exclusive_scan(v, &tot);
        if (i < n) start[i] = carry + pre;
        carry += tot;
    }
    if (threadIdx.x == 0) start[n] = carry;
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(maxc, mx);
}

__global__ void cell_scatter_kernel(const int32_t *molcellno, int nmol, const int32_t *start, int32_t *fill,
                                    int32_t *cell_mols) {
    int im = blockIdx.x * blockDim.x + threadIdx.x;
    if (im >= nmol) return;
    int c = molcellno[im] - 1;
    int p = atomicAdd(fill + c, 1);
    cell_mols[start[c] + p] = im;
}

__global__ void cell_sort_kernel(const int32_t *start, int ncell, int32_t *cell_mols) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    int a = start[c], b = start[c + 1];
    for (int i = a + 1; i < b; ++i) {
        int v = cell_mols[i];
        int j = i - 1;
        while (j >= a && cell_mols[j] > v) {
            cell_mols[j + 1] = cell_mols[j];
            --j;
        }
        cell_mols[j + 1] = v;
    }
}

// makecellneighbourlist: candidate offsets in (ic, ib, ia) order, ia fastest.
__global__ void cell_offsets_kernel(int na, int nb, int nc, float rmax, LatHost L, int32_t *offsets,
                                    int32_t *nfound) {
    const float *alatc = L.l9, *blatc = L.l9 + 3, *clatc = L.l9 + 6;
    const float cella = __fdiv_rn(1.0f, (float)na), cellb = __fdiv_rn(1.0f, (float)nb),
                cellc = __fdiv_rn(1.0f, (float)nc);
    const float cella2 = __fmul_rn(0.5f, cella), cellb2 = __fmul_rn(0.5f, cellb), cellc2 = __fmul_rn(0.5f, cellc);
    __shared__ float xc[8], yc[8], zc[8];
    if (threadIdx.x == 0) {
        int f = 0;
        for (int ic = -1; ic <= 1; ic += 2)
            for (int ib = -1; ib <= 1; ib += 2)
                for (int ia = -1; ia <= 1; ia += 2) {
                    float cx = __fmul_rn(__fmul_rn((float)ic, cellc2), clatc[0]);
                    float cy = __fmul_rn(__fmul_rn((float)ic, cellc2), clatc[1]);
                    float cz = __fmul_rn(__fmul_rn((float)ic, cellc2), clatc[2]);
                    float bx = __fmul_rn(__fmul_rn((float)ib, cellb2), blatc[0]);
                    float by = __fmul_rn(__fmul_rn((float)ib, cellb2), blatc[1]);
                    float bz = __fmul_rn(__fmul_rn((float)ib, cellb2), blatc[2]);
                    float ax = __fmul_rn(__fmul_rn((float)ia, cella2), alatc[0]);
                    float ay = __fmul_rn(__fmul_rn((float)ia, cella2), alatc[1]);
                    float az = __fmul_rn(__fmul_rn((float)ia, cella2), alatc[2]);
                    xc[f] = __fadd_rn(__fadd_rn(ax, bx), cx);
                    yc[f] = __fadd_rn(__fadd_rn(ay, by), cy);
                    zc[f] = __fadd_rn(__fadd_rn(az, bz), cz);
                    ++f;
                }
    }
    __syncthreads();
    const int nra = (na - 1) / 2, nrb = (nb - 1) / 2, nrc = (nc - 1) / 2;
    const int wa = 2 * nra + 1, wb = 2 * nrb + 1, wc = 2 * nrc + 1;
    const int total = wa * wb * wc;
    const float rmaxsq = __fmul_rn(rmax, rmax);
    int carry = 0;
    for (int base = 0; base < total; base += blockDim.x) {
        int t = base + threadIdx.x;
        int found = 0, ia = 0, ib = 0, ic = 0;
        if (t < total) {
            ia = t % wa - nra;
            ib = (t / wa) % wb - nrb;
            ic = t / (wa * wb) - nrc;
            float cx = __fmul_rn(__fmul_rn((float)ic, cellc), clatc[0]);
            float cy = __fmul_rn(__fmul_rn((float)ic, cellc), clatc[1]);
            float cz = __fmul_rn(__fmul_rn((float)ic, cellc), clatc[2]);
            float bx = __fmul_rn(__fmul_rn((float)ib, cellb), blatc[0]);
            float by = __fmul_rn(__fmul_rn((float)ib, cellb), blatc[1]);
            float bz = __fmul_rn(__fmul_rn((float)ib, cellb), blatc[2]);
            float ax = __fmul_rn(__fmul_rn((float)ia, cella), alatc[0]);
            float ay = __fmul_rn(__fmul_rn((float)ia, cella), alatc[1]);
            float az = __fmul_rn(__fmul_rn((float)ia, cella), alatc[2]);
            float xdc = __fadd_rn(__fadd_rn(ax, bx), cx);
            float ydc = __fadd_rn(__fadd_rn(ay, by), cy);
            float zdc = __fadd_rn(__fadd_rn(az, bz), cz);
            for (int f1 = 0; f1 < 8 && !found; ++f1)
                for (int f2 = 0; f2 < 8 && !found; ++f2) {
                    float xd = __fsub_rn(__fadd_rn(xdc, xc[f1]), xc[f2]);
                    float yd = __fsub_rn(__fadd_rn(ydc, yc[f1]), yc[f2]);
                    float zd = __fsub_rn(__fadd_rn(zdc, zc[f1]), zc[f2]);
                    float r2 = __fadd_rn(__fadd_rn(__fmul_rn(xd, xd), __fmul_rn(yd, yd)), __fmul_rn(zd, zd));
                    found = (r2 < rmaxsq) || (ia == 0 && ib == 0 && ic == 0);
                }
        }
        int tot;
        int pos = carry + block_exclusive_scan(found, &tot);
        if (found) {
            offsets[3 * pos + 0] = ia;
            offsets[3 * pos + 1] = ib;
            offsets[3 * pos + 2] = ic;
        }
        carry += tot;
    }
    if (threadIdx.x == 0) *nfound = carry;
}

__device__ __forceinline__ int fold(int x, int n) {
    while (x < 0) x += n;
    while (x >= n) x -= n;
    return x;
}

// per-cell neighbour count (get_nnbrefmax) and region start offsets per neighbour cell
__global__ void region_count_kernel(const int32_t *start, const int32_t *offsets, int noff, int na, int nb, int nc,
                                    int32_t *nn_out, int32_t *maxnn) {
    int c0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (c0 >= na * nb * nc) return;
    int icc = c0 / (na * nb);
    int ibb = (c0 - icc * na * nb) / na;
    int iaa = c0 - na * (ibb + nb * icc);
    int n = 0;
    for (int k = 0; k < noff; ++k) {
        int a = fold(iaa + offsets[3 * k], na), b = fold(ibb + offsets[3 * k + 1], nb),
            c = fold(icc + offsets[3 * k + 2], nc);
        int cell = a + na * (b + nb * c);
        n += start[cell + 1] - start[cell];
    }
    if (nn_out) nn_out[c0] = n;
    atomicMax(maxnn, n);
}

// nnbrefmax with the offset count read on the device (no host round trip)
__global__ void region_count_dev_kernel(const int32_t *start, const int32_t *offsets, const int32_t *noff_p, int na,
                                        int nb, int nc, int32_t *maxnn) {
    int c0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (c0 >= na * nb * nc) return;
    const int noff = *noff_p;
    int icc = c0 / (na * nb);
    int ibb = (c0 - icc * na * nb) / na;
    int iaa = c0 - na * (ibb + nb * icc);
    int n = 0;
    for (int k = 0; k < noff; ++k) {
        int a = fold(iaa + offsets[3 * k], na), b = fold(ibb + offsets[3 * k + 1], nb),
            c = fold(icc + offsets[3 * k + 2], nc);
        int cell = a + na * (b + nb * c);
        n += start[cell + 1] - start[cell];
    }
    atomicMax(maxnn, n);
}

}  // namespace epsr

using namespace epsr;

extern "C" int epsr_cell_dims(int32_t nmolcellin, int32_t nmol, const float *lat6, int32_t *dims) {
    if (!lat6 || !dims || nmol <= 0 || nmolcellin <= 0) {
        epsr_set_error("epsr_cell_dims: bad arguments");
        return EPSR_ERR_ARG;
    }
    int nmolcell = nmolcellin > nmol ? nmol : nmolcellin;
    float ratio = (float)nmol / (float)nmolcell;
    // nint(powf(ratio, 1/3)) -- the same glibc powf the reference calls
    float p = powf(ratio, 1.0f / 3.0f);
    double t = trunc((double)p), fr = (double)p - t;
    if (fr >= 0.5) t += 1.0;
    int ncelldiv = (int)t;
    if (ncelldiv < 1) ncelldiv = 1;
    float mn = lat6[0];
    if (lat6[3] < mn) mn = lat6[3];
    if (lat6[5] < mn) mn = lat6[5];
    volatile float two_mn = 2.0f * mn;
    float cellsize = two_mn / (float)ncelldiv;
    volatile float qa = lat6[0] / cellsize, qb = lat6[3] / cellsize, qc = lat6[5] / cellsize;
    dims[0] = 2 * (int)qa + 1;
    dims[1] = 2 * (int)qb + 1;
    dims[2] = 2 * (int)qc + 1;
    dims[3] = dims[0] * dims[1] * dims[2];
    return EPSR_OK;
}

extern "C" int epsr_cell_list(const float *xadd, const float *yadd, const float *zadd, int32_t nmol,
                              int32_t nmolcell, float rmax, const float *lat6, const float *lat9,
                              epsr_cells_t *cells, int32_t *scratch, int64_t scratch_len, void *stream) {
    if (!xadd || !yadd || !zadd || !cells || !lat6 || !lat9 || !scratch) {
        epsr_set_error("epsr_cell_list: null pointer");
        return EPSR_ERR_ARG;
    }
    int32_t dims[4];
    int rc = epsr_cell_dims(nmolcell, nmol, lat6, dims);
    if (rc) return rc;
    const int ncell = dims[3];
    if (scratch_len < 2LL * ncell + 4) {
        epsr_set_error("epsr_cell_list: scratch needs %lld int32, got %lld", 2LL * ncell + 4,
                       (long long)scratch_len);
        return EPSR_ERR_CAPACITY;
    }
    cudaStream_t s = (cudaStream_t)stream;
    LatHost L;
    for (int i = 0; i < 6; ++i) L.l6[i] = lat6[i];
    for (int i = 0; i < 9; ++i) L.l9[i] = lat9[i];
    int32_t *count = scratch, *fill = scratch + ncell, *misc = scratch + 2 * ncell;  // misc: maxc, nfound
    EPSR_CUDA(cudaMemsetAsync(scratch, 0, sizeof(int32_t) * (2 * ncell + 4), s));
    cell_assign_kernel<<<(nmol + 255) / 256, 256, 0, s>>>(xadd, yadd, zadd, nmol, L, dims[0], dims[1], dims[2],
                                                          cells->molcellno, count);
    scan_kernel<<<1, 1024, 0, s>>>(count, ncell, cells->cell_start, misc);
    cell_scatter_kernel<<<(nmol + 255) / 256, 256, 0, s>>>(cells->molcellno, nmol, cells->cell_start, fill,
                                                           cells->cell_mols);
    cell_sort_kernel<<<(ncell + 127) / 128, 128, 0, s>>>(cells->cell_start, ncell, cells->cell_mols);
    cell_offsets_kernel<<<1, 1024, 0, s>>>(dims[0], dims[1], dims[2], rmax, L, cells->offsets, misc + 1);
    region_count_dev_kernel<<<(ncell + 127) / 128, 128, 0, s>>>(cells->cell_start, cells->offsets, misc + 1, dims[0],
                                                                dims[1], dims[2], misc + 2);
    EPSR_CUDA(cudaGetLastError());
    int32_t host[3];
    EPSR_D2H(host, misc, sizeof(host), s);
    cells->ncelldiva = dims[0];
    cells->ncelldivb = dims[1];
    cells->ncelldivc = dims[2];
    cells->ncell = ncell;
    cells->maxcellno = host[0];
    cells->ncellneighb = host[1];
    cells->nnbrefmax = host[2];
    return EPSR_OK;
}

extern "C" int epsr_nnbrefmax(const epsr_cells_t *cells, int32_t *out, int32_t *d, void *stream) {
    if (!cells || !out || !d) {
        epsr_set_error("epsr_nnbrefmax: null pointer");
        return EPSR_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    EPSR_CUDA(cudaMemsetAsync(d, 0, sizeof(int32_t), s));
    region_count_kernel<<<(cells->ncell + 127) / 128, 128, 0, s>>>(cells->cell_start, cells->offsets,
                                                                   cells->ncellneighb, cells->ncelldiva,
                                                                   cells->ncelldivb, cells->ncelldivc, nullptr, d);
    EPSR_D2H(out, d, sizeof(int32_t), s);
    return EPSR_OK;
}
