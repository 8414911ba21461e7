// batch.cu -- many independent boxes advanced together by a parallel (checkerboard) Metropolis
// scheme, with an optional delayed-acceptance first stage from the surrogate network.
//
// Scheme.  Each sweep every box draws a random shift of its grid of ncell^3 cells and a random
// colour order; its centres are binned (counting sort, members of a cell in molecule order).
// Step t moves, in every box, one randomly chosen molecule of every cell of colour
// (colour_off + t) mod stride^3.  Cells of one colour are (stride - 1) cells apart, at least the
// interaction range, and a move that would take a centre out of its cell is rejected, so the
// moves of one step never see each other: they are exact single-molecule Metropolis moves made
// in parallel.  The proposal (rotation about a uniformly random axis by an angle uniform in
// [-rotmax, rotmax], translation uniform in the cube) is symmetric.
//
// Kernels per step: propose (one CTA per slot: the molecule, the proposal, and with the
// surrogate the radial histograms of the moved molecule before and after the move, written as
// two rows of BF16 features), the network (mlp.cu) when delayed acceptance is on, and decide
// (one CTA per slot: the first-stage test on the network's antisymmetric output, then the
// exact energy change over the partners within rint -- table lookups of molfit.py:1251-1279 --
// and the Metropolis test of molfit.py:401-408 on beta*dE - s, and the commit).  A CTA whose
// move fails the first stage returns before any pair energy: that is the work the surrogate
// saves.  All random numbers come from Philox4x32-10 counted by (sweep, step, slot).
#include <cuda_bf16.h>

#include "common.cuh"
#include "philox.cuh"

namespace epsr {

constexpr int BMC_THREADS = 256;
constexpr int BMC_MAXAT = 64;
constexpr int BMC_LIST = 6144;            // partner molecules scanned per move
constexpr int FEAT_BINS = 64, FEAT_CLASSES = 10, FEAT_HALF = FEAT_BINS * FEAT_CLASSES, FEAT_IN = 2 * FEAT_HALF;
constexpr float FEAT_RMAX = 8.0f;         // A
constexpr float FEAT_SCALE = 0.25f;       // count -> feature value
constexpr uint32_t P_BIN = 0xB1u, P_MOVE = 1u, P_DECIDE = 2u;

__device__ __forceinline__ float wrap_c(float c) { return __fsub_rn(c, nint_f(c)); }

__device__ __forceinline__ int cell_coord(float x, float shift, int n) {
    int i = __float2int_rd(__fmul_rn(__fadd_rn(__fadd_rn(x, 0.5f), shift), (float)n));
    i %= n;
    return i < 0 ? i + n : i;
}

__device__ __forceinline__ Tables box_tables(const epsr_bmc_t &B, const epsr_bmc_box_t &X) {
    Tables T;
    T.tab = (const float4 *)B.tab + X.tab0;
    T.xstar = B.xstar + X.xstar0;
    T.ld = X.ld;
    T.npt2 = X.izcut;
    T.izcut = X.izcut;
    T.stepcl = X.stepcl;
    return T;
}

__device__ __forceinline__ int feat_class(int c1, int c2) {
    const int a = c1 < c2 ? c1 : c2, b = c1 < c2 ? c2 : c1;
    return (a * (7 - a)) / 2 + b;   // (0,0)=0 ... (3,3)=9
}

// ----------------------------------------------------------------- binning
__global__ void bmc_begin_kernel(epsr_bmc_t B) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B.nbox) return;
    epsr_bmc_box_t &X = B.box[b];
    const int64_t sw = *B.sweep_counter;
    X.sweep = sw;
    const U4 r = philox4x32(U4{(uint32_t)sw, (uint32_t)(sw >> 32), P_BIN, 0u}, X.key0, X.key1);
    const float a = 1.0f / (float)X.ncell;
    X.shift[0] = u01(r.x) * a;
    X.shift[1] = u01(r.y) * a;
    X.shift[2] = u01(r.z) * a;
    const int ncol = X.stride * X.stride * X.stride;
    X.colour_off = (int)(r.w % (uint32_t)ncol);
    const int nc = X.ncell * X.ncell * X.ncell;
    for (int c = 0; c <= nc; ++c) B.cell_start[X.cell0 + b + c] = 0;
}

__global__ void bmc_count_kernel(epsr_bmc_t B) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= B.nmol) return;
    const int b = B.mol_box[m];
    const epsr_bmc_box_t &X = B.box[b];
    const int n = X.ncell;
    const int c = (cell_coord(B.xadd[m], X.shift[0], n) * n + cell_coord(B.yadd[m], X.shift[1], n)) * n +
                  cell_coord(B.zadd[m], X.shift[2], n);
    B.mol_cell[m] = c;
    atomicAdd(B.cell_start + X.cell0 + b + c + 1, 1);
}

// one CTA per box: inclusive scan of the counts into starts
__global__ void bmc_scan_kernel(epsr_bmc_t B) {
    const epsr_bmc_box_t &X = B.box[blockIdx.x];
    int *st = B.cell_start + X.cell0 + blockIdx.x;
    const int nc = X.ncell * X.ncell * X.ncell;
    __shared__ int carry;
    __shared__ int ws[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 1; base <= nc; base += blockDim.x) {
        const int i = base + threadIdx.x;
        int v = i <= nc ? st[i] : 0;
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += u;
        }
        if (lane == 31) ws[w] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            int a = 0;
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
                const int t = ws[k];
                ws[k] = a;
                a += t;
            }
        }
        __syncthreads();
        if (i <= nc) st[i] = carry + ws[w] + v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += ws[w] + v;
        __syncthreads();
    }
}

__global__ void bmc_scatter_kernel(epsr_bmc_t B, int32_t *cursor) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= B.nmol) return;
    const int b = B.mol_box[m];
    const epsr_bmc_box_t &X = B.box[b];
    const int idx = X.cell0 + b + B.mol_cell[m];
    const int p = atomicAdd(cursor + idx, 1);
    B.cell_mols[X.mol0 + B.cell_start[idx] + p] = m;
}

// members of each cell in ascending molecule order (the scatter's order is not deterministic)
__global__ void bmc_sort_kernel(epsr_bmc_t B, const int32_t *cell_box, int ncell_tot) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;   // packed cell index (without the +b)
    if (g >= ncell_tot) return;
    const int b = cell_box[g];
    const epsr_bmc_box_t &X = B.box[b];
    const int idx = g + b;
    int *mm = B.cell_mols + X.mol0;
    const int s0 = B.cell_start[idx], s1 = B.cell_start[idx + 1];
    for (int i = s0 + 1; i < s1; ++i) {
        const int v = mm[i];
        int j = i - 1;
        while (j >= s0 && mm[j] > v) {
            mm[j + 1] = mm[j];
            --j;
        }
        mm[j + 1] = v;
    }
}

__global__ void bmc_end_kernel(epsr_bmc_t B) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *B.sweep_counter += 1;
}

// ----------------------------------------------------------------- partner lists
// The molecules of the cells within `nr` of cell (ix, iy, iz) (each cell once, wrapped), in
// cell order and ascending molecule order within a cell, into list[]; returns the count (or
// -1 when the list would overflow).
__device__ int gather_partners(const epsr_bmc_t &B, const epsr_bmc_box_t &X, int b, int ix, int iy, int iz, int nr,
                               int *list, int *scan_ws) {
    const int n = X.ncell;
    const int w = 2 * nr + 1 < n ? 2 * nr + 1 : n;
    const int ox = 2 * nr + 1 < n ? ix - nr : 0, oy = 2 * nr + 1 < n ? iy - nr : 0, oz = 2 * nr + 1 < n ? iz - nr : 0;
    const int ncell = w * w * w;
    const int *st = B.cell_start + X.cell0 + b;
    const int *mm = B.cell_mols + X.mol0;
    int total = 0;
    for (int base = 0; base < ncell; base += blockDim.x) {
        const int k = base + threadIdx.x;
        int cnt = 0, s0 = 0;
        if (k < ncell) {
            const int dx = k / (w * w), dy = (k / w) % w, dz = k % w;
            const int cx = ((ox + dx) % n + n) % n, cy = ((oy + dy) % n + n) % n, cz = ((oz + dz) % n + n) % n;
            const int c = (cx * n + cy) * n + cz;
            s0 = st[c];
            cnt = st[c + 1] - s0;
        }
        // block exclusive scan of cnt
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        int v = cnt;
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += u;
        }
        if (lane == 31) scan_ws[wid] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            int a = 0;
            for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
                const int t = scan_ws[q];
                scan_ws[q] = a;
                a += t;
            }
            scan_ws[32] = a;
        }
        __syncthreads();
        const int at = total + scan_ws[wid] + v - cnt;
        for (int q = 0; q < cnt; ++q)
            if (at + q < BMC_LIST) list[at + q] = mm[s0 + q];
        total += scan_ws[32];
        __syncthreads();
    }
    return total <= BMC_LIST ? total : -1;
}

__device__ __forceinline__ float4 atom_pos(const epsr_bmc_t &B, int a) { return ((const float4 *)B.pos)[a]; }

// ----------------------------------------------------------------- propose
__global__ void __launch_bounds__(BMC_THREADS) bmc_propose_kernel(epsr_bmc_t B, int step, __nv_bfloat16 *xfeat) {
    __shared__ int list[BMC_LIST];
    __shared__ int scan_ws[33];
    __shared__ int hist[2 * FEAT_HALF];
    __shared__ float4 p_old[BMC_MAXAT], p_new[BMC_MAXAT];
    __shared__ int s_mol, s_n, s_left, s_ix, s_iy, s_iz;
    const int k = blockIdx.x;
    const int b = B.slot_box[k];
    const epsr_bmc_box_t &X = B.box[b];
    const int j = k - X.slot0;
    const int n = X.ncell, s = X.stride, na = n / s;
    const int ncol = s * s * s;
    const int colour = (X.colour_off + step) % ncol;
    const int cx = colour / (s * s), cy = (colour / s) % s, cz = colour % s;
    const int ix = cx + s * (j / (na * na)), iy = cy + s * ((j / na) % na), iz = cz + s * (j % na);
    const int c = (ix * n + iy) * n + iz;
    if (threadIdx.x == 0) {
        const int *st = B.cell_start + X.cell0 + b;
        const int s0 = st[c], cnt = st[c + 1] - s0;
        int mol = -1, left = 0;
        if (cnt > 0) {
            const U4 r0 = philox4x32(U4{(uint32_t)X.sweep, (uint32_t)step, (uint32_t)k, P_MOVE}, X.key0, X.key1);
            const U4 r1 = philox4x32(U4{(uint32_t)X.sweep, (uint32_t)step, (uint32_t)k, P_MOVE + 16u}, X.key0, X.key1);
            int pick = (int)(u01(r0.x) * (float)cnt);
            pick = pick < cnt ? pick : cnt - 1;
            mol = B.cell_mols[X.mol0 + s0 + pick];
            // rotation: axis from (u1, u2), angle from u3 (Rodrigues, in float)
            const float ct = __fsub_rn(__fmul_rn(2.0f, u01(r0.y)), 1.0f);
            const float st_ = __fsqrt_rn(fmaxf(__fsub_rn(1.0f, __fmul_rn(ct, ct)), 0.0f));
            const float ph = __fmul_rn(6.2831853071795864769f, u01(r0.z));
            const float ax = __fmul_rn(st_, cos_r(ph)), ay = __fmul_rn(st_, sin_r(ph)), az = ct;
            const float al = __fmul_rn(X.rotmax, __fsub_rn(__fmul_rn(2.0f, u01(r0.w)), 1.0f));
            const float ca = cos_r(al), sa = sin_r(al), oc = __fsub_rn(1.0f, ca);
            float ccx = B.xadd[mol], ccy = B.yadd[mol], ccz = B.zadd[mol];
            const float nx = wrap_c(__fadd_rn(ccx, __fmul_rn(X.transmax, __fsub_rn(__fmul_rn(2.0f, u01(r1.x)), 1.0f))));
            const float ny = wrap_c(__fadd_rn(ccy, __fmul_rn(X.transmax, __fsub_rn(__fmul_rn(2.0f, u01(r1.y)), 1.0f))));
            const float nz = wrap_c(__fadd_rn(ccz, __fmul_rn(X.transmax, __fsub_rn(__fmul_rn(2.0f, u01(r1.z)), 1.0f))));
            left = cell_coord(nx, X.shift[0], n) != ix || cell_coord(ny, X.shift[1], n) != iy ||
                   cell_coord(nz, X.shift[2], n) != iz;
            const int a0 = B.naf[mol], na_ = B.nato[mol];
            float4 *so = (float4 *)B.slot_off + (size_t)k * BMC_MAXAT;
            float4 *sn = (float4 *)B.slot_new + (size_t)k * BMC_MAXAT;
            for (int q = 0; q < na_; ++q) {
                const float vx = B.xa[a0 + q], vy = B.ya[a0 + q], vz = B.za[a0 + q];
                // v' = v cos + (n x v) sin + n (n.v)(1 - cos)
                const float dot = __fadd_rn(__fadd_rn(__fmul_rn(ax, vx), __fmul_rn(ay, vy)), __fmul_rn(az, vz));
                const float cxv = __fsub_rn(__fmul_rn(ay, vz), __fmul_rn(az, vy));
                const float cyv = __fsub_rn(__fmul_rn(az, vx), __fmul_rn(ax, vz));
                const float czv = __fsub_rn(__fmul_rn(ax, vy), __fmul_rn(ay, vx));
                const float dd = __fmul_rn(dot, oc);
                const float rx = __fadd_rn(__fadd_rn(__fmul_rn(vx, ca), __fmul_rn(cxv, sa)), __fmul_rn(ax, dd));
                const float ry = __fadd_rn(__fadd_rn(__fmul_rn(vy, ca), __fmul_rn(cyv, sa)), __fmul_rn(ay, dd));
                const float rz = __fadd_rn(__fadd_rn(__fmul_rn(vz, ca), __fmul_rn(czv, sa)), __fmul_rn(az, dd));
                const float4 po = atom_pos(B, a0 + q);
                so[q] = make_float4(rx, ry, rz, 0.0f);
                sn[q] = make_float4(__fadd_rn(rx, nx), __fadd_rn(ry, ny), __fadd_rn(rz, nz), po.w);
                p_old[q] = po;
                p_new[q] = sn[q];
            }
            ((float4 *)B.slot_centre)[k] = make_float4(nx, ny, nz, 0.0f);
            s_n = na_;
        } else {
            s_n = 0;
        }
        B.slot_mol[k] = mol < 0 ? -1 : (left ? -2 : mol);
        s_mol = mol;
        s_left = left;
        s_ix = ix;
        s_iy = iy;
        s_iz = iz;
    }
    __syncthreads();
    if (!xfeat) return;
    __nv_bfloat16 *row0 = xfeat + (size_t)(2 * k) * FEAT_IN, *row1 = row0 + FEAT_IN;
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.0f);
    if (s_mol < 0 || s_left) {   // nothing to screen: zero rows
        for (int i = threadIdx.x; i < FEAT_IN; i += blockDim.x) row0[i] = row1[i] = zero;
        return;
    }
    for (int i = threadIdx.x; i < 2 * FEAT_HALF; i += blockDim.x) hist[i] = 0;
    const int cnt = gather_partners(B, X, b, s_ix, s_iy, s_iz, X.nrange_feat, list, scan_ws);
    if (cnt < 0) {
        if (threadIdx.x == 0) atomicExch(B.status, 2);
        return;
    }
    Lattice L;
    L.cubic = 1;
    const int mol = s_mol, na_ = s_n;
    const float rf = X.rfeat;
    const float binf = (float)FEAT_BINS / FEAT_RMAX * X.dmax;   // bins per box unit
    const float mx = B.xadd[mol], my = B.yadd[mol], mz = B.zadd[mol];
    const float rfc2 = __fmul_rn(X.rfeat_c, X.rfeat_c);
    const float rsq_skip = (float)((double)rf * (double)rf * (1.0 + 1e-5));   // d >= rf beyond it
    // 1. the partners whose centre is within rfeat_c: no atom of a partner beyond it is within
    // 8 A of an atom of the moved molecule, before or after the move (compacted in list order)
    __shared__ int wcnt[BMC_THREADS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    int ncomp = 0;
    for (int c0 = 0; c0 < cnt; c0 += blockDim.x) {
        const int p = c0 + threadIdx.x;
        const int jm = p < cnt ? list[p] : -1;
        bool in = false;
        if (jm >= 0 && jm != mol) {
            float dx = __fsub_rn(B.xadd[jm], mx), dy = __fsub_rn(B.yadd[jm], my), dz = __fsub_rn(B.zadd[jm], mz);
            dx = __fsub_rn(dx, nint_f(dx));
            dy = __fsub_rn(dy, nint_f(dy));
            dz = __fsub_rn(dz, nint_f(dz));
            in = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)) <= rfc2;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, in);
        if (lane == 0) wcnt[wid] = __popc(bal);
        __syncthreads();
        int off = ncomp, tot = 0;
        for (int w = 0; w < nwarp; ++w) {
            if (w < wid) off += wcnt[w];
            tot += wcnt[w];
        }
        if (in) list[off + __popc(bal & ((1u << lane) - 1u))] = jm;
        ncomp += tot;
        __syncthreads();
    }
    // 2. one item per (partner, atom of the moved molecule): its distances to the partner's
    // atoms before and after the move, binned
    const int a00 = B.naf[mol];
    for (int it = threadIdx.x; it < ncomp * na_; it += blockDim.x) {
        const int jm = list[it / na_], a = it - (it / na_) * na_;
        const int b0 = B.naf[jm], nb = B.nato[jm];
        const int ca = B.fclass[a00 + a];
        const float4 po = p_old[a], pn = p_new[a];
        for (int q = 0; q < nb; ++q) {
            const float4 pb = atom_pos(B, b0 + q);
            const int fc = feat_class(ca, B.fclass[b0 + q]) * FEAT_BINS;
            // the square root only for pairs that can be within rf
            float x0 = __fsub_rn(pb.x, po.x), y0 = __fsub_rn(pb.y, po.y), z0 = __fsub_rn(pb.z, po.z);
            float x1 = __fsub_rn(pb.x, pn.x), y1 = __fsub_rn(pb.y, pn.y), z1 = __fsub_rn(pb.z, pn.z);
            minimagec(L, x0, y0, z0);
            minimagec(L, x1, y1, z1);
            const float q0 = __fadd_rn(__fadd_rn(__fmul_rn(x0, x0), __fmul_rn(y0, y0)), __fmul_rn(z0, z0));
            const float q1 = __fadd_rn(__fadd_rn(__fmul_rn(x1, x1), __fmul_rn(y1, y1)), __fmul_rn(z1, z1));
            if (q0 <= rsq_skip) {
                const float d0 = __fsqrt_rn(q0);
                if (d0 < rf) atomicAdd(&hist[fc + min((int)__fmul_rn(d0, binf), FEAT_BINS - 1)], 1);
            }
            if (q1 <= rsq_skip) {
                const float d1 = __fsqrt_rn(q1);
                if (d1 < rf) atomicAdd(&hist[FEAT_HALF + fc + min((int)__fmul_rn(d1, binf), FEAT_BINS - 1)], 1);
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < FEAT_IN; i += blockDim.x) {
        const float a = (float)hist[i] * FEAT_SCALE;
        const float bb = (float)hist[i < FEAT_HALF ? i + FEAT_HALF : i - FEAT_HALF] * FEAT_SCALE;
        row0[i] = __float2bfloat16_rn(a);
        row1[i] = __float2bfloat16_rn(bb);
    }
}

// ----------------------------------------------------------------- decide
__device__ __forceinline__ double block_sum_d(double v, double *ws) {
    v = warp_sum_d(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) ws[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0) {
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += ws[q];
        ws[32] = t;
    }
    __syncthreads();
    return ws[32];
}

__global__ void __launch_bounds__(BMC_THREADS) bmc_decide_kernel(epsr_bmc_t B, int step, int mode, const float *y,
                                                                 float *target) {
    __shared__ int list[BMC_LIST];
    __shared__ int scan_ws[33];
    __shared__ double dws[33];
    __shared__ float4 p_old[BMC_MAXAT], p_new[BMC_MAXAT];
    __shared__ int s_go;
    const int k = blockIdx.x;
    const int mol = B.slot_mol[k];
    const int b = B.slot_box[k];
    const epsr_bmc_box_t &X = B.box[b];
    long long *cnt4 = B.counters + 4 * b;
    const float qnan = __int_as_float(0x7fc00000);
    if (mol == -1) {
        if (target && threadIdx.x == 0) target[k] = qnan;
        return;
    }
    if (mol == -2) {
        if (threadIdx.x == 0) {
            atomicAdd((unsigned long long *)cnt4, 1ull);
            atomicAdd((unsigned long long *)(cnt4 + 3), 1ull);
            if (target) target[k] = qnan;
        }
        return;
    }
    const U4 r = philox4x32(U4{(uint32_t)X.sweep, (uint32_t)step, (uint32_t)k, P_DECIDE}, X.key0, X.key1);
    float sg = 0.0f;
    if (threadIdx.x == 0) {
        int go = 1;
        atomicAdd((unsigned long long *)cnt4, 1ull);
        if (mode == 1) {
            sg = 0.5f * (y[2 * k] - y[2 * k + 1]);
            sg = fminf(fmaxf(sg, -40.0f), 40.0f);
            go = sg <= 0.0f || (double)u01(r.x) < exp(-(double)sg);
        }
        if (go) atomicAdd((unsigned long long *)(cnt4 + 1), 1ull);
        else if (target) target[k] = qnan;
        s_go = go;
    }
    __syncthreads();
    if (!s_go) return;   // first stage rejected: no pair energy is evaluated
    const int a0 = B.naf[mol], na_ = B.nato[mol];
    const float4 *sn = (const float4 *)B.slot_new + (size_t)k * BMC_MAXAT;
    for (int q = threadIdx.x; q < na_; q += blockDim.x) {
        p_old[q] = atom_pos(B, a0 + q);
        p_new[q] = sn[q];
    }
    const int n = X.ncell;
    const int ix = cell_coord(B.xadd[mol], X.shift[0], n), iy = cell_coord(B.yadd[mol], X.shift[1], n),
              iz = cell_coord(B.zadd[mol], X.shift[2], n);
    const int cnt = gather_partners(B, X, b, ix, iy, iz, X.nrange, list, scan_ws);
    if (cnt < 0) {
        if (threadIdx.x == 0) atomicExch(B.status, 2);
        return;
    }
    Lattice L;
    L.cubic = 1;
    const Tables T = box_tables(B, X);
    const float dsq_skip = skip_dsq(T.stepcl, T.izcut);
    const int *pr = B.npairref + X.npairref0;
    const float cx = B.xadd[mol], cy = B.yadd[mol], cz = B.zadd[mol];
    const float rint2 = __fmul_rn(X.rint, X.rint);
    // 1. the partners whose centre is within rint of the old centre (rint covers the cutoff,
    // both molecules' extents and the largest displacement), compacted in list order
    __shared__ int wcnt[BMC_THREADS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    int ncomp = 0;
    for (int c0 = 0; c0 < cnt; c0 += blockDim.x) {
        const int p = c0 + threadIdx.x;
        const int jm = p < cnt ? list[p] : -1;
        bool in = false;
        if (jm >= 0 && jm != mol) {
            float dx = __fsub_rn(B.xadd[jm], cx), dy = __fsub_rn(B.yadd[jm], cy), dz = __fsub_rn(B.zadd[jm], cz);
            dx = __fsub_rn(dx, nint_f(dx));
            dy = __fsub_rn(dy, nint_f(dy));
            dz = __fsub_rn(dz, nint_f(dz));
            in = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)) <= rint2;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, in);
        if (lane == 0) wcnt[wid] = __popc(bal);
        __syncthreads();   // every thread has read its entry of this chunk
        int off = ncomp, tot = 0;
        for (int w = 0; w < nwarp; ++w) {
            if (w < wid) off += wcnt[w];
            tot += wcnt[w];
        }
        if (in) list[off + __popc(bal & ((1u << lane) - 1u))] = jm;   // positions below this chunk's end
        ncomp += tot;
        __syncthreads();
    }
    // 2. one item per (partner, atom of the moved molecule): the partner's atoms against that
    // atom before and after the move, float sums over the partner's atoms, the change in double
    double de = 0.0;
    const int nitems = ncomp * na_;
    for (int it = threadIdx.x; it < nitems; it += blockDim.x) {
        const int jm = list[it / na_], a = it - (it / na_) * na_;
        const int b0 = B.naf[jm], nb = B.nato[jm];
        const int *row = pr + __float_as_int(p_old[a].w) * X.ntype;
        const float4 pn = p_new[a], po = p_old[a];
        float e_new = 0.0f, e_old = 0.0f;
        for (int q = 0; q < nb; ++q) {
            const float4 pb = atom_pos(B, b0 + q);
            const int icref = row[__float_as_int(pb.w)];
            e_new = __fadd_rn(e_new, pair_energy_far(L, T, dsq_skip, pn, pb, icref));
            e_old = __fadd_rn(e_old, pair_energy_far(L, T, dsq_skip, po, pb, icref));
        }
        de += (double)e_new - (double)e_old;
    }
    de = block_sum_d(de, dws);
    if (threadIdx.x == 0) {
        const double x = (double)X.beta * de - (double)sg;
        const int acc = x <= 0.0 || (double)u01(r.y) < exp(-x);
        if (target) target[k] = (float)((double)X.beta * de - (double)sg);   // beta dE (mode 2), beta dE - s (1)
        s_go = acc;
        if (acc) {
            atomicAdd((unsigned long long *)(cnt4 + 2), 1ull);
            atomicAdd(B.energy + b, de);
            const float4 c = ((const float4 *)B.slot_centre)[k];
            B.xadd[mol] = c.x;
            B.yadd[mol] = c.y;
            B.zadd[mol] = c.z;
        }
    }
    __syncthreads();
    if (s_go) {
        const float4 *so = (const float4 *)B.slot_off + (size_t)k * BMC_MAXAT;
        for (int q = threadIdx.x; q < na_; q += blockDim.x) {
            B.xa[a0 + q] = so[q].x;
            B.ya[a0 + q] = so[q].y;
            B.za[a0 + q] = so[q].z;
            ((float4 *)B.pos)[a0 + q] = p_new[q];
        }
    }
}

// ----------------------------------------------------------------- total energy
__global__ void __launch_bounds__(BMC_THREADS) bmc_mol_energy_kernel(epsr_bmc_t B) {
    __shared__ int list[BMC_LIST];
    __shared__ int scan_ws[33];
    __shared__ double dws[33];
    const int mol = blockIdx.x;
    const int b = B.mol_box[mol];
    const epsr_bmc_box_t &X = B.box[b];
    const int n = X.ncell;
    const int ix = cell_coord(B.xadd[mol], X.shift[0], n), iy = cell_coord(B.yadd[mol], X.shift[1], n),
              iz = cell_coord(B.zadd[mol], X.shift[2], n);
    const int cnt = gather_partners(B, X, b, ix, iy, iz, X.nrange, list, scan_ws);
    if (cnt < 0) {
        if (threadIdx.x == 0) atomicExch(B.status, 2);
        return;
    }
    Lattice L;
    L.cubic = 1;
    const Tables T = box_tables(B, X);
    const float dsq_skip = skip_dsq(T.stepcl, T.izcut);
    const int *pr = B.npairref + X.npairref0;
    const int a0 = B.naf[mol], na_ = B.nato[mol];
    double e = 0.0;
    for (int p = threadIdx.x; p < cnt; p += blockDim.x) {
        const int jm = list[p];
        if (jm <= mol) continue;   // each pair once
        const int b0 = B.naf[jm], nb = B.nato[jm];
        float s = 0.0f;
        for (int a = 0; a < na_; ++a) {
            const float4 pa = atom_pos(B, a0 + a);
            const int *row = pr + __float_as_int(pa.w) * X.ntype;
            for (int q = 0; q < nb; ++q) {
                const float4 pb = atom_pos(B, b0 + q);
                s = __fadd_rn(s, pair_energy_far(L, T, dsq_skip, pa, pb, row[__float_as_int(pb.w)]));
            }
        }
        e += (double)s;
    }
    e = block_sum_d(e, dws);
    if (threadIdx.x == 0) B.emol[mol] = e;
}

__global__ void bmc_box_energy_kernel(epsr_bmc_t B) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B.nbox) return;
    const epsr_bmc_box_t &X = B.box[b];
    double e = 0.0;
    for (int m = 0; m < X.nmol; ++m) e += B.emol[X.mol0 + m];
    B.energy[b] = e;
}

// ----------------------------------------------------------------- histograms (atogen, all origins)
__global__ void bmc_hist_intra_kernel(epsr_bmc_t B, epsr_bmc_hist_t H) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= B.nmol) return;
    const int b = B.mol_box[m];
    const epsr_bmc_box_t &X = B.box[b];
    const int a0 = B.naf[m], n = B.nato[m];
    if (n <= 1) return;
    Lattice L;
    L.cubic = 1;
    const int ld = H.ldw[b], npt1 = H.npt1[b];
    unsigned long long *cnt = H.counts + H.hist0[b];
    const int *pr = B.npairref + X.npairref0;
    long long np = 0;
    for (int ia = a0; ia < a0 + n - 1; ++ia) {
        for (int ja = ia + 1; ja < a0 + n; ++ja) {
            const int icref = pr[__float_as_int(((const float4 *)B.pos)[ia].w) * X.ntype +
                                 __float_as_int(((const float4 *)B.pos)[ja].w)];
            const float d = dist_f(L, __fsub_rn(B.xa[ia], B.xa[ja]), __fsub_rn(B.ya[ia], B.ya[ja]),
                                   __fsub_rn(B.za[ia], B.za[ja]));
            const int iz1 = nint_i(__fdiv_rn(d, X.stepcl)) + 2;
            if (iz1 > 1 && iz1 <= npt1) atomicAdd(cnt + (size_t)icref * ld + iz1, 1ull);
            ++np;
        }
    }
    atomicAdd((unsigned long long *)(H.pairs + b), (unsigned long long)np);
}

__global__ void __launch_bounds__(256) bmc_hist_inter_kernel(epsr_bmc_t B, epsr_bmc_hist_t H) {
    extern __shared__ unsigned char sm[];
    const int it = blockIdx.x;
    const int b = H.items[3 * it], t0 = H.items[3 * it + 1], o0 = H.items[3 * it + 2];
    const epsr_bmc_box_t &X = B.box[b];
    const int np = H.npairs[b], ld = H.ldw[b], npt1 = H.npt1[b];
    const int nbins = np * ld;
    unsigned int *hist = (unsigned int *)sm;
    unsigned int *hpot = hist + nbins;
    const size_t tp_off = ((sizeof(unsigned int) * ((size_t)H.max_bins)) + 15) & ~(size_t)15;
    float4 *tp = (float4 *)(sm + tp_off);
    int *tm = (int *)(tp + H.tile);
    const int tn = min(H.tile, X.natom - t0);
    for (int i = threadIdx.x; i < nbins + np; i += blockDim.x) hist[i] = 0;
    const float4 *pos = (const float4 *)B.pos + X.atom0;
    const int *amol = H.atom_mol + X.atom0;
    for (int i = threadIdx.x; i < tn; i += blockDim.x) {
        tp[i] = pos[t0 + i];
        tm[i] = amol[t0 + i];
    }
    __syncthreads();
    Lattice L;
    L.cubic = 1;
    const int o = o0 + threadIdx.x;
    long long npairs_done = 0;
    if (o < X.natom) {
        const float4 p1 = pos[o];
        const int im = amol[o];
        const int *pr = B.npairref + X.npairref0 + __float_as_int(p1.w) * X.ntype;
        const float *rmx = H.rminex + H.pair0[b];
        for (int q = 0; q < tn; ++q) {
            if (tm[q] <= im) continue;
            const float4 p2 = tp[q];
            const int icref = pr[__float_as_int(p2.w)];
            // xx = x1 - x2 (ato_manipulation_rev4.py:3798)
            const float d = dist_f(L, __fsub_rn(p1.x, p2.x), __fsub_rn(p1.y, p2.y), __fsub_rn(p1.z, p2.z));
            const int iz1 = nint_i(__fdiv_rn(d, X.stepcl)) + 2;
            if (iz1 > 1 && iz1 <= npt1) atomicAdd(hist + icref * ld + iz1, 1u);
            if (__fmul_rn(d, X.dmax) < fabsf(rmx[icref])) atomicAdd(hpot + icref, 1u);
            ++npairs_done;
        }
    }
    npairs_done = (long long)warp_sum_d((double)npairs_done);
    if ((threadIdx.x & 31) == 0 && npairs_done) atomicAdd((unsigned long long *)(H.pairs + b),
                                                          (unsigned long long)npairs_done);
    __syncthreads();
    unsigned long long *cnt = H.counts + H.hist0[b];
    for (int i = threadIdx.x; i < nbins; i += blockDim.x)
        if (hist[i]) atomicAdd(cnt + (size_t)nbins + i, (unsigned long long)hist[i]);
    for (int i = threadIdx.x; i < np; i += blockDim.x)
        if (hpot[i]) atomicAdd(cnt + (size_t)2 * nbins + i, (unsigned long long)hpot[i]);
}

// normalisation (:3857-3897) of box blockIdx.y, pair blockIdx.x
__global__ void bmc_hist_norm_kernel(epsr_bmc_t B, epsr_bmc_hist_t H) {
    const int b = blockIdx.y, ic = blockIdx.x;
    const int np = H.npairs[b];
    if (ic >= np) return;
    const epsr_bmc_box_t &X = B.box[b];
    const int ld = H.ldw[b], npt1 = H.npt1[b];
    const int p0 = H.pair0[b], t0 = H.type0[b];
    const int it = H.n1extr[p0 + ic], jt = H.n2extr[p0 + ic];
    const float *cfrac = H.cfrac + t0, *csampled = H.csampled + t0;
    float cprod = __fmul_rn(__fmul_rn(cfrac[it], cfrac[jt]), (float)X.natom);
    float cprod2 = __fmul_rn(csampled[it], cfrac[jt]);
    if (it != jt) {
        cprod = __fmul_rn(cprod, 2.0f);
        cprod2 = __fadd_rn(cprod2, __fmul_rn(csampled[jt], cfrac[it]));
    }
    const unsigned long long *cnt = H.counts + H.hist0[b];
    float *wav = H.wav + H.wav0[b];
    float *w1 = wav + (size_t)ic * ld, *w2 = wav + (size_t)(np + ic) * ld;
    const unsigned long long *c1 = cnt + (size_t)ic * ld, *c2 = cnt + (size_t)(np + ic) * ld;
    for (int iz = 1 + threadIdx.x; iz <= npt1; iz += blockDim.x) {
        const float v1 = (float)(2ull * c1[iz]);
        const float v2 = __fmul_rn((float)c2[iz], 2.0f);
        w1[iz] = cprod > 0.0f ? __fdiv_rn(v1, cprod) : 0.0f;
        w2[iz] = cprod2 > 0.0f ? __fdiv_rn(v2, cprod2) : 0.0f;
    }
    const unsigned long long pc = cnt[(size_t)2 * np * ld + ic];
    if (threadIdx.x == 0) H.potex[p0 + ic] = cprod2 > 0.0f ? __fdiv_rn(__fmul_rn((float)pc, cfrac[jt]), cprod2)
                                                           : (float)pc;
}

}  // namespace epsr

using namespace epsr;

namespace {
int check_bmc(const epsr_bmc_t *b, const char *who) {
    if (!b || !b->box || !b->slot_box || !b->mol_box || !b->naf || !b->nato || !b->fclass || !b->xa || !b->xadd ||
        !b->pos || !b->tab || !b->xstar || !b->npairref || !b->cell_start || !b->cell_mols || !b->mol_cell ||
        !b->slot_mol || !b->slot_new || !b->slot_off || !b->slot_centre || !b->energy || !b->counters ||
        !b->sweep_counter || !b->status || b->nbox <= 0 || b->nmol <= 0 || b->nslot <= 0 ||
        (b->threads != 64 && b->threads != 128 && b->threads != 256)) {
        epsr_set_error("%s: null pointer or empty batch", who);
        return EPSR_ERR_ARG;
    }
    return EPSR_OK;
}
}  // namespace

extern "C" int epsr_bmc_begin_sweep(const epsr_bmc_t *b, void *stream) {
    int rc = check_bmc(b, "epsr_bmc_begin_sweep");
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    // the cursor and the cell -> box map live after the molecule-cell array in mol_cell's
    // allocation: mol_cell [nmol], cursor [ncell + nbox], cell_box [ncell]
    int32_t *cursor = b->mol_cell + b->nmol;
    const int32_t *cell_box = cursor + b->ncell + b->nbox;
    bmc_begin_kernel<<<(b->nbox + 127) / 128, 128, 0, s>>>(*b);
    EPSR_CUDA(cudaMemsetAsync(cursor, 0, sizeof(int32_t) * (size_t)(b->ncell + b->nbox), s));
    bmc_count_kernel<<<(b->nmol + 255) / 256, 256, 0, s>>>(*b);
    bmc_scan_kernel<<<b->nbox, 1024, 0, s>>>(*b);
    bmc_scatter_kernel<<<(b->nmol + 255) / 256, 256, 0, s>>>(*b, cursor);
    bmc_sort_kernel<<<(b->ncell + 255) / 256, 256, 0, s>>>(*b, cell_box, b->ncell);
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}

extern "C" int epsr_bmc_propose(const epsr_bmc_t *b, int32_t step, void *x, void *stream) {
    int rc = check_bmc(b, "epsr_bmc_propose");
    if (rc) return rc;
    if (step < 0) {
        epsr_set_error("epsr_bmc_propose: negative step");
        return EPSR_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    EPSR_TIMED("bmc_propose_kernel", s,
               bmc_propose_kernel<<<b->nslot, b->threads, 0, s>>>(*b, step, (__nv_bfloat16 *)x));
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}

extern "C" int epsr_bmc_decide(const epsr_bmc_t *b, int32_t step, int32_t mode, const float *y, float *target,
                               void *stream) {
    int rc = check_bmc(b, "epsr_bmc_decide");
    if (rc) return rc;
    if (mode < 0 || mode > 2 || (mode == 1 && !y) || (mode == 2 && !target)) {
        epsr_set_error("epsr_bmc_decide: mode %d needs %s", mode, mode == 1 ? "y" : "target");
        return EPSR_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    EPSR_TIMED("bmc_decide_kernel", s,
               bmc_decide_kernel<<<b->nslot, b->threads, 0, s>>>(*b, step, mode, y, target));
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}

extern "C" int epsr_bmc_end_sweep(const epsr_bmc_t *b, void *stream) {
    int rc = check_bmc(b, "epsr_bmc_end_sweep");
    if (rc) return rc;
    bmc_end_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(*b);
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}

extern "C" int epsr_bmc_total_energy(const epsr_bmc_t *b, void *stream) {
    int rc = check_bmc(b, "epsr_bmc_total_energy");
    if (rc) return rc;
    if (!b->emol) {
        epsr_set_error("epsr_bmc_total_energy: emol scratch missing");
        return EPSR_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    bmc_mol_energy_kernel<<<b->nmol, BMC_THREADS, 0, s>>>(*b);
    bmc_box_energy_kernel<<<(b->nbox + 127) / 128, 128, 0, s>>>(*b);
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}

extern "C" int epsr_bmc_histograms(const epsr_bmc_t *b, const epsr_bmc_hist_t *h, int64_t counts_len, void *stream) {
    int rc = check_bmc(b, "epsr_bmc_histograms");
    if (rc) return rc;
    if (!h || !h->items || !h->hist0 || !h->wav0 || !h->npairs || !h->npt1 || !h->ldw || !h->pair0 || !h->type0 ||
        !h->n1extr || !h->n2extr || !h->atom_mol || !h->rminex || !h->cfrac || !h->csampled || !h->counts || !h->wav ||
        !h->potex || !h->pairs || h->nitems <= 0 || h->tile <= 0 || h->tile > 4096 || h->max_bins <= 0 ||
        counts_len <= 0) {
        epsr_set_error("epsr_bmc_histograms: null pointer or bad sizes");
        return EPSR_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const size_t shm = (((sizeof(unsigned int) * (size_t)h->max_bins) + 15) & ~(size_t)15) +
                       (sizeof(float4) + sizeof(int)) * (size_t)h->tile;
    if (shm > 220 * 1024) {
        epsr_set_error("epsr_bmc_histograms: %zu bytes of shared histogram and tile", shm);
        return EPSR_ERR_UNSUPPORTED;
    }
    if (shm > 48 * 1024) EPSR_SMEM_OPTIN(bmc_hist_inter_kernel);
    EPSR_CUDA(cudaMemsetAsync(h->counts, 0, sizeof(unsigned long long) * (size_t)counts_len, s));
    EPSR_CUDA(cudaMemsetAsync(h->pairs, 0, sizeof(long long) * (size_t)b->nbox, s));
    bmc_hist_intra_kernel<<<(b->nmol + 127) / 128, 128, 0, s>>>(*b, *h);
    EPSR_TIMED("bmc_hist_inter_kernel", s, bmc_hist_inter_kernel<<<h->nitems, 256, shm, s>>>(*b, *h));
    bmc_hist_norm_kernel<<<dim3(64, b->nbox), 256, 0, s>>>(*b, *h);
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}
