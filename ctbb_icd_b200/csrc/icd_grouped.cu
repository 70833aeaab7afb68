// Grouped ICD: many voxel updates in flight, FP32 error sinogram.
//
// Same per-voxel update as icd_iteration.cpp:198-249 (surrogate numerator
// beta = sum a e and denominator alpha = sum a^2 over the column's in-range
// entries, the reference penalty, the positivity clamp, then e -= delta a),
// but instead of one voxel at a time a persistent kernel drains a device work
// queue of (voxel column, slice) items, one warp per item:
//
//   * warp-level dot product: lanes stride the column's SSM entries of the
//     slice's view window (contiguous thanks to the per-view offsets), gather
//     e through L2 (ld.global.cg; other SMs are updating it), accumulate in
//     FP32, reduce with shuffles;
//   * penalty: lanes 0-7 hold the 8 in-plane neighbours; the quadratic
//     update is closed form, the edge-preserving update solves the same
//     surrogate equation as penalties.cpp:88-154 by safeguarded Newton on the
//     reference's bisection bracket;
//   * scatter: e -= delta a with fire-and-forget L2 reductions (red.global.add).
//
// Visiting order (the "groups"): voxels are enumerated lattice by lattice.
// A lattice is every P-th column in x and y at offset (a, b) and every Q-th
// slice at residue r; lattice offsets are visited in a scrambled order. The
// items in flight at any moment (about `warps_in_flight` of them) are
// consecutive in this order, so they are P columns apart in-plane and Q slices
// apart in z: their footprints overlap only where two voxels are collinear
// with the source, and never through the penalty neighbourhood. Footprints of
// a whole lattice are not disjoint (any two voxels of one slice share rays at
// the views where they line up with the source), so updates of one lattice
// meet in the red.global.add scatter rather than being ordered.
//
// The warp count in flight bounds how stale a gather can be: with W warps
// and a voxel footprint crossing ~T voxels per ray, about T*W/N voxels of a
// ray change concurrently; the default keeps that near 0.4.
#include <math.h>

#include <algorithm>

#include "gpu_internal.h"

namespace {

struct GParams {
    int nx, ny, nz, nch, nr, nvsm, readings, penalty;
    int P, Q, mx, my, kq, n_offsets, stride, pstride;
    uint64_t n_items, per_offset, per_residue, nvsm1;
    float lambda, delta;
    double relax;  // step scale applied to the exact 1-D update before the positivity clamp
    double cvx, cvy, vx, vy, fov_limit;
};

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum over lanes 0..7 of a value held per neighbour (other lanes hold 0).
__device__ __forceinline__ double sum8(double v) {
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    v += __shfl_xor_sync(0xffffffffu, v, 2);
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    return __shfl_sync(0xffffffffu, v, 0);
}

template <class WT>
__device__ __forceinline__ float ldw(const WT* w, int64_t m);
template <>
__device__ __forceinline__ float ldw<float>(const float* w, int64_t m) {
    return __ldg(w + m);
}
template <>
__device__ __forceinline__ float ldw<__half>(const __half* w, int64_t m) {
    return __half2float(__ldg(w + m));
}

template <class WT>
__global__ void __launch_bounds__(256) icd_grouped_kernel(GParams P, const int64_t* __restrict__ colptr,
                                                          const uint32_t* __restrict__ vptr,
                                                          const int32_t* __restrict__ idx,
                                                          const WT* __restrict__ w, const int32_t* __restrict__ start,
                                                          float* e, float* x, unsigned long long* queue) {
    const int lane = threadIdx.x & 31;
    const double r2 = 1.0 / 1.41421356237309504880168872420969807;
    // Neighbour offsets and weights of penalties.cpp:41-52 / 67-74 (lanes 0..7).
    const int64_t nx = P.nx;
    int64_t noff = 0;
    double nw = 0.0;
    if (lane < 8) {
        const int64_t offs[8] = {-nx - 1, -nx, -nx + 1, -1, 1, nx - 1, nx, nx + 1};
        noff = offs[lane];
        nw = (lane == 1 || lane == 3 || lane == 4 || lane == 6) ? 1.0 : r2;
    }
    const double ws = 4.0 + 4.0 * r2;  // all 8 weights (the quadratic denominator always uses them)
    const int64_t nvox = (int64_t)P.nx * P.ny * P.nz;
    const uint64_t ncol = (uint64_t)P.nx * P.ny;

    for (;;) {
        unsigned long long item = 0;
        if (lane == 0) item = atomicAdd(queue, 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= P.n_items) break;
        // Decode the visiting order: offset, slice residue, lattice point, slice.
        const int o = (int)(item / P.per_offset);
        uint64_t rem = item % P.per_offset;
        const int r = (int)(rem / P.per_residue);
        rem %= P.per_residue;
        const int pt = (int)(rem / P.kq);
        const int kk = (int)(rem % P.kq);
        const int os = (int)(((uint64_t)o * P.stride) % P.n_offsets);
        // Golden-ratio stride over the lattice points spreads consecutive
        // items (and hence the items in flight) over the whole slice.
        const int ps = (int)(((uint64_t)pt * P.pstride) % (uint64_t)(P.mx * P.my));
        const int i = os % P.P + P.P * (ps % P.mx);
        const int j = os / P.P + P.P * (ps / P.mx);
        const int k = r + P.Q * kk;
        if (i >= P.nx || j >= P.ny || k >= P.nz) continue;
        const double xx = (i - P.cvx) * P.vx, yy = (j - P.cvy) * P.vy;
        if (!(xx * xx + yy * yy < P.fov_limit)) continue;
        const uint64_t col = (uint64_t)i + (uint64_t)P.nx * j;
        const int64_t q = (int64_t)col + (int64_t)ncol * k;
        const int s = start[k];
        const int v0 = max(0, -s), v1 = min(P.nvsm, P.readings - s);
        int64_t b = 0, en = 0;
        if (v1 > v0) {
            const int64_t cb = colptr[col];
            b = cb + vptr[col * P.nvsm1 + v0];
            en = cb + vptr[col * P.nvsm1 + v1];
        }
        const int off = s * P.nch * P.nr;

        // beta = sum a e, alpha = sum a^2 (FP32 accumulation per lane).
        float acc_b = 0.f, acc_a = 0.f;
        int64_t m = b + lane;
        constexpr int U = 8;
        for (; m + 32 * (U - 1) < en; m += 32 * U) {
            int qi[U];
            float wi[U], ev[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                qi[u] = __ldg(idx + m + 32 * u) + off;
                wi[u] = ldw(w, m + 32 * u);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) ev[u] = __ldcg(e + qi[u]);
#pragma unroll
            for (int u = 0; u < U; ++u) {
                acc_b = fmaf(wi[u], ev[u], acc_b);
                acc_a = fmaf(wi[u], wi[u], acc_a);
            }
        }
        for (; m < en; m += 32) {
            const float wv = ldw(w, m);
            acc_b = fmaf(wv, __ldcg(e + __ldg(idx + m) + off), acc_b);
            acc_a = fmaf(wv, wv, acc_a);
        }
        const double beta = (double)warp_sum(acc_b);
        const double alpha = (double)warp_sum(acc_a);

        // Neighbour differences x_n - x_q (lanes 0..7; weight 0 when outside).
        const double xq = (double)__ldcg(x + q);
        double diff = 0.0, wn = 0.0;
        if (lane < 8) {
            const int64_t n = q + noff;
            if (n >= 0 && n < nvox) {
                diff = (double)__ldcg(x + n) - xq;
                wn = nw;
            }
        }
        double upd;
        if (P.penalty == CTBB_PENALTY_QUADRATIC) {
            // penalties.cpp:84
            const double sum = sum8(wn * diff);
            upd = (beta + (double)P.lambda * sum) / (alpha + (double)P.lambda * ws);
        } else if (alpha == 0.0) {
            upd = 0.0;  // penalties.cpp:101-102
        } else {
            // Root of f(d) = 2 alpha d - 2 beta + lambda sum w psi(d - diff),
            // psi(t) = t / (delta + |t|), inside the reference's bracket.
            const double lam = (double)P.lambda, del = (double)P.delta;
            double lo = beta / alpha, hi = beta / alpha;
            {
                double dmin = (wn != 0.0) ? diff : lo, dmax = (wn != 0.0) ? diff : hi;
#pragma unroll
                for (int o2 = 1; o2 < 8; o2 <<= 1) {
                    dmin = fmin(dmin, __shfl_xor_sync(0xffffffffu, dmin, o2));
                    dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o2));
                }
                lo = fmin(lo, __shfl_sync(0xffffffffu, dmin, 0));
                hi = fmax(hi, __shfl_sync(0xffffffffu, dmax, 0));
            }
            double c = beta / alpha;
            for (int it = 0; it < 64; ++it) {
                const double t = c - diff;
                const double den = del + fabs(t);
                const double f = 2.0 * alpha * c - 2.0 * beta + lam * sum8(wn * t / den);
                const double fp = 2.0 * alpha + lam * sum8(wn * del / (den * den));
                if (f > 0.0)
                    hi = c;
                else
                    lo = c;
                double cn = c - f / fp;
                if (!(cn > lo && cn < hi)) cn = 0.5 * (lo + hi);
                const bool done = fabs(cn - c) <= 1e-12 * (1e-3 + fabs(c)) || (hi - lo) <= 1e-14;
                c = cn;
                if (done) break;
            }
            upd = c;
        }
        upd *= P.relax;
        if (upd + xq < 0.0) upd = -xq;  // icd_iteration.cpp:233-234
        if (lane == 0) x[q] = (float)(xq + upd);
        const float du = (float)upd;
        if (du != 0.f) {
            for (int64_t mm = b + lane; mm < en; mm += 32)
                atomicAdd(e + (__ldg(idx + mm) + off), -du * ldw(w, mm));
        }
    }
}

// Sum of in-range entries over (column inside the FOV, slice): the unit of
// work of one iteration. One warp per column.
__global__ void __launch_bounds__(256) count_entries_kernel(GParams P, const uint32_t* __restrict__ vptr,
                                                            const int32_t* __restrict__ start,
                                                            unsigned long long* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const uint64_t ncol = (uint64_t)P.nx * P.ny;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t col = warp; col < ncol; col += nwarps) {
        const int i = (int)(col % P.nx), j = (int)(col / P.nx);
        const double xx = (i - P.cvx) * P.vx, yy = (j - P.cvy) * P.vy;
        if (!(xx * xx + yy * yy < P.fov_limit)) continue;
        unsigned long long s = 0;
        for (int k = lane; k < P.nz; k += 32) {
            const int st = start[k];
            const int v0 = max(0, -st), v1 = min(P.nvsm, P.readings - st);
            if (v1 > v0) s += vptr[col * P.nvsm1 + v1] - vptr[col * P.nvsm1 + v0];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) atomicAdd(out, s);
    }
}

GParams make_params(const ctbb_recon* rc, const ctbb_ssm* ssm, const ctbb_icd_opts& o) {
    const ctbb_geom_c& g = rc->geom;
    GParams P;
    P.nx = (int)g.num_voxels_x;
    P.ny = (int)g.num_voxels_y;
    P.nz = (int)g.num_voxels_z;
    P.nch = (int)g.n_channels;
    P.nr = (int)g.Nrows_projection;
    P.nvsm = (int)ssm->nvsm;
    P.nvsm1 = ssm->nvsm + 1;
    P.readings = (int)g.Readings;
    P.penalty = g.penalty;
    P.P = o.lattice > 0 ? o.lattice : (P.nx >= 256 ? 16 : (P.nx >= 64 ? 8 : 4));
    P.P = std::min(P.P, std::max(P.nx, P.ny));
    P.Q = P.nz >= 2 ? 2 : 1;
    P.mx = (P.nx + P.P - 1) / P.P;
    P.my = (P.ny + P.P - 1) / P.P;
    P.kq = (P.nz + P.Q - 1) / P.Q;
    P.n_offsets = P.P * P.P;
    // Stride coprime with P*P scrambles the order of lattice offsets.
    int stride = P.n_offsets / 2 + 1;
    auto gcd = [](int a, int b) {
        while (b) {
            const int t = a % b;
            a = b;
            b = t;
        }
        return a;
    };
    while (gcd(stride, P.n_offsets) != 1) ++stride;
    P.stride = stride;
    const int npts = P.mx * P.my;
    int ps = std::max(1, (int)(0.6180339887 * npts));
    while (npts > 1 && gcd(ps, npts) != 1) ++ps;
    P.pstride = ps;
    P.per_residue = (uint64_t)P.mx * P.my * P.kq;
    P.per_offset = P.per_residue * P.Q;
    P.n_items = P.per_offset * P.n_offsets;
    P.lambda = (float)g.lambda;
    P.delta = (float)g.delta;
    P.relax = (o.relax > 0.0 && o.relax < 2.0) ? o.relax : 1.0;
    P.cvx = g.center_voxel_x;
    P.cvy = g.center_voxel_y;
    P.vx = g.voxel_size_x;
    P.vy = g.voxel_size_y;
    P.fov_limit = (g.acquisition_fov / 2.0) * (g.acquisition_fov / 2.0);

    return P;
}


}  // namespace

namespace ctbb {

ctbb_status inrange_entries(ctbb_recon* rc, const ctbb_ssm* ssm, double* out) {
    if (rc->entries_ssm != ssm) {
        ctbb_icd_opts o{};
        const GParams P = make_params(rc, ssm, o);
        ctbb_ctx* ctx = rc->ctx;
        unsigned long long* d = ctx->d_queue + 1;
        CTBB_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned long long), ctx->stream));
        count_entries_kernel<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(P, ssm->d_vptr, rc->d_start, d);
        CTBB_CUDA(cudaGetLastError());
        unsigned long long h = 0;
        CTBB_CUDA(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
        CTBB_CUDA(cudaStreamSynchronize(ctx->stream));
        rc->entries = (double)h;
        rc->entries_ssm = ssm;
    }
    *out = rc->entries;
    return CTBB_OK;
}

int default_warps_in_flight(const ctbb_recon* rc) {
    // Keep (voxels crossed per ray) * W / N near 0.4; a ray crosses about
    // 4 * 0.8 * nx voxels (2 in-plane bilinear taps x 2 slices per x step).
    const double n = (double)rc->nvox;
    const double per_ray = 3.2 * (double)rc->geom.num_voxels_x;
    int w = (int)(0.4 * n / per_ray);
    const int lo = 4, hi = rc->ctx->sm_count * 32;
    return std::max(lo, std::min(hi, w));
}

ctbb_status launch_icd_grouped(ctbb_recon* rc, const ctbb_ssm* ssm, const ctbb_icd_opts& o, float* ms,
                               double* entries) {
    const GParams P = make_params(rc, ssm, o);
    if (entries) CTBB_TRY(inrange_entries(rc, ssm, entries));
    const int W = o.warps_in_flight > 0 ? o.warps_in_flight : default_warps_in_flight(rc);
    const int blocks = std::max(1, (W + 7) / 8);
    ctbb_ctx* ctx = rc->ctx;
    cudaStream_t st = ctx->stream;
    CTBB_CUDA(cudaMemsetAsync(ctx->d_queue, 0, sizeof(unsigned long long), st));
    cudaEvent_t e0, e1;
    CTBB_CUDA(cudaEventCreate(&e0));
    CTBB_CUDA(cudaEventCreate(&e1));
    CTBB_CUDA(cudaEventRecord(e0, st));
    const int wsel = o.weights ? o.weights : CTBB_SSM_FP32;
    if (wsel == CTBB_SSM_FP16)
        icd_grouped_kernel<__half><<<blocks, 256, 0, st>>>(P, ssm->d_colptr, ssm->d_vptr, ssm->d_idx, ssm->d_w16,
                                                           rc->d_start, rc->d_e32, rc->d_x32, ctx->d_queue);
    else
        icd_grouped_kernel<float><<<blocks, 256, 0, st>>>(P, ssm->d_colptr, ssm->d_vptr, ssm->d_idx, ssm->d_w32,
                                                          rc->d_start, rc->d_e32, rc->d_x32, ctx->d_queue);
    CTBB_CUDA(cudaGetLastError());
    CTBB_CUDA(cudaEventRecord(e1, st));
    CTBB_CUDA(cudaEventSynchronize(e1));
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return CTBB_OK;
}

}  // namespace ctbb
