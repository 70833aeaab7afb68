// Sequential-order ICD (parity mode).
//
// Reproduces icd_iteration.cpp:149-274: voxels visited y-outer, x, z-inner;
// for each voxel alpha = sum a^2 and beta = sum a (y - y_hat) over the
// in-range entries of its column (:198-212), the penalty update
// (penalties.cpp:61-139), the positivity clamp (:233-234), x += delta and
// y_hat += delta * a (:240-249). The image and y_hat are FP64, weights and
// raw data FP32, products formed with the reference's float/double mixing.
//
// One 1024-thread block walks the voxels in order (each update depends on
// the previous one). The block splits a column's entries across threads,
// reduces alpha/beta in FP64, one warp evaluates the penalty exactly as the
// reference does (bisection included), and the block scatters the update. Only the summation order of alpha/beta differs from the
// reference's OpenMP reduction. Compiled with -fmad=false.
#include "gpu_internal.h"

namespace {

struct SeqParams {
    int nx, ny, nz, nch, nr, nvsm, readings, penalty;
    uint64_t nvsm1;
    double cvx, cvy, vx, vy, fov_limit, lambda, delta;
};

__device__ __forceinline__ double W8(int i) {
    const double r2 = 1.0 / 1.41421356237309504880168872420969807;  // penalties.cpp:15, :33-40
    return (i == 1 || i == 3 || i == 4 || i == 6) ? 1.0 : r2;
}

__device__ __forceinline__ void neighbours(int q, size_t nx, size_t nb[8]) {
    // size_t arithmetic: indices below zero wrap and fail `< array_size`.
    nb[0] = q - nx - 1;
    nb[1] = q - nx;
    nb[2] = q - nx + 1;
    nb[3] = q - 1;
    nb[4] = q + 1;
    nb[5] = q + nx - 1;
    nb[6] = q + nx;
    nb[7] = q + nx + 1;
}

// penalties.cpp:61-85
__device__ double quadratic_update(int q, double alpha, double beta, double lambda, size_t nx, size_t nvox,
                                   const double* x) {
    size_t nb[8];
    neighbours(q, nx, nb);
    double sum = 0.0;
    for (int i = 0; i < 8; ++i)
        if (nb[i] < nvox) sum += W8(i) * (x[nb[i]] - x[q]);
    double ws = 0.0;
    for (int i = 0; i < 8; ++i) ws += W8(i);
    return (beta + lambda * sum) / (alpha + lambda * ws);
}

// penalties.cpp:88-154 (bisection on func) evaluated by one warp: lanes 0-7
// compute the eight neighbour terms of func in parallel and every lane then
// adds them in the order i = 0..7, so each f(d) (and hence the bisection
// path) is bit-identical to the serial evaluation. f(a) is a pure function of
// a, so it is carried along instead of being re-evaluated each step.
__device__ double edge_update_warp(int q, double alpha, double beta, double lambda, double delta, size_t nx,
                                   size_t nvox, const double* x) {
    const int lane = threadIdx.x & 31;
    size_t nb[8];
    neighbours(q, nx, nb);
    if (alpha == 0.0) return 0.0;
    const double xq = x[q];
    double xn = 0.0, wl = 0.0;
    bool valid = false;
    if (lane < 8) {
        size_t n = nb[0];
#pragma unroll
        for (int i = 1; i < 8; ++i)
            if (lane == i) n = nb[i];
        valid = n < nvox;
        if (valid) xn = x[n];
        wl = W8(lane);
    }
    const unsigned vmask = __ballot_sync(0xffffffffu, valid);
    double a = beta / alpha, b = beta / alpha;
    for (int i = 0; i < 8; ++i) {
        const double d = __shfl_sync(0xffffffffu, xn, i) - xq;
        if (vmask & (1u << i)) {
            if (d < a) a = d;
            if (d > b) b = d;
        }
    }
    auto f = [&](double du) {
        double term = 0.0;
        if (valid) {
            const double t = du - (xn - xq);
            const double g = 1.0 - 1.0 / (1.0 + fabs(t / delta));
            term = (t >= 0) ? wl * g : -(wl * g);
        }
        double sum = 0.0;
        for (int i = 0; i < 8; ++i) {
            const double v = __shfl_sync(0xffffffffu, term, i);
            if (vmask & (1u << i)) sum = sum + v;
        }
        return 2 * alpha * du - 2 * beta + lambda * sum;
    };
    double fa = f(a);
    double c = (a + b) / 2.0;
    for (int it = 0; it < 1000000; ++it) {
        c = (a + b) / 2.0;
        const double fc = f(c);
        if (fc == 0 || (b - a) / 2 < 0.00000001) return c;
        const int sc = fc < 0 ? -1 : 1, sa = fa < 0 ? -1 : 1;
        if (sc == sa) {
            a = c;
            fa = fc;
        } else {
            b = c;
        }
    }
    return c;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(1024) icd_seq_kernel(SeqParams P, const int64_t* __restrict__ colptr,
                                                       const uint32_t* __restrict__ vptr,
                                                       const int32_t* __restrict__ idx, const float* __restrict__ w,
                                                       const float* __restrict__ raw, const int32_t* __restrict__ start,
                                                       double* est, double* x) {
    __shared__ double sa[32], sb[32];
    __shared__ double s_upd;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
    const size_t nxs = (size_t)P.nx;
    const size_t nvox = (size_t)P.nx * P.ny * P.nz;
    for (int j = 0; j < P.ny; j++) {
        const double y = (j - P.cvy) * P.vy;
        for (int i = 0; i < P.nx; i++) {
            const double xx = (i - P.cvx) * P.vx;
            if (!((xx * xx + y * y) < P.fov_limit)) continue;  // icd_iteration.cpp:181
            const uint64_t col = (uint64_t)i + nxs * j;
            const int64_t cb = colptr[col];
            for (int k = 0; k < P.nz; k++) {
                const int q = (int)(col + nxs * P.ny * k);
                const int s = start[k];
                const int v0 = max(0, -s), v1 = min(P.nvsm, P.readings - s);
                int64_t b = cb, e = cb;
                if (v1 > v0) {
                    b = cb + vptr[col * P.nvsm1 + v0];
                    e = cb + vptr[col * P.nvsm1 + v1];
                }
                const int off = s * P.nch * P.nr;
                double alpha = 0.0, beta = 0.0;
                for (int64_t m = b + tid; m < e; m += blockDim.x) {
                    const float wm = w[m];
                    const int index = idx[m] + off;
                    const float ww = wm * wm;  // float product (:208)
                    alpha += (double)ww;
                    beta += (double)wm * ((double)raw[index] - est[index]);
                }
                alpha = warp_sum(alpha);
                beta = warp_sum(beta);
                if (lane == 0) {
                    sa[wid] = alpha;
                    sb[wid] = beta;
                }
                __syncthreads();
                if (wid == 0) {
                    double A = 0.0, B = 0.0;
                    for (int t = 0; t < nw; ++t) {
                        A += sa[t];
                        B += sb[t];
                    }
                    double upd;
                    if (P.penalty == CTBB_PENALTY_QUADRATIC) {
                        upd = quadratic_update(q, A, B, P.lambda, nxs, nvox, x);
                    } else {
                        upd = edge_update_warp(q, A, B, P.lambda, P.delta, nxs, nvox, x);
                    }
                    if (lane == 0) {
                        if (upd + x[q] < 0) upd = -x[q];
                        x[q] += upd;
                        s_upd = upd;
                    }
                }
                __syncthreads();
                const double upd = s_upd;
                for (int64_t m = b + tid; m < e; m += blockDim.x) {
                    const int index = idx[m] + off;
                    est[index] += upd * (double)w[m];
                }
                __syncthreads();
            }
        }
    }
}

}  // namespace

namespace ctbb {

ctbb_status launch_icd_sequential(ctbb_recon* rc, const ctbb_ssm* ssm, int n_iter, float* ms) {
    const ctbb_geom_c& g = rc->geom;
    SeqParams P;
    P.nx = (int)g.num_voxels_x;
    P.ny = (int)g.num_voxels_y;
    P.nz = (int)g.num_voxels_z;
    P.nch = (int)g.n_channels;
    P.nr = (int)g.Nrows_projection;
    P.nvsm = (int)ssm->nvsm;
    P.nvsm1 = ssm->nvsm + 1;
    P.readings = (int)g.Readings;
    P.penalty = g.penalty;
    P.cvx = g.center_voxel_x;
    P.cvy = g.center_voxel_y;
    P.vx = g.voxel_size_x;
    P.vy = g.voxel_size_y;
    P.fov_limit = (g.acquisition_fov / 2.0) * (g.acquisition_fov / 2.0);  // icd_iteration.cpp:154
    P.lambda = g.lambda;
    P.delta = g.delta;
    cudaStream_t st = rc->ctx->stream;
    cudaEvent_t e0, e1;
    CTBB_CUDA(cudaEventCreate(&e0));
    CTBB_CUDA(cudaEventCreate(&e1));
    CTBB_CUDA(cudaEventRecord(e0, st));
    for (int it = 0; it < n_iter; ++it)
        icd_seq_kernel<<<1, 1024, 0, st>>>(P, ssm->d_colptr, ssm->d_vptr, ssm->d_idx, ssm->d_w32, rc->d_raw,
                                           rc->d_start, rc->d_est64, rc->d_x64);
    CTBB_CUDA(cudaGetLastError());
    CTBB_CUDA(cudaEventRecord(e1, st));
    CTBB_CUDA(cudaEventSynchronize(e1));
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return CTBB_OK;
}

}  // namespace ctbb
