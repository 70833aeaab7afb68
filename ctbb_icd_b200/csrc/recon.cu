// Device-resident ICD state: raw data, image, error sinogram; FP64 forward
// projection / residual refresh; FP64 cost; the iterate dispatcher and the
// one-call icd_iteration drop-in.
//
// FP64 forward projection: one warp per (voxel column, slice) scatters
// x * a into an FP64 accumulator with native double atomics (the only place
// FP64 atomics appear: the once-every-K-iterations refresh that cancels the
// drift of the FP32 incremental updates, and the setup of y_hat = A x).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "gpu_internal.h"

namespace {

struct FpParams {
    int nx, ny, nz, nch, nr, nvsm, readings;
    uint64_t nvsm1;
};

template <class XT>
__global__ void __launch_bounds__(256) forward_f64_kernel(FpParams P, const int64_t* __restrict__ colptr,
                                                          const uint32_t* __restrict__ vptr,
                                                          const int32_t* __restrict__ idx,
                                                          const float* __restrict__ w32,
                                                          const __half* __restrict__ w16,
                                                          const int32_t* __restrict__ start,
                                                          const XT* __restrict__ x, double* __restrict__ acc) {
    const int lane = threadIdx.x & 31;
    const uint64_t nitems = (uint64_t)P.nx * P.ny * P.nz;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint64_t ncol = (uint64_t)P.nx * P.ny;
    for (uint64_t it = warp; it < nitems; it += nwarps) {
        const uint64_t col = it % ncol;
        const int k = (int)(it / ncol);
        const double xv = (double)x[col + ncol * k];
        if (xv == 0.0) continue;
        const int s = start[k];
        const int v0 = max(0, -s), v1 = min(P.nvsm, P.readings - s);
        if (v1 <= v0) continue;
        const int64_t cb = colptr[col];
        const int64_t b = cb + vptr[col * P.nvsm1 + v0], e = cb + vptr[col * P.nvsm1 + v1];
        const int off = s * P.nch * P.nr;
        for (int64_t m = b + lane; m < e; m += 32) {
            const double w = w32 ? (double)w32[m] : (double)__half2float(w16[m]);
            atomicAdd(acc + (idx[m] + off), xv * w);
        }
    }
}

__global__ void residual_kernel(const float* __restrict__ raw, const double* __restrict__ acc,
                                float* __restrict__ e32, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        e32[i] = (float)((double)raw[i] - acc[i]);
}

__global__ void f64_to_f32_kernel(const double* __restrict__ a, float* __restrict__ b, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

// In-plane 2x bilinear upsampling of a coarse image onto a grid with the same
// field of view and slices and half the voxel size: fine voxel (i, j) sits
// at coarse coordinates (i/2 - 1/4, j/2 - 1/4) (both grids centred, voxel
// centres at (index - (n-1)/2) * size); clamped at the edges.
__global__ void upsample2_kernel(const float* __restrict__ xc, int ncx, int ncy, int nz, float* __restrict__ xf) {
    const int nfx = 2 * ncx, nfy = 2 * ncy;
    const uint64_t n = (uint64_t)nfx * nfy * nz;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
        const int i = (int)(t % nfx), j = (int)((t / nfx) % nfy), k = (int)(t / ((uint64_t)nfx * nfy));
        const float u = fminf(fmaxf(0.5f * i - 0.25f, 0.f), (float)(ncx - 1));
        const float v = fminf(fmaxf(0.5f * j - 0.25f, 0.f), (float)(ncy - 1));
        const int i0 = min((int)u, max(ncx - 2, 0)), j0 = min((int)v, max(ncy - 2, 0));
        const int i1 = min(i0 + 1, ncx - 1), j1 = min(j0 + 1, ncy - 1);
        const float a = u - (float)i0, b = v - (float)j0;
        const float* s = xc + (uint64_t)k * ncx * ncy;
        const float top = (1.f - a) * s[(uint64_t)j0 * ncx + i0] + a * s[(uint64_t)j0 * ncx + i1];
        const float bot = (1.f - a) * s[(uint64_t)j1 * ncx + i0] + a * s[(uint64_t)j1 * ncx + i1];
        xf[t] = (1.f - b) * top + b * bot;
    }
}

__global__ void f32_to_f64_kernel(const float* __restrict__ a, double* __restrict__ b, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        b[i] = (double)a[i];
}

// Block-level FP64 partial sums, reduced on the host in a fixed order.
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += sh[i];
    __syncthreads();
    return t;
}

// sum (raw - acc)^2 (acc may be null: sum e32^2 with e32 passed as raw).
__global__ void __launch_bounds__(256) sq_sum_kernel(const float* __restrict__ a, const double* __restrict__ acc,
                                                     uint64_t n, double* __restrict__ partials) {
    __shared__ double sh[8];
    double s = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const double d = acc ? (double)a[i] - acc[i] : (double)a[i];
        s += d * d;
    }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// Penalty sum over voxels q and their 8 in-plane flat-index neighbours
// (penalties.cpp:41-52, 67-74): quadratic w t^2, edge-preserving
// w (|t| - delta ln(1 + |t|/delta)).
template <class XT>
__global__ void __launch_bounds__(256) penalty_sum_kernel(const XT* __restrict__ x, uint64_t nvox, int64_t nx,
                                                          int penalty, double delta, double* __restrict__ partials) {
    __shared__ double sh[8];
    const double r2 = 1.0 / 1.41421356237309504880168872420969807;  // penalties.cpp:15, :33
    const double W[8] = {r2, 1.0, r2, 1.0, 1.0, r2, 1.0, r2};
    const int64_t off[8] = {-nx - 1, -nx, -nx + 1, -1, 1, nx - 1, nx, nx + 1};
    double s = 0.0;
    for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < nvox; q += (uint64_t)gridDim.x * blockDim.x) {
        const double xq = (double)x[q];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int64_t n = (int64_t)q + off[i];
            if (n < 0 || n >= (int64_t)nvox) continue;
            const double t = xq - (double)x[n];
            if (penalty == CTBB_PENALTY_QUADRATIC) {
                s += W[i] * t * t;
            } else {
                const double at = fabs(t);
                s += W[i] * (at - delta * log1p(at / delta));
            }
        }
    }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

int grid_for(const ctbb_ctx* ctx, uint64_t n, int threads, int per_sm = 16) {
    const uint64_t want = (n + threads - 1) / threads;
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)ctx->sm_count * per_sm));
}

ctbb_status reduce_partials(ctbb_ctx* ctx, int nblocks, double* out) {
    std::vector<double> h(nblocks);
    CTBB_CUDA(cudaMemcpyAsync(h.data(), ctx->d_partials, nblocks * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CTBB_CUDA(cudaStreamSynchronize(ctx->stream));
    double s = 0.0;
    for (int i = 0; i < nblocks; ++i) s += h[i];
    *out = s;
    return CTBB_OK;
}

FpParams fp_params(const ctbb_recon* rc, const ctbb_ssm* ssm) {
    FpParams P;
    P.nx = (int)rc->geom.num_voxels_x;
    P.ny = (int)rc->geom.num_voxels_y;
    P.nz = (int)rc->geom.num_voxels_z;
    P.nch = (int)rc->geom.n_channels;
    P.nr = (int)rc->geom.Nrows_projection;
    P.nvsm = (int)ssm->nvsm;
    P.readings = (int)rc->geom.Readings;
    P.nvsm1 = ssm->nvsm + 1;
    return P;
}

ctbb_status check_pair(const ctbb_recon* rc, const ctbb_ssm* ssm) {
    const ctbb_geom_c &a = rc->geom, &b = ssm->geom;
    if (a.num_voxels_x != b.num_voxels_x || a.num_voxels_y != b.num_voxels_y || a.n_channels != b.n_channels ||
        a.Nrows_projection != b.Nrows_projection || a.num_views_for_system_matrix != b.num_views_for_system_matrix)
        return ctbb::fail(CTBB_ERR_INVALID_ARG, "system matrix geometry does not match the reconstruction");
    if (rc->ctx != ssm->ctx) return ctbb::fail(CTBB_ERR_INVALID_ARG, "matrix and reconstruction use different contexts");
    return CTBB_OK;
}

}  // namespace

namespace ctbb {

ctbb_status forward_project_f64(ctbb_recon* rc, const ctbb_ssm* ssm, bool from_x32, double* d_out) {
    ctbb_ctx* ctx = rc->ctx;
    CTBB_CUDA(cudaMemsetAsync(d_out, 0, rc->data_size * sizeof(double), ctx->stream));
    const FpParams P = fp_params(rc, ssm);
    const uint64_t nitems = rc->nvox;
    const int grid = grid_for(ctx, nitems * 32, 256, 16);
    if (from_x32)
        forward_f64_kernel<float><<<grid, 256, 0, ctx->stream>>>(P, ssm->d_colptr, ssm->d_vptr, ssm->d_idx, ssm->d_w32,
                                                                 ssm->d_w16, rc->d_start, rc->d_x32, d_out);
    else
        forward_f64_kernel<double><<<grid, 256, 0, ctx->stream>>>(P, ssm->d_colptr, ssm->d_vptr, ssm->d_idx,
                                                                  ssm->d_w32, ssm->d_w16, rc->d_start, rc->d_x64, d_out);
    CTBB_CUDA(cudaGetLastError());
    return CTBB_OK;
}

ctbb_status recon_to_grouped(ctbb_recon* rc, const ctbb_ssm* ssm) {
    (void)ssm;
    if (rc->rep == 1) return CTBB_OK;
    ctbb_ctx* ctx = rc->ctx;
    f64_to_f32_kernel<<<grid_for(ctx, rc->nvox, 256), 256, 0, ctx->stream>>>(rc->d_x64, rc->d_x32, rc->nvox);
    residual_kernel<<<grid_for(ctx, rc->data_size, 256), 256, 0, ctx->stream>>>(rc->d_raw, rc->d_est64, rc->d_e32,
                                                                                  rc->data_size);
    CTBB_CUDA(cudaGetLastError());
    rc->rep = 1;
    return CTBB_OK;
}

ctbb_status recon_to_sequential(ctbb_recon* rc, const ctbb_ssm* ssm) {
    if (rc->rep == 0) return CTBB_OK;
    ctbb_ctx* ctx = rc->ctx;
    f32_to_f64_kernel<<<grid_for(ctx, rc->nvox, 256), 256, 0, ctx->stream>>>(rc->d_x32, rc->d_x64, rc->nvox);
    CTBB_CUDA(cudaGetLastError());
    CTBB_TRY(forward_project_f64(rc, ssm, false, rc->d_est64));
    rc->rep = 0;
    return CTBB_OK;
}

ctbb_status cost_f64(ctbb_recon* rc, const ctbb_ssm* ssm, bool exact, double* out) {
    ctbb_ctx* ctx = rc->ctx;
    const int nb = ctx->sm_count * 8;
    CTBB_TRY(ensure_partials(ctx, nb));
    double data = 0.0, pen = 0.0;
    const bool quad = rc->geom.penalty == CTBB_PENALTY_QUADRATIC;
    if (rc->rep == 0) {
        sq_sum_kernel<<<nb, 256, 0, ctx->stream>>>(rc->d_raw, rc->d_est64, rc->data_size, ctx->d_partials);
    } else if (exact) {
        // Recompute A x in FP64 into the (grouped-mode spare) FP64 buffer.
        CTBB_TRY(forward_project_f64(rc, ssm, true, rc->d_est64));
        sq_sum_kernel<<<nb, 256, 0, ctx->stream>>>(rc->d_raw, rc->d_est64, rc->data_size, ctx->d_partials);
    } else {
        sq_sum_kernel<<<nb, 256, 0, ctx->stream>>>(rc->d_e32, nullptr, rc->data_size, ctx->d_partials);
    }
    CTBB_CUDA(cudaGetLastError());
    CTBB_TRY(reduce_partials(ctx, nb, &data));
    if (rc->rep == 0)
        penalty_sum_kernel<double><<<nb, 256, 0, ctx->stream>>>(rc->d_x64, rc->nvox, (int64_t)rc->geom.num_voxels_x,
                                                                rc->geom.penalty, rc->geom.delta, ctx->d_partials);
    else
        penalty_sum_kernel<float><<<nb, 256, 0, ctx->stream>>>(rc->d_x32, rc->nvox, (int64_t)rc->geom.num_voxels_x,
                                                               rc->geom.penalty, rc->geom.delta, ctx->d_partials);
    CTBB_CUDA(cudaGetLastError());
    CTBB_TRY(reduce_partials(ctx, nb, &pen));
    *out = quad ? 0.5 * data + rc->geom.lambda / 4.0 * pen : data + rc->geom.lambda / 2.0 * pen;
    return CTBB_OK;
}

}  // namespace ctbb

using namespace ctbb;

extern "C" ctbb_status ctbb_gpu_recon_create(ctbb_ctx* ctx, const ctbb_geom_c* geom, const uint64_t* slice_indices,
                                             ctbb_recon** out) {
    clear_error();
    if (!ctx || !geom || !out || (!slice_indices && geom->num_voxels_z)) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    CTBB_TRY(ssm_validate_geometry(*geom));
    if (geom->num_voxels_z == 0) return fail(CTBB_ERR_INVALID_ARG, "no slices");
    CTBB_CUDA(cudaSetDevice(ctx->device));
    ctbb_recon* rc = new ctbb_recon();
    struct Guard {
        ctbb_recon* r;
        ~Guard() {
            if (r) ctbb_gpu_recon_free(r);
        }
    } guard{rc};
    rc->ctx = ctx;
    ctx_retain(ctx);
    rc->geom = *geom;
    rc->nvox = geom->num_voxels_x * geom->num_voxels_y * geom->num_voxels_z;
    rc->data_size = geom->Readings * geom->n_channels * geom->Nrows_projection;
    rc->slice_indices.assign(slice_indices, slice_indices + geom->num_voxels_z);
    std::vector<int32_t> start(geom->num_voxels_z);
    for (uint64_t k = 0; k < geom->num_voxels_z; ++k) {
        if (slice_indices[k] >= geom->Readings) return fail(CTBB_ERR_INVALID_ARG, "slice index beyond the scan");
        start[k] = (int32_t)(slice_indices[k] - geom->num_views_for_system_matrix / 2);  // icd_iteration.cpp:195
    }
    CTBB_CUDA(cudaMalloc(&rc->d_start, start.size() * sizeof(int32_t)));
    CTBB_CUDA(cudaMemcpy(rc->d_start, start.data(), start.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    CTBB_CUDA(cudaMalloc(&rc->d_raw, rc->data_size * sizeof(float)));
    CTBB_CUDA(cudaMalloc(&rc->d_est64, rc->data_size * sizeof(double)));
    CTBB_CUDA(cudaMalloc(&rc->d_e32, rc->data_size * sizeof(float)));
    CTBB_CUDA(cudaMalloc(&rc->d_x64, rc->nvox * sizeof(double)));
    CTBB_CUDA(cudaMalloc(&rc->d_x32, rc->nvox * sizeof(float)));
    CTBB_CUDA(cudaMemsetAsync(rc->d_raw, 0, rc->data_size * sizeof(float), ctx->stream));
    CTBB_CUDA(cudaMemsetAsync(rc->d_est64, 0, rc->data_size * sizeof(double), ctx->stream));
    CTBB_CUDA(cudaMemsetAsync(rc->d_e32, 0, rc->data_size * sizeof(float), ctx->stream));
    CTBB_CUDA(cudaMemsetAsync(rc->d_x64, 0, rc->nvox * sizeof(double), ctx->stream));
    CTBB_CUDA(cudaMemsetAsync(rc->d_x32, 0, rc->nvox * sizeof(float), ctx->stream));
    CTBB_CUDA(cudaStreamSynchronize(ctx->stream));
    rc->rep = 0;
    guard.r = nullptr;
    *out = rc;
    return CTBB_OK;
}

extern "C" void ctbb_gpu_recon_free(ctbb_recon* rc) {
    if (!rc) return;
    if (rc->ctx) {
        cudaSetDevice(rc->ctx->device);
        cudaStreamSynchronize(rc->ctx->stream);
    }
    cudaFree(rc->d_start);
    cudaFree(rc->d_raw);
    cudaFree(rc->d_est64);
    cudaFree(rc->d_e32);
    cudaFree(rc->d_x64);
    cudaFree(rc->d_x32);
    cudaFree(rc->d_order);
    cudaFree(rc->d_stacks);
    cudaFree(rc->d_prio);
    cudaFree(rc->d_prio_order);
    cudaFree(rc->d_prio_stacks);
    if (rc->icd_graph) cudaGraphExecDestroy(rc->icd_graph);
    ctx_release(rc->ctx);
    delete rc;
}

extern "C" ctbb_status ctbb_gpu_recon_set_raw(ctbb_recon* rc, const float* raw_host) {
    clear_error();
    if (!rc || !raw_host) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    CTBB_CUDA(cudaSetDevice(rc->ctx->device));
    CTBB_CUDA(cudaMemcpyAsync(rc->d_raw, raw_host, rc->data_size * sizeof(float), cudaMemcpyHostToDevice, rc->ctx->stream));
    CTBB_CUDA(cudaStreamSynchronize(rc->ctx->stream));
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_gpu_recon_set_raw_device(ctbb_recon* rc, const float* raw_dev) {
    clear_error();
    if (!rc || !raw_dev) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    CTBB_CUDA(cudaSetDevice(rc->ctx->device));
    if (raw_dev != rc->d_raw)
        CTBB_CUDA(cudaMemcpyAsync(rc->d_raw, raw_dev, rc->data_size * sizeof(float), cudaMemcpyDeviceToDevice,
                                  rc->ctx->stream));
    return CTBB_OK;
}

extern "C" float* ctbb_gpu_recon_raw_device(ctbb_recon* rc) { return rc ? rc->d_raw : nullptr; }

extern "C" ctbb_status ctbb_gpu_recon_get_raw(ctbb_recon* rc, float* raw_host) {
    clear_error();
    if (!rc || !raw_host) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    CTBB_CUDA(cudaSetDevice(rc->ctx->device));
    CTBB_CUDA(cudaMemcpyAsync(raw_host, rc->d_raw, rc->data_size * sizeof(float), cudaMemcpyDeviceToHost,
                              rc->ctx->stream));
    CTBB_CUDA(cudaStreamSynchronize(rc->ctx->stream));
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_gpu_recon_set_volume_estimate(ctbb_recon* rc, const ctbb_ssm* ssm, const float* vol_host,
                                                          int32_t estimate) {
    clear_error();
    if (!rc || !ssm) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (estimate != CTBB_ESTIMATE_ZERO && estimate != CTBB_ESTIMATE_FORWARD)
        return fail(CTBB_ERR_INVALID_ARG, "estimate must be CTBB_ESTIMATE_ZERO or CTBB_ESTIMATE_FORWARD");
    CTBB_TRY(check_pair(rc, ssm));
    CTBB_CUDA(cudaSetDevice(rc->ctx->device));
    cudaStream_t st = rc->ctx->stream;
    if (vol_host) {
        CTBB_CUDA(cudaMemcpyAsync(rc->d_x32, vol_host, rc->nvox * sizeof(float), cudaMemcpyHostToDevice, st));
        f32_to_f64_kernel<<<grid_for(rc->ctx, rc->nvox, 256), 256, 0, st>>>(rc->d_x32, rc->d_x64, rc->nvox);
        CTBB_CUDA(cudaGetLastError());
        if (estimate == CTBB_ESTIMATE_FORWARD)
            CTBB_TRY(forward_project_f64(rc, ssm, false, rc->d_est64));
        else  // icd_iteration.cpp:47, 63: the estimate stays zero unless a wFBP start forward-projects it
            CTBB_CUDA(cudaMemsetAsync(rc->d_est64, 0, rc->data_size * sizeof(double), st));
    } else {
        CTBB_CUDA(cudaMemsetAsync(rc->d_x32, 0, rc->nvox * sizeof(float), st));
        CTBB_CUDA(cudaMemsetAsync(rc->d_x64, 0, rc->nvox * sizeof(double), st));
        CTBB_CUDA(cudaMemsetAsync(rc->d_est64, 0, rc->data_size * sizeof(double), st));
    }
    residual_kernel<<<grid_for(rc->ctx, rc->data_size, 256), 256, 0, st>>>(rc->d_raw, rc->d_est64, rc->d_e32,
                                                                             rc->data_size);
    CTBB_CUDA(cudaGetLastError());
    CTBB_CUDA(cudaStreamSynchronize(st));
    rc->rep = 0;  // both representations are current; sequential is the canonical one
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_gpu_recon_set_volume_upsampled(ctbb_recon* fine, const ctbb_ssm* fine_ssm,
                                                            ctbb_recon* coarse) {
    clear_error();
    if (!fine || !fine_ssm || !coarse) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    CTBB_TRY(check_pair(fine, fine_ssm));
    const ctbb_geom_c& gf = fine->geom;
    const ctbb_geom_c& gc = coarse->geom;
    if (fine->ctx != coarse->ctx) return fail(CTBB_ERR_INVALID_ARG, "reconstructions on different contexts");
    if (gf.num_voxels_x != 2 * gc.num_voxels_x || gf.num_voxels_y != 2 * gc.num_voxels_y ||
        gf.num_voxels_z != gc.num_voxels_z || gf.recon_fov != gc.recon_fov || gf.Readings != gc.Readings ||
        fine->slice_indices != coarse->slice_indices)
        return fail(CTBB_ERR_INVALID_ARG,
                    "the fine grid must have twice the coarse grid's in-plane size, the same field of view, "
                    "scan and slices");
    CTBB_CUDA(cudaSetDevice(fine->ctx->device));
    cudaStream_t st = fine->ctx->stream;
    if (coarse->rep == 0) {
        f64_to_f32_kernel<<<grid_for(coarse->ctx, coarse->nvox, 256), 256, 0, st>>>(coarse->d_x64, coarse->d_x32,
                                                                                    coarse->nvox);
        CTBB_CUDA(cudaGetLastError());
    }
    upsample2_kernel<<<grid_for(fine->ctx, fine->nvox, 256), 256, 0, st>>>(
        coarse->d_x32, (int)gc.num_voxels_x, (int)gc.num_voxels_y, (int)gc.num_voxels_z, fine->d_x32);
    CTBB_CUDA(cudaGetLastError());
    f32_to_f64_kernel<<<grid_for(fine->ctx, fine->nvox, 256), 256, 0, st>>>(fine->d_x32, fine->d_x64, fine->nvox);
    CTBB_CUDA(cudaGetLastError());
    CTBB_TRY(forward_project_f64(fine, fine_ssm, false, fine->d_est64));
    residual_kernel<<<grid_for(fine->ctx, fine->data_size, 256), 256, 0, st>>>(fine->d_raw, fine->d_est64,
                                                                               fine->d_e32, fine->data_size);
    CTBB_CUDA(cudaGetLastError());
    CTBB_CUDA(cudaStreamSynchronize(st));
    fine->rep = 0;
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_gpu_recon_set_volume(ctbb_recon* rc, const ctbb_ssm* ssm, const float* vol_host) {
    return ctbb_gpu_recon_set_volume_estimate(rc, ssm, vol_host, CTBB_ESTIMATE_FORWARD);
}

extern "C" ctbb_status ctbb_gpu_recon_get_volume(ctbb_recon* rc, float* vol_host) {
    clear_error();
    if (!rc || !vol_host) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    CTBB_CUDA(cudaSetDevice(rc->ctx->device));
    cudaStream_t st = rc->ctx->stream;
    if (rc->rep == 0) {
        // icd_iteration.cpp:277-284: the FP64 image is cast to float at the end.
        f64_to_f32_kernel<<<grid_for(rc->ctx, rc->nvox, 256), 256, 0, st>>>(rc->d_x64, rc->d_x32, rc->nvox);
        CTBB_CUDA(cudaGetLastError());
    }
    CTBB_CUDA(cudaMemcpyAsync(vol_host, rc->d_x32, rc->nvox * sizeof(float), cudaMemcpyDeviceToHost, st));
    CTBB_CUDA(cudaStreamSynchronize(st));
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_gpu_recon_get_volume_f64(ctbb_recon* rc, double* vol_host) {
    clear_error();
    if (!rc || !vol_host) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    CTBB_CUDA(cudaSetDevice(rc->ctx->device));
    cudaStream_t st = rc->ctx->stream;
    if (rc->rep == 1) {
        f32_to_f64_kernel<<<grid_for(rc->ctx, rc->nvox, 256), 256, 0, st>>>(rc->d_x32, rc->d_x64, rc->nvox);
        CTBB_CUDA(cudaGetLastError());
    }
    CTBB_CUDA(cudaMemcpyAsync(vol_host, rc->d_x64, rc->nvox * sizeof(double), cudaMemcpyDeviceToHost, st));
    CTBB_CUDA(cudaStreamSynchronize(st));
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_gpu_recon_entries(ctbb_recon* rc, const ctbb_ssm* ssm, double* entries) {
    clear_error();
    if (!rc || !ssm || !entries) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    CTBB_TRY(check_pair(rc, ssm));
    CTBB_CUDA(cudaSetDevice(rc->ctx->device));
    return inrange_entries(rc, ssm, entries);
}

extern "C" ctbb_status ctbb_gpu_recon_refresh_residual(ctbb_recon* rc, const ctbb_ssm* ssm) {
    clear_error();
    if (!rc || !ssm) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    CTBB_TRY(check_pair(rc, ssm));
    CTBB_CUDA(cudaSetDevice(rc->ctx->device));
    if (rc->rep == 0) {
        CTBB_TRY(forward_project_f64(rc, ssm, false, rc->d_est64));
    } else {
        CTBB_TRY(forward_project_f64(rc, ssm, true, rc->d_est64));
        residual_kernel<<<grid_for(rc->ctx, rc->data_size, 256), 256, 0, rc->ctx->stream>>>(
            rc->d_raw, rc->d_est64, rc->d_e32, rc->data_size);
        CTBB_CUDA(cudaGetLastError());
    }
    CTBB_CUDA(cudaStreamSynchronize(rc->ctx->stream));
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_gpu_recon_cost(ctbb_recon* rc, double* cost) {
    clear_error();
    if (!rc || !cost) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    CTBB_CUDA(cudaSetDevice(rc->ctx->device));
    // Exact cost needs A x in FP64; in grouped mode the matrix is not at
    // hand here, so the FP32 error sinogram is reduced in FP64 instead.
    return cost_f64(rc, nullptr, false, cost);
}

extern "C" ctbb_status ctbb_gpu_recon_iterate(ctbb_recon* rc, const ctbb_ssm* ssm, const ctbb_icd_opts* opts,
                                              int32_t n_iter, ctbb_iter_stats* stats) {
    clear_error();
    if (!rc || !ssm || !opts) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (n_iter < 0) return fail(CTBB_ERR_INVALID_ARG, "negative iteration count");
    CTBB_TRY(check_pair(rc, ssm));
    CTBB_CUDA(cudaSetDevice(rc->ctx->device));
    ctbb_iter_stats s;
    memset(&s, 0, sizeof(s));
    double prev_cost = NAN;
    for (int it = 0; it < n_iter; ++it) {
        float ms = 0.f;
        double entries = 0.0;
        double upd = (double)rc->nvox;
        if (opts->mode == CTBB_ICD_SEQUENTIAL) {
            if (!ssm->d_w32) return fail(CTBB_ERR_INVALID_ARG, "sequential mode needs FP32 weights");
            CTBB_TRY(recon_to_sequential(rc, ssm));
            CTBB_TRY(launch_icd_sequential(rc, ssm, 1, &ms));
        } else if (opts->mode == CTBB_ICD_GROUPED) {
            const int wsel = opts->weights ? opts->weights : CTBB_SSM_FP32;
            if ((wsel == CTBB_SSM_FP32 && !ssm->d_w32) || (wsel == CTBB_SSM_FP16 && !ssm->d_w16))
                return fail(CTBB_ERR_INVALID_ARG, "requested weight format is not held by the matrix");
            CTBB_TRY(recon_to_grouped(rc, ssm));
            if (opts->refresh_every > 0 && it > 0 && it % opts->refresh_every == 0) {
                CTBB_TRY(forward_project_f64(rc, ssm, true, rc->d_est64));
                residual_kernel<<<grid_for(rc->ctx, rc->data_size, 256), 256, 0, rc->ctx->stream>>>(
                    rc->d_raw, rc->d_est64, rc->d_e32, rc->data_size);
                CTBB_CUDA(cudaGetLastError());
            }
            uint64_t items = 0;
            double scattered = 0.0;
            CTBB_TRY(launch_icd_grouped(rc, ssm, *opts, &ms, &entries, &items, &scattered));
            if (opts->priority) upd = (double)items;
            s.entries_scattered += scattered;
        } else {
            return fail(CTBB_ERR_INVALID_ARG, "unknown ICD mode %d", opts->mode);
        }
        s.iterations += 1;
        s.device_ms += ms;
        s.entries += entries;
        s.voxel_updates += upd;
        if (opts->compute_cost || opts->stop_rel_change > 0.0) {
            // Exact FP64 cost: in grouped mode A x is recomputed in FP64 (not
            // the incrementally updated FP32 e), and e is refreshed from it.
            double c = 0.0;
            CTBB_TRY(cost_f64(rc, ssm, true, &c));
            if (rc->rep == 1) {
                residual_kernel<<<grid_for(rc->ctx, rc->data_size, 256), 256, 0, rc->ctx->stream>>>(
                    rc->d_raw, rc->d_est64, rc->d_e32, rc->data_size);
                CTBB_CUDA(cudaGetLastError());
            }
            s.cost = c;
            if (!isnan(prev_cost)) {
                s.rel_change = fabs(prev_cost - c) / fmax(fabs(c), 1e-300);
                if (opts->stop_rel_change > 0.0 && s.rel_change < opts->stop_rel_change) {
                    prev_cost = c;
                    break;
                }
            }
            prev_cost = c;
        }
    }
    CTBB_CUDA(cudaStreamSynchronize(rc->ctx->stream));
    if (stats) *stats = s;
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_gpu_icd(ctbb_ctx* ctx, const ctbb_ssm* ssm, const ctbb_geom_c* geom,
                                    const uint64_t* slice_indices, const float* raw, float* recon_volume,
                                    const ctbb_icd_opts* opts, ctbb_iter_stats* stats) {
    clear_error();
    if (!ctx || !ssm || !geom || !slice_indices || !raw || !recon_volume)
        return fail(CTBB_ERR_INVALID_ARG, "null argument");
    ctbb_icd_opts o;
    memset(&o, 0, sizeof(o));
    o.mode = CTBB_ICD_SEQUENTIAL;
    if (opts) o = *opts;
    ctbb_recon* rc = nullptr;
    CTBB_TRY(ctbb_gpu_recon_create(ctx, geom, slice_indices, &rc));
    ctbb_status st = ctbb_gpu_recon_set_raw(rc, raw);
    // Sequential (parity) mode starts like icd_iteration.cpp:47-63: the
    // sinogram estimate is forward-projected only for a wFBP start, so an
    // initial image loaded from initial_recon_path starts with y_hat = 0.
    // Grouped mode always starts from a consistent e = y - A x.
    const int32_t est = (o.mode == CTBB_ICD_SEQUENTIAL && !geom->wfbp_initialize) ? CTBB_ESTIMATE_ZERO
                                                                                  : CTBB_ESTIMATE_FORWARD;
    if (st == CTBB_OK) st = ctbb_gpu_recon_set_volume_estimate(rc, ssm, recon_volume, est);
    if (st == CTBB_OK) st = ctbb_gpu_recon_iterate(rc, ssm, &o, (int32_t)geom->num_iterations, stats);
    if (st == CTBB_OK) st = ctbb_gpu_recon_get_volume(rc, recon_volume);
    ctbb_gpu_recon_free(rc);
    return st;
}

// Learned warm start: x <- max(0, x + R_fixed2rot(cnn(R_rot2fixed(x)))), then
// e = y - Ax in FP64; the per-voxel step size becomes the priority map.
extern "C" ctbb_status ctbb_gpu_recon_warm_start(ctbb_recon* rc, const ctbb_ssm* ssm, ctbb_cnn* cnn,
                                                 const double* tube_angles_deg) {
    clear_error();
    if (!rc || !ssm || !cnn || !tube_angles_deg) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    CTBB_TRY(check_pair(rc, ssm));
    if (cnn_ctx(cnn) != rc->ctx) return fail(CTBB_ERR_INVALID_ARG, "network and reconstruction use different contexts");
    CTBB_CUDA(cudaSetDevice(rc->ctx->device));
    CTBB_TRY(recon_to_grouped(rc, ssm));
    const ctbb_geom_c& g = rc->geom;
    const uint64_t n = rc->nvox;
    if (!rc->d_prio) CTBB_CUDA(cudaMalloc(&rc->d_prio, n * sizeof(float)));
    float *d_a = nullptr, *d_b = nullptr;
    CTBB_CUDA(cudaMalloc(&d_a, n * sizeof(float)));
    if (cudaMalloc(&d_b, n * sizeof(float)) != cudaSuccess) {
        cudaFree(d_a);
        return fail(CTBB_ERR_OOM, "warm start scratch");
    }
    ctbb_status st = rotate_volume(rc->ctx, g, tube_angles_deg, rc->slice_indices.data(), rc->d_x32, d_a,
                                   CTBB_ROTATE_ROTATING2FIXED);
    if (st == CTBB_OK)
        st = cnn_predict_correction(cnn, d_a, (int)g.num_voxels_x, (int)g.num_voxels_y, (int)g.num_voxels_z, d_b);
    if (st == CTBB_OK)
        st = rotate_volume(rc->ctx, g, tube_angles_deg, rc->slice_indices.data(), d_b, d_a,
                           CTBB_ROTATE_FIXED2ROTATING);
    if (st == CTBB_OK) st = apply_correction(rc->ctx, n, rc->d_x32, d_a, rc->d_prio);
    if (st == CTBB_OK) st = ctbb_gpu_recon_refresh_residual(rc, ssm);
    if (st == CTBB_OK) st = cnn_check_flag(cnn);
    cudaFree(d_a);
    cudaFree(d_b);
    cudaFree(rc->d_prio_order);
    cudaFree(rc->d_prio_stacks);
    rc->d_prio_order = nullptr;
    rc->n_prio_order = 0;
    rc->d_prio_stacks = nullptr;
    rc->n_prio_stacks = 0;
    return st;
}
