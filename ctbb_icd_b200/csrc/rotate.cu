// Slice rotation between the rotating ICD frame and the fixed frame.
//
// Replaces rotate_slices_rotating2fixed (rotate_slices.cpp:81-114),
// rotate_slices_fixed2rotating (:48-79), rotate_slice (:116-154) and interp2
// (interp.h:41-76). Each thread gathers the four bilinear taps of four
// output pixels of one row, all loads issued before any is used. (A variant
// that staged each 32 x 32 output tile's input box in shared memory measured
// slower: at 134 MB per volume the kernel is bound by its per-pixel
// arithmetic and launch, not by HBM.)
//
// Compiled with -fmad=false. The per-slice cos/sin are computed on the host
// with the reference's expressions, the rotated coordinates in double and
// rounded to float exactly where rotate_slice.cpp:142-151 rounds them, and
// the interpolation in float with the reference's operation order, so the
// output matches the reference bit for bit.
#include <limits.h>
#include <math.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "gpu_internal.h"

namespace {

// Output pixels per thread (spaced kRotBlock apart along x).
constexpr int kRotBlock = 128, kRotPix = 4;

// Grid: x = groups of kRotBlock * kRotPix pixels of a row, y = row, z = slice.
// Each thread issues the 16 bilinear loads of its 4 pixels before using any
// (the input slice, at most 1 MB at 512 x 512, stays in L2 while its rows are
// written). FLOAT_CENTRE: the centre (cvx, cvy) is exactly a float. Then
// (float)((double)xp + cvx) equals the float sum xp + (float)cvx: the exact
// sum of two floats fits in a double's 53 bits unless the smaller one is
// below about 2^-29 of the larger, and then it is far below half a float ulp
// of the larger, so both roundings return the larger. The float add saves
// two conversions per coordinate on the narrow conversion pipe.
template <bool FLOAT_CENTRE>
__global__ void __launch_bounds__(kRotBlock) rotate_kernel(const float* __restrict__ in, float* __restrict__ out,
                                                           int nx, int ny, int nz, int dim1, int dim2,
                                                           int out_stride_y, const double* __restrict__ cs,
                                                           double cvx, double cvy) {
    const int k = blockIdx.z, y_idx = blockIdx.y;
    const uint64_t npix = (uint64_t)nx * ny;
    const double c = cs[2 * k], s = cs[2 * k + 1];
    const float* a = in + (uint64_t)k * npix;
    const double y = y_idx - cvy;
    const double sy = s * y, cy = c * y;
    const float cvx_f = (float)cvx, cvy_f = (float)cvy;
    float tap[kRotPix][4], vv[kRotPix], ww[kRotPix];
    bool inside[kRotPix];
#pragma unroll
    for (int u = 0; u < kRotPix; ++u) {
        const int x_idx = blockIdx.x * (kRotBlock * kRotPix) + u * kRotBlock + threadIdx.x;
        const double x = x_idx - cvx;
        const float xp = (float)(c * x - sy);
        const float yp = (float)(s * x + cy);
        const float i1 = FLOAT_CENTRE ? __fadd_rn(xp, cvx_f) : (float)((double)xp + cvx);
        const float i2 = FLOAT_CENTRE ? __fadd_rn(yp, cvy_f) : (float)((double)yp + cvy);
        // interp.h:57-58: zero outside [0, n-2] in either index.
        inside[u] = x_idx < nx && !(i1 > (float)(dim1 - 2) || (i1 < 0) || i2 > (float)(dim2 - 2) || (i2 < 0));
        vv[u] = i1 - floorf(i1);
        ww[u] = i2 - floorf(i2);
        if (inside[u]) {
            const int f1 = (int)floorf(i1), f2 = (int)floorf(i2);
            tap[u][0] = __ldg(a + (f2 * dim1 + f1));
            tap[u][1] = __ldg(a + (f2 * dim1 + f1 + 1));
            tap[u][2] = __ldg(a + ((f2 + 1) * dim1 + f1));
            tap[u][3] = __ldg(a + ((f2 + 1) * dim1 + f1 + 1));
        }
    }
#pragma unroll
    for (int u = 0; u < kRotPix; ++u) {
        const int x_idx = blockIdx.x * (kRotBlock * kRotPix) + u * kRotBlock + threadIdx.x;
        if (x_idx >= nx) continue;
        const float v = vv[u], w = ww[u];
        // interp.h:70-73, the reference's operation order.
        const float val = inside[u] ? tap[u][0] * (1.0f - v) * (1.0f - w) + tap[u][1] * v * (1.0f - w) +
                                          tap[u][2] * (1.0f - v) * w + tap[u][3] * v * w
                                    : 0.0f;
        // rotate_slices.cpp:128 writes with stride num_voxels_y.
        out[(uint64_t)k * npix + (uint64_t)x_idx + (uint64_t)y_idx * out_stride_y] = val;
    }
}

// Launches the rotation of every slice of g on st; slices go in chunks of
// at most 65535 (the grid's z limit), each chunk with its own base pointers.
cudaError_t launch_rotate(cudaStream_t st, const ctbb_geom_c& g, const float* in, float* out, const double* cs) {
    const uint64_t npix = g.num_voxels_x * g.num_voxels_y;
    if (npix == 0 || g.num_voxels_z == 0) return cudaSuccess;
    const unsigned gx = (unsigned)((g.num_voxels_x + kRotBlock * kRotPix - 1) / (kRotBlock * kRotPix));
    const bool fc = (double)(float)g.center_voxel_x == g.center_voxel_x &&
                    (double)(float)g.center_voxel_y == g.center_voxel_y;
    for (uint64_t k0 = 0; k0 < g.num_voxels_z; k0 += 65535) {
        const unsigned nz = (unsigned)std::min<uint64_t>(65535, g.num_voxels_z - k0);
        (fc ? rotate_kernel<true> : rotate_kernel<false>)<<<dim3(gx, (unsigned)g.num_voxels_y, nz), kRotBlock, 0,
                                                          st>>>(
            in + k0 * npix, out + k0 * npix, (int)g.num_voxels_x, (int)g.num_voxels_y, (int)nz, (int)g.nx, (int)g.ny,
            (int)g.num_voxels_y, cs + 2 * k0, g.center_voxel_x, g.center_voxel_y);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

ctbb_status angles(const ctbb_geom_c& g, const double* tube_angles_deg, const uint64_t* slice_indices, int direction,
                   std::vector<double>& cs) {
    const double PI = 3.141592653589793238;  // rotate_slices.cpp:29
    cs.resize(2 * g.num_voxels_z);
    for (uint64_t k = 0; k < g.num_voxels_z; ++k) {
        if (slice_indices[k] >= g.Readings) return ctbb::fail(CTBB_ERR_INVALID_ARG, "slice index out of range");
        double a = -(tube_angles_deg[slice_indices[k]]) * 2.0 * PI / 360.0;
        if (direction == CTBB_ROTATE_FIXED2ROTATING) a = -a;
        cs[2 * k] = cos(a);
        cs[2 * k + 1] = sin(a);
    }
    return CTBB_OK;
}

ctbb_status rotate_device(ctbb_ctx* ctx, const ctbb_geom_c& g, const double* tube_angles_deg,
                          const uint64_t* slice_indices, const float* d_in, float* d_out, int direction) {
    using namespace ctbb;
    if (direction != CTBB_ROTATE_FIXED2ROTATING && direction != CTBB_ROTATE_ROTATING2FIXED)
        return fail(CTBB_ERR_INVALID_ARG, "direction must be +1 or -1");
    if (g.num_voxels_x != g.num_voxels_y)
        return fail(CTBB_ERR_INVALID_ARG, "slice rotation needs square slices (rotate_slices.cpp:128)");
    std::vector<double> cs;
    CTBB_TRY(angles(g, tube_angles_deg, slice_indices, direction, cs));
    double* d_cs = nullptr;
    CTBB_CUDA(cudaMalloc(&d_cs, cs.size() * sizeof(double)));
    cudaStream_t st = ctx->stream;
    cudaError_t e = cudaMemcpyAsync(d_cs, cs.data(), cs.size() * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        e = launch_rotate(st, g, d_in, d_out, d_cs);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    cudaFree(d_cs);
    if (e != cudaSuccess) return fail(CTBB_ERR_CUDA, "rotate: %s", cudaGetErrorString(e));
    return CTBB_OK;
}

}  // namespace

using namespace ctbb;

namespace ctbb {
ctbb_status rotate_volume(ctbb_ctx* ctx, const ctbb_geom_c& g, const double* tube_angles_deg,
                          const uint64_t* slice_indices, const float* d_in, float* d_out, int direction) {
    return rotate_device(ctx, g, tube_angles_deg, slice_indices, d_in, d_out, direction);
}
}  // namespace ctbb

extern "C" ctbb_status ctbb_gpu_rotate_device(ctbb_ctx* ctx, const ctbb_geom_c* geom, const double* tube_angles_deg,
                                              const uint64_t* slice_indices, const float* in_dev, float* out_dev,
                                              int32_t direction) {
    clear_error();
    if (!ctx || !geom || !tube_angles_deg || !slice_indices || !in_dev || !out_dev)
        return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (in_dev == out_dev) return fail(CTBB_ERR_INVALID_ARG, "in and out must not alias");
    CTBB_CUDA(cudaSetDevice(ctx->device));
    return rotate_device(ctx, *geom, tube_angles_deg, slice_indices, in_dev, out_dev, direction);
}

// ---------------------------------------------------------------------------
// Allocation-free variant of ctbb_gpu_rotate_device.
//
// Some callers cannot let a library call cudaMalloc: applications that hand
// out all device memory from their own pool up front (so a stray allocation
// could fail or fragment it), real-time reconstruction loops that must not
// hit the allocator's implicit synchronisation, and embedders that run the
// rotation between other work without wanting the driver to grow the
// process's footprint. For them the per-slice cos/sin table, the only scratch
// the rotation kernel needs, lives in this fixed device array instead of a
// cudaMalloc'd buffer.
//
// The array is a file-scope __device__ symbol (2 * kNoAllocMaxSlices doubles,
// 128 KB): it is resident on each GPU from the library's first use there
// (under CUDA's lazy module loading, the first call into it) until the
// process exits. Host code only knows the symbol's host-side shadow, so the
// device address is looked up with cudaGetSymbolAddress once per device,
// with that device current, the first time the entry point runs on it, and
// kept until exit (a caller's cudaDeviceReset would invalidate it; calls
// after one are not supported).
// ---------------------------------------------------------------------------
namespace {

constexpr uint64_t kNoAllocMaxSlices = 8192;
static __device__ __align__(256) double g_rotate_scratch[2 * kNoAllocMaxSlices];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
double* g_scratch_addr[kMaxDevices] = {};

// Device address of g_rotate_scratch on `device` (which must be current).
ctbb_status scratch_address(int device, double** out) {
    using namespace ctbb;
    if (device < 0 || device >= kMaxDevices) return fail(CTBB_ERR_INVALID_ARG, "device index %d too large", device);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_rotate_scratch);
        if (e != cudaSuccess)
            return fail(CTBB_ERR_CUDA, "cudaGetSymbolAddress(g_rotate_scratch): %s", cudaGetErrorString(e));
        g_scratch_addr[device] = (double*)p;
    }
    *out = g_scratch_addr[device];
    return CTBB_OK;
}

}  // namespace

extern "C" ctbb_status ctbb_gpu_rotate_device_noalloc(ctbb_ctx* ctx, const ctbb_geom_c* geom,
                                                      const double* tube_angles_deg, const uint64_t* slice_indices,
                                                      const float* in_dev, float* out_dev, int32_t direction) {
    clear_error();
    if (!ctx || !geom || !tube_angles_deg || !slice_indices || !in_dev || !out_dev)
        return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (in_dev == out_dev) return fail(CTBB_ERR_INVALID_ARG, "in and out must not alias");
    if (direction != CTBB_ROTATE_FIXED2ROTATING && direction != CTBB_ROTATE_ROTATING2FIXED)
        return fail(CTBB_ERR_INVALID_ARG, "direction must be +1 or -1");
    if (geom->num_voxels_z > kNoAllocMaxSlices)
        return fail(CTBB_ERR_INVALID_ARG,
                    "ctbb_gpu_rotate_device_noalloc handles at most %llu slices (got %llu); use ctbb_gpu_rotate_device",
                    (unsigned long long)kNoAllocMaxSlices, (unsigned long long)geom->num_voxels_z);
    if (geom->num_voxels_x != geom->num_voxels_y)
        return fail(CTBB_ERR_INVALID_ARG, "slice rotation needs square slices (rotate_slices.cpp:128)");
    CTBB_CUDA(cudaSetDevice(ctx->device));
    double* d_cs = nullptr;
    CTBB_TRY(scratch_address(ctx->device, &d_cs));
    // Every slice's entries are rewritten below, so nothing left by an
    // earlier call needs clearing.
    std::vector<double> cs;
    CTBB_TRY(angles(*geom, tube_angles_deg, slice_indices, direction, cs));
    if (cs.empty()) return CTBB_OK;
    cudaStream_t st = ctx->stream;
    CTBB_CUDA(cudaMemcpyAsync(d_cs, cs.data(), cs.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    const ctbb_geom_c& g = *geom;
    CTBB_CUDA(launch_rotate(st, g, in_dev, out_dev, d_cs));
    CTBB_CUDA(cudaStreamSynchronize(st));
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_gpu_rotate(ctbb_ctx* ctx, const ctbb_geom_c* geom, const double* tube_angles_deg,
                                       const uint64_t* slice_indices, float* vol_host, int32_t direction) {
    clear_error();
    if (!ctx || !geom || !tube_angles_deg || !slice_indices || !vol_host)
        return fail(CTBB_ERR_INVALID_ARG, "null argument");
    CTBB_CUDA(cudaSetDevice(ctx->device));
    const size_t bytes = geom->num_voxels_x * geom->num_voxels_y * geom->num_voxels_z * sizeof(float);
    if (bytes == 0) return CTBB_OK;
    float *d_in = nullptr, *d_out = nullptr;
    CTBB_CUDA(cudaMalloc(&d_in, bytes));
    if (cudaMalloc(&d_out, bytes) != cudaSuccess) {
        cudaFree(d_in);
        return fail(CTBB_ERR_OOM, "rotate: device allocation failed");
    }
    ctbb_status rc = CTBB_OK;
    if (cudaMemcpyAsync(d_in, vol_host, bytes, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
        rc = fail(CTBB_ERR_CUDA, "rotate: upload failed");
    if (rc == CTBB_OK) rc = rotate_device(ctx, *geom, tube_angles_deg, slice_indices, d_in, d_out, direction);
    if (rc == CTBB_OK &&
        (cudaMemcpyAsync(vol_host, d_out, bytes, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
         cudaStreamSynchronize(ctx->stream) != cudaSuccess))
        rc = fail(CTBB_ERR_CUDA, "rotate: download failed");
    cudaFree(d_in);
    cudaFree(d_out);
    return rc;
}
