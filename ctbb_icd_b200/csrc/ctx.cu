// GPU context (device + stream) and the GPU synthetic projector.
#include <string.h>

#include <algorithm>
#include <vector>

#include "gpu_internal.h"
#include "phantom.h"

namespace ctbb {

ctbb_status ensure_partials(ctbb_ctx* ctx, size_t n) {
    if (ctx->partials_cap >= n) return CTBB_OK;
    cudaFree(ctx->d_partials);
    ctx->d_partials = nullptr;
    ctx->partials_cap = 0;
    CTBB_CUDA(cudaMalloc(&ctx->d_partials, n * sizeof(double)));
    ctx->partials_cap = n;
    return CTBB_OK;
}

}  // namespace ctbb

using namespace ctbb;

extern "C" ctbb_status ctbb_gpu_init(int device, void* stream, ctbb_ctx** out) {
    clear_error();
    if (!out) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    int n = 0;
    const cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
        return fail(CTBB_ERR_NO_DEVICE, "no CUDA device available (%s)", cudaGetErrorString(e));
    if (device < 0 || device >= n) return fail(CTBB_ERR_INVALID_ARG, "device %d out of range (%d devices)", device, n);
    CTBB_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    CTBB_CUDA(cudaGetDeviceProperties(&prop, device));
    ctbb_ctx* ctx = new ctbb_ctx();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    ctx->smem_per_block_optin = prop.sharedMemPerBlockOptin;
    if (stream) {
        ctx->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete ctx;
            return fail(CTBB_ERR_CUDA, "stream creation failed");
        }
        ctx->own_stream = true;
    }
    if (cudaMalloc(&ctx->d_queue, 64 * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&ctx->d_flags, 64 * sizeof(int)) != cudaSuccess) {
        ctbb_gpu_destroy(ctx);
        return fail(CTBB_ERR_OOM, "context allocation failed");
    }
    cudaMemset(ctx->d_flags, 0, 64 * sizeof(int));
    *out = ctx;
    return CTBB_OK;
}

namespace {

void teardown(ctbb_ctx* ctx) {
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->d_partials);
    cudaFree(ctx->d_queue);
    cudaFree(ctx->d_flags);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

}  // namespace

namespace ctbb {

void ctx_retain(ctbb_ctx* ctx) {
    if (ctx) ctx->refs.fetch_add(1);
}

void ctx_release(ctbb_ctx* ctx) {
    if (!ctx) return;
    if (ctx->refs.fetch_sub(1) == 1 && ctx->closing.load()) teardown(ctx);
}

}  // namespace ctbb

// Destroying a context that still has live matrices, reconstructions or
// batches only marks it; the last of them to be freed tears it down, so the
// order in which a caller (or a garbage collector) releases objects does not
// matter.
extern "C" void ctbb_gpu_destroy(ctbb_ctx* ctx) {
    if (!ctx) return;
    if (ctx->closing.exchange(true)) return;
    if (ctx->refs.load() == 0) teardown(ctx);
}

extern "C" void* ctbb_gpu_stream(ctbb_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

extern "C" ctbb_status ctbb_gpu_synchronize(ctbb_ctx* ctx) {
    clear_error();
    if (!ctx) return fail(CTBB_ERR_INVALID_ARG, "null context");
    CTBB_CUDA(cudaSetDevice(ctx->device));
    CTBB_CUDA(cudaStreamSynchronize(ctx->stream));
    return CTBB_OK;
}

// ---------------------------------------------------------------------------
// Synthetic projector: one thread per ray, phantom objects in constant memory.
// ---------------------------------------------------------------------------
namespace {

constexpr int kMaxObjects = 96;
__constant__ ctbb_object c_objects[kMaxObjects];

__global__ void __launch_bounds__(256) synth_kernel(ctbb_ray_geom G, int n_obj, uint64_t seed, double i0_lo,
                                                    double i0_hi, double clip_lo, double clip_hi,
                                                    float* __restrict__ raw) {
    const uint64_t n = (uint64_t)G.readings * G.n_channels * G.n_rows;
    for (uint64_t ray = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; ray < n;
         ray += (uint64_t)gridDim.x * blockDim.x) {
        const int64_t r = (int64_t)(ray % G.n_rows);
        const int64_t c = (int64_t)((ray / G.n_rows) % G.n_channels);
        const int64_t v = (int64_t)(ray / ((uint64_t)G.n_rows * G.n_channels));
        const double p = ctbb_line_integral(G, c_objects, n_obj, v, c, r, clip_lo, clip_hi);
        raw[ray] = ctbb_noisy_sample(p, ctbb_view_i0(seed, v, i0_lo, i0_hi), seed, ray);
    }
}

}  // namespace

extern "C" ctbb_status ctbb_gpu_synth_raw(ctbb_ctx* ctx, const ctbb_geom_c* geom, const ctbb_phantom_spec* spec,
                                          float* raw_dev) {
    clear_error();
    if (!ctx || !geom || !spec || !raw_dev) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    // The projector needs the data-view geometry of load_raw (z_first_view,
    // table direction); derive it on a copy so the caller's geometry is untouched.
    ctbb_geom_c g = *geom;
    std::vector<double> ta(g.Readings), tp(g.Readings);
    const ctbb_status st = ctbb_slice_tables(&g, ta.data(), tp.data(), nullptr, nullptr, 0);
    if (st != CTBB_OK && st != CTBB_ERR_RANGE) return st;
    clear_error();
    std::vector<ctbb_object> objs;
    ctbb_water_phantom(objs);
    if (spec->n_ellipsoids > 0)
        ctbb_random_ellipsoids(objs, spec->n_ellipsoids, spec->seed, spec->ellipsoid_z_lo, spec->ellipsoid_z_hi);
    if ((int)objs.size() > kMaxObjects) return fail(CTBB_ERR_INVALID_ARG, "too many phantom objects");
    CTBB_CUDA(cudaSetDevice(ctx->device));
    CTBB_CUDA(cudaMemcpyToSymbolAsync(c_objects, objs.data(), objs.size() * sizeof(ctbb_object), 0,
                                      cudaMemcpyHostToDevice, ctx->stream));
    const ctbb_ray_geom G = ctbb_ray_geom_from(g);
    const uint64_t n = (uint64_t)G.readings * G.n_channels * G.n_rows;
    const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)ctx->sm_count * 32));
    synth_kernel<<<grid, 256, 0, ctx->stream>>>(G, (int)objs.size(), spec->seed, spec->i0_lo, spec->i0_hi,
                                                spec->clip_z_lo, spec->clip_z_hi, raw_dev);
    CTBB_CUDA(cudaGetLastError());
    CTBB_CUDA(cudaStreamSynchronize(ctx->stream));
    return CTBB_OK;
}
