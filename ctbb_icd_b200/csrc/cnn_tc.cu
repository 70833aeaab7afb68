// Warm-start network: the 32 -> 32 channel 3x3x3 convolution on the fifth-
// generation tensor cores (tcgen05.mma, TMEM accumulator, TMA staging).
//
// Implicit GEMM per tile of 128 output voxels along x (one line, fixed y, z):
//   D[128 voxels][32 co] = sum over 27 taps of A_t[128][32 ci] . W_t[32 co][32 ci]^T
// with BF16 operands and FP32 accumulation in TMEM (128 lanes x 32 columns).
//
// Shared memory (no swizzle, K-major canonical layout: rows of 16 bytes =
// 8 channels, row r of a region at byte 16 r):
//   weights  27 taps x 4 channel chunks x 32 rows (co)          54 KB, once
//   halo x2  9 input lines (dz, dy in -1..1), each one TMA box of
//            4 chunk regions x 130 rows (x0-1 .. x0+128): the tensor map
//            orders its dimensions (8 channels, x, chunk, y, z), so the box
//            lands chunk-major, 2080 bytes per chunk, 8320 per line
//            (a multiple of 128: every box starts 128-byte aligned)  73 KB each
// Tap (dx, dy, dz) reads line (dz, dy) starting at row 1 + dx, so the 27 A
// operands are descriptors into the same halo (start address shifted by
// 16 bytes per voxel); the borders come from the TMA's zero fill.
//
// One elected thread issues the TMA loads (9 boxes per tile) and the 54
// MMAs (27 taps x 2 K-halves of 16 channels) and commits them to an
// mbarrier; all four warps then read their 32 TMEM lanes (tcgen05.ld
// 32x32b) and apply the epilogue (+ bias, + residual, zero where mask <= 0,
// relu) as conv_mid_kernel does. Halo and accumulator are double-buffered
// and the schedule is software-pipelined: the MMAs of tile i+1 are issued
// before the epilogue of tile i, and the halo of tile i+2 is loaded as soon
// as the MMAs of tile i have read theirs. Every wait on an mbarrier is
// bounded; on expiry the kernel records a code in the device error flag and
// returns after its copies have landed and its tensor memory is released.
#include <cuda.h>
#include <cuda_bf16.h>
#include <string.h>

#include <algorithm>
#include <mutex>

#include "gpu_internal.h"

namespace {

constexpr int kC = 32;
constexpr int kTaps = 27;
constexpr int kM = 128;                         // output voxels per tile
constexpr int kLine = kM + 2;                   // input voxels per halo line
constexpr int kChunkBytes = kLine * 16;         // 2080: one 8-channel chunk of a line
constexpr int kLineBytes = 4 * kChunkBytes;     // 8320: one TMA box
constexpr int kHaloBytes = 9 * kLineBytes;      // 74880
constexpr int kTapWBytes = 4 * kC * 16;         // 2048
constexpr int kWBytes = kTaps * kTapWBytes;     // 55296
constexpr int kOffHalo0 = kWBytes;
constexpr int kOffHalo1 = kOffHalo0 + kHaloBytes;
constexpr int kOffBar = kOffHalo1 + kHaloBytes;  // 4 mbarriers (load x2, mma x2)
constexpr int kOffTmem = kOffBar + 4 * 8;
constexpr int kSmemBytes = kOffTmem + 16;
constexpr int kThreads = 128;
constexpr int kTmemCols = 64;                    // two 32-column accumulators
static_assert(kLineBytes % 128 == 0 && kHaloBytes % 128 == 0 && kWBytes % 128 == 0,
              "TMA destinations (one per halo line) must stay 128-byte aligned");
static_assert(kChunkBytes % 16 == 0, "matrix descriptor offsets are in 16-byte units");
static_assert(kSmemBytes <= 227 * 1024, "shared memory per CTA");

// Instruction descriptor of tcgen05.mma kind::f16: D FP32, A and B BF16,
// both K-major, N = 32, M = 128.
constexpr uint32_t kIdesc = (1u << 4)             // D format: F32
                            | (1u << 7)           // A format: BF16
                            | (1u << 10)          // B format: BF16
                            | ((uint32_t)(kC >> 3) << 17)
                            | ((uint32_t)(kM >> 4) << 24);

// Shared-memory matrix descriptor, no swizzle, K-major: rows 16 bytes apart
// within an 8-row core matrix, `sbo` between 8-row groups, `lbo` between the
// two 8-element halves of the 16-element K step.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of this architecture
    return d;                // base offset 0, layout type 0 (no swizzle)
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: about a second of SM clock at most.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > 2000000000ll) return false;
    return true;
}

__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int c0, int c1, int c2,
                                            int c3, int c4) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
        "%6}], [%7];" ::"r"(dst),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\ntcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            d_tmem),
        "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate));
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
        "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

struct TcDims {
    int nx, ny, nz, tiles_x;
    uint64_t n_tiles;
};

__device__ __forceinline__ void tile_coords(const TcDims& d, uint64_t t, int& x0, int& y, int& z) {
    x0 = (int)(t % d.tiles_x) * kM;
    const uint64_t r = t / d.tiles_x;
    y = (int)(r % d.ny);
    z = (int)(r / d.ny);
}

// The 9 TMA boxes of one tile's halo: line (dz, dy) -> 4 chunk regions of
// rows x0-1 .. x0+128 of input line (y+dy, z+dz), 16 bytes (8 channels) each.
__device__ __forceinline__ void issue_halo(const CUtensorMap* map, uint32_t halo, uint32_t bar, const TcDims& d,
                                           uint64_t t) {
    int x0, y, z;
    tile_coords(d, t, x0, y, z);
    mbar_expect_tx(bar, (uint32_t)kHaloBytes);
#pragma unroll 1
    for (int line = 0; line < 9; ++line) {
        const int dz = line / 3 - 1, dy = line % 3 - 1;
        tma_load_5d(halo + (uint32_t)(line * kLineBytes), map, bar, 0, x0 - 1, 0, y + dy, z + dz);
    }
}

// The 54 MMAs of one tile (27 taps x 2 K-halves) into a TMEM accumulator,
// committed to an mbarrier (one thread).
__device__ __forceinline__ void issue_mmas(uint32_t d_tmem, uint32_t halo, uint32_t s_w, uint32_t bar) {
#pragma unroll 1
    for (int tap = 0; tap < kTaps; ++tap) {
        const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;  // offsets + 1
        const uint32_t a0 = halo + (uint32_t)((dz * 3 + dy) * kLineBytes + dx * 16);
        const uint32_t w0 = s_w + (uint32_t)(tap * kTapWBytes);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint64_t ad = smem_desc(a0 + (uint32_t)(2 * h * kChunkBytes), kChunkBytes, 128);
            const uint64_t bd = smem_desc(w0 + (uint32_t)(2 * h * 512), 512, 128);
            mma_bf16(d_tmem, ad, bd, (tap | h) ? 1u : 0u);
        }
    }
    mma_commit(bar);
}

__global__ void __launch_bounds__(kThreads, 1) conv_mid_tc_kernel(const __grid_constant__ CUtensorMap in_map,
                                                                  TcDims d, const __nv_bfloat16* __restrict__ wt,
                                                                  const float* __restrict__ bias,
                                                                  const __nv_bfloat16* __restrict__ residual,
                                                                  const __nv_bfloat16* __restrict__ mask, int relu,
                                                                  __nv_bfloat16* __restrict__ out, int* err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const uint32_t s_base = (uint32_t)__cvta_generic_to_shared(smem);
    const uint32_t s_w = s_base;
    auto s_halo = [&](int b) { return s_base + (uint32_t)(b ? kOffHalo1 : kOffHalo0); };
    auto bar_load = [&](int b) { return s_base + (uint32_t)(kOffBar + 8 * b); };
    auto bar_mma = [&](int b) { return s_base + (uint32_t)(kOffBar + 16 + 8 * b); };
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(smem + kOffTmem);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // Weights [tap][co][ci] -> chunk-major K-major rows: tap t, chunk c,
    // row co at 2048 t + 512 c + 16 co.
    for (int i = tid; i < kTaps * kC * 4; i += kThreads) {
        const int c = i & 3, co = (i >> 2) % kC, t = i / (4 * kC);
        const uint4 v = *reinterpret_cast<const uint4*>(wt + ((size_t)(t * kC + co) * kC + c * 8));
        *reinterpret_cast<uint4*>(smem + t * kTapWBytes + c * 512 + co * 16) = v;
    }
    if (tid == 0) {
        for (int i = 0; i < 4; ++i) mbar_init(s_base + kOffBar + 8 * i, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // Generic-proxy stores (weights) visible to the tensor cores.
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(s_tmem)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *s_tmem;
    // Every TMA destination is the halo base plus a multiple of 128 bytes:
    // refuse to issue any copy if the base itself is not 128-byte aligned.
    if (((s_base + kOffHalo0) & 127u) != 0u) {
        if (tid == 0) atomicExch(err, 2);
        fence_before();
        __syncthreads();
        fence_after();
        if (warp == 0)
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
        return;
    }

    // Phase parity of each barrier (bit b), advanced only after a completed
    // wait. A wait that runs out in any thread ends the loop in every thread
    // (__syncthreads_or), so all threads take the same barriers.
    uint32_t ph_load = 0, ph_mma = 0;
    bool aborted = false;
    const uint64_t first = blockIdx.x, step = gridDim.x;
    // Prologue: halos of the first two tiles, MMAs of the first.
    if (first < d.n_tiles) {
        if (tid == 0) {
            issue_halo(&in_map, s_halo(0), bar_load(0), d, first);
            if (first + step < d.n_tiles) issue_halo(&in_map, s_halo(1), bar_load(1), d, first + step);
        }
        const bool ok = mbar_wait(bar_load(0), 0);
        if (ok) ph_load ^= 1u;
        aborted = __syncthreads_or(!ok) != 0;
        if (!aborted) {
            fence_after();
            if (tid == 0) issue_mmas(tmem, s_halo(0), s_w, bar_mma(0));
        }
    }
    int i = 0;
    for (uint64_t t = first; t < d.n_tiles && !aborted; t += step, ++i) {
        const int b = i & 1, nb = b ^ 1;
        const uint64_t next = t + step;
        // MMAs of tile i+1 into the other accumulator (free since tile i-1's
        // epilogue), once its halo has landed.
        if (next < d.n_tiles) {
            const bool ok = mbar_wait(bar_load(nb), (ph_load >> nb) & 1);
            if (ok) ph_load ^= 1u << nb;
            if (__syncthreads_or(!ok)) {
                aborted = true;
                break;
            }
            fence_after();
            if (tid == 0) issue_mmas(tmem + (uint32_t)(nb * kC), s_halo(nb), s_w, bar_mma(nb));
        }
        // Tile i's MMAs done: its halo buffer is free for tile i+2.
        {
            const bool ok = mbar_wait(bar_mma(b), (ph_mma >> b) & 1);
            if (ok) ph_mma ^= 1u << b;
            if (__syncthreads_or(!ok)) {
                aborted = true;
                break;
            }
        }
        fence_after();
        if (tid == 0 && next + step < d.n_tiles) issue_halo(&in_map, s_halo(b), bar_load(b), d, next + step);
        // Epilogue: warp w holds voxels 32 w .. 32 w + 31 of the tile.
        float acc[kC];
        tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(b * kC), acc);
        int x0, y, z;
        tile_coords(d, t, x0, y, z);
        const int gx = x0 + 32 * warp + lane;
        if (gx < d.nx) {
            const size_t v = ((size_t)z * d.ny + y) * d.nx + gx;
            __align__(16) __nv_bfloat162 o[kC / 2];
#pragma unroll
            for (int c2 = 0; c2 < kC / 2; ++c2) {
                float v0 = acc[2 * c2] + (bias ? bias[2 * c2] : 0.f);
                float v1 = acc[2 * c2 + 1] + (bias ? bias[2 * c2 + 1] : 0.f);
                if (residual) {
                    const __nv_bfloat162 r = *reinterpret_cast<const __nv_bfloat162*>(residual + v * kC + 2 * c2);
                    v0 += __bfloat162float(r.x);
                    v1 += __bfloat162float(r.y);
                }
                if (mask) {
                    const __nv_bfloat162 m = *reinterpret_cast<const __nv_bfloat162*>(mask + v * kC + 2 * c2);
                    if (!(__bfloat162float(m.x) > 0.f)) v0 = 0.f;
                    if (!(__bfloat162float(m.y) > 0.f)) v1 = 0.f;
                }
                if (relu) {
                    v0 = fmaxf(v0, 0.f);
                    v1 = fmaxf(v1, 0.f);
                }
                o[c2] = __floats2bfloat162_rn(v0, v1);
            }
            uint4* dst = reinterpret_cast<uint4*>(out + v * kC);
            const uint4* src = reinterpret_cast<const uint4*>(o);
#pragma unroll
            for (int q = 0; q < 4; ++q) dst[q] = src[q];
        }
        fence_before();
        __syncthreads();  // TMEM buffer b read before the MMAs of tile i+2 overwrite it
    }
    if (aborted) {
        if (tid == 0) atomicExch(err, 1);
        // Let any TMA or MMA still in flight land before the memory goes away.
        for (int k = 0; k < 2; ++k) {
            mbar_wait(bar_load(k), (ph_load >> k) & 1);
            mbar_wait(bar_mma(k), (ph_mma >> k) & 1);
        }
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static std::once_flag once;
    static EncodeTiledFn fn = nullptr;
    std::call_once(once, []() {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    });
    return fn;
}

}  // namespace

namespace ctbb {

// C -> C convolution of channels-last BF16 activations `in` [nz][ny][nx][32]
// with the kernel `wt` [27][co][ci] on the tcgen05 tensor cores; epilogue as
// conv_mid_kernel. `err` (device) receives 1 if a wait ran out, 2 if shared
// memory was not aligned for the TMA copies (nothing is computed then).
ctbb_status conv_mid_tc(ctbb_ctx* ctx, int nx, int ny, int nz, const __nv_bfloat16* in, const __nv_bfloat16* wt,
                        const float* bias, const __nv_bfloat16* residual, const __nv_bfloat16* mask, int relu,
                        __nv_bfloat16* out, int* err) {
    EncodeTiledFn enc = encode_fn();
    if (!enc) return fail(CTBB_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    if (((uintptr_t)in & 15) || ((uintptr_t)out & 15) || ((uintptr_t)wt & 15))
        return fail(CTBB_ERR_INVALID_ARG, "convolution buffers must be 16-byte aligned");
    CUtensorMap map;
    memset(&map, 0, sizeof(map));
    // (8 channels, x, 4 chunks, y, z); strides of dims 1..4 in bytes. The
    // chunk dimension comes after x so that one box lands chunk-major.
    const cuuint64_t dims[5] = {8, (cuuint64_t)nx, 4, (cuuint64_t)ny, (cuuint64_t)nz};
    const cuuint64_t strides[4] = {64, 16, (cuuint64_t)64 * nx, (cuuint64_t)64 * nx * ny};
    const cuuint32_t box[5] = {8, (cuuint32_t)kLine, 4, 1, 1};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    const CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, (void*)in, dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(CTBB_ERR_CUDA, "convolution tensor map: driver error %d", (int)r);
    TcDims d;
    d.nx = nx;
    d.ny = ny;
    d.nz = nz;
    d.tiles_x = (nx + kM - 1) / kM;
    d.n_tiles = (uint64_t)d.tiles_x * ny * nz;
    if (d.n_tiles == 0) return CTBB_OK;
    static bool attr = false;
    if (!attr) {
        CTBB_CUDA(cudaFuncSetAttribute(conv_mid_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes));
        attr = true;
    }
    const int grid = (int)std::min<uint64_t>(d.n_tiles, (uint64_t)ctx->sm_count);
    conv_mid_tc_kernel<<<grid, kThreads, kSmemBytes, ctx->stream>>>(map, d, wt, bias, residual, mask, relu, out, err);
    CTBB_CUDA(cudaGetLastError());
    return CTBB_OK;
}

}  // namespace ctbb
