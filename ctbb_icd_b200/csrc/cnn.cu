// Learned warm start: a small 3D residual CNN trained and run on the GPU.
//
// Network (C = 32 channels, B residual blocks, 3x3x3 kernels, zero padding):
//   a_0     = relu(conv_in(s_in * x) + b_in)                  1 -> C
//   h_l     = relu(conv(a_l; W1_l) + b1_l)                    C -> C
//   a_{l+1} = a_l + conv(h_l; W2_l) + b2_l                    C -> C
//   out     = conv_out(a_B) + b_out                           C -> 1
// `out` is the predicted correction (converged - input) in network units;
// the physical correction is out / s_out.
//
// Activations are channels-last BF16 ([voxel][32], 64 B per voxel). The
// C -> C convolutions (forward, and backward-data with the tap-flipped,
// transposed kernel) are implicit GEMMs on the tensor cores: BF16 operands
// staged in swizzled shared memory, FP32 accumulation (mma.m16n8k16). Their
// weight gradients are GEMMs over voxels on the same units. The 1 -> C and
// C -> 1 layers are small dot products on the FP32 cores. Adam keeps FP32
// master weights and moments; every step re-derives the BF16 copies.
//
// Parameter layout (one flat FP32 array):
//   W_in[27][C], b_in[C],
//   per block l: W1[27][C][C] (tap, ci, co), b1[C], W2[27][C][C], b2[C],
//   W_out[27][C] (tap, ci), b_out[1].
// Tap t = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1) reads the input at
// (x + dx, y + dy, z + dz).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include <cuda_bf16.h>

#include "gpu_internal.h"

namespace {

constexpr int kC = 32;
constexpr int kTaps = 27;
constexpr int kConvW = kTaps * kC * kC;  // one C -> C kernel
// Output tile of the tensor-core kernels: 16 (x) by 8 (y) by 2 (z) voxels.
constexpr int kTX = 16, kTY = 8, kTZ = 2;
constexpr int kHX = kTX + 2, kHY = kTY + 2, kHZ = kTZ + 2;
constexpr int kHalo = kHX * kHY * kHZ;  // 720 voxels
constexpr int kTileVox = kTX * kTY * kTZ;
constexpr int kRowBytes = kC * 2;  // 64 B per voxel (or per kernel row)

// 16-byte chunk c of 64-byte row r lives at chunk c ^ ((r >> 1) & 3): eight
// consecutive rows then cover all 32 banks for ldmatrix.
__device__ __forceinline__ uint32_t swz(uint32_t base, int row, int chunk) {
    return base + (uint32_t)row * kRowBytes + (uint32_t)((chunk ^ ((row >> 1) & 3)) << 4);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool valid) {
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(n));
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}
__device__ __forceinline__ void mma_bf16(float* c, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

struct Dims {
    int nx, ny, nz;
    int tiles_x, tiles_y, tiles_z;
    uint64_t n_tiles;
};

Dims make_dims(int nx, int ny, int nz) {
    Dims d;
    d.nx = nx;
    d.ny = ny;
    d.nz = nz;
    d.tiles_x = (nx + kTX - 1) / kTX;
    d.tiles_y = (ny + kTY - 1) / kTY;
    d.tiles_z = (nz + kTZ - 1) / kTZ;
    d.n_tiles = (uint64_t)d.tiles_x * d.tiles_y * d.tiles_z;
    return d;
}

__device__ __forceinline__ void tile_origin(const Dims& d, uint64_t tile, int& x0, int& y0, int& z0) {
    x0 = (int)(tile % d.tiles_x) * kTX;
    const uint64_t r = tile / d.tiles_x;
    y0 = (int)(r % d.tiles_y) * kTY;
    z0 = (int)(r / d.tiles_y) * kTZ;
}

// Stage the (kHX x kHY x kHZ) input halo of a tile, zero outside the volume.
__device__ __forceinline__ void load_halo(const Dims& d, const __nv_bfloat16* __restrict__ in, uint32_t s_halo, int x0,
                                          int y0, int z0) {
    for (int idx = threadIdx.x; idx < kHalo * 4; idx += blockDim.x) {
        const int row = idx >> 2, chunk = idx & 3;
        const int hx = row % kHX, hy = (row / kHX) % kHY, hz = row / (kHX * kHY);
        const int gx = x0 + hx - 1, gy = y0 + hy - 1, gz = z0 + hz - 1;
        const bool ok = gx >= 0 && gx < d.nx && gy >= 0 && gy < d.ny && gz >= 0 && gz < d.nz;
        const uint64_t v = ok ? ((uint64_t)gz * d.ny + gy) * d.nx + gx : 0;
        cp_async16(swz(s_halo, row, chunk), in + v * kC + chunk * 8, ok);
    }
}

// C -> C convolution (tensor cores). wt is the kernel in [tap][co][ci] BF16
// order (ci contiguous). Epilogue: + bias, + residual, * (mask > 0), relu.
// Persistent CTAs of 8 warps; warp w owns output rows 2w and 2w+1 of the
// tile (row r = y + kTY * z), 16 voxels along x each.
__global__ void __launch_bounds__(256) conv_mid_kernel(Dims d, const __nv_bfloat16* __restrict__ in,
                                                       const __nv_bfloat16* __restrict__ wt,
                                                       const float* __restrict__ bias,
                                                       const __nv_bfloat16* __restrict__ residual,
                                                       const __nv_bfloat16* __restrict__ mask, int relu,
                                                       __nv_bfloat16* __restrict__ out) {
    extern __shared__ __align__(128) unsigned char smem[];
    const uint32_t s_w = (uint32_t)__cvta_generic_to_shared(smem);
    const uint32_t s_halo = s_w + kTaps * kC * kRowBytes;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // Kernel rows (tap, co) with swizzled 16-byte chunks, loaded once.
    for (int idx = threadIdx.x; idx < kTaps * kC * 4; idx += blockDim.x) {
        const int row = idx >> 2, chunk = idx & 3;
        cp_async16(swz(s_w, row, chunk), wt + (uint64_t)row * kC + chunk * 8, true);
    }
    float bv[4][2];
#pragma unroll
    for (int n = 0; n < 4; ++n) {
        const int co = n * 8 + (lane & 3) * 2;
        bv[n][0] = bias ? bias[co] : 0.f;
        bv[n][1] = bias ? bias[co + 1] : 0.f;
    }
    const int r0 = 2 * warp;
    const int oz = r0 / kTY;
    for (uint64_t tile = blockIdx.x; tile < d.n_tiles; tile += gridDim.x) {
        int x0, y0, z0;
        tile_origin(d, tile, x0, y0, z0);
        __syncthreads();  // previous tile's halo fully consumed
        load_halo(d, in, s_halo, x0, y0, z0);
        cp_async_wait_all();
        __syncthreads();
        float acc[2][4][4];
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int n = 0; n < 4; ++n)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[j][n][q] = 0.f;
        for (int t = 0; t < kTaps; ++t) {
            const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;  // offsets + 1
#pragma unroll
            for (int kk = 0; kk < 2; ++kk) {
                uint32_t b[4][2];
#pragma unroll
                for (int p = 0; p < 2; ++p) {
                    const int row = t * kC + p * 16 + ((lane >> 4) << 3) + (lane & 7);
                    const int chunk = kk * 2 + ((lane >> 3) & 1);
                    ldsm_x4(swz(s_w, row, chunk), b[2 * p][0], b[2 * p][1], b[2 * p + 1][0], b[2 * p + 1][1]);
                }
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const int oy = (r0 + j) % kTY;
                    const int hrow = ((oz + dz) * kHY + (oy + dy)) * kHX + dx + ((lane >> 3) & 1) * 8 + (lane & 7);
                    const int chunk = kk * 2 + (lane >> 4);
                    uint32_t a0, a1, a2, a3;
                    ldsm_x4(swz(s_halo, hrow, chunk), a0, a1, a2, a3);
#pragma unroll
                    for (int n = 0; n < 4; ++n) mma_bf16(acc[j][n], a0, a1, a2, a3, b[n][0], b[n][1]);
                }
            }
        }
        // Epilogue: thread holds voxels x0 + g and x0 + g + 8 of rows r0, r0+1,
        // channels n*8 + 2*(lane&3) + {0,1}.
        const int gz = z0 + oz;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int gy = y0 + (r0 + j) % kTY;
#pragma unroll
            for (int hh = 0; hh < 2; ++hh) {
                const int gx = x0 + (lane >> 2) + hh * 8;
                if (gx >= d.nx || gy >= d.ny || gz >= d.nz) continue;
                const uint64_t v = ((uint64_t)gz * d.ny + gy) * d.nx + gx;
#pragma unroll
                for (int n = 0; n < 4; ++n) {
                    const int co = n * 8 + (lane & 3) * 2;
                    float v0 = acc[j][n][hh * 2] + bv[n][0];
                    float v1 = acc[j][n][hh * 2 + 1] + bv[n][1];
                    if (residual) {
                        const __nv_bfloat162 r = *reinterpret_cast<const __nv_bfloat162*>(residual + v * kC + co);
                        v0 += __bfloat162float(r.x);
                        v1 += __bfloat162float(r.y);
                    }
                    if (mask) {
                        const __nv_bfloat162 m = *reinterpret_cast<const __nv_bfloat162*>(mask + v * kC + co);
                        if (!(__bfloat162float(m.x) > 0.f)) v0 = 0.f;
                        if (!(__bfloat162float(m.y) > 0.f)) v1 = 0.f;
                    }
                    if (relu) {
                        v0 = fmaxf(v0, 0.f);
                        v1 = fmaxf(v1, 0.f);
                    }
                    *reinterpret_cast<__nv_bfloat162*>(out + v * kC + co) = __floats2bfloat162_rn(v0, v1);
                }
            }
        }
    }
}

// Weight gradient of a C -> C convolution (tensor cores):
//   dW[t][ci][co] += sum_v X[v + off(t)][ci] * dY[v][co].
// Work unit u = (tap t = u / 2, ci half u % 2); warp w owns units w, w+8, ...
// Per-CTA FP32 partials are added to dw with atomics once at the end.
constexpr int kUnitsPerWarp = 7;  // ceil(54 / 8)

__global__ void __launch_bounds__(256) conv_wgrad_kernel(Dims d, const __nv_bfloat16* __restrict__ x,
                                                         const __nv_bfloat16* __restrict__ dy,
                                                         float* __restrict__ dw) {
    extern __shared__ __align__(128) unsigned char smem[];
    const uint32_t s_halo = (uint32_t)__cvta_generic_to_shared(smem);
    const uint32_t s_dy = s_halo + kHalo * kRowBytes;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float acc[kUnitsPerWarp][4][4];
#pragma unroll
    for (int u = 0; u < kUnitsPerWarp; ++u)
#pragma unroll
        for (int n = 0; n < 4; ++n)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[u][n][q] = 0.f;
    for (uint64_t tile = blockIdx.x; tile < d.n_tiles; tile += gridDim.x) {
        int x0, y0, z0;
        tile_origin(d, tile, x0, y0, z0);
        __syncthreads();
        load_halo(d, x, s_halo, x0, y0, z0);
        for (int idx = threadIdx.x; idx < kTileVox * 4; idx += blockDim.x) {
            const int row = idx >> 2, chunk = idx & 3;
            const int tx = row % kTX, ty = (row / kTX) % kTY, tz = row / (kTX * kTY);
            const int gx = x0 + tx, gy = y0 + ty, gz = z0 + tz;
            const bool ok = gx < d.nx && gy < d.ny && gz < d.nz;
            const uint64_t v = ok ? ((uint64_t)gz * d.ny + gy) * d.nx + gx : 0;
            cp_async16(swz(s_dy, row, chunk), dy + v * kC + chunk * 8, ok);
        }
        cp_async_wait_all();
        __syncthreads();
        for (int ks = 0; ks < kTY * kTZ; ++ks) {  // 16 voxels along x per step
            const int oy = ks % kTY, oz = ks / kTY;
            uint32_t b[4][2];
#pragma unroll
            for (int p = 0; p < 2; ++p) {
                const int mi = lane >> 3;
                const int row = ks * kTX + (mi & 1) * 8 + (lane & 7);
                const int chunk = p * 2 + (mi >> 1);
                ldsm_x4_t(swz(s_dy, row, chunk), b[2 * p][0], b[2 * p][1], b[2 * p + 1][0], b[2 * p + 1][1]);
            }
#pragma unroll
            for (int u = 0; u < kUnitsPerWarp; ++u) {
                const int unit = warp + 8 * u;
                if (unit >= 2 * kTaps) break;
                const int t = unit >> 1, mt = unit & 1;
                const int dz = t / 9, dy_ = (t / 3) % 3, dx = t % 3;
                const int mi = lane >> 3;
                const int hrow = ((oz + dz) * kHY + (oy + dy_)) * kHX + dx + (mi >> 1) * 8 + (lane & 7);
                const int chunk = mt * 2 + (mi & 1);
                uint32_t a0, a1, a2, a3;
                ldsm_x4_t(swz(s_halo, hrow, chunk), a0, a1, a2, a3);
#pragma unroll
                for (int n = 0; n < 4; ++n) mma_bf16(acc[u][n], a0, a1, a2, a3, b[n][0], b[n][1]);
            }
        }
    }
#pragma unroll
    for (int u = 0; u < kUnitsPerWarp; ++u) {
        const int unit = warp + 8 * u;
        if (unit >= 2 * kTaps) break;
        const int t = unit >> 1, mt = unit & 1;
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            const int co = n * 8 + (lane & 3) * 2;
            const int ci = mt * 16 + (lane >> 2);
            float* p0 = dw + ((uint64_t)t * kC + ci) * kC + co;
            float* p1 = dw + ((uint64_t)t * kC + ci + 8) * kC + co;
            atomicAdd(p0, acc[u][n][0]);
            atomicAdd(p0 + 1, acc[u][n][1]);
            atomicAdd(p1, acc[u][n][2]);
            atomicAdd(p1 + 1, acc[u][n][3]);
        }
    }
}

__device__ __forceinline__ bool inside(int x, int y, int z, int nx, int ny, int nz) {
    return x >= 0 && x < nx && y >= 0 && y < ny && z >= 0 && z < nz;
}

// a_0 = relu(conv_in(s_in * x) + b_in): one thread per voxel, 32 outputs.
// w holds W_in[27][C] followed by b_in[C].
__global__ void __launch_bounds__(256) conv_in_kernel(int nx, int ny, int nz, const float* __restrict__ x,
                                                      float s_in, const float* __restrict__ w,
                                                      __nv_bfloat16* __restrict__ out) {
    __shared__ float sw[kTaps * kC + kC];
    for (int i = threadIdx.x; i < kTaps * kC + kC; i += blockDim.x) sw[i] = w[i];
    __syncthreads();
    const uint64_t n = (uint64_t)nx * ny * nz;
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
        const int ix = (int)(v % nx), iy = (int)((v / nx) % ny), iz = (int)(v / ((uint64_t)nx * ny));
        float acc[kC];
#pragma unroll
        for (int c = 0; c < kC; ++c) acc[c] = sw[kTaps * kC + c];
        for (int t = 0; t < kTaps; ++t) {
            const int jx = ix + t % 3 - 1, jy = iy + (t / 3) % 3 - 1, jz = iz + t / 9 - 1;
            if (!inside(jx, jy, jz, nx, ny, nz)) continue;
            const float xv = s_in * x[((uint64_t)jz * ny + jy) * nx + jx];
#pragma unroll
            for (int c = 0; c < kC; ++c) acc[c] = fmaf(xv, sw[t * kC + c], acc[c]);
        }
        __nv_bfloat162* o = reinterpret_cast<__nv_bfloat162*>(out + v * kC);
#pragma unroll
        for (int c = 0; c < kC; c += 2) o[c / 2] = __floats2bfloat162_rn(fmaxf(acc[c], 0.f), fmaxf(acc[c + 1], 0.f));
    }
}

// out[v] = b_out + sum_t sum_ci a[v + off(t)][ci] * W_out[t][ci]; w holds
// W_out[27][C] followed by b_out.
__global__ void __launch_bounds__(256) conv_out_kernel(int nx, int ny, int nz, const __nv_bfloat16* __restrict__ a,
                                                       const float* __restrict__ w, float* __restrict__ out) {
    __shared__ float sw[kTaps * kC + 1];
    for (int i = threadIdx.x; i < kTaps * kC + 1; i += blockDim.x) sw[i] = w[i];
    __syncthreads();
    const uint64_t n = (uint64_t)nx * ny * nz;
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
        const int ix = (int)(v % nx), iy = (int)((v / nx) % ny), iz = (int)(v / ((uint64_t)nx * ny));
        float acc = sw[kTaps * kC];
        for (int t = 0; t < kTaps; ++t) {
            const int jx = ix + t % 3 - 1, jy = iy + (t / 3) % 3 - 1, jz = iz + t / 9 - 1;
            if (!inside(jx, jy, jz, nx, ny, nz)) continue;
            const uint4* p = reinterpret_cast<const uint4*>(a + (((uint64_t)jz * ny + jy) * nx + jx) * kC);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint4 u = __ldg(p + q);
                const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const float2 f = __bfloat1622float2(h[e]);
                    acc = fmaf(f.x, sw[t * kC + q * 8 + 2 * e], acc);
                    acc = fmaf(f.y, sw[t * kC + q * 8 + 2 * e + 1], acc);
                }
            }
        }
        out[v] = acc;
    }
}

// Weighted squared error against the target (xc - x) * s_out and its
// gradient: loss = sum m (out - t)^2 / sum m, dout = 2 m (out - t) / sum m.
__global__ void __launch_bounds__(256) loss_kernel(uint64_t n, const float* __restrict__ out,
                                                   const float* __restrict__ x, const float* __restrict__ xc,
                                                   const float* __restrict__ m, float s_out, double inv_wsum,
                                                   float* __restrict__ dout, double* __restrict__ partials) {
    __shared__ double sh[8];
    double s = 0.0;
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
        const float wv = m ? m[v] : 1.f;
        const float r = out[v] - (xc[v] - x[v]) * s_out;
        s += (double)wv * r * r;
        dout[v] = (float)(2.0 * inv_wsum) * wv * r;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += sh[i];
        partials[blockIdx.x] = t * inv_wsum;
    }
}

// Sum of the loss weights, per block, for the normaliser.
__global__ void __launch_bounds__(256) weight_sum_kernel(uint64_t n, const float* __restrict__ m,
                                                         double* __restrict__ partials) {
    __shared__ double sh[8];
    double s = 0.0;
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
        s += (double)m[v];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += sh[i];
        partials[blockIdx.x] = t;
    }
}

// g[v][ci] = sum_t dout[v - off(t)] * W_out[t][ci] (backward data of conv_out).
__global__ void __launch_bounds__(256) conv_out_bwd_kernel(int nx, int ny, int nz, const float* __restrict__ dout,
                                                           const float* __restrict__ w,
                                                           __nv_bfloat16* __restrict__ g) {
    __shared__ float sw[kTaps * kC];
    for (int i = threadIdx.x; i < kTaps * kC; i += blockDim.x) sw[i] = w[i];
    __syncthreads();
    const uint64_t n = (uint64_t)nx * ny * nz;
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
        const int ix = (int)(v % nx), iy = (int)((v / nx) % ny), iz = (int)(v / ((uint64_t)nx * ny));
        float acc[kC];
#pragma unroll
        for (int c = 0; c < kC; ++c) acc[c] = 0.f;
        for (int t = 0; t < kTaps; ++t) {
            const int jx = ix - (t % 3 - 1), jy = iy - ((t / 3) % 3 - 1), jz = iz - (t / 9 - 1);
            if (!inside(jx, jy, jz, nx, ny, nz)) continue;
            const float dv = dout[((uint64_t)jz * ny + jy) * nx + jx];
#pragma unroll
            for (int c = 0; c < kC; ++c) acc[c] = fmaf(dv, sw[t * kC + c], acc[c]);
        }
        __nv_bfloat162* o = reinterpret_cast<__nv_bfloat162*>(g + v * kC);
#pragma unroll
        for (int c = 0; c < kC; c += 2) o[c / 2] = __floats2bfloat162_rn(acc[c], acc[c + 1]);
    }
}

// Weight gradients of the 1-channel layers. Thread (tq, c) of a 288-thread
// block owns taps tq, tq + 9, tq + 18 of channel c and sums over a chunk of
// voxels; per-block sums go to dw with atomics.
//   mode 0 (conv_out): dw[t][c] += sum_v a[v + off(t)][c] * dout[v];  dw[27*32] += sum dout
//   mode 1 (conv_in):  dw[t][c] += sum_v s_in x[v + off(t)] * g[v][c] * (a0[v][c] > 0);
//                      dw[27*32 + c] += sum_v g[v][c] * (a0[v][c] > 0)
constexpr int kWg1Threads = 288;
constexpr int kWg1Chunk = 1024;

__global__ void __launch_bounds__(kWg1Threads) wgrad_1ch_kernel(int mode, int nx, int ny, int nz,
                                                                 const __nv_bfloat16* __restrict__ act,
                                                                 const float* __restrict__ scal, float s_in,
                                                                 const __nv_bfloat16* __restrict__ mask,
                                                                 float* __restrict__ dw) {
    const int c = threadIdx.x & 31, tq = threadIdx.x >> 5;
    const uint64_t n = (uint64_t)nx * ny * nz;
    float acc[3] = {0.f, 0.f, 0.f};
    float accb = 0.f;
    const uint64_t v0 = (uint64_t)blockIdx.x * kWg1Chunk;
    const uint64_t v1 = min(n, v0 + kWg1Chunk);
    for (uint64_t v = v0; v < v1; ++v) {
        const int ix = (int)(v % nx), iy = (int)((v / nx) % ny), iz = (int)(v / ((uint64_t)nx * ny));
        if (mode == 0) {
            const float dv = scal[v];
            if (tq == 0 && c == 0) accb += dv;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const int t = tq + 9 * q;
                const int jx = ix + t % 3 - 1, jy = iy + (t / 3) % 3 - 1, jz = iz + t / 9 - 1;
                if (!inside(jx, jy, jz, nx, ny, nz)) continue;
                acc[q] = fmaf(__bfloat162float(act[(((uint64_t)jz * ny + jy) * nx + jx) * kC + c]), dv, acc[q]);
            }
        } else {
            float gv = __bfloat162float(act[v * kC + c]);
            if (!(__bfloat162float(mask[v * kC + c]) > 0.f)) gv = 0.f;
            if (tq == 0) accb += gv;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const int t = tq + 9 * q;
                const int jx = ix + t % 3 - 1, jy = iy + (t / 3) % 3 - 1, jz = iz + t / 9 - 1;
                if (!inside(jx, jy, jz, nx, ny, nz)) continue;
                acc[q] = fmaf(s_in * scal[((uint64_t)jz * ny + jy) * nx + jx], gv, acc[q]);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) atomicAdd(dw + (tq + 9 * q) * kC + c, acc[q]);
    if (mode == 0 && tq == 0 && c == 0) atomicAdd(dw + kTaps * kC, accb);
    if (mode == 1 && tq == 0) atomicAdd(dw + kTaps * kC + c, accb);
}

// db[c] += sum_v dy[v][c].
__global__ void __launch_bounds__(256) bias_grad_kernel(uint64_t n, const __nv_bfloat16* __restrict__ dy,
                                                        float* __restrict__ db) {
    __shared__ float sh[8][kC];
    const int c = threadIdx.x & 31, r = threadIdx.x >> 5;
    float s = 0.f;
    for (uint64_t v = blockIdx.x * 8ull + r; v < n; v += gridDim.x * 8ull) s += __bfloat162float(dy[v * kC + c]);
    sh[r][c] = s;
    __syncthreads();
    if (r == 0) {
        for (int i = 1; i < 8; ++i) s += sh[i][c];
        atomicAdd(db + c, s);
    }
}

__global__ void adam_kernel(uint64_t n, float* __restrict__ p, float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2,
                            float gscale) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const float gi = g[i] * gscale;
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        g[i] = 0.f;
    }
}

// BF16 kernels of each C -> C convolution: forward [t][co][ci] and backward
// data [t][ci][co] with the tap flipped (off(26 - t) = -off(t)).
__global__ void prep_weights_kernel(int n_conv, const float* __restrict__ params, const uint64_t* __restrict__ offs,
                                    __nv_bfloat16* __restrict__ wf, __nv_bfloat16* __restrict__ wb) {
    const uint64_t n = (uint64_t)n_conv * kConvW;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const int l = (int)(i / kConvW);
        const int r = (int)(i % kConvW);
        const int t = r / (kC * kC), ci = (r / kC) % kC, co = r % kC;
        const float w = params[offs[l] + r];
        wf[(uint64_t)l * kConvW + ((uint64_t)t * kC + co) * kC + ci] = __float2bfloat16_rn(w);
        wb[(uint64_t)l * kConvW + ((uint64_t)(kTaps - 1 - t) * kC + ci) * kC + co] = __float2bfloat16_rn(w);
    }
}

// x_new = max(0, x + d); prio = |x_new - x| (the step the warm start took).
__global__ void apply_correction_kernel(uint64_t n, float* __restrict__ x, const float* __restrict__ d,
                                        float* __restrict__ prio) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const float xo = x[i];
        const float xn = fmaxf(0.f, xo + d[i]);
        x[i] = xn;
        if (prio) prio[i] = fabsf(xn - xo);
    }
}

__global__ void scale_copy_kernel(uint64_t n, const float* __restrict__ a, float* __restrict__ b, float s) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        b[i] = a[i] * s;
}

uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

}  // namespace

struct ctbb_cnn {
    ctbb_ctx* ctx = nullptr;
    int blocks = 0;
    uint64_t n_params = 0;
    // Offsets into the flat parameter array.
    uint64_t off_win = 0, off_bin = 0, off_wout = 0, off_bout = 0;
    std::vector<uint64_t> off_w, off_b;  // per C -> C conv (2 per block)
    float s_in = 1.f, s_out = 1.f;
    long adam_t = 0;
    float *d_p = nullptr, *d_g = nullptr, *d_m = nullptr, *d_v = nullptr;
    uint64_t* d_offs = nullptr;
    __nv_bfloat16 *d_wf = nullptr, *d_wb = nullptr;
    bool weights_dirty = true;
    // C -> C convolutions: CTBB_CNN_ENGINE_TCGEN05 (cnn_tc.cu) or
    // CTBB_CNN_ENGINE_MMA_SYNC (conv_mid_kernel below).
    int engine = CTBB_CNN_ENGINE_MMA_SYNC;
    // Activation workspace, grown on demand: a_0..a_B, h_0..h_{B-1}, two
    // gradient buffers and du.
    uint64_t cap = 0;
    __nv_bfloat16* d_act = nullptr;
    float* d_out = nullptr;
    float* d_dout = nullptr;
    __nv_bfloat16* a(int l) { return d_act + (uint64_t)l * cap * kC; }
    __nv_bfloat16* h(int l) { return d_act + (uint64_t)(blocks + 1 + l) * cap * kC; }
    __nv_bfloat16* gbuf(int i) { return d_act + (uint64_t)(2 * blocks + 1 + i) * cap * kC; }
    __nv_bfloat16* du() { return d_act + (uint64_t)(2 * blocks + 3) * cap * kC; }
    int n_act() const { return 2 * blocks + 4; }
};

namespace {

using namespace ctbb;

constexpr size_t kMidSmem = (size_t)kTaps * kC * kRowBytes + (size_t)kHalo * kRowBytes;  // 101,376 B
constexpr size_t kWgSmem = (size_t)kHalo * kRowBytes + (size_t)kTileVox * kRowBytes;      // 62,464 B

ctbb_status ensure_workspace(ctbb_cnn* c, uint64_t nvox) {
    if (c->cap >= nvox) return CTBB_OK;
    cudaFree(c->d_act);
    cudaFree(c->d_out);
    cudaFree(c->d_dout);
    c->d_act = nullptr;
    c->d_out = c->d_dout = nullptr;
    c->cap = 0;
    CTBB_CUDA(cudaMalloc(&c->d_act, (uint64_t)c->n_act() * nvox * kC * sizeof(__nv_bfloat16)));
    CTBB_CUDA(cudaMalloc(&c->d_out, nvox * sizeof(float)));
    CTBB_CUDA(cudaMalloc(&c->d_dout, nvox * sizeof(float)));
    c->cap = nvox;
    return CTBB_OK;
}

int grid1(const ctbb_ctx* ctx, uint64_t n, int per_sm = 8) {
    return (int)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)ctx->sm_count * per_sm));
}

ctbb_status configure_kernels(int device) {
    static thread_local int configured_device = -1;
    if (configured_device == device) return CTBB_OK;
    CTBB_CUDA(cudaFuncSetAttribute(conv_mid_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMidSmem));
    CTBB_CUDA(cudaFuncSetAttribute(conv_wgrad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWgSmem));
    configured_device = device;
    return CTBB_OK;
}

ctbb_status prep_weights(ctbb_cnn* c) {
    if (!c->weights_dirty) return CTBB_OK;
    const int n_conv = 2 * c->blocks;
    if (n_conv > 0) {
        prep_weights_kernel<<<grid1(c->ctx, (uint64_t)n_conv * kConvW), 256, 0, c->ctx->stream>>>(
            n_conv, c->d_p, c->d_offs, c->d_wf, c->d_wb);
        CTBB_CUDA(cudaGetLastError());
    }
    c->weights_dirty = false;
    return CTBB_OK;
}

ctbb_status conv_mid(ctbb_cnn* c, const Dims& d, const __nv_bfloat16* in, const __nv_bfloat16* wt, const float* bias,
                     const __nv_bfloat16* residual, const __nv_bfloat16* mask, int relu, __nv_bfloat16* out) {
    if (c->engine == CTBB_CNN_ENGINE_TCGEN05)
        return conv_mid_tc(c->ctx, d.nx, d.ny, d.nz, in, wt, bias, residual, mask, relu, out, c->ctx->d_flags + 1);
    CTBB_TRY(configure_kernels(c->ctx->device));
    const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>(d.n_tiles, (uint64_t)c->ctx->sm_count * 2));
    conv_mid_kernel<<<grid, 256, kMidSmem, c->ctx->stream>>>(d, in, wt, bias, residual, mask, relu, out);
    CTBB_CUDA(cudaGetLastError());
    return CTBB_OK;
}

// After a synchronised call: a tensor-core convolution whose mbarrier wait
// ran out leaves 1 in the context's error flag 1 (cnn_tc.cu).
ctbb_status check_conv_flag(ctbb_cnn* c) {
    int h = 0;
    CTBB_CUDA(cudaMemcpy(&h, c->ctx->d_flags + 1, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) {
        CTBB_CUDA(cudaMemset(c->ctx->d_flags + 1, 0, sizeof(int)));
        if (h == 2) return fail(CTBB_ERR_CUDA, "tensor-core convolution: shared memory not aligned for its copies");
        return fail(CTBB_ERR_TIMEOUT, "tensor-core convolution: a wait for its loads or products expired");
    }
    return CTBB_OK;
}

ctbb_status conv_wgrad(ctbb_cnn* c, const Dims& d, const __nv_bfloat16* x, const __nv_bfloat16* dy, float* dw) {
    CTBB_TRY(configure_kernels(c->ctx->device));
    const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>(d.n_tiles, (uint64_t)c->ctx->sm_count * 2));
    conv_wgrad_kernel<<<grid, 256, kWgSmem, c->ctx->stream>>>(d, x, dy, dw);
    CTBB_CUDA(cudaGetLastError());
    return CTBB_OK;
}

ctbb_status forward(ctbb_cnn* c, const float* x, int nx, int ny, int nz) {
    const uint64_t n = (uint64_t)nx * ny * nz;
    CTBB_TRY(ensure_workspace(c, n));
    CTBB_TRY(prep_weights(c));
    const Dims d = make_dims(nx, ny, nz);
    cudaStream_t st = c->ctx->stream;
    conv_in_kernel<<<grid1(c->ctx, n), 256, 0, st>>>(nx, ny, nz, x, c->s_in, c->d_p + c->off_win, c->a(0));
    CTBB_CUDA(cudaGetLastError());
    for (int l = 0; l < c->blocks; ++l) {
        CTBB_TRY(conv_mid(c, d, c->a(l), c->d_wf + (uint64_t)(2 * l) * kConvW, c->d_p + c->off_b[2 * l], nullptr,
                          nullptr, 1, c->h(l)));
        CTBB_TRY(conv_mid(c, d, c->h(l), c->d_wf + (uint64_t)(2 * l + 1) * kConvW, c->d_p + c->off_b[2 * l + 1],
                          c->a(l), nullptr, 0, c->a(l + 1)));
    }
    conv_out_kernel<<<grid1(c->ctx, n), 256, 0, st>>>(nx, ny, nz, c->a(c->blocks), c->d_p + c->off_wout, c->d_out);
    CTBB_CUDA(cudaGetLastError());
    return CTBB_OK;
}

ctbb_status reduce(ctbb_ctx* ctx, int nb, double* out) {
    std::vector<double> h(nb);
    CTBB_CUDA(cudaMemcpyAsync(h.data(), ctx->d_partials, nb * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CTBB_CUDA(cudaStreamSynchronize(ctx->stream));
    double s = 0.0;
    for (double v : h) s += v;
    *out = s;
    return CTBB_OK;
}

}  // namespace

extern "C" ctbb_status ctbb_cnn_create(ctbb_ctx* ctx, int32_t blocks, uint64_t seed, ctbb_cnn** out) {
    clear_error();
    if (!ctx || !out) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    if (blocks < 0 || blocks > 16) return fail(CTBB_ERR_INVALID_ARG, "blocks must be in [0, 16] (got %d)", blocks);
    CTBB_CUDA(cudaSetDevice(ctx->device));
    ctbb_cnn* c = new ctbb_cnn();
    struct Guard {
        ctbb_cnn* c;
        ~Guard() {
            if (c) ctbb_cnn_free(c);
        }
    } guard{c};
    c->ctx = ctx;
    ctx_retain(ctx);
    c->blocks = blocks;
    uint64_t o = 0;
    c->off_win = o;
    o += kTaps * kC;
    c->off_bin = o;
    o += kC;
    for (int l = 0; l < 2 * blocks; ++l) {
        c->off_w.push_back(o);
        o += kConvW;
        c->off_b.push_back(o);
        o += kC;
    }
    c->off_wout = o;
    o += kTaps * kC;
    c->off_bout = o;
    o += 1;
    c->n_params = o;
    // He-style uniform initialisation; the second convolution of each block
    // and the output layer start small, so the network starts near a zero
    // correction with every block near the identity.
    std::vector<float> p(o, 0.f);
    uint64_t s = seed * 0x2545f4914f6cdd1dull + 1;
    auto uni = [&](float bound) {
        const double u = (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
        return (float)((2.0 * u - 1.0) * bound);
    };
    for (int i = 0; i < kTaps * kC; ++i) p[c->off_win + i] = uni(sqrtf(6.f / kTaps));
    for (int l = 0; l < 2 * blocks; ++l) {
        const float bound = sqrtf(6.f / (kTaps * kC)) * ((l & 1) ? 0.1f : 1.f);
        for (int i = 0; i < kConvW; ++i) p[c->off_w[l] + i] = uni(bound);
    }
    for (int i = 0; i < kTaps * kC; ++i) p[c->off_wout + i] = uni(0.1f * sqrtf(6.f / (kTaps * kC)));
    CTBB_CUDA(cudaMalloc(&c->d_p, o * sizeof(float)));
    CTBB_CUDA(cudaMalloc(&c->d_g, o * sizeof(float)));
    CTBB_CUDA(cudaMalloc(&c->d_m, o * sizeof(float)));
    CTBB_CUDA(cudaMalloc(&c->d_v, o * sizeof(float)));
    const size_t nw = std::max<size_t>(1, (size_t)2 * blocks) * kConvW;
    CTBB_CUDA(cudaMalloc(&c->d_wf, nw * sizeof(__nv_bfloat16)));
    CTBB_CUDA(cudaMalloc(&c->d_wb, nw * sizeof(__nv_bfloat16)));
    CTBB_CUDA(cudaMalloc(&c->d_offs, std::max<size_t>(1, c->off_w.size()) * sizeof(uint64_t)));
    cudaStream_t st = ctx->stream;
    CTBB_CUDA(cudaMemcpyAsync(c->d_p, p.data(), o * sizeof(float), cudaMemcpyHostToDevice, st));
    if (!c->off_w.empty())
        CTBB_CUDA(cudaMemcpyAsync(c->d_offs, c->off_w.data(), c->off_w.size() * sizeof(uint64_t),
                                  cudaMemcpyHostToDevice, st));
    CTBB_CUDA(cudaMemsetAsync(c->d_g, 0, o * sizeof(float), st));
    CTBB_CUDA(cudaMemsetAsync(c->d_m, 0, o * sizeof(float), st));
    CTBB_CUDA(cudaMemsetAsync(c->d_v, 0, o * sizeof(float), st));
    CTBB_CUDA(cudaStreamSynchronize(st));
    guard.c = nullptr;
    *out = c;
    return CTBB_OK;
}

extern "C" void ctbb_cnn_free(ctbb_cnn* c) {
    if (!c) return;
    if (c->ctx) {
        cudaSetDevice(c->ctx->device);
        cudaStreamSynchronize(c->ctx->stream);
    }
    cudaFree(c->d_p);
    cudaFree(c->d_g);
    cudaFree(c->d_m);
    cudaFree(c->d_v);
    cudaFree(c->d_wf);
    cudaFree(c->d_wb);
    cudaFree(c->d_offs);
    cudaFree(c->d_act);
    cudaFree(c->d_out);
    cudaFree(c->d_dout);
    ctx_release(c->ctx);
    delete c;
}

extern "C" uint64_t ctbb_cnn_num_params(const ctbb_cnn* c) { return c ? c->n_params : 0; }

extern "C" ctbb_status ctbb_cnn_get_params(ctbb_cnn* c, float* host, uint64_t n) {
    clear_error();
    if (!c || !host) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (n != c->n_params) return fail(CTBB_ERR_INVALID_ARG, "expected %llu parameters", (unsigned long long)c->n_params);
    CTBB_CUDA(cudaSetDevice(c->ctx->device));
    CTBB_CUDA(cudaMemcpyAsync(host, c->d_p, n * sizeof(float), cudaMemcpyDeviceToHost, c->ctx->stream));
    CTBB_CUDA(cudaStreamSynchronize(c->ctx->stream));
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_cnn_set_params(ctbb_cnn* c, const float* host, uint64_t n) {
    clear_error();
    if (!c || !host) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (n != c->n_params) return fail(CTBB_ERR_INVALID_ARG, "expected %llu parameters", (unsigned long long)c->n_params);
    CTBB_CUDA(cudaSetDevice(c->ctx->device));
    CTBB_CUDA(cudaMemcpyAsync(c->d_p, host, n * sizeof(float), cudaMemcpyHostToDevice, c->ctx->stream));
    CTBB_CUDA(cudaStreamSynchronize(c->ctx->stream));
    c->weights_dirty = true;
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_cnn_set_scaling(ctbb_cnn* c, float s_in, float s_out) {
    clear_error();
    if (!c) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (!(s_in > 0.f) || !(s_out > 0.f)) return fail(CTBB_ERR_INVALID_ARG, "scales must be positive");
    c->s_in = s_in;
    c->s_out = s_out;
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_cnn_get_scaling(const ctbb_cnn* c, float* s_in, float* s_out) {
    clear_error();
    if (!c || !s_in || !s_out) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    *s_in = c->s_in;
    *s_out = c->s_out;
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_cnn_forward(ctbb_cnn* c, const float* x_dev, int32_t nx, int32_t ny, int32_t nz,
                                        float* out_dev) {
    clear_error();
    if (!c || !x_dev || !out_dev) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (nx <= 0 || ny <= 0 || nz <= 0) return fail(CTBB_ERR_INVALID_ARG, "empty volume");
    CTBB_CUDA(cudaSetDevice(c->ctx->device));
    CTBB_TRY(forward(c, x_dev, nx, ny, nz));
    const uint64_t n = (uint64_t)nx * ny * nz;
    CTBB_CUDA(cudaMemcpyAsync(out_dev, c->d_out, n * sizeof(float), cudaMemcpyDeviceToDevice, c->ctx->stream));
    CTBB_CUDA(cudaStreamSynchronize(c->ctx->stream));
    return check_conv_flag(c);
}

extern "C" ctbb_status ctbb_cnn_set_engine(ctbb_cnn* c, int32_t engine) {
    clear_error();
    if (!c) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (engine != CTBB_CNN_ENGINE_TCGEN05 && engine != CTBB_CNN_ENGINE_MMA_SYNC)
        return fail(CTBB_ERR_INVALID_ARG, "unknown convolution engine %d", engine);
    c->engine = engine;
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_cnn_accumulate_gradient(ctbb_cnn* c, const float* x_dev, const float* xc_dev,
                                                    const float* weight_dev, int32_t nx, int32_t ny, int32_t nz,
                                                    double* loss) {
    clear_error();
    if (!c || !x_dev || !xc_dev) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (nx <= 0 || ny <= 0 || nz <= 0) return fail(CTBB_ERR_INVALID_ARG, "empty volume");
    CTBB_CUDA(cudaSetDevice(c->ctx->device));
    ctbb_ctx* ctx = c->ctx;
    cudaStream_t st = ctx->stream;
    const uint64_t n = (uint64_t)nx * ny * nz;
    const int lg = grid1(ctx, n);
    CTBB_TRY(ensure_partials(ctx, lg));
    double wsum = (double)n;
    if (weight_dev) {
        weight_sum_kernel<<<lg, 256, 0, st>>>(n, weight_dev, ctx->d_partials);
        CTBB_CUDA(cudaGetLastError());
        CTBB_TRY(reduce(ctx, lg, &wsum));
    }
    if (!(wsum > 0.0)) return fail(CTBB_ERR_INVALID_ARG, "loss weights sum to zero");
    CTBB_TRY(forward(c, x_dev, nx, ny, nz));
    const Dims d = make_dims(nx, ny, nz);
    loss_kernel<<<lg, 256, 0, st>>>(n, c->d_out, x_dev, xc_dev, weight_dev, c->s_out, 1.0 / wsum, c->d_dout,
                                    ctx->d_partials);
    CTBB_CUDA(cudaGetLastError());
    double L = 0.0;
    CTBB_TRY(reduce(ctx, lg, &L));
    const int B = c->blocks;
    // out = conv_out(a_B) + b_out
    const int wg_blocks = (int)((n + kWg1Chunk - 1) / kWg1Chunk);
    wgrad_1ch_kernel<<<wg_blocks, kWg1Threads, 0, st>>>(0, nx, ny, nz, c->a(B), c->d_dout, 0.f, nullptr,
                                                         c->d_g + c->off_wout);
    CTBB_CUDA(cudaGetLastError());
    conv_out_bwd_kernel<<<grid1(ctx, n), 256, 0, st>>>(nx, ny, nz, c->d_dout, c->d_p + c->off_wout, c->gbuf(0));
    CTBB_CUDA(cudaGetLastError());
    int gi = 0;
    for (int l = B - 1; l >= 0; --l) {
        __nv_bfloat16* g = c->gbuf(gi);
        // a_{l+1} = a_l + conv(h_l; W2) + b2
        CTBB_TRY(conv_wgrad(c, d, c->h(l), g, c->d_g + c->off_w[2 * l + 1]));
        bias_grad_kernel<<<grid1(ctx, n / 8 + 1), 256, 0, st>>>(n, g, c->d_g + c->off_b[2 * l + 1]);
        CTBB_CUDA(cudaGetLastError());
        CTBB_TRY(conv_mid(c, d, g, c->d_wb + (uint64_t)(2 * l + 1) * kConvW, nullptr, nullptr, c->h(l), 0, c->du()));
        // h_l = relu(conv(a_l; W1) + b1)
        CTBB_TRY(conv_wgrad(c, d, c->a(l), c->du(), c->d_g + c->off_w[2 * l]));
        bias_grad_kernel<<<grid1(ctx, n / 8 + 1), 256, 0, st>>>(n, c->du(), c->d_g + c->off_b[2 * l]);
        CTBB_CUDA(cudaGetLastError());
        CTBB_TRY(conv_mid(c, d, c->du(), c->d_wb + (uint64_t)(2 * l) * kConvW, nullptr, g, nullptr, 0,
                          c->gbuf(1 - gi)));
        gi = 1 - gi;
    }
    // a_0 = relu(conv_in(s_in x) + b_in)
    wgrad_1ch_kernel<<<wg_blocks, kWg1Threads, 0, st>>>(1, nx, ny, nz, c->gbuf(gi), x_dev, c->s_in, c->a(0),
                                                         c->d_g + c->off_win);
    CTBB_CUDA(cudaGetLastError());
    CTBB_CUDA(cudaStreamSynchronize(st));
    CTBB_TRY(check_conv_flag(c));
    if (loss) *loss = L;
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_cnn_get_gradient(ctbb_cnn* c, float* host, uint64_t n) {
    clear_error();
    if (!c || !host) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (n != c->n_params) return fail(CTBB_ERR_INVALID_ARG, "expected %llu parameters", (unsigned long long)c->n_params);
    CTBB_CUDA(cudaSetDevice(c->ctx->device));
    CTBB_CUDA(cudaMemcpyAsync(host, c->d_g, n * sizeof(float), cudaMemcpyDeviceToHost, c->ctx->stream));
    CTBB_CUDA(cudaStreamSynchronize(c->ctx->stream));
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_cnn_zero_gradient(ctbb_cnn* c) {
    clear_error();
    if (!c) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    CTBB_CUDA(cudaSetDevice(c->ctx->device));
    CTBB_CUDA(cudaMemsetAsync(c->d_g, 0, c->n_params * sizeof(float), c->ctx->stream));
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_cnn_adam_step(ctbb_cnn* c, float lr, float beta1, float beta2, float eps,
                                          float grad_scale) {
    clear_error();
    if (!c) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (!(lr > 0.f) || !(beta1 >= 0.f && beta1 < 1.f) || !(beta2 >= 0.f && beta2 < 1.f) || !(eps > 0.f))
        return fail(CTBB_ERR_INVALID_ARG, "invalid Adam hyper-parameters");
    CTBB_CUDA(cudaSetDevice(c->ctx->device));
    c->adam_t += 1;
    const float c1 = 1.f - powf(beta1, (float)c->adam_t), c2 = 1.f - powf(beta2, (float)c->adam_t);
    adam_kernel<<<grid1(c->ctx, c->n_params), 256, 0, c->ctx->stream>>>(
        c->n_params, c->d_p, c->d_g, c->d_m, c->d_v, lr, beta1, beta2, eps, c1, c2, grad_scale);
    CTBB_CUDA(cudaGetLastError());
    c->weights_dirty = true;
    return CTBB_OK;
}

namespace ctbb {

// Physical correction predicted for a fixed-frame volume: d = out / s_out.
ctbb_status cnn_predict_correction(ctbb_cnn* c, const float* x_dev, int nx, int ny, int nz, float* d_dev) {
    CTBB_TRY(forward(c, x_dev, nx, ny, nz));
    const uint64_t n = (uint64_t)nx * ny * nz;
    scale_copy_kernel<<<grid1(c->ctx, n), 256, 0, c->ctx->stream>>>(n, c->d_out, d_dev, 1.f / c->s_out);
    CTBB_CUDA(cudaGetLastError());
    return CTBB_OK;
}

ctbb_status apply_correction(ctbb_ctx* ctx, uint64_t n, float* x_dev, const float* d_dev, float* prio_dev) {
    apply_correction_kernel<<<grid1(ctx, n), 256, 0, ctx->stream>>>(n, x_dev, d_dev, prio_dev);
    CTBB_CUDA(cudaGetLastError());
    return CTBB_OK;
}

ctbb_ctx* cnn_ctx(const ctbb_cnn* c) { return c->ctx; }

ctbb_status cnn_check_flag(ctbb_cnn* c) { return check_conv_flag(c); }

}  // namespace ctbb
