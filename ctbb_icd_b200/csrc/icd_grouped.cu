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
// Visiting order (the "groups"). A voxel update touches ~2 short runs of
// detector rows per view, each costing a whole 32-byte sector, so what bounds
// the kernel is DRAM sectors, not bytes. The voxels whose runs share sectors
// are the ones at the same physical (x, y) position in different slices:
// they project to the same channels and to neighbouring rows. With rotating
// slices (Xu & Tsui), that physical position is a different column index in
// every slice, so the order is built from physical positions: each voxel's
// centre is rotated into the fixed frame (by the tube angle of its slice's
// central view) and snapped to a grid cell; the plane is cut into T x T-cell
// tiles, and
//
//   key = (cell rank inside its tile, slice parity, tile, slice)
//
// with cells ranked along a serpentine raster. A "round" is one cell of every
// tile (with one slice parity); the ~`warps_in_flight` items in flight are a
// part of one round: stacks of every-other slice at the same relative cell of
// many tiles, T cells apart. A stack shares sinogram sectors (its z-profiles
// are disjoint, so it is nearly uncoupled); the next round moves every tile
// to the neighbouring cell (or the other parity of the same cell), whose
// footprint is still in L2, so the sinogram is streamed from DRAM a few times
// per iteration instead of once per lattice pass. Neighbouring voxels are a
// round apart, never in flight together as long as W is below a round, and
// within a tile the sweep is the reference's raster-like order. Footprints
// still overlap where voxels line up with the source, so the scatter is an L2
// reduction rather than ordered stores.
//
// The warp count in flight bounds how stale a gather can be: with W warps
// and a voxel footprint crossing ~T voxels per ray, about T*W/N voxels of a
// ray change concurrently; the default keeps that near 0.4.
#include <math.h>

#include <string.h>

#include <algorithm>
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <type_traits>
#include <vector>

#include "gpu_internal.h"

namespace {

struct GParams {
    int nx, ny, nz, nch, nr, nvsm, readings, penalty;
    int last_slice[2];  // last slice of each parity
    uint64_t n_items, nvsm1;
    double lambda, delta;
    double relax;  // step scale applied to the exact 1-D update before the positivity clamp
    double cvx, cvy, vx, vy, fov_limit;
    int stack_align;  // CTA kernels: sweep from the slice stack's common data view
    int l2_hints;     // CTA kernels: matrix loads evict-first, e gathers evict-last;
                      // bulk kernels (stage_column 4/5): the column copy evict-first
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

// L2 eviction policies: a voxel update reads its matrix entries twice (gather,
// then scatter); the gather's loads ask L2 to keep the lines, the scatter's
// to drop them first.
__device__ __forceinline__ uint64_t l2_keep() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_drop() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_normal() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
    return p;
}
// e gather through L2 (other SMs update e) with an eviction priority.
__device__ __forceinline__ float ld_e(const float* p, uint64_t pol) {
    float v;
    asm volatile("ld.global.cg.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ int ld_idx(const int32_t* p, uint64_t pol) {
    int v;
    asm volatile("ld.global.nc.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}
template <class WT>
__device__ __forceinline__ float ldw_hint(const WT* w, int64_t m, uint64_t pol);
template <>
__device__ __forceinline__ float ldw_hint<float>(const float* w, int64_t m, uint64_t pol) {
    float v;
    asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(w + m), "l"(pol));
    return v;
}
template <>
__device__ __forceinline__ float ldw_hint<__half>(const __half* w, int64_t m, uint64_t pol) {
    unsigned short v;
    asm volatile("ld.global.nc.L2::cache_hint.b16 %0, [%1], %2;" : "=h"(v) : "l"(w + m), "l"(pol));
    return __half2float(__ushort_as_half(v));
}

// Entries m, m+32, ..., m+32(U-1) of a column: sinogram index (q + off, or
// -1 past the end) and weight (0 past the end).
template <int U, class WT>
__device__ __forceinline__ void load_chunk(const int32_t* __restrict__ idx, const WT* __restrict__ w, int64_t m,
                                           int64_t en, int off, uint64_t pol, int* q, float* wt) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int64_t mu = m + 32 * u;
        if (mu < en) {
            q[u] = ld_idx(idx + mu, pol) + off;
            wt[u] = ldw_hint(w, mu, pol);
        } else {
            q[u] = -1;
            wt[u] = 0.f;
        }
    }
}

// The two FP16 weights of an entry pair ({q, w0 | w1 << 16}).
__device__ __forceinline__ float half_lo(uint32_t w) { return __half2float(__ushort_as_half((unsigned short)(w & 0xffffu))); }
__device__ __forceinline__ float half_hi(uint32_t w) { return __half2float(__ushort_as_half((unsigned short)(w >> 16))); }

constexpr int kU = 8;       // entries per lane in flight per chunk (default)
constexpr int kStack = 16;  // same-parity slices that sweep the sinogram together

// Matrix view where slice k's sweep starts so that the members of its slice
// stack (up to kStack same-parity slices at one physical position) read and
// update each sinogram sector at about the same time: the data view where
// the stack's last member's window begins, clamped to k's window [v0, v1).
__device__ __forceinline__ int stack_start_view(const GParams& P, const int32_t* __restrict__ start, int k, int s,
                                                int v0, int v1) {
    const int kl = min(k - (k % (2 * kStack)) + (k % 2) + 2 * (kStack - 1),
                       ((k & 1) ? P.last_slice[1] : P.last_slice[0]));
    return min(max(start[kl] - s, v0), v1);
}

// Gather beta += a e and alpha += a^2 over entries [b, en) of a column: chunks
// of 32 x U entries, the next chunk's indices and weights fetched while this
// chunk's e gathers are in flight (one DRAM round trip per chunk).
template <class WT, int U>
__device__ __forceinline__ void gather_range(const int32_t* __restrict__ idx, const WT* __restrict__ w,
                                             const float* e, int64_t b, int64_t en, int off, int lane,
                                             uint64_t pol, float& acc_b, float& acc_a) {
    if (b >= en) return;
    int qa[U];
    float wa[U];
    load_chunk<U>(idx, w, b + lane, en, off, pol, qa, wa);
    for (int64_t base = b; base < en; base += 32 * U) {
        float ev[U];
#pragma unroll
        for (int u = 0; u < U; ++u) ev[u] = (qa[u] >= 0) ? __ldcg(e + qa[u]) : 0.f;
        int qb[U];
        float wb[U];
        load_chunk<U>(idx, w, base + 32 * U + lane, en, off, pol, qb, wb);
#pragma unroll
        for (int u = 0; u < U; ++u) {
            acc_b = fmaf(wa[u], ev[u], acc_b);
            acc_a = fmaf(wa[u], wa[u], acc_a);
            qa[u] = qb[u];
            wa[u] = wb[u];
        }
    }
}

// e -= du * a over entries [b, en): U independent index/weight loads per
// lane per chunk, then U fire-and-forget L2 reductions. Chunks run from the
// end of the range back to its start: the entries gathered last are the ones
// whose matrix lines and e sectors are likeliest to still be in L2.
template <class WT, int U>
__device__ __forceinline__ void scatter_range(const int32_t* __restrict__ idx, const WT* __restrict__ w, float* e,
                                              int64_t b, int64_t en, int off, int lane, uint64_t pol, float du) {
    if (b >= en) return;
    const int64_t nchunk = (en - b + 32 * U - 1) / (32 * U);
    for (int64_t c = nchunk - 1; c >= 0; --c) {
        const int64_t base = b + c * (32 * U);
        int qs[U];
        float ws[U];
        load_chunk<U>(idx, w, base + lane, en, off, pol, qs, ws);
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (qs[u] >= 0) atomicAdd(e + qs[u], -du * ws[u]);
    }
}

// Raw weight bits for the shared-memory stage, and their value.
template <class WT>
struct WBits;
template <>
struct WBits<float> {
    using T = float;
    __device__ static __forceinline__ float load(const float* w, int64_t m, uint64_t pol) { return ldw_hint(w, m, pol); }
    __device__ static __forceinline__ float value(float v) { return v; }
};
template <>
struct WBits<__half> {
    using T = unsigned short;
    __device__ static __forceinline__ unsigned short load(const __half* w, int64_t m, uint64_t pol) {
        unsigned short v;
        asm volatile("ld.global.nc.L2::cache_hint.b16 %0, [%1], %2;" : "=h"(v) : "l"(w + m), "l"(pol));
        return v;
    }
    __device__ static __forceinline__ float value(unsigned short v) { return __half2float(__ushort_as_half(v)); }
};

// Gather over entries [m0, m1) of a column, which occupy stage positions
// p0 + (m - m0): the entry's sinogram index (slice offset applied) and raw
// weight go to the warp's shared-memory stage (positions below `cap`) while
// its e value is gathered; chunks of 32 x U entries, the next chunk's matrix
// entries fetched while this chunk's e gathers are in flight.
template <class WT, int U>
__device__ __forceinline__ void stage_gather(const int32_t* __restrict__ idx, const WT* __restrict__ w,
                                             const float* e, int64_t m0, int64_t m1, int64_t p0, int off, int lane,
                                             uint64_t pol, int32_t* sq, typename WBits<WT>::T* sw, int64_t cap,
                                             float& acc_b, float& acc_a) {
    using B = WBits<WT>;
    if (m0 >= m1) return;
    int qa[U];
    typename B::T wa[U];
    auto load = [&](int64_t base, int* q, typename B::T* wv) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t m = base + lane + 32 * u;
            if (m < m1) {
                q[u] = ld_idx(idx + m, pol) + off;
                wv[u] = B::load(w, m, pol);
            } else {
                q[u] = -1;
                wv[u] = typename B::T(0);
            }
        }
    };
    load(m0, qa, wa);
    for (int64_t base = m0; base < m1; base += 32 * U) {
        float ev[U];
#pragma unroll
        for (int u = 0; u < U; ++u) ev[u] = (qa[u] >= 0) ? __ldcg(e + qa[u]) : 0.f;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t p = p0 + (base - m0) + lane + 32 * u;
            if (qa[u] >= 0 && p < cap) {
                sq[p] = qa[u];
                sw[p] = wa[u];
            }
        }
        int qb[U];
        typename B::T wb[U];
        load(base + 32 * U, qb, wb);
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const float wf = B::value(wa[u]);
            acc_b = fmaf(wf, ev[u], acc_b);
            acc_a = fmaf(wf, wf, acc_a);
            qa[u] = qb[u];
            wa[u] = wb[u];
        }
    }
}

// Device-side view of one scan for the batched kernel.
template <class WT>
struct ScanRefs {
    GParams P;
    const uint32_t* order;
    const int64_t* colptr;
    const uint32_t* vptr;
    const int32_t* idx;
    const WT* w;
    const int32_t* start;
    float* e;
    float* x;
};

constexpr double kInvSqrt2 = 1.0 / 1.41421356237309504880168872420969807;

// Weight of neighbour lane 0-7 in the order {-nx-1, -nx, -nx+1, -1, +1,
// nx-1, nx, nx+1} (penalties.cpp:39-59): 1 for edges, 1/sqrt(2) for corners.
__device__ __forceinline__ double neighbour_weight(int lane) {
    return (lane == 1 || lane == 3 || lane == 4 || lane == 6) ? 1.0 : kInvSqrt2;
}

// The penalised 1-D surrogate solve of one voxel by one warp. Lanes 0-7 hold
// a neighbour's difference x_n - x_q and its weight (0 for a neighbour
// outside the volume); other lanes hold zeros. Returns the step before the
// positivity clamp; every lane gets the same value.
__device__ __forceinline__ double penalty_solve(int penalty, double lam, double del, double alpha, double beta,
                                                double diff, double wn) {
    if (penalty == CTBB_PENALTY_QUADRATIC) {
        // penalties.cpp:84 (the denominator always uses all 8 weights)
        const double sum = sum8(wn * diff);
        return (beta + lam * sum) / (alpha + lam * (4.0 + 4.0 * kInvSqrt2));
    }
    if (alpha == 0.0) return 0.0;  // penalties.cpp:101-102
    // Root of f(d) = 2 alpha d - 2 beta + lambda sum w psi(d - diff),
    // psi(t) = t / (delta + |t|), inside the reference's bracket.
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
    // Newton from beta / alpha, kept inside the bracket: a step that leaves
    // it, or that would not at least halve the step before last, is replaced
    // by bisection (Numerical Recipes' rtsafe rule), so every iteration
    // shrinks the bracket or converges quadratically. A Newton step landing
    // on the bracket's end is kept (an exact root, f = 0, ends there).
    double c = beta / alpha;
    double step_old = hi - lo, step = step_old;
    for (int it = 0; it < 64; ++it) {
        const double t = c - diff;
        const double r = 1.0 / (del + fabs(t));  // one division per lane and iteration
        const double wr = wn * r;
        const double f = 2.0 * alpha * c - 2.0 * beta + lam * sum8(wr * t);
        const double fp = 2.0 * alpha + lam * sum8(wr * del * r);
        if (f > 0.0)
            hi = c;
        else
            lo = c;
        double cn = c - f / fp;
        if (!(cn >= lo && cn <= hi) || fabs(2.0 * f) > fabs(step_old * fp)) cn = 0.5 * (lo + hi);
        step_old = step;
        step = cn - c;
        const bool done = fabs(cn - c) <= 1e-12 * (1e-3 + fabs(c)) || (hi - lo) <= 1e-14;
        c = cn;
        if (done) break;
    }
    return c;
}

// Penalised 1-D update of voxel q by one warp (lanes 0-7 hold the 8 in-plane
// neighbours of penalties.cpp:41-52 / 67-74, flat-index offsets, a neighbour
// outside [0, nvox) dropped).
// The neighbour of voxel q that lane 0-7 holds, as loaded from x (lane
// >= 8 or outside [0, nvox): *w = 0). Loaded before the update's gather so
// the value is in a register when the penalty solve starts.
__device__ __forceinline__ float neighbour_value(const GParams& P, const float* x, int64_t q, int lane, double* w) {
    *w = 0.0;
    if (lane >= 8) return 0.f;
    const int64_t nx = P.nx;
    const int64_t nvox = (int64_t)P.nx * P.ny * P.nz;
    const int64_t dr = lane < 3 ? -1 : (lane < 5 ? 0 : 1);
    const int64_t dc = lane < 3 ? lane - 1 : (lane < 5 ? 2 * lane - 7 : lane - 6);
    const int64_t n = q + dr * nx + dc;
    if (n < 0 || n >= nvox) return 0.f;
    *w = neighbour_weight(lane);
    return __ldcg(x + n);
}

__device__ __forceinline__ double penalty_step(const GParams& P, const float* x, int64_t q, double xq, double alpha,
                                               double beta, int lane) {
    const int64_t nx = P.nx;
    const int64_t nvox = (int64_t)P.nx * P.ny * P.nz;
    double diff = 0.0, wn = 0.0;
    if (lane < 8) {
        // Lane -> flat-index offset {-nx-1, -nx, -nx+1, -1, +1, nx-1, nx, nx+1}.
        const int64_t dr = lane < 3 ? -1 : (lane < 5 ? 0 : 1);
        const int64_t dc = lane < 3 ? lane - 1 : (lane < 5 ? 2 * lane - 7 : lane - 6);
        const int64_t n = q + dr * nx + dc;
        if (n >= 0 && n < nvox) {
            diff = (double)__ldcg(x + n) - xq;
            wn = neighbour_weight(lane);
        }
    }
    return penalty_solve(P.penalty, P.lambda, P.delta, alpha, beta, diff, wn);
}

// One warp per voxel: the grouped update's penalty solve on given inputs
// (ctbb_gpu_penalty_steps). x9[9 i] is the voxel, x9[9 i + 1 + l] its
// neighbour l (NaN: outside the volume).
__global__ void __launch_bounds__(256) penalty_steps_kernel(int penalty, double lam, double del, uint64_t n,
                                                            const double* __restrict__ alpha,
                                                            const double* __restrict__ beta,
                                                            const float* __restrict__ x9, double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = warp; i < n; i += nwarps) {
        const double xq = (double)x9[9 * i];
        double diff = 0.0, wn = 0.0;
        if (lane < 8) {
            const float xn = x9[9 * i + 1 + lane];
            if (!isnan(xn)) {
                diff = (double)xn - xq;
                wn = neighbour_weight(lane);
            }
        }
        const double d = penalty_solve(penalty, lam, del, alpha[i], beta[i], diff, wn);
        if (lane == 0) out[i] = d;
    }
}

// One voxel update (work item `item` of a scan's visiting order) by one warp.
template <class WT, int U = kU>
__device__ __forceinline__ void process_item(const GParams& P, const uint32_t* __restrict__ order,
                                             const int64_t* __restrict__ colptr, const uint32_t* __restrict__ vptr,
                                             const int32_t* __restrict__ idx, const WT* __restrict__ w,
                                             const int32_t* __restrict__ start, float* e, float* x, uint64_t item,
                                             int lane, unsigned long long* scattered = nullptr) {
    const uint64_t ncol = (uint64_t)P.nx * P.ny;
    const uint32_t packed = __ldg(order + item);
    const uint64_t col = packed / (uint32_t)P.nz;
    const int k = (int)(packed % (uint32_t)P.nz);
    const int64_t q = (int64_t)col + (int64_t)ncol * k;
    const int s = start[k];
    const int v0 = max(0, -s), v1 = min(P.nvsm, P.readings - s);
    int64_t b = 0, en = 0, mid = 0;
    if (v1 > v0) {
        const int64_t cb = colptr[col];
        const uint32_t* vp = vptr + col * P.nvsm1;
        b = cb + vp[v0];
        en = cb + vp[v1];
        // Members of a slice stack (up to 16 same-parity slices at this
        // physical position) all start their sweep at the data view where the
        // stack's last member's window begins, then wrap around, so they read
        // and update each sinogram sector at about the same time.
        const int kl = min(k - (k % (2 * kStack)) + (k % 2) + 2 * (kStack - 1), ((k & 1) ? P.last_slice[1] : P.last_slice[0]));
        const int vs = min(max(start[kl] - s, v0), v1);
        mid = cb + vp[vs];
    }
    const int off = s * P.nch * P.nr;

    // beta = sum a e, alpha = sum a^2 (FP32 accumulation per lane) over
    // [mid, en) then [b, mid).
    float acc_b = 0.f, acc_a = 0.f;
    const uint64_t keep = l2_keep();
    gather_range<WT, U>(idx, w, e, mid, en, off, lane, keep, acc_b, acc_a);
    gather_range<WT, U>(idx, w, e, b, mid, off, lane, keep, acc_b, acc_a);
    const double beta = (double)warp_sum(acc_b);
    const double alpha = (double)warp_sum(acc_a);

    const double xq = (double)__ldcg(x + q);
    double upd = penalty_step(P, x, q, xq, alpha, beta, lane) * P.relax;
    if (upd + xq < 0.0) upd = -xq;  // icd_iteration.cpp:233-234
    if (lane == 0) x[q] = (float)(xq + upd);
    const float du = (float)upd;
    if (du != 0.f) {
        // Reverse of the gather order: [b, mid) backwards, then [mid, en).
        const uint64_t drop = l2_drop();
        scatter_range<WT, U>(idx, w, e, b, mid, off, lane, drop, du);
        scatter_range<WT, U>(idx, w, e, mid, en, off, lane, drop, du);
        if (scattered) *scattered += (unsigned long long)(en - b);
    }
}

// Scatter counters of one launch, summed once per warp at exit:
// [0] updates that scattered (du != 0), [1] matrix entries they scattered.
__device__ __forceinline__ void flush_counts(unsigned long long* stats, unsigned long long upd,
                                             unsigned long long ent, int lane) {
    if (stats && lane == 0 && upd) {
        atomicAdd(stats, upd);
        atomicAdd(stats + 1, ent);
    }
}

template <class WT, int U>
__global__ void __launch_bounds__(256) icd_grouped_kernel(GParams P, const uint32_t* __restrict__ order,
                                                          const int64_t* __restrict__ colptr,
                                                          const uint32_t* __restrict__ vptr,
                                                          const int32_t* __restrict__ idx,
                                                          const WT* __restrict__ w, const int32_t* __restrict__ start,
                                                          float* e, float* x, unsigned long long* queue,
                                                          unsigned long long* stats) {
    const int lane = threadIdx.x & 31;
    unsigned long long n_ent = 0, n_upd = 0;
    for (;;) {
        unsigned long long item = 0;
        if (lane == 0) item = atomicAdd(queue, 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= P.n_items) break;
        const unsigned long long before = n_ent;
        process_item<WT, U>(P, order, colptr, vptr, idx, w, start, e, x, item, lane, &n_ent);
        n_upd += n_ent != before;
    }
    flush_counts(stats, n_upd, n_ent, lane);
}

// One warp per update over the matrix's entry pairs (the streamed kernel's
// order, stack start view and round trips). Lanes 2j and 2j+1 share pair j of
// a row of 16 pairs: both load the same 8 bytes (one request) and each takes
// one of its two entries, so a warp's gathers touch consecutive sinogram
// rows as with single entries (coalesced in the same sectors) while the
// matrix costs 4 bytes per entry instead of 6. Position p of a lane in row u
// of a chunk: pair base + 16 u + lane / 2, entry lane & 1.
template <int U, int STRIDE = 16>
__device__ __forceinline__ void load_pair_entries(const uint2* __restrict__ pairs, int64_t m, int64_t en, int off,
                                                  int half, uint64_t pol, int* q, float* wt) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int64_t mu = m + (int64_t)STRIDE * u;
        q[u] = -1;
        wt[u] = 0.f;
        if (mu < en) {
            uint32_t a, bb;
            asm volatile("ld.global.nc.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;"
                         : "=r"(a), "=r"(bb)
                         : "l"(pairs + mu), "l"(pol));
            if (!half || (bb >> 16)) {
                q[u] = (int)a + off + half;
                wt[u] = half ? half_hi(bb) : half_lo(bb);
            }
        }
    }
}

// Pair positions p, p + STRIDE, ... of an item's sweep: pair p + hi for
// p < n1, else p + lo; -1 / 0 past n (the sweep's length).
template <int U, int STRIDE>
__device__ __forceinline__ void load_seq_pairs(const uint2* __restrict__ pairs, int p0, int n, int n1, int64_t hi,
                                               int64_t lo, int off, int half, uint64_t pol, int* q, float* wt) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int p = p0 + STRIDE * u;
        q[u] = -1;
        wt[u] = 0.f;
        if (p < n) {
            const int64_t m = (p < n1 ? hi : lo) + p;
            uint32_t a, bb;
            asm volatile("ld.global.nc.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;"
                         : "=r"(a), "=r"(bb)
                         : "l"(pairs + m), "l"(pol));
            if (!half || (bb >> 16)) {
                q[u] = (int)a + off + half;
                wt[u] = half ? half_hi(bb) : half_lo(bb);
            }
        }
    }
}

template <int U>
__device__ __forceinline__ void gather_pairs(const uint2* __restrict__ pairs, const float* e, int64_t b, int64_t en,
                                             int off, int lane, uint64_t pol, float& acc_b, float& acc_a) {
    if (b >= en) return;
    const int half = lane & 1, j = lane >> 1;
    int qa[U];
    float wa[U];
    load_pair_entries<U>(pairs, b + j, en, off, half, pol, qa, wa);
    for (int64_t base = b; base < en; base += 16 * U) {
        float ev[U];
#pragma unroll
        for (int u = 0; u < U; ++u) ev[u] = qa[u] >= 0 ? __ldcg(e + qa[u]) : 0.f;
        int qb[U];
        float wb[U];
        load_pair_entries<U>(pairs, base + 16 * U + j, en, off, half, pol, qb, wb);
#pragma unroll
        for (int u = 0; u < U; ++u) {
            acc_b = fmaf(wa[u], ev[u], acc_b);
            acc_a = fmaf(wa[u], wa[u], acc_a);
            qa[u] = qb[u];
            wa[u] = wb[u];
        }
    }
}

template <int U>
__device__ __forceinline__ void scatter_pairs(const uint2* __restrict__ pairs, float* e, int64_t b, int64_t en,
                                              int off, int lane, uint64_t pol, float du) {
    if (b >= en) return;
    const int half = lane & 1, j = lane >> 1;
    const int64_t nchunk = (en - b + 16 * U - 1) / (16 * U);
    for (int64_t c = nchunk - 1; c >= 0; --c) {
        int qs[U];
        float ws[U];
        load_pair_entries<U>(pairs, b + c * (16 * U) + j, en, off, half, pol, qs, ws);
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (qs[u] >= 0) atomicAdd(e + qs[u], -du * ws[u]);
    }
}

template <int U>
__global__ void __launch_bounds__(256) icd_grouped_pairs_kernel(
    GParams P, const uint32_t* __restrict__ order, const int64_t* __restrict__ pcolptr,
    const uint32_t* __restrict__ pvptr, const uint2* __restrict__ pairs, const uint32_t* __restrict__ vptr,
    const int32_t* __restrict__ start, float* e, float* x, unsigned long long* queue, unsigned long long* stats) {
    const int lane = threadIdx.x & 31;
    const uint64_t ncol = (uint64_t)P.nx * P.ny;
    unsigned long long n_ent = 0, n_upd = 0;
    for (;;) {
        unsigned long long item = 0;
        if (lane == 0) item = atomicAdd(queue, 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= P.n_items) break;
        const uint32_t packed = __ldg(order + item);
        const uint64_t col = packed / (uint32_t)P.nz;
        const int k = (int)(packed % (uint32_t)P.nz);
        const int64_t q = (int64_t)col + (int64_t)ncol * k;
        const int s = start[k];
        const int v0 = max(0, -s), v1 = min(P.nvsm, P.readings - s);
        int64_t b = 0, en = 0, mid = 0, n_entries = 0;
        if (v1 > v0) {
            const int64_t cb = pcolptr[col];
            const uint32_t* vp = pvptr + col * P.nvsm1;
            b = cb + vp[v0];
            en = cb + vp[v1];
            // Same common start view for the members of a slice stack as
            // process_item.
            const int kl = min(k - (k % (2 * kStack)) + (k % 2) + 2 * (kStack - 1),
                               ((k & 1) ? P.last_slice[1] : P.last_slice[0]));
            mid = cb + vp[min(max(start[kl] - s, v0), v1)];
            n_entries = (int64_t)vptr[col * P.nvsm1 + v1] - (int64_t)vptr[col * P.nvsm1 + v0];
        }
        const int off = s * P.nch * P.nr;
        float acc_b = 0.f, acc_a = 0.f;
        const uint64_t keep = l2_keep();
        gather_pairs<U>(pairs, e, mid, en, off, lane, keep, acc_b, acc_a);
        gather_pairs<U>(pairs, e, b, mid, off, lane, keep, acc_b, acc_a);
        const double beta = (double)warp_sum(acc_b);
        const double alpha = (double)warp_sum(acc_a);
        const double xq = (double)__ldcg(x + q);
        double upd = penalty_step(P, x, q, xq, alpha, beta, lane) * P.relax;
        if (upd + xq < 0.0) upd = -xq;  // icd_iteration.cpp:233-234
        if (lane == 0) x[q] = (float)(xq + upd);
        const float du = (float)upd;
        if (du != 0.f) {
            const uint64_t drop = l2_drop();
            scatter_pairs<U>(pairs, e, b, mid, off, lane, drop, du);
            scatter_pairs<U>(pairs, e, mid, en, off, lane, drop, du);
            n_ent += (unsigned long long)n_entries;
            ++n_upd;
        }
    }
    flush_counts(stats, n_upd, n_ent, lane);
}

// Entries p0, p0+32, ..., p0+32(U-1) of an item's entry sequence: positions
// [0, n1) are matrix entries [mid, en) (the stack's common start view to the
// end of the slice's window), positions [n1, n) entries [b, mid); hi = mid,
// lo = b - n1, so entry = position + (position < n1 ? hi : lo).
template <int U, class WT>
__device__ __forceinline__ void load_seq(const int32_t* __restrict__ idx, const WT* __restrict__ w, int p0, int n,
                                         int n1, int64_t hi, int64_t lo, int off, uint64_t pol, int* q, float* wt) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int p = p0 + 32 * u;
        if (p < n) {
            const int64_t m = (int64_t)p + (p < n1 ? hi : lo);
            q[u] = ld_idx(idx + m, pol) + off;
            wt[u] = ldw_hint(w, m, pol);
        } else {
            q[u] = -1;
            wt[u] = 0.f;
        }
    }
}

// One voxel update per CTA of WPV warps over the matrix's entry pairs
// ({q, w0 | w1 << 16}: rows q and q + 1 of one (view, channel), w1 = 0 for a
// lone entry). Threads 2j and 2j+1 share pair j (one 8-byte request) and
// take one entry each, so the gathers stay coalesced as with single entries;
// each thread keeps R entries in registers from the gather to the scatter, so
// a column of up to 32 * WPV * R / 2 pairs is read from HBM once; longer
// columns re-read their tail. Same update as icd_cta_kernel (including its
// sweep order and L2 hints); the entry counts (for the statistics) come from
// the entry offsets.
template <int WPV, int R>
__global__ void __launch_bounds__(32 * WPV, 16 / WPV) icd_cta_pairs_kernel(
    GParams P, const uint32_t* __restrict__ order, const int64_t* __restrict__ pcolptr,
    const uint32_t* __restrict__ pvptr, const uint2* __restrict__ pairs, const uint32_t* __restrict__ vptr,
    const int32_t* __restrict__ start, float* e, float* x, unsigned long long* queue, unsigned long long* stats) {
    constexpr int NT = 32 * WPV;
    constexpr int NP = NT / 2;  // pairs per row of the CTA
    constexpr int64_t CAP = (int64_t)NP * R;
    unsigned long long n_ent = 0, n_upd = 0;
    __shared__ unsigned long long s_item;
    __shared__ float s_red[2 * WPV + 1];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int half = tid & 1, j = tid >> 1;
    const uint64_t ncol = (uint64_t)P.nx * P.ny;
    const uint64_t pol_m = P.l2_hints ? l2_drop() : l2_normal();
    const uint64_t pol_e = P.l2_hints ? l2_keep() : l2_normal();
    for (;;) {
        if (tid == 0) s_item = atomicAdd(queue, 1ull);
        __syncthreads();
        const uint64_t item = s_item;
        if (item >= P.n_items) break;
        const uint32_t packed = __ldg(order + item);
        const uint64_t col = packed / (uint32_t)P.nz;
        const int k = (int)(packed % (uint32_t)P.nz);
        const int64_t q = (int64_t)col + (int64_t)ncol * k;
        const int s = start[k];
        const int v0 = max(0, -s), v1 = min(P.nvsm, P.readings - s);
        int64_t b = 0, en = 0, mid = 0, n_entries = 0;
        if (v1 > v0) {
            const int64_t cb = pcolptr[col];
            const uint32_t* vp = pvptr + col * P.nvsm1;
            b = cb + vp[v0];
            en = cb + vp[v1];
            mid = P.stack_align ? cb + vp[stack_start_view(P, start, k, s, v0, v1)] : b;
            if (tid == 0) n_entries = (int64_t)vptr[col * P.nvsm1 + v1] - (int64_t)vptr[col * P.nvsm1 + v0];
        }
        const int off = s * P.nch * P.nr;
        // Sweep position p (pairs) -> pair p + hi for p < n1 ([mid, en)), else
        // p + lo ([b, mid)).
        const int n = (int)(en - b), n1 = (int)(en - mid);
        const int64_t hi = mid, lo = b - n1;
        const int nreg = min(n, (int)CAP);
        int qr[R];
        float wr[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int p = j + NP * r;
            qr[r] = -1;
            wr[r] = 0.f;
            if (p < nreg) {
                const int64_t m = (p < n1 ? hi : lo) + p;
                uint32_t a, bb;
                asm volatile("ld.global.nc.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;"
                             : "=r"(a), "=r"(bb)
                             : "l"(pairs + m), "l"(pol_m));
                if (!half || (bb >> 16)) {
                    qr[r] = (int)a + off + half;
                    wr[r] = half ? half_hi(bb) : half_lo(bb);
                }
            }
        }
        float acc_b = 0.f, acc_a = 0.f;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const float ev = qr[r] >= 0 ? ld_e(e + qr[r], pol_e) : 0.f;
            acc_b = fmaf(wr[r], ev, acc_b);
            acc_a = fmaf(wr[r], wr[r], acc_a);
        }
        for (int base = (int)CAP; base < n; base += NP * kU) {
            int qo[kU];
            float wo[kU];
            load_seq_pairs<kU, NP>(pairs, base + j, n, n1, hi, lo, off, half, pol_m, qo, wo);
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const float ev = qo[u] >= 0 ? ld_e(e + qo[u], pol_e) : 0.f;
                acc_b = fmaf(wo[u], ev, acc_b);
                acc_a = fmaf(wo[u], wo[u], acc_a);
            }
        }
        acc_b = warp_sum(acc_b);
        acc_a = warp_sum(acc_a);
        if (lane == 0) {
            s_red[wid] = acc_b;
            s_red[WPV + wid] = acc_a;
        }
        __syncthreads();
        if (wid == 0) {
            double beta = 0.0, alpha = 0.0;
#pragma unroll
            for (int i = 0; i < WPV; ++i) {
                beta += (double)s_red[i];
                alpha += (double)s_red[WPV + i];
            }
            const double xq = (double)__ldcg(x + q);
            double upd = penalty_step(P, x, q, xq, alpha, beta, lane) * P.relax;
            if (upd + xq < 0.0) upd = -xq;  // icd_iteration.cpp:233-234
            if (lane == 0) {
                x[q] = (float)(xq + upd);
                s_red[2 * WPV] = (float)upd;
            }
        }
        __syncthreads();
        const float du = s_red[2 * WPV];
        if (du != 0.f) {
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (qr[r] >= 0) atomicAdd(e + qr[r], -du * wr[r]);
            for (int base = (int)CAP; base < n; base += NP * kU) {
                int qo[kU];
                float wo[kU];
                load_seq_pairs<kU, NP>(pairs, base + j, n, n1, hi, lo, off, half, pol_m, qo, wo);
#pragma unroll
                for (int u = 0; u < kU; ++u)
                    if (qo[u] >= 0) atomicAdd(e + qo[u], -du * wo[u]);
            }
            n_ent += (unsigned long long)n_entries;
            ++n_upd;
        }
        __syncthreads();  // s_item / s_red reused by the next item
    }
    flush_counts(stats, n_upd, n_ent, tid);
}

// ---------------------------------------------------------------------------
// Bulk-staged CTA kernel: one voxel update per CTA of 8 warps, the update's
// entry pairs copied into shared memory by the TMA engine
// (cp.async.bulk, completion on an mbarrier) instead of per-thread loads.
// The copy of the next item's pairs is issued as soon as a stage is free, so
// with two stages it runs while the current update gathers, solves and
// scatters; the column is read from HBM once (gather and scatter both read
// the stage), and a thread issues all of its ~28 e gathers back to back (one
// round trip instead of a chain of index-then-gather chunks). Windows longer
// than the stage stream their tail from global memory twice, as the CTA pairs
// kernel does. Same per-voxel update as icd_cta_pairs_kernel.
// ---------------------------------------------------------------------------
constexpr int kBulkThreads = 256;
constexpr int kBulkNP = kBulkThreads / 2;        // pairs per row (two threads per pair)
constexpr int kBulkRows = 28;                    // rows of pairs staged per update
constexpr int kBulkCap = kBulkNP * kBulkRows;    // 3584 pairs (7168 entries)
constexpr int kBulkStagePairs = kBulkCap + 2;    // + slack for the 16-byte-aligned start
constexpr int kBulkHeader = 256;                 // mbarriers and item records
constexpr uint32_t kBulkChunk = 16384;           // bytes per bulk copy instruction
constexpr size_t bulk_smem_bytes(int stages) { return kBulkHeader + (size_t)stages * kBulkStagePairs * 8; }
static_assert((kBulkStagePairs * 8) % 16 == 0, "stage size must keep 16-byte alignment");

struct BulkItem {
    int64_t b, en;       // pair range of the slice's view window
    int64_t q;           // voxel index
    int64_t n_entries;   // matrix entries of the window (statistics)
    int off, d, ns, valid;  // sinogram offset, stage skew (0/1), staged pairs, item present
};
static_assert(2 * sizeof(BulkItem) + 16 <= kBulkHeader, "item records overflow the header");

__device__ __forceinline__ void bulk_mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void bulk_mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bulk_mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait (about a second of SM clock); false if it gave up.
__device__ __forceinline__ bool bulk_mbar_wait(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    while (!bulk_mbar_try_wait(bar, parity))
        if (clock64() - t0 > 2000000000ll) return false;
    return true;
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
// The same copy with an L2 eviction policy (createpolicy) for the source lines.
__device__ __forceinline__ void bulk_g2s_hint(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar,
                                              uint64_t pol) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
            dst),
        "l"(src), "r"(bytes), "r"(bar), "l"(pol)
        : "memory");
}

// Thread 0: take the next work item and start the copy of its pairs into
// the stage at `dst` (bytes counted on `bar`). Pairs [b0, e1) are copied with
// b0 = b rounded down and e1 rounded up to even (16-byte boundaries; the pair
// array has two pairs of padding past its end); the item's first pair sits at
// stage position d = b - b0.
__device__ __forceinline__ void bulk_issue(const GParams& P, const uint32_t* __restrict__ order,
                                           const int64_t* __restrict__ pcolptr, const uint32_t* __restrict__ pvptr,
                                           const uint2* __restrict__ pairs, const uint32_t* __restrict__ vptr,
                                           const int32_t* __restrict__ start, unsigned long long* queue,
                                           BulkItem* it, uint32_t dst, uint32_t bar) {
    const uint64_t item = atomicAdd(queue, 1ull);
    if (item >= P.n_items) {
        it->valid = 0;
        return;
    }
    const uint64_t ncol = (uint64_t)P.nx * P.ny;
    const uint32_t packed = __ldg(order + item);
    const uint64_t col = packed / (uint32_t)P.nz;
    const int k = (int)(packed % (uint32_t)P.nz);
    const int s = start[k];
    const int v0 = max(0, -s), v1 = min(P.nvsm, P.readings - s);
    int64_t b = 0, en = 0, ne = 0;
    if (v1 > v0) {
        const int64_t cb = pcolptr[col];
        const uint32_t* vp = pvptr + col * P.nvsm1;
        b = cb + vp[v0];
        en = cb + vp[v1];
        ne = (int64_t)vptr[col * P.nvsm1 + v1] - (int64_t)vptr[col * P.nvsm1 + v0];
    }
    const int ns = (int)min(en - b, (int64_t)kBulkCap);
    const int64_t b0 = b & ~(int64_t)1;
    const int64_t e1 = (b + ns + 1) & ~(int64_t)1;
    const uint32_t bytes = ns > 0 ? (uint32_t)((e1 - b0) * 8) : 0u;
    it->b = b;
    it->en = en;
    it->q = (int64_t)col + (int64_t)ncol * k;
    it->n_entries = ne;
    it->off = s * P.nch * P.nr;
    it->d = (int)(b - b0);
    it->ns = ns;
    it->valid = 1;
    // The stage was last read through the generic proxy; order those reads
    // before the async-proxy writes of the copy.
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    bulk_mbar_expect_tx(bar, bytes);
    const char* src = reinterpret_cast<const char*>(pairs + b0);
    if (P.l2_hints) {
        // The column is read once per update and kept in shared memory for
        // the scatter: mark its L2 lines first to go, leaving L2 to e.
        const uint64_t pol = l2_drop();
        for (uint32_t o = 0; o < bytes; o += kBulkChunk)
            bulk_g2s_hint(dst + o, src + o, min(kBulkChunk, bytes - o), bar, pol);
    } else {
        for (uint32_t o = 0; o < bytes; o += kBulkChunk) bulk_g2s(dst + o, src + o, min(kBulkChunk, bytes - o), bar);
    }
}

template <int STAGES>
__global__ void __launch_bounds__(kBulkThreads, STAGES == 1 ? 4 : 3) icd_bulk_kernel(
    GParams P, const uint32_t* __restrict__ order, const int64_t* __restrict__ pcolptr,
    const uint32_t* __restrict__ pvptr, const uint2* __restrict__ pairs, const uint32_t* __restrict__ vptr,
    const int32_t* __restrict__ start, float* e, float* x, unsigned long long* queue, unsigned long long* stats,
    unsigned long long* err) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ float s_red[2 * (kBulkThreads / 32) + 1];
    constexpr int NW = kBulkThreads / 32;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int j = tid >> 1, half = tid & 1;
    const uint32_t base = (uint32_t)__cvta_generic_to_shared(smem);
    BulkItem* items = reinterpret_cast<BulkItem*>(smem + 16);
    auto bar = [&](int s) { return base + 8u * (uint32_t)s; };
    auto stage_addr = [&](int s) { return base + (uint32_t)kBulkHeader + (uint32_t)s * (uint32_t)(kBulkStagePairs * 8); };
    const uint64_t pol = l2_normal();
    unsigned long long n_ent = 0, n_upd = 0;
    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) bulk_mbar_init(bar(s), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        for (int s = 0; s < STAGES; ++s)
            bulk_issue(P, order, pcolptr, pvptr, pairs, vptr, start, queue, &items[s], stage_addr(s), bar(s));
    }
    uint32_t parity = 0;  // bit s: phase of stage s's barrier to wait for
    int cur = 0;
    bool failed = false;
    for (;;) {
        __syncthreads();
        const BulkItem it = items[cur];
        if (!it.valid) break;
        const bool ok = bulk_mbar_wait(bar(cur), (parity >> cur) & 1u);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        parity ^= 1u << cur;
        const uint2* stp = reinterpret_cast<const uint2*>(smem + kBulkHeader + (size_t)cur * kBulkStagePairs * 8) + it.d;
        const int n = (int)(it.en - it.b);
        // Warp 0 loads the voxel and its in-plane neighbours now; they are in
        // registers when the penalty solve starts after the gather.
        double wn = 0.0;
        float xn = 0.f, xqf = 0.f;
        if (wid == 0) {
            xn = neighbour_value(P, x, it.q, lane, &wn);
            xqf = __ldcg(x + it.q);
        }
        float ev[kBulkRows];
#pragma unroll
        for (int i = 0; i < kBulkRows; ++i) {
            const int p = j + kBulkNP * i;
            float v = 0.f;
            if (p < it.ns) {
                const uint2 pr = stp[p];
                if (!half || (pr.y >> 16)) v = __ldcg(e + ((int)pr.x + it.off + half));
            }
            ev[i] = v;
        }
        float acc_b = 0.f, acc_a = 0.f;
#pragma unroll
        for (int i = 0; i < kBulkRows; ++i) {
            const int p = j + kBulkNP * i;
            if (p < it.ns) {
                const uint32_t wb = stp[p].y;
                const float wv = half ? half_hi(wb) : half_lo(wb);
                acc_b = fmaf(wv, ev[i], acc_b);
                acc_a = fmaf(wv, wv, acc_a);
            }
        }
        for (int b2 = it.ns; b2 < n; b2 += kBulkNP * kU) {
            int qo[kU];
            float wo[kU];
            load_pair_entries<kU, kBulkNP>(pairs, it.b + b2 + j, it.en, it.off, half, pol, qo, wo);
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const float evu = qo[u] >= 0 ? __ldcg(e + qo[u]) : 0.f;
                acc_b = fmaf(wo[u], evu, acc_b);
                acc_a = fmaf(wo[u], wo[u], acc_a);
            }
        }
        acc_b = warp_sum(acc_b);
        acc_a = warp_sum(acc_a);
        if (lane == 0) {
            s_red[wid] = acc_b;
            s_red[NW + wid] = acc_a;
        }
        __syncthreads();
        if (wid == 0) {
            double beta = 0.0, alpha = 0.0;
#pragma unroll
            for (int i = 0; i < NW; ++i) {
                beta += (double)s_red[i];
                alpha += (double)s_red[NW + i];
            }
            const double xq = (double)xqf;
            const double diff = wn != 0.0 ? (double)xn - xq : 0.0;
            double upd = penalty_solve(P.penalty, P.lambda, P.delta, alpha, beta, diff, wn) * P.relax;
            if (upd + xq < 0.0) upd = -xq;  // icd_iteration.cpp:233-234
            if (lane == 0) {
                x[it.q] = (float)(xq + upd);
                s_red[2 * NW] = (float)upd;
            }
        }
        __syncthreads();
        const float du = s_red[2 * NW];
        if (du != 0.f) {
#pragma unroll
            for (int i = 0; i < kBulkRows; ++i) {
                const int p = j + kBulkNP * i;
                if (p < it.ns) {
                    const uint2 pr = stp[p];
                    if (!half || (pr.y >> 16))
                        atomicAdd(e + ((int)pr.x + it.off + half), -du * (half ? half_hi(pr.y) : half_lo(pr.y)));
                }
            }
            for (int b2 = it.ns; b2 < n; b2 += kBulkNP * kU) {
                int qo[kU];
                float wo[kU];
                load_pair_entries<kU, kBulkNP>(pairs, it.b + b2 + j, it.en, it.off, half, pol, qo, wo);
#pragma unroll
                for (int u = 0; u < kU; ++u)
                    if (qo[u] >= 0) atomicAdd(e + qo[u], -du * wo[u]);
            }
            n_ent += (unsigned long long)it.n_entries;
            ++n_upd;
        }
        __syncthreads();  // the stage, the item record and s_red are free
        if (tid == 0)
            bulk_issue(P, order, pcolptr, pvptr, pairs, vptr, start, queue, &items[cur], stage_addr(cur), bar(cur));
        cur = cur + 1 == STAGES ? 0 : cur + 1;
    }
    if (failed) {
        // A copy that never completed: record it, then wait (bounded) for any
        // copy still writing this CTA's shared memory before exiting.
        if (tid == 0) {
            atomicExch(err, 1ull);
            for (int c = 0; c < STAGES; ++c)
                if (items[c].valid) bulk_mbar_wait(bar(c), (parity >> c) & 1u);
        }
        __syncthreads();
    }
    flush_counts(stats, n_upd, n_ent, tid);
}

// ---------------------------------------------------------------------------
// Claim-ahead bulk-staged kernel (stage_column 6): the update of
// icd_bulk_kernel<1> with the work-queue claim taken off the critical path.
// In the one-stage kernel every update waits, before its copy can even be
// issued, for a chain of dependent global round trips: the work-queue claim,
// the visiting-order entry it names, then the column's pair offsets. Here
// warp 1, idle while warp 0 solves the current update's penalty, claims the
// next item and resolves its record; after the scatter only the copy is left
// to issue. A CTA holds two claimed items (one being updated, one claimed),
// so the launch keeps twice the CTAs within the visiting order's concurrency
// bound. (Issuing the next copy right after the gather, with the scatter
// re-reading the pairs from global memory, measured slower: the re-read
// column mostly missed L2 and DRAM bytes per entry rose by 39 %.)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void bulk_claim(const GParams& P, const uint32_t* __restrict__ order,
                                           const int64_t* __restrict__ pcolptr, const uint32_t* __restrict__ pvptr,
                                           const uint32_t* __restrict__ vptr, const int32_t* __restrict__ start,
                                           unsigned long long* queue, BulkItem* it) {
    const uint64_t item = atomicAdd(queue, 1ull);
    if (item >= P.n_items) {
        it->valid = 0;
        return;
    }
    const uint64_t ncol = (uint64_t)P.nx * P.ny;
    const uint32_t packed = __ldg(order + item);
    const uint64_t col = packed / (uint32_t)P.nz;
    const int k = (int)(packed % (uint32_t)P.nz);
    const int s = start[k];
    const int v0 = max(0, -s), v1 = min(P.nvsm, P.readings - s);
    int64_t b = 0, en = 0, ne = 0;
    if (v1 > v0) {
        const int64_t cb = pcolptr[col];
        const uint32_t* vp = pvptr + col * P.nvsm1;
        b = cb + vp[v0];
        en = cb + vp[v1];
        ne = (int64_t)vptr[col * P.nvsm1 + v1] - (int64_t)vptr[col * P.nvsm1 + v0];
    }
    const int ns = (int)min(en - b, (int64_t)kBulkCap);
    it->b = b;
    it->en = en;
    it->q = (int64_t)col + (int64_t)ncol * k;
    it->n_entries = ne;
    it->off = s * P.nch * P.nr;
    it->d = (int)(b - (b & ~(int64_t)1));
    it->ns = ns;
    it->valid = 1;
}

// Start the copy of a claimed item's staged pairs [b0, e1) (b0 = b rounded
// down, e1 = b + ns rounded up to even: 16-byte boundaries; the pair array
// has two pairs of padding past its end) into the stage at `dst`.
__device__ __forceinline__ void bulk_copy(const uint2* __restrict__ pairs, const BulkItem& it, uint32_t dst,
                                          uint32_t bar) {
    const int64_t b0 = it.b - it.d;
    const int64_t e1 = (it.b + it.ns + 1) & ~(int64_t)1;
    const uint32_t bytes = it.ns > 0 ? (uint32_t)((e1 - b0) * 8) : 0u;
    // The stage was last read through the generic proxy; order those reads
    // before the async-proxy writes of the copy.
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    bulk_mbar_expect_tx(bar, bytes);
    const char* src = reinterpret_cast<const char*>(pairs + b0);
    for (uint32_t o = 0; o < bytes; o += kBulkChunk) bulk_g2s(dst + o, src + o, min(kBulkChunk, bytes - o), bar);
}

__global__ void __launch_bounds__(kBulkThreads, 4) icd_bulk_pipe_kernel(
    GParams P, const uint32_t* __restrict__ order, const int64_t* __restrict__ pcolptr,
    const uint32_t* __restrict__ pvptr, const uint2* __restrict__ pairs, const uint32_t* __restrict__ vptr,
    const int32_t* __restrict__ start, float* e, float* x, unsigned long long* queue, unsigned long long* stats,
    unsigned long long* err) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ float s_red[2 * (kBulkThreads / 32) + 1];
    constexpr int NW = kBulkThreads / 32;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int j = tid >> 1, half = tid & 1;
    const uint32_t base = (uint32_t)__cvta_generic_to_shared(smem);
    BulkItem* ring = reinterpret_cast<BulkItem*>(smem + 16);  // current item, next item
    const uint32_t bar = base;
    const uint32_t stage = base + (uint32_t)kBulkHeader;
    const uint2* stp0 = reinterpret_cast<const uint2*>(smem + kBulkHeader);
    const uint64_t pol = l2_normal();
    unsigned long long n_ent = 0, n_upd = 0;
    if (tid == 0) {
        bulk_mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        bulk_claim(P, order, pcolptr, pvptr, vptr, start, queue, &ring[0]);
        if (ring[0].valid) bulk_copy(pairs, ring[0], stage, bar);
    }
    uint32_t parity = 0;
    int cur = 0;
    bool failed = false;
    for (;;) {
        __syncthreads();
        const BulkItem it = ring[cur];
        const int nxt = cur ^ 1;
        if (!it.valid) break;
        const bool ok = bulk_mbar_wait(bar, parity);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        parity ^= 1u;
        const uint2* stp = stp0 + it.d;
        const int n = (int)(it.en - it.b);
        double wn = 0.0;
        float xn = 0.f, xqf = 0.f;
        if (wid == 0) {
            xn = neighbour_value(P, x, it.q, lane, &wn);
            xqf = __ldcg(x + it.q);
        }
        float ev[kBulkRows];
#pragma unroll
        for (int i = 0; i < kBulkRows; ++i) {
            const int p = j + kBulkNP * i;
            float v = 0.f;
            if (p < it.ns) {
                const uint2 pr = stp[p];
                if (!half || (pr.y >> 16)) v = __ldcg(e + ((int)pr.x + it.off + half));
            }
            ev[i] = v;
        }
        float acc_b = 0.f, acc_a = 0.f;
#pragma unroll
        for (int i = 0; i < kBulkRows; ++i) {
            const int p = j + kBulkNP * i;
            if (p < it.ns) {
                const uint32_t wb = stp[p].y;
                const float wv = half ? half_hi(wb) : half_lo(wb);
                acc_b = fmaf(wv, ev[i], acc_b);
                acc_a = fmaf(wv, wv, acc_a);
            }
        }
        for (int b2 = it.ns; b2 < n; b2 += kBulkNP * kU) {
            int qo[kU];
            float wo[kU];
            load_pair_entries<kU, kBulkNP>(pairs, it.b + b2 + j, it.en, it.off, half, pol, qo, wo);
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const float evu = qo[u] >= 0 ? __ldcg(e + qo[u]) : 0.f;
                acc_b = fmaf(wo[u], evu, acc_b);
                acc_a = fmaf(wo[u], wo[u], acc_a);
            }
        }
        acc_b = warp_sum(acc_b);
        acc_a = warp_sum(acc_a);
        if (lane == 0) {
            s_red[wid] = acc_b;
            s_red[NW + wid] = acc_a;
        }
        __syncthreads();
        if (wid == 0) {
            double beta = 0.0, alpha = 0.0;
#pragma unroll
            for (int i = 0; i < NW; ++i) {
                beta += (double)s_red[i];
                alpha += (double)s_red[NW + i];
            }
            const double xq = (double)xqf;
            const double diff = wn != 0.0 ? (double)xn - xq : 0.0;
            double upd = penalty_solve(P.penalty, P.lambda, P.delta, alpha, beta, diff, wn) * P.relax;
            if (upd + xq < 0.0) upd = -xq;  // icd_iteration.cpp:233-234
            if (lane == 0) {
                x[it.q] = (float)(xq + upd);
                s_red[2 * NW] = (float)upd;
            }
        } else if (tid == 32) {
            // The next item, claimed while warp 0 solves (the slot held the
            // item finished last round, no longer read).
            bulk_claim(P, order, pcolptr, pvptr, vptr, start, queue, &ring[nxt]);
        }
        __syncthreads();
        const float du = s_red[2 * NW];
        if (du != 0.f) {
#pragma unroll
            for (int i = 0; i < kBulkRows; ++i) {
                const int p = j + kBulkNP * i;
                if (p < it.ns) {
                    const uint2 pr = stp[p];
                    if (!half || (pr.y >> 16))
                        atomicAdd(e + ((int)pr.x + it.off + half), -du * (half ? half_hi(pr.y) : half_lo(pr.y)));
                }
            }
            for (int b2 = it.ns; b2 < n; b2 += kBulkNP * kU) {
                int qo[kU];
                float wo[kU];
                load_pair_entries<kU, kBulkNP>(pairs, it.b + b2 + j, it.en, it.off, half, pol, qo, wo);
#pragma unroll
                for (int u = 0; u < kU; ++u)
                    if (qo[u] >= 0) atomicAdd(e + qo[u], -du * wo[u]);
            }
            n_ent += (unsigned long long)it.n_entries;
            ++n_upd;
        }
        __syncthreads();  // the stage and s_red are free
        if (tid == 0 && ring[nxt].valid) bulk_copy(pairs, ring[nxt], stage, bar);
        cur = nxt;
    }
    if (failed) {
        // A copy that never completed: record it, then wait (bounded) for it
        // before exiting, so no copy still writes this CTA's shared memory.
        if (tid == 0) {
            atomicExch(err, 1ull);
            bulk_mbar_wait(bar, parity);
        }
        __syncthreads();
    }
    flush_counts(stats, n_upd, n_ent, tid);
}

// Lockstep stacks: one CTA of kStack warps per slice stack (the same-parity
// slices of one physical cell, consecutive in the visiting order; the stack
// table lists where each starts). Members start at the stack's common data
// view and wrap around (as in process_item), so at equal positions of their
// entry sequences they are at about the same data view; a CTA barrier after
// every chunk of 32 x U entries keeps them within a chunk of one another, so
// the sinogram sectors they share are fetched from DRAM once and hit in L2
// for the others (items of one stack drifting apart by more than the L2's
// residence time was what made the streamed kernel re-read them). The
// scatter walks the chunks back in the same lockstep.
template <class WT, int U>
__global__ void __launch_bounds__(32 * kStack, U == 8 ? 2 : 1) icd_lockstep_kernel(
    GParams P, const uint32_t* __restrict__ order, const uint32_t* __restrict__ stacks, uint64_t n_stacks,
    const int64_t* __restrict__ colptr, const uint32_t* __restrict__ vptr, const int32_t* __restrict__ idx,
    const WT* __restrict__ w, const int32_t* __restrict__ start, float* e, float* x, unsigned long long* queue,
    unsigned long long* stats) {
    __shared__ unsigned long long s_stack;
    __shared__ int s_chunks[kStack];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint64_t ncol = (uint64_t)P.nx * P.ny;
    unsigned long long n_ent = 0, n_upd = 0;
    for (;;) {
        if (threadIdx.x == 0) s_stack = atomicAdd(queue, 1ull);
        __syncthreads();
        const unsigned long long sid = s_stack;
        if (sid >= n_stacks) break;
        const uint32_t i0 = __ldg(stacks + sid), i1 = __ldg(stacks + sid + 1);
        // A stack holds at most kStack items; longer runs go in blocks.
        for (uint32_t j0 = i0; j0 < i1; j0 += kStack) {
            const uint32_t item = j0 + (uint32_t)wid;
            int64_t hi = 0, lo = 0, q = 0;
            int n = 0, n1 = 0, off = 0;
            if (item < i1) {
                const uint32_t packed = __ldg(order + item);
                const uint64_t col = packed / (uint32_t)P.nz;
                const int k = (int)(packed % (uint32_t)P.nz);
                q = (int64_t)col + (int64_t)ncol * k;
                const int s = start[k];
                const int v0 = max(0, -s), v1 = min(P.nvsm, P.readings - s);
                if (v1 > v0) {
                    const int64_t cb = colptr[col];
                    const uint32_t* vp = vptr + col * P.nvsm1;
                    const uint32_t b = vp[v0], en = vp[v1];
                    const int kl = min(k - (k % (2 * kStack)) + (k % 2) + 2 * (kStack - 1),
                                       ((k & 1) ? P.last_slice[1] : P.last_slice[0]));
                    const uint32_t mid = vp[min(max(start[kl] - s, v0), v1)];
                    n = (int)(en - b);
                    n1 = (int)(en - mid);
                    hi = cb + mid;
                    lo = cb + b - n1;
                }
                off = s * P.nch * P.nr;
            }
            const int chunks = (n + 32 * U - 1) / (32 * U);
            if (lane == 0) s_chunks[wid] = chunks;
            __syncthreads();
            int maxc = 0;
#pragma unroll
            for (int i = 0; i < kStack; ++i) maxc = max(maxc, s_chunks[i]);
            // (maxc is the same in every warp.) With no chunk loop below,
            // this barrier keeps s_chunks from being rewritten while read.
            if (maxc == 0) __syncthreads();

            float acc_b = 0.f, acc_a = 0.f;
            {
                const uint64_t keep = l2_keep();
                int qa[U];
                float wa[U];
                load_seq<U>(idx, w, lane, n, n1, hi, lo, off, keep, qa, wa);
                for (int c = 0; c < maxc; ++c) {
                    if (c < chunks) {
                        float ev[U];
#pragma unroll
                        for (int u = 0; u < U; ++u) ev[u] = (qa[u] >= 0) ? __ldcg(e + qa[u]) : 0.f;
                        int qb[U];
                        float wb[U];
                        load_seq<U>(idx, w, (c + 1) * (32 * U) + lane, n, n1, hi, lo, off, keep, qb, wb);
#pragma unroll
                        for (int u = 0; u < U; ++u) {
                            acc_b = fmaf(wa[u], ev[u], acc_b);
                            acc_a = fmaf(wa[u], wa[u], acc_a);
                            qa[u] = qb[u];
                            wa[u] = wb[u];
                        }
                    }
                    __syncthreads();
                }
            }
            float du = 0.f;
            if (item < i1) {
                const double beta = (double)warp_sum(acc_b);
                const double alpha = (double)warp_sum(acc_a);
                const double xq = (double)__ldcg(x + q);
                double upd = penalty_step(P, x, q, xq, alpha, beta, lane) * P.relax;
                if (upd + xq < 0.0) upd = -xq;  // icd_iteration.cpp:233-234
                if (lane == 0) x[q] = (float)(xq + upd);
                du = (float)upd;
            }
            {
                const uint64_t drop = l2_drop();
                for (int c = maxc - 1; c >= 0; --c) {
                    if (du != 0.f && c < chunks) {
                        int qs[U];
                        float ws[U];
                        load_seq<U>(idx, w, c * (32 * U) + lane, n, n1, hi, lo, off, drop, qs, ws);
#pragma unroll
                        for (int u = 0; u < U; ++u)
                            if (qs[u] >= 0) atomicAdd(e + qs[u], -du * ws[u]);
                    }
                    __syncthreads();
                }
            }
            if (du != 0.f) {
                n_ent += (unsigned long long)n;
                ++n_upd;
            }
        }
    }
    flush_counts(stats, n_upd, n_ent, lane);
}

// Shared-memory staged variant: one warp per voxel update, NW warps per CTA,
// each warp owning `cap` stage positions in shared memory. The gather reads
// the column's matrix entries from HBM once, with a streaming (evict-first)
// L2 policy so they do not displace the error sinogram, keeps each entry's
// sinogram index (slice offset applied) and weight in the stage and gathers
// e; after the penalty step the scatter reads the entries back from shared
// memory, latest-gathered first (their e sectors are the likeliest to still
// be in L2). Columns longer than `cap` re-read their tail from HBM.
// One voxel update by one warp with the column staged in shared memory
// (sq / sw: this warp's `cap` stage positions); counts an update that
// scattered in n_upd / n_ent.
template <class WT, int U>
__device__ __forceinline__ void staged_item(const GParams& P, const uint32_t* __restrict__ order,
                                            const int64_t* __restrict__ colptr, const uint32_t* __restrict__ vptr,
                                            const int32_t* __restrict__ idx, const WT* __restrict__ w,
                                            const int32_t* __restrict__ start, float* e, float* x, uint64_t item,
                                            int lane, int32_t* sq, typename WBits<WT>::T* sw, int cap,
                                            uint64_t stream, unsigned long long& n_ent, unsigned long long& n_upd) {
    const uint64_t ncol = (uint64_t)P.nx * P.ny;
    const uint32_t packed = __ldg(order + item);
    const uint64_t col = packed / (uint32_t)P.nz;
    const int k = (int)(packed % (uint32_t)P.nz);
    const int64_t q = (int64_t)col + (int64_t)ncol * k;
    const int s = start[k];
    const int v0 = max(0, -s), v1 = min(P.nvsm, P.readings - s);
    int64_t b = 0, en = 0, mid = 0;
    if (v1 > v0) {
        const int64_t cb = colptr[col];
        const uint32_t* vp = vptr + col * P.nvsm1;
        b = cb + vp[v0];
        en = cb + vp[v1];
        // Same common start view for the members of a slice stack as
        // process_item.
        const int kl = min(k - (k % (2 * kStack)) + (k % 2) + 2 * (kStack - 1),
                           ((k & 1) ? P.last_slice[1] : P.last_slice[0]));
        const int vs = min(max(start[kl] - s, v0), v1);
        mid = cb + vp[vs];
    }
    const int off = s * P.nch * P.nr;
    const int64_t n1 = en - mid, n = en - b;

    float acc_b = 0.f, acc_a = 0.f;
    stage_gather<WT, U>(idx, w, e, mid, en, 0, off, lane, stream, sq, sw, cap, acc_b, acc_a);
    stage_gather<WT, U>(idx, w, e, b, mid, n1, off, lane, stream, sq, sw, cap, acc_b, acc_a);
    const double beta = (double)warp_sum(acc_b);
    const double alpha = (double)warp_sum(acc_a);

    const double xq = (double)__ldcg(x + q);
    double upd = penalty_step(P, x, q, xq, alpha, beta, lane) * P.relax;
    if (upd + xq < 0.0) upd = -xq;  // icd_iteration.cpp:233-234
    if (lane == 0) x[q] = (float)(xq + upd);
    const float du = (float)upd;
    __syncwarp();  // stage writes of every lane visible to the scatter
    if (du != 0.f) {
        // Positions [cap, n) were not staged: re-read them (last first).
        for (int64_t p = n - 1 - lane; p >= cap; p -= 32) {
            const int64_t m = p < n1 ? mid + p : b + (p - n1);
            atomicAdd(e + (ld_idx(idx + m, stream) + off), -du * WBits<WT>::value(WBits<WT>::load(w, m, stream)));
        }
        const int64_t ns = n < cap ? n : cap;
        int64_t p = ns - 1 - lane;
        for (; p >= 32 * 3; p -= 32 * 4) {
            const int32_t q0 = sq[p], q1 = sq[p - 32], q2 = sq[p - 64], q3 = sq[p - 96];
            const float w0 = WBits<WT>::value(sw[p]), w1 = WBits<WT>::value(sw[p - 32]);
            const float w2 = WBits<WT>::value(sw[p - 64]), w3 = WBits<WT>::value(sw[p - 96]);
            atomicAdd(e + q0, -du * w0);
            atomicAdd(e + q1, -du * w1);
            atomicAdd(e + q2, -du * w2);
            atomicAdd(e + q3, -du * w3);
        }
        for (; p >= 0; p -= 32) atomicAdd(e + sq[p], -du * WBits<WT>::value(sw[p]));
        n_ent += (unsigned long long)n;
        ++n_upd;
    }
    __syncwarp();  // stage reads done before the next item overwrites it
}

template <class WT, int U, int NW>
__global__ void __launch_bounds__(32 * NW, 1) icd_staged_kernel(GParams P, const uint32_t* __restrict__ order,
                                                                const int64_t* __restrict__ colptr,
                                                                const uint32_t* __restrict__ vptr,
                                                                const int32_t* __restrict__ idx,
                                                                const WT* __restrict__ w,
                                                                const int32_t* __restrict__ start, float* e, float* x,
                                                                unsigned long long* queue, int cap,
                                                                unsigned long long* stats) {
    using SW = typename WBits<WT>::T;
    extern __shared__ __align__(16) unsigned char stage_smem[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int32_t* sq = reinterpret_cast<int32_t*>(stage_smem) + (size_t)wid * cap;
    SW* sw = reinterpret_cast<SW*>(reinterpret_cast<int32_t*>(stage_smem) + (size_t)NW * cap) + (size_t)wid * cap;
    const uint64_t stream = l2_drop();
    unsigned long long n_ent = 0, n_upd = 0;
    for (;;) {
        unsigned long long item = 0;
        if (lane == 0) item = atomicAdd(queue, 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= P.n_items) break;
        staged_item<WT, U>(P, order, colptr, vptr, idx, w, start, e, x, item, lane, sq, sw, cap, stream, n_ent, n_upd);
    }
    flush_counts(stats, n_upd, n_ent, lane);
}

// CTA-per-voxel variant: WPV warps share one voxel update. Each thread keeps
// up to R of the item's entries (sinogram index and weight) in registers
// from the gather to the scatter, so the matrix column is read from memory
// once per update and the reductions hit e's lines while they are still in
// L2; with one item per CTA, one to a few updates per SM are in flight.
// Entries beyond 32 * WPV * R (rare) are streamed twice. With
// P.stack_align the sweep starts at the slice stack's common data view and
// wraps around (as in process_item), so the stack's members, consecutive in
// the visiting order, touch each shared sinogram sector within microseconds
// of one another; with P.l2_hints the matrix loads (read once) are marked
// evict-first and the e gathers evict-last.
template <class WT, int WPV, int R>
__global__ void __launch_bounds__(32 * WPV, 16 / WPV) icd_cta_kernel(GParams P, const uint32_t* __restrict__ order,
                                                        const int64_t* __restrict__ colptr,
                                                        const uint32_t* __restrict__ vptr,
                                                        const int32_t* __restrict__ idx, const WT* __restrict__ w,
                                                        const int32_t* __restrict__ start, float* e, float* x,
                                                        unsigned long long* queue, unsigned long long* stats) {
    constexpr int NT = 32 * WPV;
    unsigned long long n_ent = 0, n_upd = 0;
    constexpr int64_t CAP = (int64_t)NT * R;
    __shared__ unsigned long long s_item;
    __shared__ float s_red[2 * WPV + 1];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const uint64_t ncol = (uint64_t)P.nx * P.ny;
    const uint64_t pol_m = P.l2_hints ? l2_drop() : l2_normal();
    const uint64_t pol_e = P.l2_hints ? l2_keep() : l2_normal();
    for (;;) {
        if (tid == 0) s_item = atomicAdd(queue, 1ull);
        __syncthreads();
        const uint64_t item = s_item;
        if (item >= P.n_items) break;
        const uint32_t packed = __ldg(order + item);
        const uint64_t col = packed / (uint32_t)P.nz;
        const int k = (int)(packed % (uint32_t)P.nz);
        const int64_t q = (int64_t)col + (int64_t)ncol * k;
        const int s = start[k];
        const int v0 = max(0, -s), v1 = min(P.nvsm, P.readings - s);
        int64_t b = 0, en = 0, mid = 0;
        if (v1 > v0) {
            const int64_t cb = colptr[col];
            const uint32_t* vp = vptr + col * P.nvsm1;
            b = cb + vp[v0];
            en = cb + vp[v1];
            mid = P.stack_align ? cb + vp[stack_start_view(P, start, k, s, v0, v1)] : b;
        }
        const int off = s * P.nch * P.nr;
        // Sweep position p -> entry p + hi for p < n1 ([mid, en)), else p + lo
        // ([b, mid)).
        const int n = (int)(en - b), n1 = (int)(en - mid);
        const int64_t hi = mid, lo = b - n1;
        const int nreg = min(n, (int)CAP);
        int qr[R];
        float wr[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int p = tid + NT * r;
            if (p < nreg) {
                const int64_t m = (p < n1 ? hi : lo) + p;
                qr[r] = ld_idx(idx + m, pol_m) + off;
                wr[r] = ldw_hint(w, m, pol_m);
            } else {
                qr[r] = -1;
                wr[r] = 0.f;
            }
        }
        float acc_b = 0.f, acc_a = 0.f;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const float ev = qr[r] >= 0 ? ld_e(e + qr[r], pol_e) : 0.f;
            acc_b = fmaf(wr[r], ev, acc_b);
            acc_a = fmaf(wr[r], wr[r], acc_a);
        }
        for (int base = (int)CAP; base < n; base += NT * kU) {
            int qo[kU];
            float wo[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int p = base + tid + NT * u;
                qo[u] = -1;
                wo[u] = 0.f;
                if (p < n) {
                    const int64_t m = (p < n1 ? hi : lo) + p;
                    qo[u] = ld_idx(idx + m, pol_m) + off;
                    wo[u] = ldw_hint(w, m, pol_m);
                }
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const float ev = qo[u] >= 0 ? ld_e(e + qo[u], pol_e) : 0.f;
                acc_b = fmaf(wo[u], ev, acc_b);
                acc_a = fmaf(wo[u], wo[u], acc_a);
            }
        }
        acc_b = warp_sum(acc_b);
        acc_a = warp_sum(acc_a);
        if (lane == 0) {
            s_red[wid] = acc_b;
            s_red[WPV + wid] = acc_a;
        }
        __syncthreads();
        if (wid == 0) {
            double beta = 0.0, alpha = 0.0;
#pragma unroll
            for (int i = 0; i < WPV; ++i) {
                beta += (double)s_red[i];
                alpha += (double)s_red[WPV + i];
            }
            const double xq = (double)__ldcg(x + q);
            double upd = penalty_step(P, x, q, xq, alpha, beta, lane) * P.relax;
            if (upd + xq < 0.0) upd = -xq;  // icd_iteration.cpp:233-234
            if (lane == 0) {
                x[q] = (float)(xq + upd);
                s_red[2 * WPV] = (float)upd;
            }
        }
        __syncthreads();
        const float du = s_red[2 * WPV];
        if (du != 0.f) {
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (qr[r] >= 0) atomicAdd(e + qr[r], -du * wr[r]);
            for (int base = (int)CAP; base < n; base += NT * kU) {
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    const int p = base + tid + NT * u;
                    if (p < n) {
                        const int64_t m = (p < n1 ? hi : lo) + p;
                        atomicAdd(e + (ld_idx(idx + m, pol_m) + off), -du * ldw_hint(w, m, pol_m));
                    }
                }
            }
            n_ent += (unsigned long long)(en - b);
            ++n_upd;
        }
        __syncthreads();  // s_item / s_red reused by the next item
    }
    flush_counts(stats, n_upd, n_ent, tid);
}

// Batched variant: one persistent launch drains the merged queue of several
// independent scans (`merged[t]` = scan << 40 | item within that scan).
template <class WT>
__global__ void __launch_bounds__(256) icd_batch_kernel(const ScanRefs<WT>* __restrict__ scans,
                                                        const uint64_t* __restrict__ merged, uint64_t n_total,
                                                        double relax, unsigned long long* queue) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(queue, 1ull);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= n_total) break;
        const uint64_t m = __ldg(merged + t);
        const ScanRefs<WT>& S = scans[m >> 40];
        GParams P = S.P;
        P.relax = relax;
        process_item(P, S.order, S.colptr, S.vptr, S.idx, S.w, S.start, S.e, S.x, m & ((1ull << 40) - 1), lane);
    }
}

// Batched variant of icd_staged_kernel (the column of each update staged in
// shared memory, 4 updates per CTA).
template <class WT>
__global__ void __launch_bounds__(128, 1) icd_batch_staged_kernel(const ScanRefs<WT>* __restrict__ scans,
                                                                  const uint64_t* __restrict__ merged,
                                                                  uint64_t n_total, double relax,
                                                                  unsigned long long* queue, int cap) {
    using SW = typename WBits<WT>::T;
    extern __shared__ __align__(16) unsigned char stage_smem[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int32_t* sq = reinterpret_cast<int32_t*>(stage_smem) + (size_t)wid * cap;
    SW* sw = reinterpret_cast<SW*>(reinterpret_cast<int32_t*>(stage_smem) + (size_t)4 * cap) + (size_t)wid * cap;
    const uint64_t stream = l2_drop();
    unsigned long long n_ent = 0, n_upd = 0;
    for (;;) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(queue, 1ull);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= n_total) break;
        const uint64_t m = __ldg(merged + t);
        const ScanRefs<WT>& S = scans[m >> 40];
        GParams P = S.P;
        P.relax = relax;
        staged_item<WT, 16>(P, S.order, S.colptr, S.vptr, S.idx, S.w, S.start, S.e, S.x, m & ((1ull << 40) - 1), lane,
                            sq, sw, cap, stream, n_ent, n_upd);
    }
}

// Merge keys: scan s's j-th item at fractional position (j + 0.5) / n_s, so
// every scan has a share of the items in flight proportional to its size.
__global__ void merge_keys_kernel(uint64_t n_s, uint32_t scan, uint64_t base, uint64_t* __restrict__ keys,
                                  uint64_t* __restrict__ vals) {
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n_s; j += (uint64_t)gridDim.x * blockDim.x) {
        keys[base + j] = (uint64_t)(((double)j + 0.5) / (double)n_s * 4294967296.0) * 64ull + scan;
        vals[base + j] = ((uint64_t)scan << 40) | j;
    }
}

// Sort keys of the visiting order (see the file comment); voxels outside the
// scanner FOV (icd_iteration.cpp:181) get the largest key and are dropped.
//   key = ((cell-in-tile rank * Q + slice parity) * n_tiles + tile) * nz + slice
// Tiles are T x T cells of the fixed frame; inside a tile cells follow a
// serpentine raster, so consecutive stacks of a tile are neighbours.
struct OrderParams {
    int nx, ny, nz, T, Q, margin, lx;
    uint64_t n_tiles;
    double cvx, cvy, vx, vy, fov_limit;
};

__global__ void order_keys_kernel(OrderParams O, const double* __restrict__ cs, const float* __restrict__ prio,
                                  float thr, uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const uint64_t ncol = (uint64_t)O.nx * O.ny, n = ncol * O.nz;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
        const int k = (int)(t / ncol);
        const uint64_t col = t % ncol;
        const int i = (int)(col % O.nx), j = (int)(col / O.nx);
        vals[t] = (uint32_t)(col * O.nz + k);
        const double xx = (i - O.cvx) * O.vx, yy = (j - O.cvy) * O.vy;
        if (!(xx * xx + yy * yy < O.fov_limit) || (prio && !(prio[t] >= thr))) {
            keys[t] = ~0ull;
            continue;
        }
        // Voxel centre in the fixed frame, in voxel units, snapped to the grid.
        const double c = cs[2 * k], s = cs[2 * k + 1];
        const double px = c * (i - O.cvx) - s * (j - O.cvy) + O.cvx;
        const double py = s * (i - O.cvx) + c * (j - O.cvy) + O.cvy;
        const int a = (int)llrint(px) + O.margin, b = (int)llrint(py) + O.margin;
        const int u = a % O.T, v = b % O.T;
        const uint64_t rank_in_tile = (uint64_t)v * O.T + (uint64_t)((v & 1) ? (O.T - 1 - u) : u);
        const uint64_t tile = (uint64_t)(a / O.T) + (uint64_t)O.lx * (uint64_t)(b / O.T);
        keys[t] = ((rank_in_tile * O.Q + (uint64_t)(k % O.Q)) * O.n_tiles + tile) * (uint64_t)O.nz + (uint64_t)k;
    }
}

// Rotated voxel centres snapped to the fixed grid can land two (rarely three)
// in-plane neighbours of one slice on the same cell: equal keys, adjacent in
// the sorted order, so they would be updated concurrently although they share
// nearly all of their rays. Every occupant after the first moves to a
// sub-phase after its cell's rank (key = rank * M + rest becomes
// (2 rank + 1) * M + rest, M = Q * n_tiles * nz), a whole rank sweep away.
__global__ void split_collisions_kernel(const uint64_t* __restrict__ sorted, uint64_t n, uint64_t M,
                                        uint64_t* __restrict__ keys_out) {
    for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < n; p += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = sorted[p];
        if (k == ~0ull) {
            keys_out[p] = k;
            continue;
        }
        const uint64_t dup = (p > 0 && sorted[p - 1] == k) ? 1ull : 0ull;
        keys_out[p] = (2ull * (k / M) + dup) * M + k % M;
    }
}

// Slice stacks of the sorted order: a stack is a run of items with the same
// key apart from the slice, and the same block of 2 kStack slices (kStack
// slices of one parity). flags[p] = 1 where a stack starts.
__global__ void stack_heads_kernel(const uint64_t* __restrict__ sorted, uint64_t n, uint64_t nz,
                                   uint8_t* __restrict__ flags) {
    for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < n; p += (uint64_t)gridDim.x * blockDim.x) {
        bool head = p == 0;
        if (!head) {
            const uint64_t a = sorted[p - 1], b = sorted[p];
            head = a / nz != b / nz || (a % nz) / (2 * kStack) != (b % nz) / (2 * kStack);
        }
        flags[p] = head ? 1 : 0;
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
    memset(&P, 0, sizeof(P));  // compared bytewise as part of the graph key
    P.nx = (int)g.num_voxels_x;
    P.ny = (int)g.num_voxels_y;
    P.nz = (int)g.num_voxels_z;
    P.nch = (int)g.n_channels;
    P.nr = (int)g.Nrows_projection;
    P.nvsm = (int)ssm->nvsm;
    P.nvsm1 = ssm->nvsm + 1;
    P.readings = (int)g.Readings;
    P.penalty = g.penalty;
    P.last_slice[(P.nz - 1) % 2] = P.nz - 1;
    P.last_slice[P.nz % 2] = P.nz >= 2 ? P.nz - 2 : P.nz - 1;
    P.n_items = rc->n_order;
    P.lambda = g.lambda;
    P.delta = g.delta;
    P.relax = (o.relax > 0.0 && o.relax < 2.0) ? o.relax : 1.0;
    P.cvx = g.center_voxel_x;
    P.cvy = g.center_voxel_y;
    P.vx = g.voxel_size_x;
    P.vy = g.voxel_size_y;
    P.fov_limit = (g.acquisition_fov / 2.0) * (g.acquisition_fov / 2.0);
    P.stack_align = o.stack_align == 1 ? 1 : 0;
    P.l2_hints = o.l2_hints == 1 ? 1 : 0;
    return P;
}

}  // namespace

namespace ctbb {

// Concurrency bound of the visiting order. Items are sorted by (cell rank in
// tile, slice parity, tile, slice): the items of one cell rank (about n / T^2,
// both parities) lie a whole tile apart in-plane; the next rank holds their
// in-plane neighbours, which share nearly all of their rays. With at most one
// rank's worth of updates in flight, no two in-plane neighbours of a slice
// are updated together. Adjacent slices of one cell (the two parities of a
// rank) may be: they overlap in about half of their detector rows, and
// updating them together keeps their sinogram sectors in L2 once.
uint64_t max_items_in_flight(uint64_t n_items, int nz, int T) {
    (void)nz;
    return std::max<uint64_t>(1, n_items / ((uint64_t)T * (uint64_t)T));
}

// Voxel updates the options ask to keep in flight (warps_in_flight counts
// warps; an update takes warps_per_voxel of them).
uint64_t requested_items(const ctbb_recon* rc, const ctbb_icd_opts& o) {
    // The staged kernel keeps one CTA of 4 (or 8) updates per SM (its stage
    // fills the SM's shared memory).
    const int staged = rc->ctx->sm_count * (o.stage_column == 2 ? 8 : 4);
    // The lockstep kernel keeps two CTAs of kStack updates per SM with 8
    // entries per lane in flight (one with 16).
    const int lockstep = rc->ctx->sm_count * (o.entries_per_lane == 16 ? 1 : 2) * kStack;
    // Unless the caller sets the count, the coupling bound (default_warps_in_
    // flight) caps every kernel: on a small volume a CTA-shaped default would
    // put a large share of the voxels on each ray in flight at once, and the
    // edge-preserving iteration then oscillates.
    const int coupling = default_warps_in_flight(rc);
    // The bulk-staged kernel keeps four CTAs (one stage, also the pipelined
    // form) or three (two stages) of 8 warps per SM.
    const int bulk = rc->ctx->sm_count * (o.stage_column == 5 ? 3 : 4) * (kBulkThreads / 32);
    const int W = o.warps_in_flight > 0 ? o.warps_in_flight
                  : o.stage_column >= 4 ? std::min(bulk, coupling)
                  : o.stage_column == 3 ? std::min(lockstep, coupling)
                  : (o.stage_column ? std::min(staged, coupling) : coupling);
    const int wpv = o.stage_column >= 4 ? kBulkThreads / 32 : o.warps_per_voxel > 1 ? o.warps_per_voxel : 1;
    return std::max<uint64_t>(1, (uint64_t)(W / wpv));
}

// Tile edge T (cells); `lattice` overrides it. Default: the largest power of
// two up to nx/4 whose cell ranks hold at least the requested in-flight
// updates (longer raster sweeps converge faster per iteration, measured on
// the 512 x 512 x 64 workload).
int lattice_spacing(const ctbb_recon* rc, const ctbb_icd_opts& o) {
    const int nx = (int)rc->geom.num_voxels_x;
    if (o.lattice > 0) return std::max(1, std::min(o.lattice, nx));
    const uint64_t items = requested_items(rc, o);
    const int nz = (int)rc->geom.num_voxels_z;
    int T = 4;
    while (2 * T <= std::max(4, nx / 4) && max_items_in_flight(rc->nvox, nz, 2 * T) >= items) T *= 2;
    return std::min(T, nx);
}

}  // namespace ctbb

namespace {

using namespace ctbb;

// Visiting order for tile edge P_lat, optionally restricted to the voxels
// whose priority is at least thr.
ctbb_status build_order_into(ctbb_recon* rc, int P_lat, const float* prio, float thr, uint32_t** out,
                             uint64_t* n_out, uint32_t** stacks_out, uint64_t* n_stacks_out) {
    using namespace ctbb;
    const ctbb_geom_c& g = rc->geom;
    ctbb_ctx* ctx = rc->ctx;
    cudaStream_t st = ctx->stream;
    const uint64_t ncol = g.num_voxels_x * g.num_voxels_y, n = ncol * g.num_voxels_z;
    if (n >= (1ull << 32)) return fail(CTBB_ERR_INVALID_ARG, "volume too large for the 32-bit visiting order");
    // Rotation of each slice's frame: the tube angle of its central view.
    std::vector<double> cs(2 * g.num_voxels_z);
    const double PI = 3.141592653589793238;
    for (uint64_t k = 0; k < g.num_voxels_z; ++k) {
        const double deg = fmod((360.0 / g.num_views_per_turn) * (double)rc->slice_indices[k], 360.0);
        cs[2 * k] = cos(deg * PI / 180.0);
        cs[2 * k + 1] = sin(deg * PI / 180.0);
    }
    OrderParams O;
    O.nx = (int)g.num_voxels_x;
    O.ny = (int)g.num_voxels_y;
    O.nz = (int)g.num_voxels_z;
    O.T = P_lat;
    O.Q = O.nz >= 2 ? 2 : 1;
    // Rotated voxel centres stay within (sqrt(2) - 1)/2 of the extent outside it.
    O.margin = P_lat * ((std::max(O.nx, O.ny) / 4 + P_lat) / P_lat);
    O.lx = (O.nx + 2 * O.margin + P_lat - 1) / P_lat;
    const int ly = (O.ny + 2 * O.margin + P_lat - 1) / P_lat;
    O.n_tiles = (uint64_t)O.lx * ly;
    O.cvx = g.center_voxel_x;
    O.cvy = g.center_voxel_y;
    O.vx = g.voxel_size_x;
    O.vy = g.voxel_size_y;
    O.fov_limit = (g.acquisition_fov / 2.0) * (g.acquisition_fov / 2.0);

    double* d_cs = nullptr;
    uint64_t *d_k0 = nullptr, *d_k1 = nullptr;
    uint32_t *d_v0 = nullptr, *d_v1 = nullptr;
    void* d_tmp = nullptr;
    size_t tmp_bytes = 0;
    ctbb_status rcode = CTBB_OK;
    auto cleanup = [&]() {
        cudaFree(d_cs);
        cudaFree(d_k0);
        cudaFree(d_k1);
        cudaFree(d_v0);
        cudaFree(d_tmp);
    };
    cudaError_t e = cudaMalloc(&d_cs, cs.size() * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_k0, n * sizeof(uint64_t));
    if (e == cudaSuccess) e = cudaMalloc(&d_k1, n * sizeof(uint64_t));
    if (e == cudaSuccess) e = cudaMalloc(&d_v0, n * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&d_v1, n * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_cs, cs.data(), cs.size() * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)ctx->sm_count * 16));
        order_keys_kernel<<<grid, 256, 0, st>>>(O, d_cs, prio, thr, d_k0, d_v0);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, d_k0, d_k1, d_v0, d_v1, (int)n, 0, 64, st);
    if (e == cudaSuccess) e = cudaMalloc(&d_tmp, tmp_bytes);
    if (e == cudaSuccess)
        e = cub::DeviceRadixSort::SortPairs(d_tmp, tmp_bytes, d_k0, d_k1, d_v0, d_v1, (int)n, 0, 64, st);
    if (e == cudaSuccess) {
        const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)ctx->sm_count * 16));
        const uint64_t M = (uint64_t)O.Q * O.n_tiles * (uint64_t)O.nz;
        split_collisions_kernel<<<grid, 256, 0, st>>>(d_k1, n, M, d_k0);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cub::DeviceRadixSort::SortPairs(d_tmp, tmp_bytes, d_k0, d_k1, d_v1, d_v0, (int)n, 0, 64, st);
    if (e == cudaSuccess) std::swap(d_v0, d_v1);  // sorted values back in d_v1
    // Items outside the FOV sort last with key ~0; count the valid prefix.
    uint64_t n_valid = n;
    if (e == cudaSuccess) {
        // Scan the sorted keys back from the end in chunks (few voxels lie
        // outside the FOV, so this usually reads one chunk).
        const uint64_t chunk = 1 << 20;
        std::vector<uint64_t> buf;
        uint64_t hi = n;
        while (e == cudaSuccess && hi > 0) {
            const uint64_t lo = hi > chunk ? hi - chunk : 0;
            buf.resize(hi - lo);
            e = cudaMemcpyAsync(buf.data(), d_k1 + lo, (hi - lo) * sizeof(uint64_t), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) break;
            uint64_t p = hi - lo;
            while (p > 0 && buf[p - 1] == ~0ull) --p;
            n_valid = lo + p;
            if (p > 0) break;
            hi = lo;
        }
    }
    // Stack table: where each slice stack starts in the order, then n_valid.
    uint32_t* d_st = nullptr;
    uint64_t n_st = 0;
    if (e == cudaSuccess && stacks_out) {
        uint8_t* d_flags = nullptr;
        int* d_num = nullptr;
        void* d_tmp2 = nullptr;
        size_t tmp2 = 0;
        e = cudaMalloc(&d_st, (n_valid + 1) * sizeof(uint32_t));
        if (e == cudaSuccess && n_valid > 0) {
            e = cudaMalloc(&d_flags, n_valid);
            if (e == cudaSuccess) e = cudaMalloc(&d_num, sizeof(int));
            if (e == cudaSuccess) {
                const int grid =
                    (int)std::max<uint64_t>(1, std::min<uint64_t>((n_valid + 255) / 256, (uint64_t)ctx->sm_count * 16));
                stack_heads_kernel<<<grid, 256, 0, st>>>(d_k1, n_valid, (uint64_t)O.nz, d_flags);
                e = cudaGetLastError();
            }
            const thrust::counting_iterator<uint32_t> pos(0);
            if (e == cudaSuccess)
                e = cub::DeviceSelect::Flagged(nullptr, tmp2, pos, d_flags, d_st, d_num, (int)n_valid, st);
            if (e == cudaSuccess) e = cudaMalloc(&d_tmp2, tmp2);
            if (e == cudaSuccess)
                e = cub::DeviceSelect::Flagged(d_tmp2, tmp2, pos, d_flags, d_st, d_num, (int)n_valid, st);
            int h_num = 0;
            if (e == cudaSuccess) e = cudaMemcpyAsync(&h_num, d_num, sizeof(int), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            n_st = (uint64_t)h_num;
        }
        const uint32_t nv = (uint32_t)n_valid;
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_st + n_st, &nv, sizeof(uint32_t), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaFree(d_flags);
        cudaFree(d_num);
        cudaFree(d_tmp2);
    }
    if (e != cudaSuccess) {
        rcode = fail(e == cudaErrorMemoryAllocation ? CTBB_ERR_OOM : CTBB_ERR_CUDA, "visiting order: %s",
                     cudaGetErrorString(e));
        cudaFree(d_v1);
        cudaFree(d_st);
        cleanup();
        return rcode;
    }
    *out = d_v1;
    *n_out = n_valid;
    if (stacks_out) {
        *stacks_out = d_st;
        *n_stacks_out = n_st;
    }
    cleanup();
    return CTBB_OK;
}

// prepare: only raise the kernel's dynamic shared-memory limit (done before
// a stream capture, outside it); otherwise launch on `st`.
template <class WT, int U, int NW>
ctbb_status launch_staged(const GParams& P, const uint32_t* order, const ctbb_ssm* ssm, const WT* w, ctbb_recon* rc,
                          uint64_t in_flight, unsigned long long* stats, cudaStream_t st, bool prepare) {
    ctbb_ctx* ctx = rc->ctx;
    const int cap = stage_capacity(ctx, NW, (int)sizeof(WT));
    const size_t smem = (size_t)NW * (size_t)cap * (4 + sizeof(WT));
    if (prepare) {
        CTBB_CUDA(cudaFuncSetAttribute(icd_staged_kernel<WT, U, NW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
        return CTBB_OK;
    }
    // One CTA per SM is resident (the stage takes the SM's shared memory);
    // a persistent grid larger than that would only add idle CTAs.
    const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>((in_flight + NW - 1) / NW, ctx->sm_count));
    icd_staged_kernel<WT, U, NW><<<blocks, 32 * NW, smem, st>>>(P, order, ssm->d_colptr, ssm->d_vptr, ssm->d_idx, w,
                                                                rc->d_start, rc->d_e32, rc->d_x32, ctx->d_queue, cap,
                                                                stats);
    return CTBB_OK;
}

// What a captured iteration depends on: a graph is reused while the key is
// unchanged (byte comparison; the struct is zero-filled before use).
struct GraphKey {
    GParams P;
    const void* order;
    const void* stacks;
    const void* w;
    const void* idx;
    const float* e;
    const float* x;
    uint64_t in_flight;
    int stage, pairs, wpv, epl, h;
};


// Build (or reuse) the full visiting order for tile edge P_lat.
ctbb_status build_order(ctbb_recon* rc, int P_lat) {
    if (rc->d_order && rc->order_P == P_lat) return CTBB_OK;
    uint32_t *o = nullptr, *stk = nullptr;
    uint64_t n = 0, n_stk = 0;
    CTBB_TRY(build_order_into(rc, P_lat, nullptr, 0.f, &o, &n, &stk, &n_stk));
    cudaFree(rc->d_order);
    cudaFree(rc->d_stacks);
    rc->d_order = o;
    rc->n_order = n;
    rc->d_stacks = stk;
    rc->n_stacks = n_stk;
    rc->order_P = P_lat;
    return CTBB_OK;
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
    // Keep (voxels crossed per ray) * W / N near 0.4 (a ray crosses about
    // 4 * 0.8 * nx voxels: 2 in-plane bilinear taps x 2 slices per x step),
    // W = warps = voxel updates in flight.
    const double n = (double)rc->nvox;
    const double per_ray = 3.2 * (double)rc->geom.num_voxels_x;
    const int w = (int)(0.4 * n / per_ray);
    return std::max(4, std::min(rc->ctx->sm_count * 32, w));
}

// Stage positions per warp of the shared-memory staged kernel: what NW
// warps' stages of (4-byte index + weight) entries fit in the opt-in shared
// memory of one CTA, in whole warps' worth of entries.
int stage_capacity(const ctbb_ctx* ctx, int nw, int wbytes) {
    const size_t smem = ctx->smem_per_block_optin ? ctx->smem_per_block_optin : 48 * 1024;
    const size_t per = smem / ((size_t)nw * (size_t)(4 + wbytes));
    return (int)(per / 32 * 32);
}


ctbb_status launch_icd_grouped(ctbb_recon* rc, const ctbb_ssm* ssm, const ctbb_icd_opts& o, float* ms,
                               double* entries, uint64_t* items, double* scattered) {
    const int T = lattice_spacing(rc, o);
    CTBB_TRY(build_order(rc, T));
    if (o.priority && !rc->d_prio_order)
        return fail(CTBB_ERR_INVALID_ARG, "priority pass requested but no priority set (ctbb_gpu_recon_set_priority)");
    const bool prio = o.priority != 0;
    GParams P = make_params(rc, ssm, o);
    if (prio) P.n_items = rc->n_prio_order;
    const uint32_t* order = prio ? rc->d_prio_order : rc->d_order;
    if (items) *items = P.n_items;
    // Updates in flight: as requested, within the order's concurrency bound.
    const uint64_t order_bound = max_items_in_flight(P.n_items, P.nz, prio ? rc->prio_P : T);
    const uint64_t in_flight = std::min<uint64_t>(requested_items(rc, o), order_bound);
    if (entries) {
        CTBB_TRY(inrange_entries(rc, ssm, entries));
        // A priority pass visits a subset; scale by the share of items.
        if (prio && rc->n_order > 0) *entries *= (double)rc->n_prio_order / (double)rc->n_order;
    }
    const int wpv = o.warps_per_voxel > 1 ? o.warps_per_voxel : 1;
    if (wpv != 1 && wpv != 4 && wpv != 8)
        return fail(CTBB_ERR_INVALID_ARG, "warps_per_voxel must be 1, 4 or 8 (got %d)", wpv);
    const int stage = o.stage_column;
    if (stage < 0 || stage > 6)
        return fail(CTBB_ERR_INVALID_ARG, "stage_column must be 0 to 6 (got %d)", stage);
    if (stage >= 1 && stage <= 3 && wpv != 1)
        return fail(CTBB_ERR_INVALID_ARG, "stage_column 1-3 needs one warp per voxel update");
    const uint32_t* stacks = prio ? rc->d_prio_stacks : rc->d_stacks;
    const uint64_t n_stacks = prio ? rc->n_prio_stacks : rc->n_stacks;
    if (stage == 3 && !stacks) return fail(CTBB_ERR_INVALID_ARG, "visiting order has no stack table");
    const int epl = o.entries_per_lane > 0 ? o.entries_per_lane : kU;
    if (epl != 8 && epl != 16) return fail(CTBB_ERR_INVALID_ARG, "entries_per_lane must be 8 or 16 (got %d)", epl);
    ctbb_ctx* ctx = rc->ctx;
    cudaStream_t st = ctx->stream;
    unsigned long long* stats = ctx->d_queue + 2;
    const int wsel = o.weights ? o.weights : CTBB_SSM_FP32;
    const bool h = wsel == CTBB_SSM_FP16;
    // Entry pairs for the CTA-per-update kernels with FP16 weights (built
    // here, outside any stream capture, on first use).
    const bool want_pairs = h && (stage >= 4 || (o.entry_pairs == 0 && (wpv > 1 || stage == 0)));
    if (want_pairs) CTBB_TRY(ssm_build_pairs(const_cast<ctbb_ssm*>(ssm)));
    const bool pairs = want_pairs && ssm->d_pairs;
    if (stage >= 4 && !pairs)
        return fail(CTBB_ERR_INVALID_ARG,
                    "stage_column 4-6 reads entry pairs: needs FP16 weights and a matrix whose detector-row runs "
                    "pair up (no z flying focal spot)");
    const int64_t* cp = ssm->d_colptr;
    const uint32_t* vp = ssm->d_vptr;
    const int32_t* ix = ssm->d_idx;

    // One iteration: reset the work queue and the scatter counters, then the
    // persistent kernel (prepare: only the launch attributes, no work).
    auto issue = [&](cudaStream_t s, bool prepare) -> ctbb_status {
        if (!prepare) CTBB_CUDA(cudaMemsetAsync(ctx->d_queue, 0, 5 * sizeof(unsigned long long), s));
        if (stage == 6) {
            // Claim-ahead bulk-staged kernel: one stage, two claimed items
            // per CTA, so half the order's bound in CTAs.
            const size_t smem = bulk_smem_bytes(1);
            if (prepare) {
                CTBB_CUDA(cudaFuncSetAttribute(icd_bulk_pipe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem));
                return CTBB_OK;
            }
            const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>(in_flight, order_bound / 2));
            icd_bulk_pipe_kernel<<<blocks, kBulkThreads, smem, s>>>(P, order, ssm->d_pcolptr, ssm->d_pvptr,
                                                                     ssm->d_pairs, vp, rc->d_start, rc->d_e32,
                                                                     rc->d_x32, ctx->d_queue, stats, stats + 2);
            CTBB_CUDA(cudaGetLastError());
            return CTBB_OK;
        }
        if (stage >= 4) {
            // One update per CTA of 8 warps; 4: one pair stage, 5: two.
            const int stages = stage == 4 ? 1 : 2;
            const size_t smem = bulk_smem_bytes(stages);
            if (prepare) {
                if (stages == 1)
                    CTBB_CUDA(cudaFuncSetAttribute(icd_bulk_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)smem));
                else
                    CTBB_CUDA(cudaFuncSetAttribute(icd_bulk_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)smem));
                return CTBB_OK;
            }
            const int blocks = (int)std::max<uint64_t>(1, in_flight);
            if (stages == 1)
                icd_bulk_kernel<1><<<blocks, kBulkThreads, smem, s>>>(P, order, ssm->d_pcolptr, ssm->d_pvptr,
                                                                      ssm->d_pairs, vp, rc->d_start, rc->d_e32,
                                                                      rc->d_x32, ctx->d_queue, stats, stats + 2);
            else
                icd_bulk_kernel<2><<<blocks, kBulkThreads, smem, s>>>(P, order, ssm->d_pcolptr, ssm->d_pvptr,
                                                                      ssm->d_pairs, vp, rc->d_start, rc->d_e32,
                                                                      rc->d_x32, ctx->d_queue, stats, stats + 2);
            CTBB_CUDA(cudaGetLastError());
            return CTBB_OK;
        }
        if (stage == 3) {
            if (prepare) return CTBB_OK;
            // One CTA (kStack warps) per stack: at most in_flight / kStack
            // stacks in flight keeps within the order's concurrency bound.
            const int blocks = (int)std::max<uint64_t>(1, in_flight / kStack);
            if (epl == 16) {
                if (h)
                    icd_lockstep_kernel<__half, 16><<<blocks, 32 * kStack, 0, s>>>(
                        P, order, stacks, n_stacks, cp, vp, ix, ssm->d_w16, rc->d_start, rc->d_e32, rc->d_x32,
                        ctx->d_queue, stats);
                else
                    icd_lockstep_kernel<float, 16><<<blocks, 32 * kStack, 0, s>>>(
                        P, order, stacks, n_stacks, cp, vp, ix, ssm->d_w32, rc->d_start, rc->d_e32, rc->d_x32,
                        ctx->d_queue, stats);
            } else {
                if (h)
                    icd_lockstep_kernel<__half, 8><<<blocks, 32 * kStack, 0, s>>>(
                        P, order, stacks, n_stacks, cp, vp, ix, ssm->d_w16, rc->d_start, rc->d_e32, rc->d_x32,
                        ctx->d_queue, stats);
                else
                    icd_lockstep_kernel<float, 8><<<blocks, 32 * kStack, 0, s>>>(
                        P, order, stacks, n_stacks, cp, vp, ix, ssm->d_w32, rc->d_start, rc->d_e32, rc->d_x32,
                        ctx->d_queue, stats);
            }
            CTBB_CUDA(cudaGetLastError());
            return CTBB_OK;
        }
        if (stage) {
            // stage_column 1: 4 warps (updates) per CTA, 2: 8 (half the stage each).
            if (stage == 1) {
                if (h)
                    return (epl == 16 ? launch_staged<__half, 16, 4> : launch_staged<__half, 8, 4>)(
                        P, order, ssm, ssm->d_w16, rc, in_flight, stats, s, prepare);
                return (epl == 16 ? launch_staged<float, 16, 4> : launch_staged<float, 8, 4>)(
                    P, order, ssm, ssm->d_w32, rc, in_flight, stats, s, prepare);
            }
            if (h)
                return (epl == 16 ? launch_staged<__half, 16, 8> : launch_staged<__half, 8, 8>)(
                    P, order, ssm, ssm->d_w16, rc, in_flight, stats, s, prepare);
            return (epl == 16 ? launch_staged<float, 16, 8> : launch_staged<float, 8, 8>)(
                P, order, ssm, ssm->d_w32, rc, in_flight, stats, s, prepare);
        }
        if (prepare) return CTBB_OK;
        if (wpv == 1 && pairs) {
            const int blocks = (int)std::max<uint64_t>(1, (in_flight + 7) / 8);
            if (epl == 16)
                icd_grouped_pairs_kernel<16><<<blocks, 256, 0, s>>>(P, order, ssm->d_pcolptr, ssm->d_pvptr,
                                                                    ssm->d_pairs, vp, rc->d_start, rc->d_e32,
                                                                    rc->d_x32, ctx->d_queue, stats);
            else
                icd_grouped_pairs_kernel<8><<<blocks, 256, 0, s>>>(P, order, ssm->d_pcolptr, ssm->d_pvptr,
                                                                   ssm->d_pairs, vp, rc->d_start, rc->d_e32,
                                                                   rc->d_x32, ctx->d_queue, stats);
        } else if (wpv == 1) {
            const int blocks = (int)std::max<uint64_t>(1, (in_flight + 7) / 8);
            if (epl == 16) {
                if (h)
                    icd_grouped_kernel<__half, 16><<<blocks, 256, 0, s>>>(P, order, cp, vp, ix, ssm->d_w16, rc->d_start,
                                                                          rc->d_e32, rc->d_x32, ctx->d_queue, stats);
                else
                    icd_grouped_kernel<float, 16><<<blocks, 256, 0, s>>>(P, order, cp, vp, ix, ssm->d_w32, rc->d_start,
                                                                         rc->d_e32, rc->d_x32, ctx->d_queue, stats);
            } else {
                if (h)
                    icd_grouped_kernel<__half, 8><<<blocks, 256, 0, s>>>(P, order, cp, vp, ix, ssm->d_w16, rc->d_start,
                                                                         rc->d_e32, rc->d_x32, ctx->d_queue, stats);
                else
                    icd_grouped_kernel<float, 8><<<blocks, 256, 0, s>>>(P, order, cp, vp, ix, ssm->d_w32, rc->d_start,
                                                                        rc->d_e32, rc->d_x32, ctx->d_queue, stats);
            }
        } else if (pairs) {
            const int blocks = (int)in_flight;
            if (wpv == 8)
                icd_cta_pairs_kernel<8, 32><<<blocks, 256, 0, s>>>(P, order, ssm->d_pcolptr, ssm->d_pvptr,
                                                                   ssm->d_pairs, vp, rc->d_start, rc->d_e32,
                                                                   rc->d_x32, ctx->d_queue, stats);
            else
                icd_cta_pairs_kernel<4, 32><<<blocks, 128, 0, s>>>(P, order, ssm->d_pcolptr, ssm->d_pvptr,
                                                                   ssm->d_pairs, vp, rc->d_start, rc->d_e32,
                                                                   rc->d_x32, ctx->d_queue, stats);
        } else {
            const int blocks = (int)in_flight;
            if (wpv == 8) {
                if (h)
                    icd_cta_kernel<__half, 8, 32><<<blocks, 256, 0, s>>>(P, order, cp, vp, ix, ssm->d_w16, rc->d_start,
                                                                         rc->d_e32, rc->d_x32, ctx->d_queue, stats);
                else
                    icd_cta_kernel<float, 8, 32><<<blocks, 256, 0, s>>>(P, order, cp, vp, ix, ssm->d_w32, rc->d_start,
                                                                        rc->d_e32, rc->d_x32, ctx->d_queue, stats);
            } else {
                if (h)
                    icd_cta_kernel<__half, 4, 32><<<blocks, 128, 0, s>>>(P, order, cp, vp, ix, ssm->d_w16, rc->d_start,
                                                                         rc->d_e32, rc->d_x32, ctx->d_queue, stats);
                else
                    icd_cta_kernel<float, 4, 32><<<blocks, 128, 0, s>>>(P, order, cp, vp, ix, ssm->d_w32, rc->d_start,
                                                                        rc->d_e32, rc->d_x32, ctx->d_queue, stats);
            }
        }
        CTBB_CUDA(cudaGetLastError());
        return CTBB_OK;
    };

    // The iteration is captured once in a CUDA graph per launch shape and
    // replayed; a stream that cannot be captured (the legacy default stream)
    // issues the same two operations directly.
    GraphKey key;
    memset(&key, 0, sizeof(key));
    key.P = P;
    key.order = order;
    key.stacks = stacks;
    key.w = pairs ? (const void*)ssm->d_pairs : h ? (const void*)ssm->d_w16 : (const void*)ssm->d_w32;
    key.idx = ix;
    key.e = rc->d_e32;
    key.x = rc->d_x32;
    key.in_flight = in_flight;
    key.stage = stage;
    key.pairs = pairs ? 1 : 0;
    key.wpv = wpv;
    key.epl = epl;
    key.h = h;
    const bool have = rc->icd_graph && rc->icd_graph_key.size() == sizeof(key) &&
                      memcmp(rc->icd_graph_key.data(), &key, sizeof(key)) == 0;
    if (!have) {
        if (rc->icd_graph) cudaGraphExecDestroy(rc->icd_graph);
        rc->icd_graph = nullptr;
        rc->icd_graph_key.clear();
        CTBB_TRY(issue(st, true));
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        CTBB_CUDA(cudaStreamIsCapturing(st, &cs));
        if (st != nullptr && cs == cudaStreamCaptureStatusNone &&
            cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            const ctbb_status is = issue(st, false);
            cudaGraph_t g = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(st, &g);
            if (is != CTBB_OK || ce != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                return is != CTBB_OK ? is : fail(CTBB_ERR_CUDA, "ICD iteration capture: %s", cudaGetErrorString(ce));
            }
            const cudaError_t ie = cudaGraphInstantiate(&rc->icd_graph, g, 0);
            cudaGraphDestroy(g);
            if (ie != cudaSuccess) {
                rc->icd_graph = nullptr;
                return fail(CTBB_ERR_CUDA, "ICD iteration graph: %s", cudaGetErrorString(ie));
            }
            rc->icd_graph_key.assign((const unsigned char*)&key, (const unsigned char*)&key + sizeof(key));
        } else {
            cudaGetLastError();  // a refused capture leaves no lasting error
        }
    }
    cudaEvent_t e0, e1;
    CTBB_CUDA(cudaEventCreate(&e0));
    CTBB_CUDA(cudaEventCreate(&e1));
    CTBB_CUDA(cudaEventRecord(e0, st));
    if (rc->icd_graph)
        CTBB_CUDA(cudaGraphLaunch(rc->icd_graph, st));
    else
        CTBB_TRY(issue(st, false));
    CTBB_CUDA(cudaEventRecord(e1, st));
    CTBB_CUDA(cudaEventSynchronize(e1));
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (scattered || stage >= 4) {
        unsigned long long h3[3] = {0, 0, 0};
        CTBB_CUDA(cudaMemcpyAsync(h3, stats, sizeof(h3), cudaMemcpyDeviceToHost, st));
        CTBB_CUDA(cudaStreamSynchronize(st));
        if (scattered) *scattered = (double)h3[1];
        if (h3[2]) return fail(CTBB_ERR_CUDA, "bulk-staged ICD kernel: a matrix copy into shared memory did not "
                                              "complete within its wait limit");
    }
    return CTBB_OK;
}

}  // namespace ctbb

// ---------------------------------------------------------------------------
// Batched independent scans (one persistent launch per iteration for all of
// them, replayed from a CUDA graph).
// ---------------------------------------------------------------------------
struct ctbb_batch {
    ctbb_ctx* ctx = nullptr;
    std::vector<ctbb_recon*> recons;
    std::vector<const ctbb_ssm*> ssms;
    uint64_t* d_merged = nullptr;
    uint64_t n_total = 0;
    std::vector<int> merged_T;  // tile edge per scan when d_merged was built
    void* d_scans = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_warps = 0, graph_weights = 0, graph_stage = 0;
    double graph_relax = 0.0;
};

namespace {

using namespace ctbb;

template <class WT>
ctbb_status upload_scans(ctbb_batch* b, const ctbb_icd_opts& o) {
    std::vector<ScanRefs<WT>> h(b->recons.size());
    for (size_t i = 0; i < h.size(); ++i) {
        ctbb_recon* rc = b->recons[i];
        const ctbb_ssm* s = b->ssms[i];
        h[i].P = make_params(rc, s, o);
        h[i].order = rc->d_order;
        h[i].colptr = s->d_colptr;
        h[i].vptr = s->d_vptr;
        h[i].idx = s->d_idx;
        h[i].w = std::is_same<WT, __half>::value ? (const WT*)s->d_w16 : (const WT*)s->d_w32;
        h[i].start = rc->d_start;
        h[i].e = rc->d_e32;
        h[i].x = rc->d_x32;
    }
    cudaFree(b->d_scans);
    b->d_scans = nullptr;
    CTBB_CUDA(cudaMalloc(&b->d_scans, h.size() * sizeof(ScanRefs<WT>)));
    CTBB_CUDA(cudaMemcpyAsync(b->d_scans, h.data(), h.size() * sizeof(ScanRefs<WT>), cudaMemcpyHostToDevice,
                              b->ctx->stream));
    return CTBB_OK;
}

ctbb_status build_merged(ctbb_batch* b) {
    cudaStream_t st = b->ctx->stream;
    uint64_t n = 0;
    for (ctbb_recon* rc : b->recons) n += rc->n_order;
    uint64_t *k0 = nullptr, *k1 = nullptr, *v0 = nullptr, *v1 = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    cudaError_t e = cudaMalloc(&k0, std::max<uint64_t>(1, n) * 8);
    if (e == cudaSuccess) e = cudaMalloc(&k1, std::max<uint64_t>(1, n) * 8);
    if (e == cudaSuccess) e = cudaMalloc(&v0, std::max<uint64_t>(1, n) * 8);
    if (e == cudaSuccess) e = cudaMalloc(&v1, std::max<uint64_t>(1, n) * 8);
    uint64_t base = 0;
    for (size_t i = 0; e == cudaSuccess && i < b->recons.size(); ++i) {
        const uint64_t ns = b->recons[i]->n_order;
        if (ns) {
            const int grid = (int)std::min<uint64_t>((ns + 255) / 256, (uint64_t)b->ctx->sm_count * 16);
            merge_keys_kernel<<<grid, 256, 0, st>>>(ns, (uint32_t)i, base, k0, v0);
            e = cudaGetLastError();
        }
        base += ns;
    }
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, k0, k1, v0, v1, (int)n, 0, 64, st);
    if (e == cudaSuccess) e = cudaMalloc(&tmp, tmp_bytes);
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, k0, k1, v0, v1, (int)n, 0, 64, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(k0);
    cudaFree(k1);
    cudaFree(v0);
    cudaFree(tmp);
    if (e != cudaSuccess) {
        cudaFree(v1);
        return fail(e == cudaErrorMemoryAllocation ? CTBB_ERR_OOM : CTBB_ERR_CUDA, "batch queue: %s",
                    cudaGetErrorString(e));
    }
    cudaFree(b->d_merged);
    b->d_merged = v1;
    b->n_total = n;
    return CTBB_OK;
}

void drop_graph(ctbb_batch* b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
}

template <class WT>
ctbb_status capture_iteration(ctbb_batch* b, int warps, double relax, int stage) {
    drop_graph(b);
    cudaStream_t st = b->ctx->stream;
    const int cap = stage_capacity(b->ctx, 4, (int)sizeof(WT));
    const size_t smem = (size_t)4 * cap * (4 + sizeof(WT));
    if (stage)
        CTBB_CUDA(cudaFuncSetAttribute(icd_batch_staged_kernel<WT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    cudaGraph_t g = nullptr;
    CTBB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(b->ctx->d_queue, 0, sizeof(unsigned long long), st);
    if (stage) {
        // One CTA of 4 staged updates per SM.
        const int blocks = std::max(1, std::min(b->ctx->sm_count, (warps + 3) / 4));
        icd_batch_staged_kernel<WT><<<blocks, 128, smem, st>>>((const ScanRefs<WT>*)b->d_scans, b->d_merged,
                                                               b->n_total, relax, b->ctx->d_queue, cap);
    } else {
        const int blocks = std::max(1, (warps + 7) / 8);
        icd_batch_kernel<WT><<<blocks, 256, 0, st>>>((const ScanRefs<WT>*)b->d_scans, b->d_merged, b->n_total,
                                                     relax, b->ctx->d_queue);
    }
    const cudaError_t le = cudaGetLastError();
    const cudaError_t ce = cudaStreamEndCapture(st, &g);
    if (le != cudaSuccess || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return fail(CTBB_ERR_CUDA, "batch graph capture: %s",
                    cudaGetErrorString(le != cudaSuccess ? le : ce));
    }
    const cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return fail(CTBB_ERR_CUDA, "batch graph instantiate: %s", cudaGetErrorString(ie));
    return CTBB_OK;
}

}  // namespace

using namespace ctbb;

extern "C" ctbb_status ctbb_gpu_batch_create(ctbb_ctx* ctx, int32_t n, ctbb_recon* const* recons,
                                             const ctbb_ssm* const* ssms, ctbb_batch** out) {
    clear_error();
    if (!ctx || !recons || !ssms || !out || n <= 0) return fail(CTBB_ERR_INVALID_ARG, "null argument or empty batch");
    if (n > 64) return fail(CTBB_ERR_INVALID_ARG, "a batch holds at most 64 scans (got %d)", n);
    for (int i = 0; i < n; ++i) {
        const ctbb_recon* rc = recons[i];
        const ctbb_ssm* s = ssms[i];
        if (!rc || !s) return fail(CTBB_ERR_INVALID_ARG, "scan %d: null reconstruction or matrix", i);
        if (rc->ctx != ctx || s->ctx != ctx) return fail(CTBB_ERR_INVALID_ARG, "scan %d belongs to another context", i);
        if (rc->geom.num_voxels_x != s->geom.num_voxels_x || rc->geom.num_voxels_y != s->geom.num_voxels_y ||
            rc->geom.n_channels != s->geom.n_channels || rc->geom.Nrows_projection != s->geom.Nrows_projection ||
            rc->geom.num_views_for_system_matrix != s->geom.num_views_for_system_matrix)
            return fail(CTBB_ERR_INVALID_ARG, "scan %d: matrix geometry does not match the reconstruction", i);
        for (int j = 0; j < i; ++j)
            if (recons[j] == rc) return fail(CTBB_ERR_INVALID_ARG, "scan %d appears twice", i);
    }
    ctbb_batch* b = new ctbb_batch();
    b->ctx = ctx;
    ctx_retain(ctx);
    b->recons.assign(recons, recons + n);
    b->ssms.assign(ssms, ssms + n);
    *out = b;
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_gpu_batch_iterate(ctbb_batch* b, const ctbb_icd_opts* opts, int32_t n_iter,
                                              ctbb_iter_stats* stats) {
    clear_error();
    if (!b || !opts) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (n_iter < 0) return fail(CTBB_ERR_INVALID_ARG, "negative iteration count");
    CTBB_CUDA(cudaSetDevice(b->ctx->device));
    const ctbb_icd_opts& o = *opts;
    const int wsel = o.weights ? o.weights : CTBB_SSM_FP32;
    if (wsel != CTBB_SSM_FP16 && wsel != CTBB_SSM_FP32) return fail(CTBB_ERR_INVALID_ARG, "weights must be FP16 or FP32");
    double entries = 0.0;
    int nx_max = 1;
    double n_sum = 0.0;
    for (ctbb_recon* rc : b->recons) {
        n_sum += (double)rc->nvox;
        nx_max = std::max(nx_max, (int)rc->geom.num_voxels_x);
    }
    // Each scan gets a share of the in-flight items proportional to its size,
    // so the per-scan coupling bound uses the whole batch's item count.
    int warps = o.warps_in_flight > 0
                    ? o.warps_in_flight
                    : std::max(4, std::min(b->ctx->sm_count * 32, (int)(0.4 * n_sum / (3.2 * nx_max))));
    bool orders_changed = b->d_merged == nullptr || b->merged_T.size() != b->recons.size();
    std::vector<int> T(b->recons.size());
    for (size_t i = 0; i < b->recons.size(); ++i) {
        ctbb_recon* rc = b->recons[i];
        const ctbb_ssm* s = b->ssms[i];
        if ((wsel == CTBB_SSM_FP16 && !s->d_w16) || (wsel == CTBB_SSM_FP32 && !s->d_w32))
            return fail(CTBB_ERR_INVALID_ARG, "scan %zu: matrix does not hold the requested weights", i);
        CTBB_TRY(recon_to_grouped(rc, s));
        ctbb_icd_opts oi = o;
        oi.warps_per_voxel = 1;
        oi.warps_in_flight = std::max(1, (int)((double)warps * (double)rc->nvox / n_sum));
        T[i] = lattice_spacing(rc, oi);
        CTBB_TRY(build_order(rc, T[i]));
        double en = 0.0;
        CTBB_TRY(inrange_entries(rc, s, &en));
        entries += en;
        if (!orders_changed && b->merged_T[i] != T[i]) orders_changed = true;
    }
    if (orders_changed) {
        CTBB_TRY(build_merged(b));
        b->merged_T = T;
        drop_graph(b);
    }
    const double relax = (o.relax > 0.0 && o.relax < 2.0) ? o.relax : 1.0;
    // Within every scan's order concurrency bound (its share of the items).
    for (size_t i = 0; i < b->recons.size(); ++i) {
        const ctbb_recon* rc = b->recons[i];
        if (rc->n_order == 0) continue;
        const double cap = (double)max_items_in_flight(rc->n_order, (int)rc->geom.num_voxels_z, T[i]) *
                           (double)b->n_total / (double)rc->n_order;
        warps = std::max(1, std::min(warps, (int)cap));
    }
    const int stage = o.stage_column ? 1 : 0;
    if (stage) warps = std::min(warps, b->ctx->sm_count * 4);
    if (!b->graph || b->graph_warps != warps || b->graph_relax != relax || b->graph_weights != wsel ||
        b->graph_stage != stage) {
        if (wsel == CTBB_SSM_FP16) {
            CTBB_TRY(upload_scans<__half>(b, o));
            CTBB_TRY(capture_iteration<__half>(b, warps, relax, stage));
        } else {
            CTBB_TRY(upload_scans<float>(b, o));
            CTBB_TRY(capture_iteration<float>(b, warps, relax, stage));
        }
        b->graph_stage = stage;
        b->graph_warps = warps;
        b->graph_relax = relax;
        b->graph_weights = wsel;
    }
    cudaStream_t st = b->ctx->stream;
    cudaEvent_t e0, e1;
    CTBB_CUDA(cudaEventCreate(&e0));
    CTBB_CUDA(cudaEventCreate(&e1));
    CTBB_CUDA(cudaEventRecord(e0, st));
    for (int it = 0; it < n_iter; ++it) CTBB_CUDA(cudaGraphLaunch(b->graph, st));
    CTBB_CUDA(cudaEventRecord(e1, st));
    CTBB_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->iterations = n_iter;
        stats->device_ms = ms;
        stats->voxel_updates = (double)b->n_total * n_iter;
        stats->entries = entries * n_iter;
    }
    return CTBB_OK;
}

extern "C" void ctbb_gpu_batch_free(ctbb_batch* b) {
    if (!b) return;
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    drop_graph(b);
    cudaFree(b->d_merged);
    cudaFree(b->d_scans);
    ctx_release(b->ctx);
    delete b;
}

// ---------------------------------------------------------------------------
// Priority subset (voxels with the largest predicted change first).
// ---------------------------------------------------------------------------
extern "C" ctbb_status ctbb_gpu_recon_set_priority(ctbb_recon* rc, const ctbb_icd_opts* opts, double fraction) {
    clear_error();
    if (!rc) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (!rc->d_prio) return fail(CTBB_ERR_INVALID_ARG, "no priority map (run ctbb_gpu_recon_warm_start first)");
    if (!(fraction > 0.0 && fraction <= 1.0)) return fail(CTBB_ERR_INVALID_ARG, "fraction must be in (0, 1]");
    CTBB_CUDA(cudaSetDevice(rc->ctx->device));
    ctbb_icd_opts o{};
    if (opts) o = *opts;
    cudaStream_t st = rc->ctx->stream;
    const uint64_t n = rc->nvox;
    // Threshold: the (1 - fraction) quantile of the priority map.
    float* d_sorted = nullptr;
    void* d_tmp = nullptr;
    size_t tmp_bytes = 0;
    float thr = 0.f;
    cudaError_t e = cudaMalloc(&d_sorted, n * sizeof(float));
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, rc->d_prio, d_sorted, (int)n, 0, 32, st);
    if (e == cudaSuccess) e = cudaMalloc(&d_tmp, tmp_bytes);
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortKeys(d_tmp, tmp_bytes, rc->d_prio, d_sorted, (int)n, 0, 32, st);
    if (e == cudaSuccess) {
        const uint64_t q = std::min<uint64_t>(n - 1, (uint64_t)((1.0 - fraction) * (double)n));
        e = cudaMemcpyAsync(&thr, d_sorted + q, sizeof(float), cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d_sorted);
    cudaFree(d_tmp);
    if (e != cudaSuccess) return fail(CTBB_ERR_CUDA, "priority threshold: %s", cudaGetErrorString(e));
    uint32_t* order = nullptr;
    uint64_t n_order = 0;
    const int T = lattice_spacing(rc, o);
    uint32_t* stk = nullptr;
    uint64_t n_stk = 0;
    CTBB_TRY(build_order_into(rc, T, rc->d_prio, thr, &order, &n_order, &stk, &n_stk));
    cudaFree(rc->d_prio_order);
    cudaFree(rc->d_prio_stacks);
    rc->d_prio_order = order;
    rc->n_prio_order = n_order;
    rc->d_prio_stacks = stk;
    rc->n_prio_stacks = n_stk;
    rc->prio_P = T;
    return CTBB_OK;
}

// ---------------------------------------------------------------------------
// The grouped update's penalised 1-D solve on caller-given inputs.
// ---------------------------------------------------------------------------
extern "C" ctbb_status ctbb_gpu_penalty_steps(ctbb_ctx* ctx, int32_t penalty, double lambda, double delta,
                                              uint64_t n, const double* alpha, const double* beta, const float* x9,
                                              double* step) {
    clear_error();
    if (!ctx || (n && (!alpha || !beta || !x9 || !step))) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (penalty != CTBB_PENALTY_QUADRATIC && penalty != CTBB_PENALTY_EDGE_PRESERVING)
        return fail(CTBB_ERR_INVALID_ARG, "unknown penalty %d", penalty);
    if (n == 0) return CTBB_OK;
    CTBB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    double *d_a = nullptr, *d_b = nullptr, *d_out = nullptr;
    float* d_x = nullptr;
    auto cleanup = [&]() {
        cudaFree(d_a);
        cudaFree(d_b);
        cudaFree(d_x);
        cudaFree(d_out);
    };
    cudaError_t e = cudaMalloc(&d_a, n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_b, n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_x, 9 * n * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&d_out, n * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_a, alpha, n * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_b, beta, n * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_x, x9, 9 * n * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        const int grid = (int)std::min<uint64_t>((n + 7) / 8, (uint64_t)ctx->sm_count * 16);
        penalty_steps_kernel<<<grid, 256, 0, st>>>(penalty, lambda, delta, n, d_a, d_b, d_x, d_out);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(step, d_out, n * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cleanup();
    if (e != cudaSuccess)
        return fail(e == cudaErrorMemoryAllocation ? CTBB_ERR_OOM : CTBB_ERR_CUDA, "penalty steps: %s",
                    cudaGetErrorString(e));
    return CTBB_OK;
}
