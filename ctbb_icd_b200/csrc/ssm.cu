// Stored-system-matrix builder on the GPU.
//
// Replaces generate_system_matrix (generate_system_matrix.cpp:54-209) and
// generate_system_matrix_ffs (generate_system_matrix_ffs.cpp:60-239).
//
// The reference walks rays (view, channel, row) and pushes modified-Joseph
// weights into per-column sparse vectors, spilling them to matrix.bin every
// 300 views. Here the same weights are produced column-major directly: one
// thread owns one (voxel column, SSM view) cell, finds the few channels and
// rows whose rays can touch that column (conservative geometric bound, a few
// channels/rows of margin), and evaluates each candidate ray with the
// reference's exact double-precision arithmetic to decide membership and
// weight. Entries of a cell come out in (channel, row) order, cells in view
// order, so every column is sorted by q like the reference's push_back order.
//
// Two passes over the cells (count, then fill) with a per-column scan in
// between; the per-(column, view) offsets are kept (vptr) so ICD can clip a
// slice's view window without testing every entry.
//
// This file is compiled with -fmad=false: each multiply and add rounds on its
// own, like the reference's x86-64 build. Trigonometric values come from
// host-side tables computed with the same libm calls as the reference, so
// the device evaluates only +, -, *, /, sqrt and floor (all correctly
// rounded) and reproduces the reference's indices and float weights bit for bit.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "gpu_internal.h"

namespace {

struct ViewTab {
    double src0, src1, src2;  // (deflected) source position, slice frame
    double ew0, ew1, eu0, eu1;
    double off0, off1, off2;  // FFS deflection (zero without FFS)
};

struct SsmParams {
    int nx, ny, nch, nr, nvsm, ffs;
    double vx, vy, vz, cvx, cvy, cvz;
    double cc, dgam;  // channel centre and angular pitch (candidate search only)
    double sa, cr;    // axial detector spacing and centre row (candidate search only)
};

// One candidate ray evaluated with the reference's arithmetic. Returns true
// and the float weight when the ray contributes to column (ic, jc).
__device__ __forceinline__ bool ray_weight(const SsmParams& P, const ViewTab& V, double A, double B,
                                           double ap, double nrm, int ic, int jc, float* wout) {
    // generate_system_matrix.cpp:111-114 / _ffs.cpp:147-151 element by element.
    double d0 = (A * V.ew0 - B * V.eu0) - ap * 0.0;
    double d1 = (A * V.ew1 - B * V.eu1) - ap * 0.0;
    double d2 = (A * 0.0 - B * 0.0) - ap * 1.0;
    double n = nrm;
    if (P.ffs) {
        d0 = d0 - V.off0;
        d1 = d1 - V.off1;
        d2 = d2 - V.off2;
        double t = 0.0;
        t += fabs(d0) * fabs(d0);
        t += fabs(d1) * fabs(d1);
        t += fabs(d2) * fabs(d2);
        n = sqrt(t);
    }
    d0 = d0 / n;
    d1 = d1 / n;
    d2 = d2 / n;
    const double aax = fabs(d0), aay = fabs(d1);
    if (aax > aay) {
        // x-major: the ray is sampled on the line x = x_ic (generate_system_matrix.cpp:127-155).
        const double x = (ic - P.cvx) * P.vx;
        const double y_hat = V.src1 + d1 / d0 * (x - V.src0);
        const double j_hat = y_hat / P.vy + P.cvy;
        const int jj = (int)floor(j_hat);
        if (jj != jc && jj != jc - 1) return false;
        if (!(jj >= 0 && jj <= P.ny - 2)) return false;
        const double z_hat = V.src2 + d2 / d0 * (x - V.src0);
        const double k_hat = z_hat / P.vz + P.cvz;
        const int kk = (int)floor(k_hat);
        if (kk != -1 && kk != 0) return false;
        const double scale = P.vx / aax;
        const double wz = (kk == -1) ? scale * (k_hat - kk) : scale * (1 - (k_hat - kk));
        *wout = (jj == jc) ? (float)(wz * (1 - (j_hat - jj))) : (float)(wz * (j_hat - jj));
        return true;
    } else {
        // y-major: sampled on the line y = y_jc (generate_system_matrix.cpp:156-184).
        const double y = (jc - P.cvy) * P.vy;
        const double x_hat = V.src0 + d0 / d1 * (y - V.src1);
        const double i_hat = x_hat / P.vx + P.cvx;
        const int ii = (int)floor(i_hat);
        if (ii != ic && ii != ic - 1) return false;
        if (!(ii >= 0 && ii <= P.nx - 2)) return false;
        const double z_hat = V.src2 + d2 / d1 * (y - V.src1);
        const double k_hat = z_hat / P.vz + P.cvz;
        const int kk = (int)floor(k_hat);
        if (kk != -1 && kk != 0) return false;
        const double scale = P.vy / aay;
        const double wz = (kk == -1) ? scale * (k_hat - kk) : scale * (1 - (k_hat - kk));
        *wout = (ii == ic) ? (float)(wz * (1 - (i_hat - ii))) : (float)(wz * (i_hat - ii));
        return true;
    }
}

// Approximate (fractional) channel whose ray passes through slice-frame point (px, py).
__device__ __forceinline__ double chan_of(const SsmParams& P, const ViewTab& V, double px, double py) {
    const double rx = px - V.src0, ry = py - V.src1;
    const double a = -(rx * V.ew0 + ry * V.ew1);
    const double b = -(rx * V.eu0 + ry * V.eu1);
    return atan2(b, a) / P.dgam + P.cc;
}

// Candidate rows for a ray with unnormalised in-plane component D (along
// the sampling axis) reaching the sampling line at coordinate s from source
// coordinate s0: z(k) = src2 - (k - cr) * sa * L with L = (s - s0) / D.
__device__ __forceinline__ void row_range(const SsmParams& P, const ViewTab& V, double D, double s,
                                          double s0, int* r_lo, int* r_hi) {
    const double L = (s - s0) / D;
    if (!(fabs(L) > 1e-12)) {
        *r_lo = 0;
        *r_hi = P.nr - 1;
        return;
    }
    // z(k) = src2 - ((k - cr) sa + off2) L: the z deflection of a z flying
    // focal spot shifts the rows by -off2 / sa.
    double a = V.src2 - P.vz, b = V.src2 + P.vz;  // k_hat in [-1, 1)  <=>  z in [-vz, vz)
    double k0 = P.cr + a / (P.sa * L) - V.off2 / P.sa, k1 = P.cr + b / (P.sa * L) - V.off2 / P.sa;
    if (k0 > k1) {
        const double t = k0;
        k0 = k1;
        k1 = t;
    }
    int lo = (int)floor(k0) - 1, hi = (int)ceil(k1) + 1;
    *r_lo = max(lo, 0);
    *r_hi = min(hi, P.nr - 1);
}

template <bool FILL>
__global__ void __launch_bounds__(256) ssm_cells_kernel(
    SsmParams P, const ViewTab* __restrict__ vt, const double* __restrict__ chA,
    const double* __restrict__ chB, const double* __restrict__ rowAp, const double* __restrict__ rowN,
    uint16_t* __restrict__ cnt, const int64_t* __restrict__ colptr, const uint32_t* __restrict__ vptr,
    int32_t* __restrict__ idx, float* __restrict__ w32, __half* __restrict__ w16) {
    const uint64_t ncell = (uint64_t)P.nx * P.ny * P.nvsm;
    for (uint64_t cell = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; cell < ncell;
         cell += (uint64_t)gridDim.x * blockDim.x) {
        const int v = (int)(cell % P.nvsm);
        const uint64_t col = cell / P.nvsm;
        const int ic = (int)(col % P.nx), jc = (int)(col / P.nx);
        const ViewTab V = vt[v];
        // Candidate channels: rays through the two sampling segments of this
        // column (vertical at x_ic for x-major rays, horizontal at y_jc for
        // y-major rays), padded by one channel for rounding and by three with
        // a flying focal spot (the deflected source shifts a ray by about a
        // channel at the fan edge relative to the nominal fan model used for
        // the bound).
        const double xc = (ic - P.cvx) * P.vx, yc = (jc - P.cvy) * P.vy;
        const double c0 = chan_of(P, V, xc, yc - P.vy), c1 = chan_of(P, V, xc, yc + P.vy);
        const double c2 = chan_of(P, V, xc - P.vx, yc), c3 = chan_of(P, V, xc + P.vx, yc);
        const double cmin = fmin(fmin(c0, c1), fmin(c2, c3)), cmax = fmax(fmax(c0, c1), fmax(c2, c3));
        const int pad = P.ffs ? 3 : 1;
        const int ch_lo = max((int)floor(cmin) - pad, 0);
        const int ch_hi = min((int)ceil(cmax) + pad, P.nch - 1);
        uint32_t n = 0;
        int64_t base = 0;
        if (FILL) base = colptr[col] + (int64_t)vptr[col * (uint64_t)(P.nvsm + 1) + v];
        const int q_view = P.nr * P.nch * v;
        for (int ch = ch_lo; ch <= ch_hi; ++ch) {
            const double A = chA[ch], B = chB[ch];
            const double D0 = (A * V.ew0 - B * V.eu0) - V.off0;
            const double D1 = (A * V.ew1 - B * V.eu1) - V.off1;
            int r_lo, r_hi;
            const double ad0 = fabs(D0), ad1 = fabs(D1);
            if (fabs(ad0 - ad1) <= 1e-9 * fmax(ad0, ad1)) {
                r_lo = 0;  // near 45 degrees: the major axis may differ per row
                r_hi = P.nr - 1;
            } else if (ad0 > ad1) {
                row_range(P, V, D0, xc, V.src0, &r_lo, &r_hi);
            } else {
                row_range(P, V, D1, yc, V.src1, &r_lo, &r_hi);
            }
            for (int r = r_lo; r <= r_hi; ++r) {
                float w;
                if (ray_weight(P, V, A, B, rowAp[r], rowN[r], ic, jc, &w)) {
                    if (FILL) {
                        const int64_t o = base + n;
                        idx[o] = r + P.nr * ch + q_view;
                        if (w32) w32[o] = w;
                        if (w16) w16[o] = __float2half_rn(w);
                    }
                    ++n;
                }
            }
        }
        if (!FILL) cnt[cell] = (uint16_t)n;
    }
}

// Per-column exclusive scan of the cell counts: vptr[c][v] and column totals.
__global__ void __launch_bounds__(256) ssm_column_scan_kernel(const uint16_t* __restrict__ cnt, int nvsm,
                                                              uint64_t ncol, uint32_t* __restrict__ vptr,
                                                              uint64_t* __restrict__ coltot) {
    __shared__ uint32_t warp_sums[8];
    __shared__ uint32_t carry;
    for (uint64_t col = blockIdx.x; col < ncol; col += gridDim.x) {
        const uint16_t* c = cnt + col * (uint64_t)nvsm;
        uint32_t* vp = vptr + col * (uint64_t)(nvsm + 1);
        if (threadIdx.x == 0) carry = 0;
        __syncthreads();
        for (int base = 0; base < nvsm; base += 256) {
            const int v = base + threadIdx.x;
            const uint32_t x = (v < nvsm) ? c[v] : 0u;
            uint32_t s = x;
            const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            if (lane == 31) warp_sums[wid] = s;
            __syncthreads();
            uint32_t wpre = 0;
            for (int i = 0; i < wid; ++i) wpre += warp_sums[i];
            const uint32_t excl = carry + wpre + s - x;
            if (v < nvsm) vp[v] = excl;
            __syncthreads();
            if (threadIdx.x == 255) carry = excl + x;
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            vp[nvsm] = carry;
            coltot[col] = carry;
        }
        __syncthreads();
    }
}

// colptr = exclusive scan of column totals (single block, sequential chunks).
__global__ void __launch_bounds__(1024) ssm_colptr_kernel(const uint64_t* __restrict__ coltot, uint64_t ncol,
                                                          int64_t* __restrict__ colptr,
                                                          unsigned long long* __restrict__ maxcol) {
    __shared__ int64_t sums[1024];
    const uint64_t per = (ncol + 1023) / 1024;
    const uint64_t b = threadIdx.x * per, e = min(ncol, b + per);
    int64_t s = 0;
    unsigned long long mx = 0;
    for (uint64_t i = b; i < e; ++i) {
        s += (int64_t)coltot[i];
        mx = max(mx, (unsigned long long)coltot[i]);
    }
    sums[threadIdx.x] = s;
    atomicMax(maxcol, mx);
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t run = 0;
        for (int i = 0; i < 1024; ++i) {
            const int64_t t = sums[i];
            sums[i] = run;
            run += t;
        }
        colptr[ncol] = run;
    }
    __syncthreads();
    int64_t run = sums[threadIdx.x];
    for (uint64_t i = b; i < e; ++i) {
        colptr[i] = run;
        run += (int64_t)coltot[i];
    }
}

__global__ void f32_to_f16_kernel(const float* __restrict__ in, __half* __restrict__ out, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = __float2half_rn(in[i]);
}

// Entry pairs: the modified-Joseph z interpolation gives every (view,
// channel) of a column two adjacent detector rows, so its entries come in
// runs of two consecutive sinogram indices. A pair {q, w0 | w1 << 16} holds
// both FP16 weights of a run in 8 bytes (4 per entry instead of 6); a lone
// entry has w1 = 0. One thread per (column, view) cell: pair count, then
// (after the same per-column / per-matrix scans as the entries) the fill.
template <bool FILL>
__global__ void __launch_bounds__(256) ssm_pairs_kernel(uint64_t ncol, int nvsm, const int64_t* __restrict__ colptr,
                                                        const uint32_t* __restrict__ vptr,
                                                        const int32_t* __restrict__ idx,
                                                        const __half* __restrict__ w16, uint16_t* __restrict__ cnt,
                                                        const int64_t* __restrict__ pcolptr,
                                                        const uint32_t* __restrict__ pvptr, uint2* __restrict__ pairs) {
    const uint64_t ncell = ncol * (uint64_t)nvsm;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < ncell; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t col = t / (uint64_t)nvsm;
        const int v = (int)(t % (uint64_t)nvsm);
        const uint32_t* vp = vptr + col * (uint64_t)(nvsm + 1);
        const int64_t b = colptr[col] + vp[v], en = colptr[col] + vp[v + 1];
        uint2* out = nullptr;
        if (FILL) out = pairs + pcolptr[col] + pvptr[col * (uint64_t)(nvsm + 1) + v];
        int n = 0;
        for (int64_t m = b; m < en;) {
            const bool two = m + 1 < en && idx[m + 1] == idx[m] + 1;
            if (FILL) {
                const uint32_t lo = __half_as_ushort(w16[m]);
                const uint32_t hi = two ? __half_as_ushort(w16[m + 1]) : 0u;
                out[n] = make_uint2((uint32_t)idx[m], lo | (hi << 16));
            }
            ++n;
            m += two ? 2 : 1;
        }
        if (!FILL) cnt[t] = (uint16_t)n;
    }
}

void free_pairs(ctbb_ssm* s) {
    cudaFree(s->d_pcolptr);
    cudaFree(s->d_pvptr);
    cudaFree(s->d_pairs);
    s->d_pcolptr = nullptr;
    s->d_pvptr = nullptr;
    s->d_pairs = nullptr;
    s->npairs = 0;
}

void free_ssm(ctbb_ssm* s) {
    if (!s) return;
    free_pairs(s);
    cudaFree(s->d_colptr);
    cudaFree(s->d_vptr);
    cudaFree(s->d_idx);
    cudaFree(s->d_w32);
    cudaFree(s->d_w16);
    ctbb::ctx_release(s->ctx);
    delete s;
}

// Host tables: trig values computed with the reference's expressions.
void host_tables(const ctbb_geom_c& g, std::vector<ViewTab>& vt, std::vector<double>& A, std::vector<double>& B,
                 std::vector<double>& ap, std::vector<double>& nrm, bool ffs) {
    const size_t nvsm = g.num_views_for_system_matrix;
    const double SDD = g.source_detector_distance, R = g.focal_spot_radius;
    const double da = SDD * R * sin(g.fan_angle_increment) / (4.0 * (SDD - R));  // generate_system_matrix_ffs.cpp:67
    // generate_system_matrix_ffs.cpp:66, with that file's PI (3.14159265359)
    const double dr = SDD * g.CollSlicewidth / (4.0 * (SDD - R) * tan(g.anode_angle * 3.14159265359 / 180.0));
    vt.resize(nvsm);
    for (int i = 0; i < (int)nvsm; ++i) {
        const double ta = (i - 0.5 * nvsm) * g.tube_angle_increment;  // generate_system_matrix.cpp:85
        ViewTab& V = vt[i];
        V.ew0 = cos(ta);
        V.ew1 = sin(ta);
        V.eu0 = -sin(ta);
        V.eu1 = cos(ta);
        const double zs = g.table_direction * ((double)i - 0.5 * (double)nvsm) * g.tube_z_increment;
        V.src0 = R * V.ew0 + zs * 0.0;  // generate_system_matrix.cpp:100
        V.src1 = R * V.ew1 + zs * 0.0;
        V.src2 = R * 0.0 + zs * 1.0;
        V.off0 = V.off1 = V.off2 = 0.0;
        if (ffs && !g.Zffs) {
            const double s = (i % 2 == 0) ? da : -da;  // generate_system_matrix_ffs.cpp:253-259
            V.off0 = s * V.eu0;
            V.off1 = s * V.eu1;
            V.off2 = s * 0.0;
        } else if (ffs && !g.Phiffs) {
            // generate_system_matrix_ffs.cpp:262-270: -/+dr e_w -/+dr tan(anode_angle) e_z
            // (the anode angle passed in degrees to tan, as the reference does)
            const double r = (i % 2 == 0) ? -dr : dr;
            const double t = tan(g.anode_angle);
            V.off0 = r * V.ew0 + (r * t) * 0.0;
            V.off1 = r * V.ew1 + (r * t) * 0.0;
            V.off2 = r * 0.0 + (r * t) * 1.0;
        } else if (ffs) {
            // generate_system_matrix_ffs.cpp:272-284: four deflections per cycle
            const int rho = i % 4;
            const double r = rho < 2 ? -dr : dr, a = (rho % 2 == 0) ? -da : da;
            const double t = tan(g.anode_angle);
            V.off0 = (r * V.ew0 + a * V.eu0) + (r * t) * 0.0;
            V.off1 = (r * V.ew1 + a * V.eu1) + (r * t) * 0.0;
            V.off2 = (r * 0.0 + a * 0.0) + (r * t) * 1.0;
        }
        if (ffs) {
            V.src0 = V.src0 + V.off0;  // generate_system_matrix_ffs.cpp:134
            V.src1 = V.src1 + V.off1;
            V.src2 = V.src2 + V.off2;
        }
    }
    const size_t nch = g.n_channels, nr = g.Nrows_projection;
    A.resize(nch);
    B.resize(nch);
    for (int j = 0; j < (int)nch; ++j) {
        double tang;
        if (ffs)
            tang = (j - g.center_channel_non_ffs) * g.fan_angle_increment;  // generate_system_matrix_ffs.cpp:138
        else
            tang = ((j - g.center_channel_non_ffs) * g.transaxial_detector_spacing) / SDD;  // generate_system_matrix.cpp:103-104
        A[j] = -SDD * cos(tang);
        B[j] = SDD * sin(tang);
    }
    ap.resize(nr);
    nrm.resize(nr);
    for (int k = 0; k < (int)nr; ++k) {
        ap[k] = (k - g.center_row) * g.axial_detector_spacing;  // generate_system_matrix.cpp:109
        nrm[k] = sqrt(ap[k] * ap[k] + SDD * SDD);
    }
}

template <class T>
ctbb_status upload(const std::vector<T>& h, T** d, cudaStream_t s) {
    CTBB_CUDA(cudaMalloc((void**)d, std::max<size_t>(1, h.size()) * sizeof(T)));
    CTBB_CUDA(cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    return CTBB_OK;
}

struct Scoped {
    std::vector<void*> ptrs;
    ~Scoped() {
        for (void* p : ptrs) cudaFree(p);
    }
};

int grid_for(const ctbb_ctx* ctx, uint64_t n, int threads) {
    const uint64_t want = (n + threads - 1) / threads;
    const uint64_t cap = (uint64_t)ctx->sm_count * 16;
    return (int)std::max<uint64_t>(1, std::min(want, cap));
}

}  // namespace

namespace ctbb {

ctbb_status ssm_validate_geometry(const ctbb_geom_c& g) {
    if (g.num_voxels_x < 2 || g.num_voxels_y < 2)
        return fail(CTBB_ERR_INVALID_ARG, "need at least 2x2 voxels per slice");
    if (g.n_channels == 0 || g.Nrows_projection == 0 || g.num_views_for_system_matrix == 0)
        return fail(CTBB_ERR_INVALID_ARG, "empty detector or system-matrix window");
    if (g.Zffs > 1 || g.Phiffs > 1) return fail(CTBB_ERR_INVALID_ARG, "Zffs and Phiffs are 0 or 1");
    const double q = (double)g.num_views_for_system_matrix * g.n_channels * g.Nrows_projection;
    const double ds = (double)g.Readings * g.n_channels * g.Nrows_projection;
    if (q >= 2147483647.0 || ds >= 2147483647.0)
        return fail(CTBB_ERR_INVALID_ARG, "sinogram index exceeds int32 (the reference's index type)");
    if (g.voxel_size_x <= 0 || g.voxel_size_y <= 0 || g.voxel_size_z <= 0)
        return fail(CTBB_ERR_INVALID_ARG, "non-positive voxel size");
    return CTBB_OK;
}

// Build (once) the pair form of an FP16 matrix (ssm_pairs_kernel).
ctbb_status ssm_build_pairs(ctbb_ssm* s) {
    if (s->d_pairs || s->pairs_checked) return CTBB_OK;
    if (!s->d_w16) return fail(CTBB_ERR_INVALID_ARG, "entry pairs need the matrix's FP16 weights");
    ctbb_ctx* ctx = s->ctx;
    cudaStream_t st = ctx->stream;
    const uint64_t ncell = s->ncol * s->nvsm;
    uint16_t* d_cnt = nullptr;
    uint64_t* d_tot = nullptr;
    unsigned long long* d_max = nullptr;
    struct Tmp {
        void* p[3] = {nullptr, nullptr, nullptr};
        ~Tmp() {
            for (void* q : p) cudaFree(q);
        }
    } tmp;
    ctbb_status rc = CTBB_OK;
    auto run = [&]() -> ctbb_status {
        CTBB_CUDA(cudaMalloc(&d_cnt, std::max<uint64_t>(1, ncell) * sizeof(uint16_t)));
        tmp.p[0] = d_cnt;
        CTBB_CUDA(cudaMalloc(&d_tot, std::max<uint64_t>(1, s->ncol) * sizeof(uint64_t)));
        tmp.p[1] = d_tot;
        CTBB_CUDA(cudaMalloc(&d_max, sizeof(unsigned long long)));
        tmp.p[2] = d_max;
        CTBB_CUDA(cudaMemsetAsync(d_max, 0, sizeof(unsigned long long), st));
        CTBB_CUDA(cudaMalloc(&s->d_pcolptr, (s->ncol + 1) * sizeof(int64_t)));
        CTBB_CUDA(cudaMalloc(&s->d_pvptr, s->ncol * (s->nvsm + 1) * sizeof(uint32_t)));
        const int grid = grid_for(ctx, ncell, 256);
        ssm_pairs_kernel<false><<<grid, 256, 0, st>>>(s->ncol, (int)s->nvsm, s->d_colptr, s->d_vptr, s->d_idx,
                                                      s->d_w16, d_cnt, nullptr, nullptr, nullptr);
        CTBB_CUDA(cudaGetLastError());
        ssm_column_scan_kernel<<<(int)std::min<uint64_t>(s->ncol, (uint64_t)ctx->sm_count * 32), 256, 0, st>>>(
            d_cnt, (int)s->nvsm, s->ncol, s->d_pvptr, d_tot);
        CTBB_CUDA(cudaGetLastError());
        ssm_colptr_kernel<<<1, 1024, 0, st>>>(d_tot, s->ncol, s->d_pcolptr, d_max);
        CTBB_CUDA(cudaGetLastError());
        int64_t np = 0;
        CTBB_CUDA(cudaMemcpyAsync(&np, s->d_pcolptr + s->ncol, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        CTBB_CUDA(cudaStreamSynchronize(st));
        s->npairs = (uint64_t)np;
        // Two pairs of padding: the bulk-staged ICD kernel copies whole 16-byte
        // units and may read one pair past the last.
        CTBB_CUDA(cudaMalloc(&s->d_pairs, (s->npairs + 2) * sizeof(uint2)));
        CTBB_CUDA(cudaMemsetAsync(s->d_pairs + s->npairs, 0, 2 * sizeof(uint2), st));
        ssm_pairs_kernel<true><<<grid, 256, 0, st>>>(s->ncol, (int)s->nvsm, s->d_colptr, s->d_vptr, s->d_idx,
                                                     s->d_w16, nullptr, s->d_pcolptr, s->d_pvptr, s->d_pairs);
        CTBB_CUDA(cudaGetLastError());
        CTBB_CUDA(cudaStreamSynchronize(st));
        return CTBB_OK;
    };
    rc = run();
    s->pairs_checked = true;
    // Pairs pay only where most runs are two rows long (8 bytes per pair
    // against 6 per entry): with fewer than 4 entries per 3 pairs (the z
    // flying focal spot splits the runs) the single entries are kept.
    if (rc != CTBB_OK || 4 * s->npairs > 3 * s->nnz) free_pairs(s);
    return rc;
}

}  // namespace ctbb

using namespace ctbb;

static ctbb_status finish_common(ctbb_ctx* ctx, ctbb_ssm* s, int weights) {
    (void)ctx;
    s->weights = weights;
    s->bytes = (s->ncol + 1) * sizeof(int64_t) + s->ncol * (s->nvsm + 1) * sizeof(uint32_t) +
               s->nnz * sizeof(int32_t) + (s->d_w32 ? s->nnz * 4 : 0) + (s->d_w16 ? s->nnz * 2 : 0);
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_gpu_generate_ssm(ctbb_ctx* ctx, const ctbb_geom_c* geom, int32_t weights,
                                             ctbb_ssm** out) {
    clear_error();
    if (!ctx || !geom || !out) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (weights < CTBB_SSM_FP32 || weights > CTBB_SSM_BOTH) return fail(CTBB_ERR_INVALID_ARG, "bad weight format");
    const ctbb_geom_c& g = *geom;
    CTBB_TRY(ssm_validate_geometry(g));
    CTBB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const bool ffs = (g.Zffs || g.Phiffs);

    std::vector<ViewTab> hv;
    std::vector<double> hA, hB, hap, hn;
    host_tables(g, hv, hA, hB, hap, hn, ffs);

    SsmParams P;
    P.nx = (int)g.num_voxels_x;
    P.ny = (int)g.num_voxels_y;
    P.nch = (int)g.n_channels;
    P.nr = (int)g.Nrows_projection;
    P.nvsm = (int)g.num_views_for_system_matrix;
    P.ffs = ffs ? 1 : 0;
    P.vx = g.voxel_size_x;
    P.vy = g.voxel_size_y;
    P.vz = g.voxel_size_z;
    P.cvx = g.center_voxel_x;
    P.cvy = g.center_voxel_y;
    P.cvz = g.center_voxel_z;
    P.cc = g.center_channel_non_ffs;
    P.dgam = ffs ? g.fan_angle_increment : g.transaxial_detector_spacing / g.source_detector_distance;
    P.sa = g.axial_detector_spacing;
    P.cr = g.center_row;

    Scoped tmp;
    ViewTab* d_vt = nullptr;
    double *d_A = nullptr, *d_B = nullptr, *d_ap = nullptr, *d_n = nullptr;
    CTBB_TRY(upload(hv, &d_vt, st));
    tmp.ptrs.push_back(d_vt);
    CTBB_TRY(upload(hA, &d_A, st));
    tmp.ptrs.push_back(d_A);
    CTBB_TRY(upload(hB, &d_B, st));
    tmp.ptrs.push_back(d_B);
    CTBB_TRY(upload(hap, &d_ap, st));
    tmp.ptrs.push_back(d_ap);
    CTBB_TRY(upload(hn, &d_n, st));
    tmp.ptrs.push_back(d_n);

    ctbb_ssm* s = new ctbb_ssm();
    s->ctx = ctx;
    ctbb::ctx_retain(ctx);
    s->geom = g;
    s->ncol = (uint64_t)P.nx * P.ny;
    s->nvsm = (uint64_t)P.nvsm;
    s->ffs = ffs ? 1 : 0;
    struct Guard {
        ctbb_ssm* s;
        ~Guard() {
            if (s) free_ssm(s);
        }
    } guard{s};

    const uint64_t ncell = s->ncol * s->nvsm;
    uint16_t* d_cnt = nullptr;
    uint64_t* d_tot = nullptr;
    unsigned long long* d_max = nullptr;
    CTBB_CUDA(cudaMalloc(&d_cnt, ncell * sizeof(uint16_t)));
    tmp.ptrs.push_back(d_cnt);
    CTBB_CUDA(cudaMalloc(&d_tot, s->ncol * sizeof(uint64_t)));
    tmp.ptrs.push_back(d_tot);
    CTBB_CUDA(cudaMalloc(&d_max, sizeof(unsigned long long)));
    tmp.ptrs.push_back(d_max);
    CTBB_CUDA(cudaMemsetAsync(d_max, 0, sizeof(unsigned long long), st));
    CTBB_CUDA(cudaMalloc(&s->d_colptr, (s->ncol + 1) * sizeof(int64_t)));
    CTBB_CUDA(cudaMalloc(&s->d_vptr, s->ncol * (s->nvsm + 1) * sizeof(uint32_t)));

    cudaEvent_t e0, e1;
    CTBB_CUDA(cudaEventCreate(&e0));
    CTBB_CUDA(cudaEventCreate(&e1));
    CTBB_CUDA(cudaEventRecord(e0, st));
    const int grid = grid_for(ctx, ncell, 256);
    ssm_cells_kernel<false><<<grid, 256, 0, st>>>(P, d_vt, d_A, d_B, d_ap, d_n, d_cnt, nullptr, nullptr,
                                                  nullptr, nullptr, nullptr);
    CTBB_CUDA(cudaGetLastError());
    ssm_column_scan_kernel<<<(int)std::min<uint64_t>(s->ncol, (uint64_t)ctx->sm_count * 32), 256, 0, st>>>(
        d_cnt, P.nvsm, s->ncol, s->d_vptr, d_tot);
    CTBB_CUDA(cudaGetLastError());
    ssm_colptr_kernel<<<1, 1024, 0, st>>>(d_tot, s->ncol, s->d_colptr, d_max);
    CTBB_CUDA(cudaGetLastError());
    int64_t nnz = 0;
    unsigned long long mx = 0;
    CTBB_CUDA(cudaMemcpyAsync(&nnz, s->d_colptr + s->ncol, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CTBB_CUDA(cudaMemcpyAsync(&mx, d_max, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    CTBB_CUDA(cudaStreamSynchronize(st));
    s->nnz = (uint64_t)nnz;
    s->max_col_nnz = mx;
    const size_t nalloc = std::max<uint64_t>(1, s->nnz);
    CTBB_CUDA(cudaMalloc(&s->d_idx, nalloc * sizeof(int32_t)));
    if (weights & CTBB_SSM_FP32) CTBB_CUDA(cudaMalloc(&s->d_w32, nalloc * sizeof(float)));
    if (weights & CTBB_SSM_FP16) CTBB_CUDA(cudaMalloc(&s->d_w16, nalloc * sizeof(__half)));
    ssm_cells_kernel<true><<<grid, 256, 0, st>>>(P, d_vt, d_A, d_B, d_ap, d_n, nullptr, s->d_colptr,
                                                 s->d_vptr, s->d_idx, s->d_w32, s->d_w16);
    CTBB_CUDA(cudaGetLastError());
    CTBB_CUDA(cudaEventRecord(e1, st));
    CTBB_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    s->build_ms = ms;
    CTBB_TRY(finish_common(ctx, s, weights));
    guard.s = nullptr;
    *out = s;
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_gpu_ssm_info(const ctbb_ssm* s, ctbb_ssm_info* info) {
    clear_error();
    if (!s || !info) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    info->n_columns = s->ncol;
    info->n_views = s->nvsm;
    info->nnz = s->nnz;
    info->max_col_nnz = s->max_col_nnz;
    info->bytes_device = s->bytes;
    info->weights = s->weights;
    info->ffs = s->ffs;
    info->build_ms = s->build_ms;
    info->n_pairs = s->npairs;
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_gpu_ssm_column(const ctbb_ssm* s, uint64_t column, int32_t* idx, float* w,
                                           uint64_t cap, uint64_t* nnz) {
    clear_error();
    if (!s || !nnz) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (column >= s->ncol) return fail(CTBB_ERR_INVALID_ARG, "column %llu out of range", (unsigned long long)column);
    CTBB_CUDA(cudaSetDevice(s->ctx->device));
    int64_t cp[2];
    CTBB_CUDA(cudaMemcpy(cp, s->d_colptr + column, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost));
    const uint64_t n = (uint64_t)(cp[1] - cp[0]);
    *nnz = n;
    if (!idx && !w) return CTBB_OK;
    if (cap < n) return fail(CTBB_ERR_INVALID_ARG, "buffer too small");
    if (idx) CTBB_CUDA(cudaMemcpy(idx, s->d_idx + cp[0], n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (w) {
        if (s->d_w32) {
            CTBB_CUDA(cudaMemcpy(w, s->d_w32 + cp[0], n * sizeof(float), cudaMemcpyDeviceToHost));
        } else {
            std::vector<__half> h(n);
            CTBB_CUDA(cudaMemcpy(h.data(), s->d_w16 + cp[0], n * sizeof(__half), cudaMemcpyDeviceToHost));
            for (uint64_t i = 0; i < n; ++i) w[i] = __half2float(h[i]);
        }
    }
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_gpu_ssm_export_reference(const ctbb_ssm* s, const char* path) {
    clear_error();
    if (!s || !path) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    CTBB_CUDA(cudaSetDevice(s->ctx->device));
    std::vector<int64_t> cp(s->ncol + 1);
    CTBB_CUDA(cudaMemcpy(cp.data(), s->d_colptr, cp.size() * sizeof(int64_t), cudaMemcpyDeviceToHost));
    FILE* f = fopen(path, "wb");
    if (!f) return fail(CTBB_ERR_IO, "cannot create %s", path);
    // Stream column chunks of up to ~64M entries through host memory.
    const uint64_t chunk_entries = 64ull << 20;
    std::vector<int32_t> hi;
    std::vector<float> hw;
    std::vector<__half> hh;
    std::vector<char> rec;
    uint64_t c0 = 0;
    ctbb_status rc = CTBB_OK;
    while (c0 < s->ncol && rc == CTBB_OK) {
        uint64_t c1 = c0 + 1;
        while (c1 < s->ncol && (uint64_t)(cp[c1 + 1] - cp[c0]) <= chunk_entries) ++c1;
        const uint64_t b = (uint64_t)cp[c0], n = (uint64_t)(cp[c1] - cp[c0]);
        hi.resize(n);
        hw.resize(n);
        if (cudaMemcpy(hi.data(), s->d_idx + b, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
            rc = fail(CTBB_ERR_CUDA, "device copy failed");
            break;
        }
        if (s->d_w32) {
            cudaMemcpy(hw.data(), s->d_w32 + b, n * 4, cudaMemcpyDeviceToHost);
        } else {
            hh.resize(n);
            cudaMemcpy(hh.data(), s->d_w16 + b, n * 2, cudaMemcpyDeviceToHost);
            for (uint64_t i = 0; i < n; ++i) hw[i] = __half2float(hh[i]);
        }
        for (uint64_t c = c0; c < c1; ++c) {
            const uint64_t cb = (uint64_t)cp[c] - b, cn = (uint64_t)(cp[c + 1] - cp[c]);
            const size_t cnt = (size_t)cn;  // size_t count, then {int32, float32} pairs
            rec.resize(sizeof(size_t) + cn * 8);
            memcpy(rec.data(), &cnt, sizeof(size_t));
            for (uint64_t i = 0; i < cn; ++i) {
                memcpy(rec.data() + sizeof(size_t) + i * 8, &hi[cb + i], 4);
                memcpy(rec.data() + sizeof(size_t) + i * 8 + 4, &hw[cb + i], 4);
            }
            if (fwrite(rec.data(), 1, rec.size(), f) != rec.size()) {
                rc = fail(CTBB_ERR_IO, "short write to %s", path);
                break;
            }
        }
        c0 = c1;
    }
    if (fclose(f) != 0 && rc == CTBB_OK) rc = fail(CTBB_ERR_IO, "close failed for %s", path);
    return rc;
}

extern "C" ctbb_status ctbb_gpu_ssm_import_reference(ctbb_ctx* ctx, const ctbb_geom_c* geom, const char* path,
                                                     int32_t weights, ctbb_ssm** out) {
    clear_error();
    if (!ctx || !geom || !path || !out) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (weights < CTBB_SSM_FP32 || weights > CTBB_SSM_BOTH) return fail(CTBB_ERR_INVALID_ARG, "bad weight format");
    CTBB_TRY(ssm_validate_geometry(*geom));
    CTBB_CUDA(cudaSetDevice(ctx->device));
    const ctbb_geom_c& g = *geom;
    const uint64_t ncol = g.num_voxels_x * g.num_voxels_y, nvsm = g.num_views_for_system_matrix;
    const uint64_t per_view = g.n_channels * g.Nrows_projection;
    FILE* f = fopen(path, "rb");
    if (!f) return fail(CTBB_ERR_IO, "matrix file not found: %s", path);
    std::vector<int64_t> cp(ncol + 1, 0);
    std::vector<uint32_t> vp(ncol * (nvsm + 1), 0);
    std::vector<int32_t> hi;
    std::vector<float> hw;
    std::vector<char> buf;
    ctbb_status rc = CTBB_OK;
    for (uint64_t c = 0; c < ncol && rc == CTBB_OK; ++c) {
        size_t n = 0;
        if (fread(&n, sizeof(size_t), 1, f) != 1) {
            rc = fail(CTBB_ERR_FORMAT, "%s: truncated at column %llu", path, (unsigned long long)c);
            break;
        }
        if (n > nvsm * per_view) {
            rc = fail(CTBB_ERR_FORMAT, "%s: column %llu claims %zu entries", path, (unsigned long long)c, n);
            break;
        }
        buf.resize(n * 8);
        if (n && fread(buf.data(), 8, n, f) != n) {
            rc = fail(CTBB_ERR_FORMAT, "%s: truncated in column %llu", path, (unsigned long long)c);
            break;
        }
        cp[c + 1] = cp[c] + (int64_t)n;
        uint32_t* v = vp.data() + c * (nvsm + 1);
        int32_t last = -1;
        for (size_t i = 0; i < n; ++i) {
            int32_t q;
            float w;
            memcpy(&q, buf.data() + i * 8, 4);
            memcpy(&w, buf.data() + i * 8 + 4, 4);
            if (q <= last || (uint64_t)q >= nvsm * per_view) {
                rc = fail(CTBB_ERR_FORMAT, "%s: column %llu index %d unsorted or out of range", path,
                          (unsigned long long)c, q);
                break;
            }
            last = q;
            v[q / per_view + 1] += 1;
            hi.push_back(q);
            hw.push_back(w);
        }
        for (uint64_t k = 0; k < nvsm; ++k) v[k + 1] += v[k];
    }
    if (rc == CTBB_OK) {
        char extra;
        if (fread(&extra, 1, 1, f) == 1) rc = fail(CTBB_ERR_FORMAT, "%s: trailing bytes (geometry mismatch?)", path);
    }
    fclose(f);
    if (rc != CTBB_OK) return rc;

    ctbb_ssm* s = new ctbb_ssm();
    struct Guard {
        ctbb_ssm* s;
        ~Guard() {
            if (s) free_ssm(s);
        }
    } guard{s};
    s->ctx = ctx;
    ctbb::ctx_retain(ctx);
    s->geom = g;
    s->ncol = ncol;
    s->nvsm = nvsm;
    s->nnz = (uint64_t)cp[ncol];
    s->ffs = (g.Zffs || g.Phiffs) ? 1 : 0;
    for (uint64_t c = 0; c < ncol; ++c) s->max_col_nnz = std::max<uint64_t>(s->max_col_nnz, cp[c + 1] - cp[c]);
    cudaStream_t st = ctx->stream;
    const size_t nalloc = std::max<uint64_t>(1, s->nnz);
    CTBB_CUDA(cudaMalloc(&s->d_colptr, cp.size() * sizeof(int64_t)));
    CTBB_CUDA(cudaMalloc(&s->d_vptr, vp.size() * sizeof(uint32_t)));
    CTBB_CUDA(cudaMalloc(&s->d_idx, nalloc * sizeof(int32_t)));
    CTBB_CUDA(cudaMemcpy(s->d_colptr, cp.data(), cp.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
    CTBB_CUDA(cudaMemcpy(s->d_vptr, vp.data(), vp.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    CTBB_CUDA(cudaMemcpy(s->d_idx, hi.data(), s->nnz * sizeof(int32_t), cudaMemcpyHostToDevice));
    float* d_w = nullptr;
    CTBB_CUDA(cudaMalloc(&d_w, nalloc * sizeof(float)));
    CTBB_CUDA(cudaMemcpy(d_w, hw.data(), s->nnz * sizeof(float), cudaMemcpyHostToDevice));
    if (weights & CTBB_SSM_FP16) {
        CTBB_CUDA(cudaMalloc(&s->d_w16, nalloc * sizeof(__half)));
        f32_to_f16_kernel<<<grid_for(ctx, s->nnz, 256), 256, 0, st>>>(d_w, s->d_w16, s->nnz);
        CTBB_CUDA(cudaGetLastError());
        CTBB_CUDA(cudaStreamSynchronize(st));
    }
    if (weights & CTBB_SSM_FP32)
        s->d_w32 = d_w;
    else
        cudaFree(d_w);
    CTBB_TRY(finish_common(ctx, s, weights));
    guard.s = nullptr;
    *out = s;
    return CTBB_OK;
}

extern "C" void ctbb_gpu_ssm_free(ctbb_ssm* s) {
    if (s && s->ctx) cudaSetDevice(s->ctx->device);
    free_ssm(s);
}
