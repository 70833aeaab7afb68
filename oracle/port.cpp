// CPU restatement of the CTBB_ICD reconstruction path. TEST INFRASTRUCTURE
// ONLY: see port.h. Compiled with -ffp-contract=off so every operation rounds
// like the reference's own x86-64 build (which has no FMA instructions).
#include "port.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "phantom.h"

namespace {

// penalties.cpp:15 and :39-59 — SQRT2 literal and the 8 in-plane weights, in
// the neighbour order {-nx-1, -nx, -nx+1, -1, +1, +nx-1, +nx, +nx+1}.
const double kSqrt2 = 1.41421356237309504880168872420969807;
const double kW[8] = {1.0 / kSqrt2, 1.0, 1.0 / kSqrt2, 1.0, 1.0, 1.0 / kSqrt2, 1.0, 1.0 / kSqrt2};

double weights_scale() {
    double s = 0.0;
    for (int i = 0; i < 8; ++i) s += kW[i];
    return s;
}

// Flat-index neighbours as size_t, so indices below zero wrap to huge values
// and fail the `< array_size` test exactly like penalties.cpp:67-74, 92-99.
void neighbours(int q, size_t nx, size_t out[8]) {
    out[0] = q - nx - 1;
    out[1] = q - nx;
    out[2] = q - nx + 1;
    out[3] = q - 1;
    out[4] = q + 1;
    out[5] = q + nx - 1;
    out[6] = q + nx;
    out[7] = q + nx + 1;
}

// penalties.cpp:61-85
double quadratic_update(int q, double alpha, double beta, double lambda, size_t nx, size_t nvox,
                        const double* x) {
    size_t nb[8];
    neighbours(q, nx, nb);
    double sum = 0.0;
    for (int i = 0; i < 8; ++i)
        if (nb[i] < nvox) sum += kW[i] * (x[nb[i]] - x[q]);
    return (beta + lambda * sum) / (alpha + lambda * weights_scale());
}

// penalties.cpp:141-154 (sign(0) = +1 via the t >= 0 branch)
double edge_f(double du, double alpha, double beta, double delta, double lambda, const double* x,
              const size_t* nb, int q, size_t nvox) {
    double sum = 0.0;
    for (int i = 0; i < 8; ++i) {
        if (nb[i] < nvox) {
            const double t = du - (x[nb[i]] - x[q]);
            if (t >= 0)
                sum = sum + kW[i] * (1.0 - 1.0 / (1.0 + fabs(t / delta)));
            else
                sum = sum - kW[i] * (1.0 - 1.0 / (1.0 + fabs(t / delta)));
        }
    }
    return 2 * alpha * du - 2 * beta + lambda * sum;
}

inline int sgn(double v) { return v < 0 ? -1 : 1; }

// penalties.cpp:88-139: bisection on the surrogate derivative.
double edge_update(int q, double alpha, double beta, double lambda, double delta, size_t nx,
                   size_t nvox, const double* x) {
    size_t nb[8];
    neighbours(q, nx, nb);
    if (alpha == 0.0) return 0.0;
    double a = beta / alpha, b = beta / alpha;
    for (int i = 0; i < 8; ++i) {
        if (nb[i] < nvox) {
            const double d = x[nb[i]] - x[q];
            if (d < a) a = d;
            if (d > b) b = d;
        }
    }
    double c = (a + b) / 2.0;
    for (int it = 0; it < 1000000; ++it) {
        c = (a + b) / 2.0;
        const double fc = edge_f(c, alpha, beta, delta, lambda, x, nb, q, nvox);
        const double fa = edge_f(a, alpha, beta, delta, lambda, x, nb, q, nvox);
        if (fc == 0 || (b - a) / 2 < 0.00000001) return c;
        if (sgn(fc) == sgn(fa))
            a = c;
        else
            b = c;
    }
    return c;
}

}  // namespace

struct port_ssm {
    std::vector<std::vector<int32_t>> idx;
    std::vector<std::vector<float>> w;
};

extern "C" port_ssm* port_ssm_build(const ctbb_geom_c* g) {
    const size_t nx = g->num_voxels_x, ny = g->num_voxels_y;
    const size_t nch = g->n_channels, nr = g->Nrows_projection, nvsm = g->num_views_for_system_matrix;
    const bool ffs = (g->Zffs || g->Phiffs);
    port_ssm* s = new port_ssm();
    s->idx.resize(nx * ny);
    s->w.resize(nx * ny);
    const double SDD = g->source_detector_distance, R = g->focal_spot_radius;
    const double vx = g->voxel_size_x, vy = g->voxel_size_y, vz = g->voxel_size_z;
    const double cvx = g->center_voxel_x, cvy = g->center_voxel_y, cvz = g->center_voxel_z;
    // generate_system_matrix_ffs.cpp:67
    const double da = SDD * R * sin(g->fan_angle_increment) / (4.0 * (SDD - R));

    auto push = [&](size_t col, int q, double val) {
        s->idx[col].push_back(q);
        s->w[col].push_back((float)val);
    };

    for (int i = 0; i < (int)nvsm; i++) {
        // gsm.cpp:210-225 (ffs.cpp:112-128)
        const double ta = (i - 0.5 * nvsm) * g->tube_angle_increment;
        const double ew0 = cos(ta), ew1 = sin(ta), ew2 = 0.0;
        const double eu0 = -sin(ta), eu1 = cos(ta), eu2 = 0.0;
        const double ez0 = 0.0, ez1 = 0.0, ez2 = 1.0;
        const double zs = g->table_direction * ((double)i - 0.5 * (double)nvsm) * g->tube_z_increment;
        double src0 = R * ew0 + zs * ez0;
        double src1 = R * ew1 + zs * ez1;
        double src2 = R * ew2 + zs * ez2;
        // ffs.cpp:131-134, 250-259: Phi-only offset +da*e_u on even views, -da*e_u on odd.
        double off0 = 0.0, off1 = 0.0, off2 = 0.0;
        if (ffs) {
            const double sdx = (i % 2 == 0) ? da : -da;
            off0 = sdx * eu0;
            off1 = sdx * eu1;
            off2 = sdx * eu2;
            src0 = src0 + off0;
            src1 = src1 + off1;
            src2 = src2 + off2;
        }
        for (int j = 0; j < (int)nch; j++) {
            double tang;
            if (ffs)
                tang = (j - g->center_channel_non_ffs) * g->fan_angle_increment;  // ffs.cpp:138
            else
                tang = ((j - g->center_channel_non_ffs) * g->transaxial_detector_spacing) / SDD;  // gsm.cpp:228-229
            const double cg = cos(tang), sg = sin(tang);
            for (int k = 0; k < (int)nr; k++) {
                const double ap = (k - g->center_row) * g->axial_detector_spacing;
                const double A = -SDD * cg, B = SDD * sg;
                double d0 = (A * ew0 - B * eu0) - ap * ez0;
                double d1 = (A * ew1 - B * eu1) - ap * ez1;
                double d2 = (A * ew2 - B * eu2) - ap * ez2;
                if (ffs) {
                    // ffs.cpp:147-151: subtract the offset, then divide by norm_2.
                    d0 = d0 - off0;
                    d1 = d1 - off1;
                    d2 = d2 - off2;
                    double t = 0.0;
                    t += fabs(d0) * fabs(d0);
                    t += fabs(d1) * fabs(d1);
                    t += fabs(d2) * fabs(d2);
                    const double n = sqrt(t);
                    d0 = d0 / n;
                    d1 = d1 / n;
                    d2 = d2 / n;
                } else {
                    // gsm.cpp:236-239
                    const double n = sqrt(ap * ap + SDD * SDD);
                    d0 = d0 / n;
                    d1 = d1 / n;
                    d2 = d2 / n;
                }
                const int q = k + (int)nr * j + (int)nr * (int)nch * i;  // gsm.cpp:241
                const double aax = fabs(d0), aay = fabs(d1);
                if (aax > aay) {
                    // gsm.cpp:256-279: x-major, step over x columns.
                    for (int ii = 0; ii < (int)nx; ii++) {
                        const double x = (ii - cvx) * vx;
                        const double y_hat = src1 + d1 / d0 * (x - src0);
                        const double j_hat = y_hat / vy + cvy;
                        const int jj = (int)floor(j_hat);
                        const double z_hat = src2 + d2 / d0 * (x - src0);
                        const double k_hat = z_hat / vz + cvz;
                        const int kk = (int)floor(k_hat);
                        if (jj >= 0 && jj <= (int)(ny - 2)) {
                            const double scale = vx / aax;
                            if (kk == -1) {
                                push(ii + nx * jj, q, scale * (k_hat - kk) * (1 - (j_hat - jj)));
                                push(ii + nx * (jj + 1), q, scale * (k_hat - kk) * (j_hat - jj));
                            }
                            if (kk == 0) {
                                push(ii + nx * jj, q, scale * (1 - (k_hat - kk)) * (1 - (j_hat - jj)));
                                push(ii + nx * (jj + 1), q, scale * (1 - (k_hat - kk)) * (j_hat - jj));
                            }
                        }
                    }
                } else {
                    // gsm.cpp:285-308: y-major, step over y rows.
                    for (int jj = 0; jj < (int)ny; jj++) {
                        const double y = (jj - cvy) * vy;
                        const double x_hat = src0 + d0 / d1 * (y - src1);
                        const double i_hat = x_hat / vx + cvx;
                        const int ii = (int)floor(i_hat);
                        const double z_hat = src2 + d2 / d1 * (y - src1);
                        const double k_hat = z_hat / vz + cvz;
                        const int kk = (int)floor(k_hat);
                        if (ii >= 0 && ii <= (int)(nx - 2)) {
                            const double scale = vy / aay;
                            if (kk == -1) {
                                push(ii + nx * jj, q, scale * (k_hat - kk) * (1 - (i_hat - ii)));
                                push((ii + 1) + nx * jj, q, scale * (k_hat - kk) * (i_hat - ii));
                            }
                            if (kk == 0) {
                                push(ii + nx * jj, q, scale * (1 - (k_hat - kk)) * (1 - (i_hat - ii)));
                                push((ii + 1) + nx * jj, q, scale * (1 - (k_hat - kk)) * (i_hat - ii));
                            }
                        }
                    }
                }
            }
        }
    }
    return s;
}

extern "C" uint64_t port_ssm_nnz(const port_ssm* s) {
    uint64_t n = 0;
    for (size_t c = 0; c < s->idx.size(); ++c) n += s->idx[c].size();
    return n;
}

extern "C" void port_ssm_copy(const port_ssm* s, int64_t* colptr, int32_t* idx, float* w) {
    int64_t p = 0;
    for (size_t c = 0; c < s->idx.size(); ++c) {
        colptr[c] = p;
        const size_t n = s->idx[c].size();
        if (n) {
            memcpy(idx + p, s->idx[c].data(), n * sizeof(int32_t));
            memcpy(w + p, s->w[c].data(), n * sizeof(float));
        }
        p += (int64_t)n;
    }
    colptr[s->idx.size()] = p;
}

extern "C" void port_ssm_free(port_ssm* s) { delete s; }

// icd_iteration.cpp:42-286 (sequential order: y outer, x, z inner).
extern "C" void port_icd(const ctbb_geom_c* g, const uint64_t* slice_indices, const float* raw,
                         const int64_t* colptr, const int32_t* idx, const float* w, double* x,
                         double* est, int n_iter, double* dumps) {
    const size_t nx = g->num_voxels_x, ny = g->num_voxels_y, nz = g->num_voxels_z;
    const size_t nvox = nx * ny * nz;
    const size_t data_size = g->Readings * g->n_channels * g->Nrows_projection;
    const double fov_limit = (g->acquisition_fov / 2.0) * (g->acquisition_fov / 2.0);
    for (int n = 0; n < n_iter; n++) {
        for (int j = 0; j < (int)ny; j++) {
            const double y = (j - g->center_voxel_y) * g->voxel_size_y;
            for (int i = 0; i < (int)nx; i++) {
                const double xx = (i - g->center_voxel_x) * g->voxel_size_x;
                const size_t col = i + nx * j;
                if (!(xx * xx + y * y < fov_limit)) continue;
                const int64_t b = colptr[col], e = colptr[col + 1];
                for (int k = 0; k < (int)nz; k++) {
                    const int q = (int)(col + nx * ny * k);
                    const int start = (int)(slice_indices[k] - g->num_views_for_system_matrix / 2);
                    const int offset = (int)(start * g->n_channels * g->Nrows_projection);
                    double alpha = 0.0, beta = 0.0;
                    for (int64_t m = b; m < e; m++) {
                        const int index = idx[m] + offset;
                        if (index > -1 && (size_t)index < data_size) {
                            alpha += w[m] * w[m];  // float product, as in :208
                            beta += w[m] * ((double)raw[index] - est[index]);
                        }
                    }
                    double upd;
                    if (g->penalty == CTBB_PENALTY_QUADRATIC)
                        upd = quadratic_update(q, alpha, beta, g->lambda, nx, nvox, x);
                    else
                        upd = edge_update(q, alpha, beta, g->lambda, g->delta, nx, nvox, x);
                    if (upd + x[q] < 0) upd = -x[q];  // :233-234
                    x[q] += upd;
                    for (int64_t m = b; m < e; m++) {
                        const int index = idx[m] + offset;
                        if (index > -1 && (size_t)index < data_size) est[index] += upd * w[m];
                    }
                }
            }
        }
        if (dumps) memcpy(dumps + (size_t)n * nvox, x, nvox * sizeof(double));
    }
}

namespace {
// interp.h:41-76 (zero "border" outside [0, n-2]).
float interp2(const float* a, int n1, int n2, float i1, float i2) {
    if (i1 > (n1 - 2) || (i1 < 0) || i2 > (n2 - 2) || (i2 < 0)) return 0.0f;
    const float v = i1 - floorf(i1);
    const float ww = i2 - floorf(i2);
    const int a1 = (int)floorf(i2) * n1 + (int)floorf(i1);
    const int a2 = (int)floorf(i2) * n1 + (int)floorf(i1) + 1;
    const int a3 = ((int)floorf(i2) + 1) * n1 + (int)floorf(i1);
    const int a4 = ((int)floorf(i2) + 1) * n1 + (int)floorf(i1) + 1;
    return a[a1] * (1.0f - v) * (1.0f - ww) + a[a2] * v * (1.0f - ww) + a[a3] * (1.0f - v) * ww +
           a[a4] * v * ww;
}
}  // namespace

// rotate_slices.cpp:48-154
extern "C" void port_rotate(const ctbb_geom_c* g, const double* tube_angles,
                            const uint64_t* slice_indices, float* vol, int direction) {
    const double PI = 3.141592653589793238;
    const size_t nx = g->num_voxels_x, ny = g->num_voxels_y, npix = nx * ny;
    std::vector<float> tmp(npix);
    for (size_t k = 0; k < g->num_voxels_z; ++k) {
        double angle = -(tube_angles[slice_indices[k]]) * 2.0 * PI / 360.0;
        if (direction > 0) angle = -angle;
        memcpy(tmp.data(), vol + k * npix, npix * sizeof(float));
        float* out = vol + k * npix;
        for (int xi = 0; xi < (int)nx; xi++) {
            for (int yi = 0; yi < (int)ny; yi++) {
                const size_t o = xi + yi * ny;
                const double x = xi - g->center_voxel_x;
                const double y = yi - g->center_voxel_y;
                const float xp = cos(angle) * x - sin(angle) * y;
                const float yp = sin(angle) * x + cos(angle) * y;
                out[o] = interp2(tmp.data(), (int)g->nx, (int)g->ny, (float)(xp + g->center_voxel_x),
                                 (float)(yp + g->center_voxel_y));
            }
        }
    }
}

extern "C" void port_forward(const ctbb_geom_c* g, const uint64_t* slice_indices,
                             const int64_t* colptr, const int32_t* idx, const float* w,
                             const double* x, double* out) {
    const size_t nx = g->num_voxels_x, ny = g->num_voxels_y, nz = g->num_voxels_z;
    const size_t data_size = g->Readings * g->n_channels * g->Nrows_projection;
    memset(out, 0, data_size * sizeof(double));
    for (size_t col = 0; col < nx * ny; ++col) {
        for (size_t k = 0; k < nz; ++k) {
            const double xv = x[col + nx * ny * k];
            if (xv == 0.0) continue;
            const int start = (int)(slice_indices[k] - g->num_views_for_system_matrix / 2);
            const int offset = (int)(start * g->n_channels * g->Nrows_projection);
            for (int64_t m = colptr[col]; m < colptr[col + 1]; ++m) {
                const int index = idx[m] + offset;
                if (index > -1 && (size_t)index < data_size) out[index] += xv * w[m];
            }
        }
    }
}

extern "C" double port_cost(const ctbb_geom_c* g, const uint64_t* slice_indices, const float* raw,
                            const int64_t* colptr, const int32_t* idx, const float* w,
                            const double* x, double* data_term, double* penalty_term) {
    const size_t nx = g->num_voxels_x, ny = g->num_voxels_y, nz = g->num_voxels_z;
    const size_t nvox = nx * ny * nz;
    const size_t data_size = g->Readings * g->n_channels * g->Nrows_projection;
    std::vector<double> ax(data_size);
    port_forward(g, slice_indices, colptr, idx, w, x, ax.data());
    double ee = 0.0;
    for (size_t i = 0; i < data_size; ++i) {
        const double e = (double)raw[i] - ax[i];
        ee += e * e;
    }
    double pen = 0.0;
    for (size_t q = 0; q < nvox; ++q) {
        size_t nb[8];
        neighbours((int)q, nx, nb);
        for (int i = 0; i < 8; ++i) {
            if (nb[i] >= nvox) continue;
            const double t = x[q] - x[nb[i]];
            if (g->penalty == CTBB_PENALTY_QUADRATIC) {
                pen += kW[i] * t * t;
            } else {
                const double at = fabs(t);
                pen += kW[i] * (at - g->delta * log1p(at / g->delta));
            }
        }
    }
    double d, p;
    if (g->penalty == CTBB_PENALTY_QUADRATIC) {
        d = 0.5 * ee;
        p = g->lambda / 4.0 * pen;
    } else {
        d = ee;
        p = g->lambda / 2.0 * pen;
    }
    if (data_term) *data_term = d;
    if (penalty_term) *penalty_term = p;
    return d + p;
}

extern "C" void port_synth(const ctbb_geom_c* g, const ctbb_phantom_spec* spec, float* raw) {
    std::vector<ctbb_object> objs;
    ctbb_water_phantom(objs);
    if (spec->n_ellipsoids > 0)
        ctbb_random_ellipsoids(objs, spec->n_ellipsoids, spec->seed, spec->ellipsoid_z_lo,
                               spec->ellipsoid_z_hi);
    const ctbb_ray_geom G = ctbb_ray_geom_from(*g);
    const int64_t nch = G.n_channels, nr = G.n_rows, nv = G.readings;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t v = 0; v < nv; ++v) {
        const double i0 = ctbb_view_i0(spec->seed, v, spec->i0_lo, spec->i0_hi);
        for (int64_t c = 0; c < nch; ++c)
            for (int64_t r = 0; r < nr; ++r) {
                const uint64_t ray = (uint64_t)((v * nch + c) * nr + r);
                const double p = ctbb_line_integral(G, objs.data(), (int)objs.size(), v, c, r, spec->clip_z_lo, spec->clip_z_hi);
                raw[ray] = ctbb_noisy_sample(p, i0, spec->seed, ray);
            }
    }
}
