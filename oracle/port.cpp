// CPU restatement of the CTBB_ICD reconstruction path. TEST INFRASTRUCTURE
// ONLY: see port.h. Compiled with -ffp-contract=off so every operation rounds
// like the reference's own x86-64 build (which has no FMA instructions).
#include "port.h"

#include <math.h>

#include <cmath>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

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

// The updates below take the 8 neighbour differences d[i] = x_n - x_q (in
// the neighbour order above) and whether each neighbour lies inside the
// volume; the volume-based forms gather them with the reference's flat-index
// test (penalties.cpp:67-74, 92-99).

// penalties.cpp:61-85
double quadratic_update_d(double alpha, double beta, double lambda, const double* d, const bool* in) {
    double sum = 0.0;
    for (int i = 0; i < 8; ++i)
        if (in[i]) sum += kW[i] * d[i];
    return (beta + lambda * sum) / (alpha + lambda * weights_scale());
}

// penalties.cpp:141-154 (sign(0) = +1 via the t >= 0 branch)
double edge_f_d(double du, double alpha, double beta, double delta, double lambda, const double* d, const bool* in) {
    double sum = 0.0;
    for (int i = 0; i < 8; ++i) {
        if (in[i]) {
            const double t = du - d[i];
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
double edge_update_d(double alpha, double beta, double lambda, double delta, const double* d, const bool* in) {
    if (alpha == 0.0) return 0.0;
    double a = beta / alpha, b = beta / alpha;
    for (int i = 0; i < 8; ++i) {
        if (in[i]) {
            if (d[i] < a) a = d[i];
            if (d[i] > b) b = d[i];
        }
    }
    double c = (a + b) / 2.0;
    for (int it = 0; it < 1000000; ++it) {
        c = (a + b) / 2.0;
        const double fc = edge_f_d(c, alpha, beta, delta, lambda, d, in);
        const double fa = edge_f_d(a, alpha, beta, delta, lambda, d, in);
        if (fc == 0 || (b - a) / 2 < 0.00000001) return c;
        if (sgn(fc) == sgn(fa))
            a = c;
        else
            b = c;
    }
    return c;
}

void gather_neighbours(int q, size_t nx, size_t nvox, const double* x, double* d, bool* in) {
    size_t nb[8];
    neighbours(q, nx, nb);
    for (int i = 0; i < 8; ++i) {
        in[i] = nb[i] < nvox;
        d[i] = in[i] ? x[nb[i]] - x[q] : 0.0;
    }
}

double quadratic_update(int q, double alpha, double beta, double lambda, size_t nx, size_t nvox,
                        const double* x) {
    double d[8];
    bool in[8];
    gather_neighbours(q, nx, nvox, x, d, in);
    return quadratic_update_d(alpha, beta, lambda, d, in);
}

double edge_update(int q, double alpha, double beta, double lambda, double delta, size_t nx,
                   size_t nvox, const double* x) {
    double d[8];
    bool in[8];
    gather_neighbours(q, nx, nvox, x, d, in);
    return edge_update_d(alpha, beta, lambda, delta, d, in);
}

}  // namespace

struct port_ssm {
    std::vector<std::vector<int32_t>> idx;
    std::vector<std::vector<float>> w;
};

namespace {

// One ray of the stored-system-matrix window: source position, unit direction
// and its matrix row q, with the reference's arithmetic.
struct Ray {
    double src0, src1, src2, d0, d1, d2, aax, aay;
    int q;
};

// View geometry shared by every ray of view i: generate_system_matrix.cpp:85-100
// (generate_system_matrix_ffs.cpp:112-134 with the Phi-only offset of
// generate_ffs_offset, :242-290: +da*e_u on even views, -da*e_u on odd).
struct ViewGeom {
    double ew0, ew1, ew2, eu0, eu1, eu2, ez0, ez1, ez2;
    double src0, src1, src2, off0, off1, off2;
};

// generate_system_matrix_ffs.cpp:66 (PI there is 3.14159265359)
double ffs_dr(const ctbb_geom_c* g) {
    const double SDD = g->source_detector_distance, R = g->focal_spot_radius;
    return SDD * g->CollSlicewidth / (4.0 * (SDD - R) * tan(g->anode_angle * 3.14159265359 / 180.0));
}

ViewGeom view_geom(const ctbb_geom_c* g, int i, bool ffs, double da) {
    ViewGeom v;
    const double nvsm = (double)g->num_views_for_system_matrix;
    const double ta = (i - 0.5 * nvsm) * g->tube_angle_increment;
    v.ew0 = cos(ta), v.ew1 = sin(ta), v.ew2 = 0.0;
    v.eu0 = -sin(ta), v.eu1 = cos(ta), v.eu2 = 0.0;
    v.ez0 = 0.0, v.ez1 = 0.0, v.ez2 = 1.0;
    const double zs = g->table_direction * ((double)i - 0.5 * nvsm) * g->tube_z_increment;
    v.src0 = g->focal_spot_radius * v.ew0 + zs * v.ez0;
    v.src1 = g->focal_spot_radius * v.ew1 + zs * v.ez1;
    v.src2 = g->focal_spot_radius * v.ew2 + zs * v.ez2;
    v.off0 = v.off1 = v.off2 = 0.0;
    if (ffs && !g->Zffs) {
        // generate_ffs_offset, Phi only (:253-259): +da e_u on even views.
        const double sdx = (i % 2 == 0) ? da : -da;
        v.off0 = sdx * v.eu0;
        v.off1 = sdx * v.eu1;
        v.off2 = sdx * v.eu2;
    } else if (ffs && !g->Phiffs) {
        // Z only (:262-270): -dr e_w - dr tan(anode_angle) e_z on even views,
        // + on odd; tan of the angle as given (degrees).
        const double dr = ffs_dr(g);
        const double c = (i % 2 == 0) ? -dr : dr;
        const double ct = c * tan(g->anode_angle);
        v.off0 = c * v.ew0 + ct * v.ez0;
        v.off1 = c * v.ew1 + ct * v.ez1;
        v.off2 = c * v.ew2 + ct * v.ez2;
    } else if (ffs) {
        // Z and Phi (:272-284): (-dr, -da), (-dr, +da), (+dr, -da), (+dr, +da).
        const double dr = ffs_dr(g);
        const int rho = i % 4;
        const double c = rho < 2 ? -dr : dr, a = (rho % 2 == 0) ? -da : da;
        const double ct = c * tan(g->anode_angle);
        v.off0 = (c * v.ew0 + a * v.eu0) + ct * v.ez0;
        v.off1 = (c * v.ew1 + a * v.eu1) + ct * v.ez1;
        v.off2 = (c * v.ew2 + a * v.eu2) + ct * v.ez2;
    }
    if (ffs) {
        v.src0 = v.src0 + v.off0;
        v.src1 = v.src1 + v.off1;
        v.src2 = v.src2 + v.off2;
    }
    return v;
}

// Ray (view i, channel j, row k). Channel angle: generate_system_matrix.cpp:103-106
// (ffs.cpp:138-140); row offset :109 (ffs :143); direction :111-114, the
// expression divided element-wise by sqrt(z^2 + SDD^2) (ffs :147-151: offset
// subtracted, then divided by norm_2); q :116 (ffs :153).
Ray make_ray(const ctbb_geom_c* g, const ViewGeom& v, int i, int j, int k, bool ffs) {
    const double SDD = g->source_detector_distance;
    double tang;
    if (ffs)
        tang = (j - g->center_channel_non_ffs) * g->fan_angle_increment;
    else
        tang = ((j - g->center_channel_non_ffs) * g->transaxial_detector_spacing) / SDD;
    const double cg = cos(tang), sg = sin(tang);
    const double ap = (k - g->center_row) * g->axial_detector_spacing;
    const double A = -SDD * cg, B = SDD * sg;
    double d0 = (A * v.ew0 - B * v.eu0) - ap * v.ez0;
    double d1 = (A * v.ew1 - B * v.eu1) - ap * v.ez1;
    double d2 = (A * v.ew2 - B * v.eu2) - ap * v.ez2;
    if (ffs) {
        d0 = d0 - v.off0;
        d1 = d1 - v.off1;
        d2 = d2 - v.off2;
        double t = 0.0;
        t += fabs(d0) * fabs(d0);
        t += fabs(d1) * fabs(d1);
        t += fabs(d2) * fabs(d2);
        const double n = sqrt(t);
        d0 = d0 / n;
        d1 = d1 / n;
        d2 = d2 / n;
    } else {
        const double n = sqrt(ap * ap + SDD * SDD);
        d0 = d0 / n;
        d1 = d1 / n;
        d2 = d2 / n;
    }
    Ray r;
    r.src0 = v.src0, r.src1 = v.src1, r.src2 = v.src2;
    r.d0 = d0, r.d1 = d1, r.d2 = d2;
    r.aax = fabs(d0), r.aay = fabs(d1);
    r.q = k + (int)g->Nrows_projection * j + (int)g->Nrows_projection * (int)g->n_channels * i;
    return r;
}

// One Joseph step of a ray: the two bilinear taps it deposits at step `s`
// (x index when x-major, y index when y-major). Returns false when the step
// deposits nothing. Columns c0, c1 and FP32 weights w0, w1 follow
// generate_system_matrix.cpp:131-153 (x-major, taps at rows j and j+1) and
// :160-182 (y-major, taps at columns i and i+1); ffs.cpp:167-189 / :196-218.
bool joseph_step(const ctbb_geom_c* g, const Ray& r, int s, int64_t* c0, int64_t* c1, float* w0, float* w1) {
    const int nx = (int)g->num_voxels_x, ny = (int)g->num_voxels_y;
    const double vx = g->voxel_size_x, vy = g->voxel_size_y, vz = g->voxel_size_z;
    const double cvx = g->center_voxel_x, cvy = g->center_voxel_y, cvz = g->center_voxel_z;
    if (r.aax > r.aay) {
        const double x = (s - cvx) * vx;
        const double y_hat = r.src1 + r.d1 / r.d0 * (x - r.src0);
        const double j_hat = y_hat / vy + cvy;
        const int jj = (int)floor(j_hat);
        const double z_hat = r.src2 + r.d2 / r.d0 * (x - r.src0);
        const double k_hat = z_hat / vz + cvz;
        const int kk = (int)floor(k_hat);
        if (!(jj >= 0 && jj <= ny - 2) || (kk != -1 && kk != 0)) return false;
        const double scale = vx / r.aax;
        *c0 = s + (int64_t)nx * jj;
        *c1 = s + (int64_t)nx * (jj + 1);
        if (kk == -1) {
            *w0 = (float)(scale * (k_hat - kk) * (1 - (j_hat - jj)));
            *w1 = (float)(scale * (k_hat - kk) * (j_hat - jj));
        } else {
            *w0 = (float)(scale * (1 - (k_hat - kk)) * (1 - (j_hat - jj)));
            *w1 = (float)(scale * (1 - (k_hat - kk)) * (j_hat - jj));
        }
        return true;
    }
    const double y = (s - cvy) * vy;
    const double x_hat = r.src0 + r.d0 / r.d1 * (y - r.src1);
    const double i_hat = x_hat / vx + cvx;
    const int ii = (int)floor(i_hat);
    const double z_hat = r.src2 + r.d2 / r.d1 * (y - r.src1);
    const double k_hat = z_hat / vz + cvz;
    const int kk = (int)floor(k_hat);
    if (!(ii >= 0 && ii <= nx - 2) || (kk != -1 && kk != 0)) return false;
    const double scale = vy / r.aay;
    *c0 = ii + (int64_t)nx * s;
    *c1 = (ii + 1) + (int64_t)nx * s;
    if (kk == -1) {
        *w0 = (float)(scale * (k_hat - kk) * (1 - (i_hat - ii)));
        *w1 = (float)(scale * (k_hat - kk) * (i_hat - ii));
    } else {
        *w0 = (float)(scale * (1 - (k_hat - kk)) * (1 - (i_hat - ii)));
        *w1 = (float)(scale * (1 - (k_hat - kk)) * (i_hat - ii));
    }
    return true;
}

double ffs_da(const ctbb_geom_c* g) {
    // generate_system_matrix_ffs.cpp:67
    const double SDD = g->source_detector_distance, R = g->focal_spot_radius;
    return SDD * R * sin(g->fan_angle_increment) / (4.0 * (SDD - R));
}

}  // namespace

// Ray-driven like the reference: views, channels, rows in order, every Joseph
// step of each ray pushing its two taps (generate_system_matrix.cpp:80-186,
// generate_system_matrix_ffs.cpp:104-222).
// Views are split into contiguous ranges built in parallel; each column's
// parts are then concatenated in view order, which is the reference's push
// order, so the result does not depend on the thread count.
extern "C" port_ssm* port_ssm_build(const ctbb_geom_c* g) {
    const size_t nx = g->num_voxels_x, ny = g->num_voxels_y, ncol = nx * ny;
    const size_t nch = g->n_channels, nr = g->Nrows_projection, nvsm = g->num_views_for_system_matrix;
    const bool ffs = (g->Zffs || g->Phiffs);
    const double da = ffs_da(g);
    port_ssm* s = new port_ssm();
    s->idx.resize(ncol);
    s->w.resize(ncol);
    int nparts = 1;
#ifdef _OPENMP
    nparts = omp_get_max_threads();
#endif
    nparts = (int)std::max<size_t>(1, std::min<size_t>((size_t)nparts, nvsm));
    std::vector<port_ssm> parts(nparts);
#pragma omp parallel for schedule(static, 1) num_threads(nparts)
    for (int p = 0; p < nparts; p++) {
        port_ssm& part = parts[p];
        part.idx.resize(ncol);
        part.w.resize(ncol);
        const int v0 = (int)(nvsm * p / nparts), v1 = (int)(nvsm * (p + 1) / nparts);
        for (int i = v0; i < v1; i++) {
            const ViewGeom v = view_geom(g, i, ffs, da);
            for (int j = 0; j < (int)nch; j++)
                for (int k = 0; k < (int)nr; k++) {
                    const Ray r = make_ray(g, v, i, j, k, ffs);
                    const int nsteps = (int)(r.aax > r.aay ? nx : ny);
                    for (int st = 0; st < nsteps; st++) {
                        int64_t c0, c1;
                        float w0, w1;
                        if (!joseph_step(g, r, st, &c0, &c1, &w0, &w1)) continue;
                        part.idx[c0].push_back(r.q);
                        part.w[c0].push_back(w0);
                        part.idx[c1].push_back(r.q);
                        part.w[c1].push_back(w1);
                    }
                }
        }
    }
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < (int64_t)ncol; c++) {
        size_t n = 0;
        for (int p = 0; p < nparts; p++) n += parts[p].idx[c].size();
        s->idx[c].reserve(n);
        s->w[c].reserve(n);
        for (int p = 0; p < nparts; p++) {
            s->idx[c].insert(s->idx[c].end(), parts[p].idx[c].begin(), parts[p].idx[c].end());
            s->w[c].insert(s->w[c].end(), parts[p].w[c].begin(), parts[p].w[c].end());
            std::vector<int32_t>().swap(parts[p].idx[c]);
            std::vector<float>().swap(parts[p].w[c]);
        }
    }
    return s;
}

// Entries of the selected columns on the selected (ascending) views only:
// for each ray of those views, the one Joseph step that can reach each
// selected column (its x index when the ray is x-major, its y index when
// y-major), with the same arithmetic as port_ssm_build. Output per
// (column, view) in that order: counts[c * n_views + v], then the entries of
// every (column, view) concatenated, sorted by q like the reference's.
extern "C" uint64_t port_ssm_subset(const ctbb_geom_c* g, int n_cols, const int64_t* cols, int n_views,
                                    const int32_t* views, uint32_t* counts, int32_t* idx, float* w,
                                    uint64_t capacity) {
    const size_t nx = g->num_voxels_x;
    const size_t nch = g->n_channels, nr = g->Nrows_projection;
    const bool ffs = (g->Zffs || g->Phiffs);
    const double da = ffs_da(g);
    std::vector<std::vector<int32_t>> qi((size_t)n_cols * n_views);
    std::vector<std::vector<float>> wi((size_t)n_cols * n_views);
#pragma omp parallel for schedule(dynamic, 1)
    for (int vv = 0; vv < n_views; vv++) {
        const int i = views[vv];
        const ViewGeom v = view_geom(g, i, ffs, da);
        for (int j = 0; j < (int)nch; j++)
            for (int k = 0; k < (int)nr; k++) {
                const Ray r = make_ray(g, v, i, j, k, ffs);
                for (int c = 0; c < n_cols; c++) {
                    const int64_t col = cols[c];
                    const int ic = (int)(col % (int64_t)nx), jc = (int)(col / (int64_t)nx);
                    const int st = r.aax > r.aay ? ic : jc;
                    int64_t c0, c1;
                    float w0, w1;
                    if (!joseph_step(g, r, st, &c0, &c1, &w0, &w1)) continue;
                    const size_t slot = (size_t)c * n_views + vv;
                    if (c0 == col) {
                        qi[slot].push_back(r.q);
                        wi[slot].push_back(w0);
                    }
                    if (c1 == col) {
                        qi[slot].push_back(r.q);
                        wi[slot].push_back(w1);
                    }
                }
            }
    }
    uint64_t n = 0;
    for (size_t slot = 0; slot < qi.size(); ++slot) {
        counts[slot] = (uint32_t)qi[slot].size();
        for (size_t e = 0; e < qi[slot].size(); ++e, ++n)
            if (n < capacity) {
                idx[n] = qi[slot][e];
                w[n] = wi[slot][e];
            }
    }
    return n;
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

// penalties.cpp:61-154 on given inputs: x9[9 i] the voxel, x9[9 i + 1 + l]
// neighbour l (NaN: outside the volume); FP32 values widened to FP64 as the
// grouped mode reads its FP32 image.
extern "C" void port_penalty_steps(int penalty, double lambda, double delta, uint64_t n, const double* alpha,
                                   const double* beta, const float* x9, double* step) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        double d[8];
        bool in[8];
        const double xq = (double)x9[9 * i];
        for (int l = 0; l < 8; ++l) {
            const float xn = x9[9 * i + 1 + l];
            in[l] = !std::isnan(xn);
            d[l] = in[l] ? (double)xn - xq : 0.0;
        }
        step[i] = penalty == CTBB_PENALTY_QUADRATIC ? quadratic_update_d(alpha[i], beta[i], lambda, d, in)
                                                    : edge_update_d(alpha[i], beta[i], lambda, delta, d, in);
    }
}
