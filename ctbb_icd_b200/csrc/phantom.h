// Seeded synthetic CT data: analytic phantoms, line integrals along the
// reference's ray geometry, and Poisson noise. This replaces the private
// ctbb_read raw-data library (called at setup.cpp:288 of the CTBB_ICD
// reference) as the source of raw frames.
//
// Shared by the host library, the CUDA projector kernel and the CPU oracle, so
// every consumer uses one definition of the phantom and of the rays. Results
// of the CPU and GPU projectors agree to libm rounding (exp/log/lgamma), not
// bit for bit; parity tests always feed the same raw buffer to both sides.
//
// Ray geometry (matches the stored-system-matrix model of
// generate_system_matrix.cpp:85-116 and generate_system_matrix_ffs.cpp:112-153,
// expressed in the fixed frame):
//   view g:   theta_g = g * tube_angle_increment, source z = table_positions[g]
//             S = (R cos theta_g, R sin theta_g, z_g)
//             e_w = (cos, sin, 0), e_u = (-sin, cos, 0)
//   channel j: gamma_j = (j - cc) * s_t / SDD            (no flying focal spot)
//              gamma_j = (j - cc) * fan_angle_increment  (in-plane FFS)
//   row r:     axial_r = (r - cr) * s_a
//   detector point b = S - SDD cos(gamma) e_w - SDD sin(gamma) e_u - axial e_z
//   FFS:       the ray starts at S + off, off = +da e_u (even g) / -da e_u (odd g),
//              da = SDD R sin(fan_inc) / (4 (SDD - R))   (generate_system_matrix_ffs.cpp:67, :250-259)
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define CTBB_HD __host__ __device__ __forceinline__
#else
#define CTBB_HD inline
#endif

#ifdef __cplusplus
#include <vector>
#endif

// ---------------------------------------------------------------------------
// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw, SC'11).
// ---------------------------------------------------------------------------
struct ctbb_u4 {
    uint32_t x, y, z, w;
};

CTBB_HD ctbb_u4 ctbb_philox(ctbb_u4 c, uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
        ctbb_u4 n;
        n.x = (uint32_t)(p1 >> 32) ^ c.y ^ k0;
        n.y = (uint32_t)p1;
        n.z = (uint32_t)(p0 >> 32) ^ c.w ^ k1;
        n.w = (uint32_t)p0;
        c = n;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// Two uniform doubles in (0,1) from one Philox block.
CTBB_HD void ctbb_uniform2(uint64_t seed, uint32_t stream, uint64_t index, uint32_t draw,
                           double* u0, double* u1) {
    ctbb_u4 c;
    c.x = (uint32_t)index;
    c.y = (uint32_t)(index >> 32);
    c.z = draw;
    c.w = stream;
    const ctbb_u4 r = ctbb_philox(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint64_t a = ((uint64_t)r.x << 21) ^ (uint64_t)(r.y >> 11);
    const uint64_t b = ((uint64_t)r.z << 21) ^ (uint64_t)(r.w >> 11);
    *u0 = ((double)(a & ((1ull << 53) - 1)) + 0.5) * (1.0 / 9007199254740992.0);
    *u1 = ((double)(b & ((1ull << 53) - 1)) + 0.5) * (1.0 / 9007199254740992.0);
}

// Poisson variate with mean lam. lam < 10: multiplication (Knuth); otherwise the
// PTRS transformed-rejection method (W. Hormann, "The transformed rejection
// method for generating Poisson random variables", 1993).
CTBB_HD double ctbb_poisson(double lam, uint64_t seed, uint64_t index) {
    uint32_t draw = 0;
    if (lam <= 0.0) return 0.0;
    if (lam < 10.0) {
        const double L = exp(-lam);
        double p = 1.0;
        double k = -1.0;
        for (;;) {
            double u0, u1;
            ctbb_uniform2(seed, 7u, index, draw++, &u0, &u1);
            p *= u0;
            k += 1.0;
            if (p <= L) return k;
            p *= u1;
            k += 1.0;
            if (p <= L) return k;
        }
    }
    const double slam = sqrt(lam);
    const double loglam = log(lam);
    const double b = 0.931 + 2.53 * slam;
    const double a = -0.059 + 0.02483 * b;
    const double invalpha = 1.1239 + 1.1328 / (b - 3.4);
    const double vr = 0.9277 - 3.6224 / (b - 2.0);
    for (int it = 0; it < 1000; ++it) {
        double U, V;
        ctbb_uniform2(seed, 7u, index, draw++, &U, &V);
        U -= 0.5;
        const double us = 0.5 - fabs(U);
        const double k = floor((2.0 * a / us + b) * U + lam + 0.43);
        if (us >= 0.07 && V <= vr) return k;
        if (k < 0.0 || (us < 0.013 && V > us)) continue;
        if (log(V) + log(invalpha) - log(a / (us * us) + b) <= -lam + k * loglam - lgamma(k + 1.0))
            return k;
    }
    return floor(lam + 0.5);
}

// ---------------------------------------------------------------------------
// Phantom objects. Values are additive attenuation (cm^-1) on top of the
// objects beneath, as in the Shepp-Logan convention.
// ---------------------------------------------------------------------------
enum { CTBB_OBJ_ZCYLINDER = 0, CTBB_OBJ_ELLIPSOID = 1 };

struct ctbb_object {
    int32_t kind;      // CTBB_OBJ_*
    int32_t pad;
    double c[3];       // centre (cm)
    double axes[3];    // semi-axes (cm); z-cylinder uses axes[0] as radius
    double rot[9];     // row-major R; body frame = R^T (p - c)
    double value;      // additive attenuation (cm^-1)
};

// Parameter interval [*t0, *t1] of the unit ray s + t u inside the object;
// returns false when the ray misses it.
CTBB_HD bool ctbb_object_interval(const ctbb_object& o, const double s[3], const double u[3], double* t0,
                                  double* t1) {
    double A, B, C;
    if (o.kind == CTBB_OBJ_ZCYLINDER) {
        const double dx = s[0] - o.c[0], dy = s[1] - o.c[1];
        A = u[0] * u[0] + u[1] * u[1];
        B = 2.0 * (dx * u[0] + dy * u[1]);
        C = dx * dx + dy * dy - o.axes[0] * o.axes[0];
    } else {
        const double d[3] = {s[0] - o.c[0], s[1] - o.c[1], s[2] - o.c[2]};
        double p[3], q[3];
        for (int i = 0; i < 3; ++i) {
            // body coordinate i = (column i of R) . d, scaled by the semi-axis
            const double ri0 = o.rot[0 * 3 + i], ri1 = o.rot[1 * 3 + i], ri2 = o.rot[2 * 3 + i];
            p[i] = (ri0 * d[0] + ri1 * d[1] + ri2 * d[2]) / o.axes[i];
            q[i] = (ri0 * u[0] + ri1 * u[1] + ri2 * u[2]) / o.axes[i];
        }
        A = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
        B = 2.0 * (p[0] * q[0] + p[1] * q[1] + p[2] * q[2]);
        C = p[0] * p[0] + p[1] * p[1] + p[2] * p[2] - 1.0;
    }
    if (A <= 0.0) return false;
    const double disc = B * B - 4.0 * A * C;
    if (disc <= 0.0) return false;
    const double h = sqrt(disc);
    *t0 = (-B - h) / (2.0 * A);
    *t1 = (-B + h) / (2.0 * A);
    return true;
}

// Chord length of the unit ray inside the object (the parameter span, |u| = 1).
CTBB_HD double ctbb_object_chord(const ctbb_object& o, const double s[3], const double u[3]) {
    double t0, t1;
    if (!ctbb_object_interval(o, s, u, &t0, &t1)) return 0.0;
    return t1 - t0;
}

// Scanner/ray geometry needed by the projector (derived recon_params values).
struct ctbb_ray_geom {
    double R, SDD, cc, cr, s_t, s_a, fan_inc, da;
    double tube_angle_increment, z_first_view, tube_z_increment;
    int32_t table_direction, phi_ffs;
    int64_t n_channels, n_rows, readings;
    // z flying focal spot (generate_system_matrix_ffs.cpp:66, :266-285): the
    // source moves by -/+dr along e_w and -/+dz along z (dz = dr * tan of the
    // anode angle taken in radians, as the reference evaluates it); with both
    // spots the in-plane offset cycles over four views.
    int32_t z_ffs, any_ffs;
    double dr, dz;
};

// Unit ray (start s, direction u) of data view g, channel j, row r.
CTBB_HD void ctbb_ray(const ctbb_ray_geom& G, int64_t g, int64_t j, int64_t r, double s[3],
                      double u[3]) {
    const double th = (double)g * G.tube_angle_increment;
    const double ct = cos(th), st = sin(th);
    const double zg = G.z_first_view + (double)g * (double)G.table_direction * G.tube_z_increment;
    const double gam = G.any_ffs ? ((double)j - G.cc) * G.fan_inc : ((double)j - G.cc) * G.s_t / G.SDD;
    const double cg = cos(gam), sg = sin(gam);
    const double ax = ((double)r - G.cr) * G.s_a;
    double off = 0.0;
    if (G.phi_ffs) off = (g % 2 == 0) ? G.da : -G.da;
    // nominal source and detector point (fixed frame)
    const double S0 = G.R * ct, S1 = G.R * st, S2 = zg;
    const double b0 = S0 - G.SDD * cg * ct + G.SDD * sg * st;
    const double b1 = S1 - G.SDD * cg * st - G.SDD * sg * ct;
    const double b2 = S2 - ax;
    if (G.z_ffs) {
        // generate_system_matrix_ffs.cpp:266-285
        double sr, sa;
        if (G.phi_ffs) {
            const int64_t rho = g % 4;
            sr = rho < 2 ? -1.0 : 1.0;
            sa = (rho % 2 == 0) ? -1.0 : 1.0;
        } else {
            sr = (g % 2 == 0) ? -1.0 : 1.0;
            sa = 0.0;
        }
        const double ow = sr * G.dr, ou = sa * G.da, oz = sr * G.dz;
        s[0] = S0 + ow * ct - ou * st;
        s[1] = S1 + ow * st + ou * ct;
        s[2] = S2 + oz;
    } else {
        s[0] = S0 - off * st;
        s[1] = S1 + off * ct;
        s[2] = S2;
    }
    double d0 = b0 - s[0], d1 = b1 - s[1], d2 = b2 - s[2];
    const double n = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    u[0] = d0 / n;
    u[1] = d1 / n;
    u[2] = d2 / n;
}

// Noise-free line integral of the phantom along ray (g, j, r). With
// clip_hi > clip_lo every object is cut to the slab clip_lo <= z <= clip_hi
// (a phantom of finite length).
CTBB_HD double ctbb_line_integral(const ctbb_ray_geom& G, const ctbb_object* objs, int n_obj,
                                  int64_t g, int64_t j, int64_t r, double clip_lo = 0.0, double clip_hi = 0.0) {
    double s[3], u[3];
    ctbb_ray(G, g, j, r, s, u);
    double zt0 = -INFINITY, zt1 = INFINITY;
    if (clip_hi > clip_lo) {
        if (u[2] != 0.0) {
            const double a = (clip_lo - s[2]) / u[2], b = (clip_hi - s[2]) / u[2];
            zt0 = a < b ? a : b;
            zt1 = a < b ? b : a;
        } else if (s[2] < clip_lo || s[2] > clip_hi) {
            return 0.0;
        }
    }
    double p = 0.0;
    for (int k = 0; k < n_obj; ++k) {
        double t0, t1;
        if (!ctbb_object_interval(objs[k], s, u, &t0, &t1)) continue;
        if (!(clip_hi > clip_lo)) {
            p += objs[k].value * (t1 - t0);
            continue;
        }
        t0 = t0 > zt0 ? t0 : zt0;
        t1 = t1 < zt1 ? t1 : zt1;
        if (t1 > t0) p += objs[k].value * (t1 - t0);
    }
    return p;
}

// Incident photon count of view g: constant when lo == hi, else uniform in [lo, hi].
CTBB_HD double ctbb_view_i0(uint64_t seed, int64_t g, double lo, double hi) {
    if (hi <= lo) return lo;
    double u0, u1;
    ctbb_uniform2(seed, 3u, (uint64_t)g, 0u, &u0, &u1);
    return lo + (hi - lo) * u0;
}

// One noisy raw sample: -ln(max(N,1)/I0), N ~ Poisson(I0 exp(-p)). i0 <= 0
// means noise-free.
CTBB_HD float ctbb_noisy_sample(double p, double i0, uint64_t seed, uint64_t ray_index) {
    if (i0 <= 0.0) return (float)p;
    const double n = ctbb_poisson(i0 * exp(-p), seed, ray_index);
    return (float)(-log((n < 1.0 ? 1.0 : n) / i0));
}

#ifdef __cplusplus
// Projector geometry from any struct carrying the recon_params field names
// (recon_params itself or its POD mirror ctbb_geom_c).
template <class G>
inline ctbb_ray_geom ctbb_ray_geom_from(const G& g) {
    ctbb_ray_geom r;
    r.R = g.focal_spot_radius;
    r.SDD = g.source_detector_distance;
    r.cc = g.center_channel_non_ffs;
    r.cr = g.center_row;
    r.s_t = g.transaxial_detector_spacing;
    r.s_a = g.axial_detector_spacing;
    r.fan_inc = g.fan_angle_increment;
    // generate_system_matrix_ffs.cpp:67
    r.da = g.source_detector_distance * g.focal_spot_radius * sin(g.fan_angle_increment) /
           (4.0 * (g.source_detector_distance - g.focal_spot_radius));
    r.tube_angle_increment = g.tube_angle_increment;
    r.z_first_view = g.z_first_view;
    r.tube_z_increment = g.tube_z_increment;
    r.table_direction = (int32_t)g.table_direction;
    r.phi_ffs = g.Phiffs != 0 ? 1 : 0;
    r.z_ffs = g.Zffs != 0 ? 1 : 0;
    r.any_ffs = (g.Phiffs != 0 || g.Zffs != 0) ? 1 : 0;
    // generate_system_matrix_ffs.cpp:66 (its PI is 3.14159265359) and the
    // tan(anode_angle) of :272 with the angle in degrees.
    r.dr = g.source_detector_distance * g.CollSlicewidth /
           (4.0 * (g.source_detector_distance - g.focal_spot_radius) * tan(g.anode_angle * 3.14159265359 / 180.0));
    r.dz = r.dr * tan(g.anode_angle);
    r.n_channels = (int64_t)g.n_channels;
    r.n_rows = (int64_t)g.Nrows_projection;
    r.readings = (int64_t)g.Readings;
    return r;
}

// ---------------------------------------------------------------------------
// Phantom builders (host only).
// ---------------------------------------------------------------------------
static const double CTBB_MU_WATER = 0.192;  // cm^-1 (0.0192 / mm)

inline ctbb_object ctbb_make_zcylinder(double cx, double cy, double radius, double value) {
    ctbb_object o = {};
    o.kind = CTBB_OBJ_ZCYLINDER;
    o.c[0] = cx;
    o.c[1] = cy;
    o.axes[0] = o.axes[1] = o.axes[2] = radius;
    o.rot[0] = o.rot[4] = o.rot[8] = 1.0;
    o.value = value;
    return o;
}

// Water cylinder (r = 10 cm) with six r = 1.5 cm inserts at -200, -100, -50,
// +50, +100, +1000 HU on a 6 cm ring at 60 degree spacing.
inline void ctbb_water_phantom(std::vector<ctbb_object>& out) {
    out.push_back(ctbb_make_zcylinder(0.0, 0.0, 10.0, CTBB_MU_WATER));
    const double hu[6] = {-200.0, -100.0, -50.0, 50.0, 100.0, 1000.0};
    for (int i = 0; i < 6; ++i) {
        const double a = i * (3.14159265358979323846 / 3.0);
        out.push_back(ctbb_make_zcylinder(6.0 * cos(a), 6.0 * sin(a), 1.5, CTBB_MU_WATER * hu[i] / 1000.0));
    }
}

// n random ellipsoids (seeded): centres uniform over the r < 8 cm disc and
// z in [z_lo, z_hi]; semi-axes uniform in 0.3..4 cm; values uniform in
// -300..+1500 HU (relative to water); orientation R = Rz(a) Ry(b) Rz(c).
inline void ctbb_random_ellipsoids(std::vector<ctbb_object>& out, int n, uint64_t seed,
                                   double z_lo, double z_hi) {
    for (int i = 0; i < n; ++i) {
        double u[8];
        for (int k = 0; k < 4; ++k) ctbb_uniform2(seed, 11u, (uint64_t)i, (uint32_t)k, &u[2 * k], &u[2 * k + 1]);
        ctbb_object o = {};
        o.kind = CTBB_OBJ_ELLIPSOID;
        const double rr = 8.0 * sqrt(u[0]), ph = 2.0 * 3.14159265358979323846 * u[1];
        o.c[0] = rr * cos(ph);
        o.c[1] = rr * sin(ph);
        o.c[2] = z_lo + (z_hi - z_lo) * u[2];
        o.axes[0] = 0.3 + 3.7 * u[3];
        o.axes[1] = 0.3 + 3.7 * u[4];
        o.axes[2] = 0.3 + 3.7 * u[5];
        const double hu = -300.0 + 1800.0 * u[6];
        o.value = CTBB_MU_WATER * hu / 1000.0;
        double u8, u9;
        ctbb_uniform2(seed, 12u, (uint64_t)i, 0u, &u8, &u9);
        const double a = 2.0 * 3.14159265358979323846 * u[7], b = 3.14159265358979323846 * u8,
                     c = 2.0 * 3.14159265358979323846 * u9;
        const double ca = cos(a), sa = sin(a), cb = cos(b), sb = sin(b), cc = cos(c), sc = sin(c);
        // Rz(a) * Ry(b) * Rz(c), row-major
        o.rot[0] = ca * cb * cc - sa * sc;
        o.rot[1] = -ca * cb * sc - sa * cc;
        o.rot[2] = ca * sb;
        o.rot[3] = sa * cb * cc + ca * sc;
        o.rot[4] = -sa * cb * sc + ca * cc;
        o.rot[5] = sa * sb;
        o.rot[6] = -sb * cc;
        o.rot[7] = sb * sc;
        o.rot[8] = cb;
        out.push_back(o);
    }
}
#endif
