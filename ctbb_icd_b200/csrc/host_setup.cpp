// Host side of the drop-in boundary: parameter file, checks and derived
// geometry, rotating-slice tables, FileType 0 raw reading, the CPU synthetic
// projector, and status/error reporting.
//
// Behaviour follows the reference's parse_config.cpp:34-111 and
// setup.cpp:69-420, with `exit(1)` replaced by status codes. Every derived
// value is computed with the same expression (same operation order and
// float/double mixing) so the results are bit-identical to the reference's.
#include <errno.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <fstream>
#include <map>
#include <string>
#include <vector>

#include <cuda_runtime_api.h>

#include "common.h"
#include "phantom.h"

namespace ctbb {

static thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
    char buf[2048];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

void clear_error() { g_last_error.clear(); }

ctbb_status fail(ctbb_status st, const char* fmt, ...) {
    char buf[2048];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    // A failed allocation is reported here; the CUDA runtime would otherwise
    // keep it as its last error and a later launch check would return it.
    if (st == CTBB_ERR_OOM) cudaGetLastError();
    return st;
}

namespace {

std::string trim(const std::string& s) {
    const char* ws = " \t\r\n";
    const size_t b = s.find_first_not_of(ws);
    if (b == std::string::npos) return "";
    const size_t e = s.find_last_not_of(ws);
    return s.substr(b, e - b + 1);
}

// Flat `key: value  # comment` YAML subset (the only form parameter files use).
bool load_prm(const char* path, std::map<std::string, std::string>& kv) {
    std::ifstream f(path);
    if (!f.good()) return false;
    std::string line;
    while (std::getline(f, line)) {
        for (size_t i = 0; i < line.size(); ++i) {
            if (line[i] == '#' && (i == 0 || line[i - 1] == ' ' || line[i - 1] == '\t')) {
                line.erase(i);
                break;
            }
        }
        const size_t colon = line.find(':');
        if (colon == std::string::npos) continue;
        std::string key = trim(line.substr(0, colon));
        std::string val = trim(line.substr(colon + 1));
        if (val.size() >= 2 && ((val.front() == '"' && val.back() == '"') ||
                                (val.front() == '\'' && val.back() == '\'')))
            val = val.substr(1, val.size() - 2);
        if (!key.empty()) kv[key] = val;
    }
    return true;
}

// parse_item (parse_config.cpp:27-32): a key that is absent, empty or not
// convertible leaves the field untouched ("NOT FOUND").
bool get_str(const std::map<std::string, std::string>& kv, const char* key, std::string* out) {
    auto it = kv.find(key);
    if (it == kv.end() || it->second.empty()) return false;
    *out = it->second;
    return true;
}

bool get_double(const std::map<std::string, std::string>& kv, const char* key, double* out) {
    std::string s;
    if (!get_str(kv, key, &s)) return false;
    char* end = nullptr;
    errno = 0;
    const double v = strtod(s.c_str(), &end);
    if (end == s.c_str() || *end != '\0' || errno == ERANGE) return false;
    *out = v;
    return true;
}

bool get_size(const std::map<std::string, std::string>& kv, const char* key, uint64_t* out) {
    std::string s;
    if (!get_str(kv, key, &s)) return false;
    if (s[0] == '-') return false;
    char* end = nullptr;
    errno = 0;
    const unsigned long long v = strtoull(s.c_str(), &end, 10);
    if (end == s.c_str() || *end != '\0' || errno == ERANGE) return false;
    *out = (uint64_t)v;
    return true;
}

void copy_str(char* dst, size_t cap, const std::string& s) {
    snprintf(dst, cap, "%s", s.c_str());
}

const double kPI = 3.141592653589793238;  // setup.cpp:35

}  // namespace
}  // namespace ctbb

using namespace ctbb;

extern "C" const char* ctbb_last_error(void) { return g_last_error.c_str(); }

extern "C" const char* ctbb_status_str(ctbb_status s) {
    switch (s) {
        case CTBB_OK: return "ok";
        case CTBB_ERR_INVALID_ARG: return "invalid argument";
        case CTBB_ERR_CONFIG: return "invalid or missing parameter";
        case CTBB_ERR_IO: return "i/o error";
        case CTBB_ERR_RANGE: return "reconstruction range outside the scanned data";
        case CTBB_ERR_CUDA: return "CUDA error";
        case CTBB_ERR_NO_DEVICE: return "no CUDA device";
        case CTBB_ERR_OOM: return "out of memory";
        case CTBB_ERR_TIMEOUT: return "device wait timed out";
        case CTBB_ERR_UNSUPPORTED: return "unsupported";
        case CTBB_ERR_FORMAT: return "bad matrix file";
        default: return "unknown status";
    }
}

// setup.cpp:69-243 and parse_config.cpp:34-111
extern "C" ctbb_status ctbb_configure_recon_params(const char* prm_path, ctbb_geom_c* g,
                                                   ctbb_prm_strings* strings) {
    clear_error();
    if (!prm_path || !g) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    std::map<std::string, std::string> kv;
    if (!load_prm(prm_path, kv)) return fail(CTBB_ERR_IO, "Parameter file not found: %s", prm_path);

    memset(g, 0, sizeof(*g));
    const uint64_t kUnset = (uint64_t)-1;  // setup.cpp:91-96 sentinels for zero-allowed fields
    g->FileType = g->FileSubType = g->RawOffset = g->Zffs = g->Phiffs = g->wfbp_initialize = kUnset;

    std::string initial_recon_path, matrix_path, output_dir, output_file, potential, recon_path,
        sinogram_path, penalty;
    get_str(kv, "initial_recon_path", &initial_recon_path);
    get_str(kv, "matrix_path", &matrix_path);
    get_str(kv, "output_dir", &output_dir);
    get_str(kv, "output_file", &output_file);
    get_str(kv, "potential", &potential);
    get_str(kv, "recon_path", &recon_path);
    get_str(kv, "sinogram_path", &sinogram_path);

    get_double(kv, "acquisition_fov", &g->acquisition_fov);
    get_double(kv, "anode_angle", &g->anode_angle);
    get_double(kv, "axial_detector_spacing", &g->axial_detector_spacing);
    get_double(kv, "axial_focal_spot_shift", &g->axial_focal_spot_shift);
    get_double(kv, "center_channel_non_ffs", &g->center_channel_non_ffs);
    get_double(kv, "center_row", &g->center_row);
    get_double(kv, "focal_spot_radius", &g->focal_spot_radius);
    get_size(kv, "n_channels", &g->n_channels);
    get_size(kv, "num_views_per_turn_without_ffs", &g->num_views_per_turn_without_ffs);
    get_double(kv, "source_detector_distance", &g->source_detector_distance);
    get_double(kv, "transaxial_detector_spacing", &g->transaxial_detector_spacing);
    get_double(kv, "transaxial_focal_spot_shift", &g->transaxial_focal_spot_shift);
    get_double(kv, "fan_angle_increment", &g->fan_angle_increment);

    get_str(kv, "penalty", &penalty);
    get_double(kv, "lambda", &g->lambda);
    get_double(kv, "delta", &g->delta);
    get_size(kv, "num_iterations", &g->num_iterations);
    get_size(kv, "num_views_for_system_matrix", &g->num_views_for_system_matrix);

    get_double(kv, "first_view_angle", &g->first_view_angle);
    get_size(kv, "num_z_ffs", &g->num_z_ffs);
    get_size(kv, "num_phi_ffs", &g->num_phi_ffs);
    get_size(kv, "num_views", &g->num_views);
    get_double(kv, "table_feed_per_rotation", &g->table_feed_per_rotation);
    get_double(kv, "tube_angle_increment", &g->tube_angle_increment);
    get_double(kv, "z_end", &g->z_end);
    get_double(kv, "z_first_view", &g->z_first_view);
    get_double(kv, "z_good_slice", &g->z_good_slice);
    get_double(kv, "z_matrix_start", &g->z_matrix_start);
    get_double(kv, "z_start", &g->z_start);

    get_double(kv, "recon_fov", &g->recon_fov);
    get_size(kv, "nx", &g->nx);
    get_size(kv, "ny", &g->ny);
    get_double(kv, "slice_thickness", &g->slice_thickness);

    get_size(kv, "FileType", &g->FileType);
    get_size(kv, "FileSubType", &g->FileSubType);
    get_size(kv, "RawOffset", &g->RawOffset);
    get_size(kv, "Readings", &g->Readings);
    get_size(kv, "Zffs", &g->Zffs);
    get_size(kv, "Phiffs", &g->Phiffs);
    get_double(kv, "CollSlicewidth", &g->CollSlicewidth);
    get_size(kv, "Nrows", &g->Nrows);
    get_size(kv, "wfbp_initialize", &g->wfbp_initialize);

    // setup.cpp:108-179 — required fields and defaults.
    std::string missing;
    auto need_s = [&](const char* n, const std::string& v) { if (v.empty()) missing += std::string(" ") + n; };
    auto need_d = [&](const char* n, double v) { if (v == 0.0) missing += std::string(" ") + n; };
    auto need_z = [&](const char* n, uint64_t v) { if (v == 0) missing += std::string(" ") + n; };
    auto need_u = [&](const char* n, uint64_t v) { if (v == kUnset) missing += std::string(" ") + n; };
    need_s("sinogram_path", sinogram_path);
    need_s("output_dir", output_dir);
    need_s("output_file", output_file);
    need_d("acquisition_fov", g->acquisition_fov);
    need_z("num_views_per_turn_without_ffs", g->num_views_per_turn_without_ffs);
    need_d("focal_spot_radius", g->focal_spot_radius);
    need_d("source_detector_distance", g->source_detector_distance);
    need_d("anode_angle", g->anode_angle);
    need_z("n_channels", g->n_channels);
    need_z("Nrows", g->Nrows);
    need_d("axial_detector_spacing", g->axial_detector_spacing);
    need_d("axial_focal_spot_shift", g->axial_focal_spot_shift);
    need_d("center_channel_non_ffs", g->center_channel_non_ffs);
    need_d("center_row", g->center_row);
    need_d("transaxial_detector_spacing", g->transaxial_detector_spacing);
    need_d("transaxial_focal_spot_shift", g->transaxial_focal_spot_shift);
    need_d("fan_angle_increment", g->fan_angle_increment);
    need_d("table_feed_per_rotation", g->table_feed_per_rotation);
    if (g->recon_fov == 0.0) g->recon_fov = 25.0;
    if (g->nx == 0) g->nx = 512;
    if (g->ny == 0) g->ny = 512;
    need_d("z_start", g->z_start);
    need_d("z_end", g->z_end);
    if (g->slice_thickness == 0.0) g->slice_thickness = 1.0;
    if (penalty.empty()) penalty = "quadratic";
    if (g->lambda == 0.0) g->lambda = 0.3;
    if (g->delta == 0.0) g->delta = 0.005;
    need_z("num_iterations", g->num_iterations);
    need_u("FileType", g->FileType);
    need_u("FileSubType", g->FileSubType);
    need_u("RawOffset", g->RawOffset);
    need_z("Readings", g->Readings);
    need_u("Zffs", g->Zffs);
    need_u("Phiffs", g->Phiffs);
    need_u("wfbp_initialize", g->wfbp_initialize);
    need_d("CollSlicewidth", g->CollSlicewidth);
    if (penalty == "quadratic")
        g->penalty = CTBB_PENALTY_QUADRATIC;
    else if (penalty == "edge-preserving")
        g->penalty = CTBB_PENALTY_EDGE_PRESERVING;
    else
        missing += " penalty(\"" + penalty + "\" is not quadratic or edge-preserving)";
    if (!missing.empty())
        return fail(CTBB_ERR_CONFIG, "Missing or invalid required parameters:%s", missing.c_str());
    if (g->Zffs > 1 || g->Phiffs > 1)
        return fail(CTBB_ERR_CONFIG, "Zffs and Phiffs must be 0 or 1");

    // setup.cpp:183-237 — derived values.
    g->center_voxel_x = (g->nx - 1.0) / 2.0;
    g->center_voxel_y = (g->ny - 1.0) / 2.0;
    g->dx = g->recon_fov / (double)g->nx;
    g->dy = g->recon_fov / (double)g->ny;
    g->dz = g->slice_thickness;
    g->fov_radius = g->recon_fov / 2.0;
    g->voxel_size_x = g->dx;
    g->voxel_size_y = g->dy;
    g->voxel_size_z = g->dz;
    g->num_voxels_x = g->nx;
    g->num_voxels_y = g->ny;
    g->num_voxels_z = g->nz;
    const int nffs = (int)((size_t)pow(2.0, (double)g->Zffs) * (size_t)pow(2.0, (double)g->Phiffs));
    g->num_views_per_turn = g->num_views_per_turn_without_ffs * (size_t)pow(2.0, (double)g->Zffs) *
                            (size_t)pow(2.0, (double)g->Phiffs);
    g->tube_angle_increment = 2.0 * kPI / g->num_views_per_turn;
    g->tube_z_increment = g->table_feed_per_rotation / g->num_views_per_turn;
    g->voxel_size_z = round(g->voxel_size_z / (nffs * g->tube_z_increment)) * (nffs * g->tube_z_increment);
    g->views_per_slice = (uint64_t)(g->voxel_size_z / g->tube_z_increment);
    g->beam_width = (double)g->Nrows * g->axial_detector_spacing;
    g->beam_width_at_roi_edge =
        g->beam_width * (g->focal_spot_radius + g->fov_radius) / g->source_detector_distance;
    g->num_views_for_system_matrix = (uint64_t)(2.0 * kPI / (g->table_feed_per_rotation * g->tube_angle_increment) *
                                                g->beam_width_at_roi_edge);
    if (g->num_views_for_system_matrix % 2 == 1) g->num_views_for_system_matrix += 1;
    while ((g->num_views_for_system_matrix / 2) % (uint64_t)nffs > 0) g->num_views_for_system_matrix += 1;
    g->Nrows_projection = g->Nrows / (size_t)pow(2.0, (double)g->Zffs);
    g->center_voxel_z = 0.0;
    if (matrix_path.empty()) matrix_path = output_dir + "/matrix.bin";
    g->num_voxels_z = (uint64_t)(fabs(g->z_end - g->z_start) / g->voxel_size_z);

    if (strings) {
        memset(strings, 0, sizeof(*strings));
        copy_str(strings->initial_recon_path, sizeof(strings->initial_recon_path), initial_recon_path);
        copy_str(strings->matrix_path, sizeof(strings->matrix_path), matrix_path);
        copy_str(strings->output_dir, sizeof(strings->output_dir), output_dir);
        copy_str(strings->output_file, sizeof(strings->output_file), output_file);
        copy_str(strings->potential, sizeof(strings->potential), potential);
        copy_str(strings->recon_path, sizeof(strings->recon_path), recon_path);
        copy_str(strings->sinogram_path, sizeof(strings->sinogram_path), sinogram_path);
        copy_str(strings->penalty, sizeof(strings->penalty), penalty);
    }
    return CTBB_OK;
}

// setup.cpp:273-285 (FileType 0 angles and positions) and :348-409.
extern "C" ctbb_status ctbb_slice_tables(ctbb_geom_c* g, double* tube_angles, double* table_positions,
                                         double* slice_locations, uint64_t* slice_indices,
                                         uint64_t max_slices) {
    clear_error();
    if (!g || !tube_angles || !table_positions) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (g->FileType != 0)
        return fail(CTBB_ERR_UNSUPPORTED, "FileType %llu: only FileType 0 (binary) readers are available",
                    (unsigned long long)g->FileType);
    if (g->Readings == 0 || g->num_views_per_turn == 0) return fail(CTBB_ERR_INVALID_ARG, "empty scan");
    g->first_view_angle = 0.0;
    g->table_direction = -1;
    for (uint64_t i = 0; i < g->Readings; i++) {
        tube_angles[i] = fmod(((360.0f / g->num_views_per_turn) * (int)i + g->first_view_angle), 360.0f);
        table_positions[i] = ((float)g->Readings / (float)g->num_views_per_turn) * g->table_feed_per_rotation -
                             (float)(int)i * g->table_feed_per_rotation / (float)g->num_views_per_turn;
    }
    const int direction = g->table_direction;
    g->z_first_view = table_positions[0] / 10.0;
    for (uint64_t i = 0; i < g->Readings; i++)
        table_positions[i] = g->z_first_view + (double)(int)i * (double)direction * g->tube_z_increment;

    const double half = ceil(0.5 * g->beam_width_at_roi_edge / g->voxel_size_z);
    double allowed_start = g->z_first_view + direction * half * g->voxel_size_z;
    double allowed_end = table_positions[g->Readings - 1] - direction * half * g->voxel_size_z;
    if (allowed_start > allowed_end) {
        const double t = allowed_start;
        allowed_start = allowed_end;
        allowed_end = t;
    }
    if (!((g->z_start > allowed_start) && (g->z_start < allowed_end) && (g->z_end > allowed_start) &&
          (g->z_end < allowed_end)))
        return fail(CTBB_ERR_RANGE, "Requested reconstruction range (%g : %g) is invalid; allowed range is %g : %g",
                    g->z_start, g->z_end, allowed_start, allowed_end);

    g->num_voxels_z = (uint64_t)(fabs(g->z_end - g->z_start) / g->voxel_size_z);
    g->nz = g->num_voxels_z;
    if (!slice_locations || !slice_indices) return CTBB_OK;
    if (g->num_voxels_z > max_slices)
        return fail(CTBB_ERR_INVALID_ARG, "slice table capacity %llu < %llu slices",
                    (unsigned long long)max_slices, (unsigned long long)g->num_voxels_z);
    const int recon_direction = (int)((g->z_end - g->z_start) / fabs(g->z_end - g->z_start));
    const uint64_t nffs = (uint64_t)n_ffs(*g);
    for (int i = 0; i < (int)g->num_voxels_z; i++) {
        slice_locations[i] = g->z_start + i * g->voxel_size_z * recon_direction;
        uint64_t c = 0;
        const double loc = slice_locations[i];
        if (g->table_direction > 0) {
            while (c < g->Readings && table_positions[c] < loc) c += nffs;
        } else {
            while (c < g->Readings && table_positions[c] > loc) c += nffs;
        }
        if (c >= g->Readings) return fail(CTBB_ERR_RANGE, "slice %d lies beyond the last view", i);
        slice_indices[i] = c;
    }
    return CTBB_OK;
}

// setup.cpp:271-299 and :334-344. FileType 0 frames are channel-major with the
// row fastest; the reference's two transposes cancel, so frame v lands at
// raw[v][channel][row] unchanged.
extern "C" ctbb_status ctbb_read_raw(const char* path, const ctbb_geom_c* g, float* raw) {
    clear_error();
    if (!path || !g || !raw) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (g->FileType != 0) return fail(CTBB_ERR_UNSUPPORTED, "only FileType 0 raw files can be read");
    FILE* f = fopen(path, "rb");
    if (!f) return fail(CTBB_ERR_IO, "Raw data file not found: %s", path);
    const size_t frame = g->n_channels * g->Nrows_projection;
    for (uint64_t v = 0; v < g->Readings; ++v) {
        const long long pos = (long long)g->RawOffset + (long long)v * (long long)(frame * sizeof(float));
        if (fseeko(f, (off_t)pos, SEEK_SET) != 0 || fread(raw + v * frame, sizeof(float), frame, f) != frame) {
            fclose(f);
            return fail(CTBB_ERR_IO, "short read of frame %llu in %s", (unsigned long long)v, path);
        }
    }
    fclose(f);
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_write_raw_file(const char* path, const ctbb_geom_c* g, const float* raw) {
    clear_error();
    if (!path || !g || !raw) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    FILE* f = fopen(path, "wb");
    if (!f) return fail(CTBB_ERR_IO, "cannot create %s", path);
    const size_t n = g->Readings * g->n_channels * g->Nrows_projection;
    const size_t w = fwrite(raw, sizeof(float), n, f);
    if (fclose(f) != 0 || w != n) return fail(CTBB_ERR_IO, "short write to %s", path);
    return CTBB_OK;
}

extern "C" ctbb_status ctbb_synth_raw_host(const ctbb_geom_c* g, const ctbb_phantom_spec* spec,
                                           float* raw, int n_threads) {
    clear_error();
    if (!g || !spec || !raw) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    std::vector<ctbb_object> objs;
    ctbb_water_phantom(objs);
    if (spec->n_ellipsoids > 0)
        ctbb_random_ellipsoids(objs, spec->n_ellipsoids, spec->seed, spec->ellipsoid_z_lo, spec->ellipsoid_z_hi);
    const ctbb_ray_geom G = ctbb_ray_geom_from(*g);
    const int64_t nch = G.n_channels, nr = G.n_rows, nv = G.readings;
    if (n_threads <= 0) n_threads = 1;
#pragma omp parallel for schedule(dynamic, 4) num_threads(n_threads)
    for (int64_t v = 0; v < nv; ++v) {
        const double i0 = ctbb_view_i0(spec->seed, v, spec->i0_lo, spec->i0_hi);
        for (int64_t c = 0; c < nch; ++c)
            for (int64_t r = 0; r < nr; ++r) {
                const uint64_t ray = (uint64_t)((v * nch + c) * nr + r);
                const double p = ctbb_line_integral(G, objs.data(), (int)objs.size(), v, c, r, spec->clip_z_lo, spec->clip_z_hi);
                raw[ray] = ctbb_noisy_sample(p, i0, spec->seed, ray);
            }
    }
    return CTBB_OK;
}
