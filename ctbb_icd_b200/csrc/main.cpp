// ctbb_icd — command-line drop-in for the reference program (src/main.cpp):
// same usage and stage order (configure_recon_params → load_raw →
// initialize_recon_volume → generate_system_matrix[_ffs] unless matrix_path
// exists → icd_iteration → rotate_slices_rotating2fixed → clean_up), every
// numerical stage on the B200 through the C ABI of libctbb_icd_b200.
//
// Outputs as the reference writes them: output_dir/reconstructions/
// iteration<n>.rcn (FP64 image before the first and after each iteration,
// rotating frame; skipped, like the reference, when that directory does not
// exist; the reference's raw-sized FP64 sino_estimation.rcn is not written) and
// output_dir/output_file (float32, fixed frame; reconstruction_final.img when
// output_file is empty). Errors print the library's message and exit 1, as
// the reference's checks do.
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include <chrono>
#include <string>
#include <vector>

#include "ctbb_icd_b200.h"

namespace {

struct Flags {
    bool verbose = false, timing = false, sequential = false, fp32 = false, autotune = true;
    int device = 0;
};

void usage() {
    printf("\n");
    printf("usage: ctbb_icd [options] input_prm_file\n\n");
    printf("    Options:\n");
    printf("           -v: verbose\n");
    printf("     --timing: time each stage of the reconstruction\n");
    printf("  --empty-prm: print an empty parameter file to stdout\n");
    printf(" --sequential: the reference's voxel visiting order (FP64 image, FP32 matrix)\n");
    printf("       --fp32: FP32 matrix weights in grouped mode (default FP16)\n");
    printf("--no-autotune: keep the default grouped-ICD launch settings\n");
    printf("  --device N : CUDA device (default 0)\n");
    printf("           -t: accepted for compatibility, no effect\n\n");
    exit(0);
}

// Parameter-file keys understood by ctbb_configure_recon_params, grouped as
// in recon_params (recon_structs.h). Values left empty or 0 take the
// reference's defaults or are reported missing.
void empty_parameter_file() {
    static const char* const lines[] = {
        "# Parameter file for ctbb_icd (flat YAML: key: value, no tabs).",
        "# Units: cm, radians, pixels.",
        "",
        "# Paths",
        "sinogram_path:          # raw projection file (required)",
        "output_dir:             # output directory (required); make <output_dir>/reconstructions",
        "                        # to keep the per-iteration images",
        "output_file:            # name of the final image inside output_dir (required)",
        "initial_recon_path:     # optional float32 start image (rotating frame)",
        "matrix_path:            # optional stored system matrix (matrix.bin layout) to reuse",
        "",
        "# Raw data",
        "FileType:               # 0: binary frames (PTR/IMA readers are not part of this build)",
        "FileSubType:",
        "RawOffset:",
        "Readings:               # number of projections (required)",
        "",
        "# Scanner",
        "acquisition_fov:",
        "n_channels:",
        "num_views_per_turn_without_ffs:",
        "focal_spot_radius:",
        "source_detector_distance:",
        "anode_angle:",
        "axial_detector_spacing:",
        "axial_focal_spot_shift:",
        "center_channel_non_ffs:",
        "center_row:",
        "transaxial_detector_spacing:",
        "transaxial_focal_spot_shift:",
        "fan_angle_increment:",
        "",
        "# Scan",
        "table_feed_per_rotation:",
        "Zffs:",
        "Phiffs:",
        "Nrows:",
        "CollSlicewidth:",
        "",
        "# Reconstruction",
        "recon_fov:",
        "nx:",
        "ny:",
        "slice_thickness:",
        "z_start:",
        "z_end:",
        "wfbp_initialize: 0      # 1 needs the external wFBP program (not part of this build)",
        "penalty: quadratic      # quadratic or edge-preserving",
        "lambda:",
        "delta:",
        "num_iterations:",
    };
    for (const char* l : lines) printf("%s\n", l);
    exit(0);
}

void die(ctbb_status s, const char* what) {
    if (s == CTBB_OK) return;
    const char* msg = ctbb_last_error();
    printf("%s failed (%s): %s\n", what, ctbb_status_str(s), msg && *msg ? msg : "");
    exit(1);
}

bool exists(const std::string& p) {
    struct stat st;
    return !p.empty() && stat(p.c_str(), &st) == 0;
}

bool is_dir(const std::string& p) {
    struct stat st;
    return stat(p.c_str(), &st) == 0 && S_ISDIR(st.st_mode);
}

struct Clock {
    bool on;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    void lap(const char* stage) {
        const auto t1 = std::chrono::steady_clock::now();
        if (on) printf("  %-28s %9.3f s\n", stage, std::chrono::duration<double>(t1 - t0).count());
        t0 = t1;
    }
};

bool write_file(const std::string& path, const void* p, size_t bytes) {
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) return false;
    const size_t w = fwrite(p, 1, bytes, f);
    return fclose(f) == 0 && w == bytes;
}

}  // namespace

int main(int argc, char** argv) {
    Flags fl;
    if (argc < 2) usage();
    if (argc == 2 && strcmp(argv[1], "--empty-prm") == 0) empty_parameter_file();
    for (int i = 1; i < argc - 1; ++i) {
        const std::string a = argv[i];
        if (a == "-v") fl.verbose = true;
        else if (a == "--timing") fl.timing = true;
        else if (a == "-t") {
        } else if (a == "--sequential") fl.sequential = true;
        else if (a == "--fp32") fl.fp32 = true;
        else if (a == "--no-autotune") fl.autotune = false;
        else if (a == "--device" && i + 1 < argc - 1) fl.device = atoi(argv[++i]);
        else usage();
    }
    const std::string prm = argv[argc - 1];
    Clock clk{fl.timing};

    // configure_recon_params (setup.cpp:69)
    ctbb_geom_c g;
    ctbb_prm_strings s;
    memset(&g, 0, sizeof(g));
    memset(&s, 0, sizeof(s));
    die(ctbb_configure_recon_params(prm.c_str(), &g, &s), "configure_recon_params");

    // load_raw (setup.cpp:245): tables, then FileType 0 frames
    std::vector<double> tube_angles(g.Readings), table_positions(g.Readings);
    const uint64_t cap = 1 + (uint64_t)(fabs(g.z_end - g.z_start) / g.voxel_size_z) + 2;
    std::vector<double> slice_locations(cap);
    std::vector<uint64_t> slice_indices(cap);
    die(ctbb_slice_tables(&g, tube_angles.data(), table_positions.data(), slice_locations.data(),
                          slice_indices.data(), cap),
        "load_raw");
    const uint64_t nz = g.num_voxels_z, nvox = g.num_voxels_x * g.num_voxels_y * nz;
    std::vector<float> raw(g.Readings * g.n_channels * g.Nrows_projection);
    die(ctbb_read_raw(s.sinogram_path, &g, raw.data()), "load_raw");
    if (fl.verbose)
        printf("%llu x %llu x %llu voxels, %llu views, %llu channels x %llu rows\n",
               (unsigned long long)g.num_voxels_x, (unsigned long long)g.num_voxels_y, (unsigned long long)nz,
               (unsigned long long)g.Readings, (unsigned long long)g.n_channels,
               (unsigned long long)g.Nrows_projection);
    clk.lap("load_raw");

    // initialize_recon_volume (initialize_recon_volume.cpp:51)
    std::vector<float> vol(nvox, 0.f);
    if (s.initial_recon_path[0]) {
        FILE* f = fopen(s.initial_recon_path, "rb");
        if (!f) {
            printf("Specified initial reconstruction file not found. Exiting\n");
            return 1;
        }
        const size_t got = fread(vol.data(), sizeof(float), nvox, f);
        fclose(f);
        if (got != nvox) {
            printf("Could not initialize reconstruction volume from given file. Exiting\n");
            return 1;
        }
    } else if (g.wfbp_initialize) {
        printf("wFBP initialisation needs the external wFBP program, which is not part of this build. Exiting\n");
        return 1;
    }
    clk.lap("initialize_recon_volume");

    ctbb_ctx* ctx = nullptr;
    die(ctbb_gpu_init(fl.device, nullptr, &ctx), "ctbb_gpu_init");

    // generate_system_matrix[_ffs] unless matrix_path exists (main.cpp:103-113)
    ctbb_ssm* ssm = nullptr;
    const int32_t wfmt = fl.sequential || fl.fp32 ? CTBB_SSM_FP32 : CTBB_SSM_FP16;
    if (exists(s.matrix_path)) {
        printf("Existing matrix file FOUND.\nUsing matrix file: %s\n", s.matrix_path);
        die(ctbb_gpu_ssm_import_reference(ctx, &g, s.matrix_path, CTBB_SSM_BOTH, &ssm), "matrix import");
    } else {
        printf("No existing matrix file found for reconstruction.\n");
        die(ctbb_gpu_generate_ssm(ctx, &g, wfmt == CTBB_SSM_FP16 ? CTBB_SSM_BOTH : CTBB_SSM_FP32,
                                  &ssm),
            g.Phiffs ? "generate_system_matrix_ffs" : "generate_system_matrix");
    }
    clk.lap("system matrix");

    // icd_iteration (icd_iteration.cpp:42)
    ctbb_recon* rc = nullptr;
    die(ctbb_gpu_recon_create(ctx, &g, slice_indices.data(), &rc), "icd_iteration");
    die(ctbb_gpu_recon_set_raw(rc, raw.data()), "icd_iteration");
    ctbb_icd_opts o;
    memset(&o, 0, sizeof(o));
    o.mode = fl.sequential ? CTBB_ICD_SEQUENTIAL : CTBB_ICD_GROUPED;
    // icd_iteration.cpp:47-63: the reference forward-projects the start only
    // for a wFBP image; in parity mode an initial_recon_path image starts
    // against a zero estimate as it does there.
    const int32_t est =
        (fl.sequential && !g.wfbp_initialize) ? CTBB_ESTIMATE_ZERO : CTBB_ESTIMATE_FORWARD;
    die(ctbb_gpu_recon_set_volume_estimate(rc, ssm, vol.data(), est), "icd_iteration");
    o.weights = wfmt;
    o.refresh_every = fl.sequential ? 0 : 10;
    const std::string dump_dir = std::string(s.output_dir) + "/reconstructions";
    const bool dumps = is_dir(dump_dir);
    std::vector<double> x64(dumps ? nvox : 0);
    if (dumps) {
        die(ctbb_gpu_recon_get_volume_f64(rc, x64.data()), "icd_iteration");
        write_file(dump_dir + "/iteration0.rcn", x64.data(), nvox * sizeof(double));
    }
    for (uint64_t it = 0; it < g.num_iterations; ++it) {
        if (!fl.sequential && fl.autotune && it == 1 && g.num_iterations >= 3) {
            // Tune from an early iterate; the tuner leaves it unchanged.
            ctbb_icd_opts tuned;
            die(ctbb_gpu_recon_autotune(rc, ssm, &o, 2, &tuned, nullptr), "autotune");
            tuned.refresh_every = o.refresh_every;
            o = tuned;
            if (fl.verbose)
                printf("autotune: %d warps per voxel, %d warps in flight, tile edge %d\n", o.warps_per_voxel,
                       o.warps_in_flight, o.lattice);
        }
        ctbb_iter_stats st;
        die(ctbb_gpu_recon_iterate(rc, ssm, &o, 1, &st), "icd_iteration");
        if (!fl.sequential && o.refresh_every > 0 && (it + 1) % (uint64_t)o.refresh_every == 0)
            die(ctbb_gpu_recon_refresh_residual(rc, ssm), "icd_iteration");
        if (fl.verbose) printf("iteration %llu: %.3f ms\n", (unsigned long long)(it + 1), st.device_ms);
        if (dumps) {
            die(ctbb_gpu_recon_get_volume_f64(rc, x64.data()), "icd_iteration");
            const std::string p = dump_dir + "/iteration" + std::to_string(it + 1) + ".rcn";
            if (!write_file(p, x64.data(), nvox * sizeof(double)) && fl.verbose)
                printf("could not write %s\n", p.c_str());
        }
    }
    die(ctbb_gpu_recon_get_volume(rc, vol.data()), "icd_iteration");
    ctbb_gpu_recon_free(rc);
    clk.lap("icd_iteration");

    // rotate_slices_rotating2fixed (rotate_slices.cpp:81)
    die(ctbb_gpu_rotate(ctx, &g, tube_angles.data(), slice_indices.data(), vol.data(), CTBB_ROTATE_ROTATING2FIXED),
        "rotate_slices_rotating2fixed");
    clk.lap("rotate_slices_rotating2fixed");

    // clean_up (setup.cpp:422)
    const std::string out = std::string(s.output_dir) + "/" +
                            (s.output_file[0] ? std::string(s.output_file) : std::string("reconstruction_final.img"));
    printf("Writing final reconstruction to: %s\n", out.c_str());
    if (!write_file(out, vol.data(), nvox * sizeof(float))) {
        printf("could not write %s\n", out.c_str());
        return 1;
    }
    ctbb_gpu_ssm_free(ssm);
    ctbb_gpu_destroy(ctx);
    clk.lap("clean_up");
    return 0;
}
