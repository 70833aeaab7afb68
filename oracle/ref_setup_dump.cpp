// Runs the reference's own configure_recon_params (setup.cpp:69) and load_raw
// (setup.cpp:245) on a parameter file and prints every numeric recon_params
// field and the slice tables at full precision, one `name value` per line.
// TEST INFRASTRUCTURE ONLY: linked against the unmodified reference sources by
// oracle/Makefile (target ref) into oracle/_ref/ref_setup_dump.
#include <cstdio>
#include <string>

#include "recon_structs.h"
#include "setup.h"

#define P_D(f) std::printf(#f " %.17g\n", (double)rp.f)
#define P_U(f) std::printf(#f " %llu\n", (unsigned long long)rp.f)
#define P_I(f) std::printf(#f " %d\n", (int)rp.f)

int main(int argc, char** argv) {
    if (argc != 2) {
        std::fprintf(stderr, "usage: ref_setup_dump prm.yaml\n");
        return 2;
    }
    struct recon_params rp = configure_recon_params(argv[1]);
    struct ct_data data = {};
    load_raw(&rp, &data);
    std::printf("===DUMP===\n");
    P_D(acquisition_fov); P_D(anode_angle); P_D(axial_detector_spacing); P_D(axial_focal_spot_shift);
    P_D(center_channel_non_ffs); P_D(center_row); P_D(focal_spot_radius); P_U(n_channels);
    P_U(num_views_per_turn); P_U(num_views_per_turn_without_ffs); P_D(source_detector_distance);
    P_D(transaxial_detector_spacing); P_D(transaxial_focal_spot_shift); P_D(fan_angle_increment);
    P_D(lambda); P_D(delta); P_U(num_iterations); P_U(Nrows); P_D(first_view_angle);
    P_D(table_feed_per_rotation); P_D(tube_angle_increment); P_D(z_end); P_D(z_first_view);
    P_D(z_start); P_I(table_direction); P_D(fov_radius); P_D(center_voxel_x); P_D(center_voxel_y);
    P_D(center_voxel_z); P_D(dx); P_D(dy); P_D(dz); P_U(nx); P_U(ny); P_U(FileType); P_U(Readings);
    P_U(Zffs); P_U(Phiffs); P_D(CollSlicewidth); P_U(Nrows_projection); P_U(views_per_slice);
    P_D(voxel_size_x); P_D(voxel_size_y); P_D(voxel_size_z); P_D(tube_z_increment); P_D(beam_width);
    P_D(beam_width_at_roi_edge); P_U(num_views_for_system_matrix); P_U(num_voxels_x);
    P_U(num_voxels_y); P_U(num_voxels_z); P_D(slice_thickness); P_D(recon_fov);
    std::printf("penalty %s\n", rp.penalty.c_str());
    std::printf("matrix_path %s\n", rp.matrix_path.c_str());
    for (size_t i = 0; i < rp.Readings; ++i)
        std::printf("view %zu %.17g %.17g\n", i, data.tube_angles[i], data.table_positions[i]);
    for (size_t k = 0; k < rp.num_voxels_z; ++k)
        std::printf("slice %zu %.17g %zu\n", k, data.slice_locations[k], data.slice_indices[k]);
    return 0;
}
