/*
 * ctbb_icd_b200 — C ABI of the B200 reconstruction path for CTBB_ICD.
 *
 * The reference program (CTBB_ICD) runs one host-thread pipeline of C++ free
 * functions  void stage(const recon_params*, ct_data*)  in this order
 * (src/main.cpp:88-128):
 *
 *   configure_recon_params -> load_raw -> initialize_recon_volume
 *     -> generate_system_matrix[_ffs] -> icd_iteration
 *     -> rotate_slices_rotating2fixed -> clean_up
 *
 * This header is the drop-in boundary for the numerical stages of that flow.
 * Every entry point is extern "C", takes plain pointers and sizes, returns a
 * ctbb_status (never exits), and names the reference function it replaces.
 * recon_params is not POD (std::string members, src/recon_structs.h:27-33),
 * so its numeric fields cross the boundary as ctbb_geom_c, in the same order,
 * with the same names and units (cm, radians; tube angles in degrees).
 *
 * Threading: one host thread per context. Device memory is owned by the
 * context / ssm / recon objects; host buffers are only borrowed for the call.
 */
#ifndef CTBB_ICD_B200_H
#define CTBB_ICD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------- */
/* Status codes                                                              */
/* ------------------------------------------------------------------------- */
typedef int32_t ctbb_status;
enum {
    CTBB_OK = 0,
    CTBB_ERR_INVALID_ARG = 1, /* null pointer, bad size, inconsistent geometry   */
    CTBB_ERR_CONFIG = 2,      /* missing/invalid parameter-file field            */
    CTBB_ERR_IO = 3,          /* file missing, short read, write failure         */
    CTBB_ERR_RANGE = 4,       /* requested z-range outside the scanned data      */
    CTBB_ERR_CUDA = 5,        /* CUDA runtime error (message in ctbb_last_error) */
    CTBB_ERR_NO_DEVICE = 6,   /* no CUDA device / library built without CUDA     */
    CTBB_ERR_OOM = 7,         /* device or host allocation failed                */
    CTBB_ERR_TIMEOUT = 8,     /* a bounded device wait gave up                   */
    CTBB_ERR_UNSUPPORTED = 9, /* feature not available (e.g. PTR/IMA readers)    */
    CTBB_ERR_FORMAT = 10      /* corrupt or mismatched matrix file               */
};

/* Penalty selector (recon_params.penalty string, src/setup.cpp:169-174). */
enum { CTBB_PENALTY_QUADRATIC = 0, CTBB_PENALTY_EDGE_PRESERVING = 1 };

/*
 * Numeric fields of recon_params (src/recon_structs.h:25-114), same order,
 * names and units. size_t fields are uint64_t; the `penalty` string becomes
 * an enum at the position the string occupied.
 */
typedef struct ctbb_geom_c {
    /* Scanner geometry */
    double acquisition_fov;
    double anode_angle;
    double axial_detector_spacing;
    double axial_focal_spot_shift;
    double center_channel_non_ffs;
    double center_row;
    double focal_spot_radius;
    uint64_t n_channels;
    uint64_t num_views_per_turn;
    uint64_t num_views_per_turn_without_ffs;
    double source_detector_distance;
    double transaxial_detector_spacing;
    double transaxial_focal_spot_shift;
    double fan_angle_increment;
    /* Iterative recon parameters */
    int32_t penalty; /* CTBB_PENALTY_* */
    int32_t reserved0;
    double lambda;
    double delta;
    uint64_t num_iterations;
    /* Scan specific parameters */
    uint64_t Nrows;
    double first_view_angle;
    uint64_t num_z_ffs;
    uint64_t num_phi_ffs;
    uint64_t num_views;
    double table_feed_per_rotation;
    double tube_angle_increment;
    double z_end;
    double z_first_view;
    double z_good_slice;
    double z_matrix_start;
    double z_start;
    int32_t table_direction;
    int32_t reserved1;
    /* Recon geometry */
    double fov_radius;
    double center_voxel_x;
    double center_voxel_y;
    double center_voxel_z;
    double dx;
    double dy;
    double dz;
    uint64_t nx;
    uint64_t ny;
    uint64_t nz;
    /* Raw-file and scan mode fields */
    uint64_t FileType;
    uint64_t FileSubType;
    uint64_t RawOffset;
    uint64_t Readings;
    uint64_t Zffs;
    uint64_t Phiffs;
    double CollSlicewidth;
    uint64_t wfbp_initialize;
    /* Derived values */
    uint64_t Nrows_projection;
    uint64_t views_per_slice;
    double voxel_size_x;
    double voxel_size_y;
    double voxel_size_z;
    double tube_z_increment;
    double beam_width;
    double beam_width_at_roi_edge;
    uint64_t num_views_for_system_matrix;
    uint64_t num_voxels_x;
    uint64_t num_voxels_y;
    uint64_t num_voxels_z;
    double slice_thickness;
    double recon_fov;
} ctbb_geom_c;

/* ------------------------------------------------------------------------- */
/* Host-side setup (no GPU needed)                                           */
/* ------------------------------------------------------------------------- */

/* Last error message of the calling thread (empty string if none). */
const char* ctbb_last_error(void);
const char* ctbb_status_str(ctbb_status s);

/*
 * Parse a parameter file, apply the reference's required-field checks and
 * defaults, and compute the derived values.
 * Replaces configure_recon_params (src/setup.cpp:69-243) and parse_config
 * (src/parse_config.cpp:34-111). String fields are returned through the
 * optional buffers (NULL to skip, each `cap` bytes).
 */
typedef struct ctbb_prm_strings {
    char initial_recon_path[1024];
    char matrix_path[1024];
    char output_dir[1024];
    char output_file[1024];
    char potential[64];
    char recon_path[1024];
    char sinogram_path[1024];
    char penalty[64];
} ctbb_prm_strings;

ctbb_status ctbb_configure_recon_params(const char* prm_path, ctbb_geom_c* geom,
                                        ctbb_prm_strings* strings);

/*
 * Tube angles, table positions and the rotating-slice tables, plus the final
 * table_direction / z_first_view / num_voxels_z, for FileType 0 data.
 * Replaces the geometry part of load_raw (src/setup.cpp:273-285, 348-409).
 * tube_angles / table_positions hold Readings values; slice_locations /
 * slice_indices hold up to max_slices values (the count is geom->num_voxels_z
 * on return). Returns CTBB_ERR_RANGE for the reference's invalid-range exit.
 */
ctbb_status ctbb_slice_tables(ctbb_geom_c* geom, double* tube_angles, double* table_positions,
                              double* slice_locations, uint64_t* slice_indices,
                              uint64_t max_slices);

/*
 * Read FileType 0 frames into raw[Readings][n_channels][Nrows_projection]
 * (row fastest). Replaces the ReadBinaryFrame loop and the two transposes of
 * load_raw (src/setup.cpp:271-299, 334-344).
 */
ctbb_status ctbb_read_raw(const char* path, const ctbb_geom_c* geom, float* raw);

/* ------------------------------------------------------------------------- */
/* Synthetic data (stands in for the private ctbb_read library)              */
/* ------------------------------------------------------------------------- */
typedef struct ctbb_phantom_spec {
    int32_t n_ellipsoids;  /* random ellipsoids added to the water phantom   */
    int32_t reserved;
    uint64_t seed;         /* phantom and noise seed                        */
    double ellipsoid_z_lo; /* z range (cm, fixed frame) of ellipsoid centres */
    double ellipsoid_z_hi;
    double i0_lo;          /* incident photons per ray; <= 0 -> noise free  */
    double i0_hi;          /* > i0_lo -> drawn per view in [i0_lo, i0_hi]   */
    double clip_z_lo;      /* clip_z_hi > clip_z_lo: every object is cut to  */
    double clip_z_hi;      /* this z range (cm), a phantom of finite length  */
} ctbb_phantom_spec;

/* CPU projector: writes raw[Readings][n_channels][Nrows_projection]. */
ctbb_status ctbb_synth_raw_host(const ctbb_geom_c* geom, const ctbb_phantom_spec* spec,
                                float* raw, int n_threads);
/* Write raw as a FileType 0 file (frames channel-major, row fastest). */
ctbb_status ctbb_write_raw_file(const char* path, const ctbb_geom_c* geom, const float* raw);

/* ------------------------------------------------------------------------- */
/* GPU context                                                               */
/* ------------------------------------------------------------------------- */
typedef struct ctbb_ctx ctbb_ctx;
typedef struct ctbb_ssm ctbb_ssm;
typedef struct ctbb_recon ctbb_recon;

/* stream: a cudaStream_t to run on, or NULL for a context-owned stream. */
ctbb_status ctbb_gpu_init(int device, void* stream, ctbb_ctx** out);
void ctbb_gpu_destroy(ctbb_ctx* ctx);
/* The cudaStream_t all work of this context is issued on. */
void* ctbb_gpu_stream(ctbb_ctx* ctx);
ctbb_status ctbb_gpu_synchronize(ctbb_ctx* ctx);

/* GPU projector writing a device buffer raw_dev of Readings*n_ch*n_rows floats. */
ctbb_status ctbb_gpu_synth_raw(ctbb_ctx* ctx, const ctbb_geom_c* geom,
                               const ctbb_phantom_spec* spec, float* raw_dev);

/* ------------------------------------------------------------------------- */
/* Stored system matrix                                                      */
/* ------------------------------------------------------------------------- */
enum { CTBB_SSM_FP32 = 1, CTBB_SSM_FP16 = 2, CTBB_SSM_BOTH = 3 };

typedef struct ctbb_ssm_info {
    uint64_t n_columns;     /* num_voxels_x * num_voxels_y                 */
    uint64_t n_views;       /* num_views_for_system_matrix                 */
    uint64_t nnz;           /* stored entries                              */
    uint64_t max_col_nnz;   /* largest column                              */
    uint64_t bytes_device;  /* device bytes held by the matrix             */
    int32_t weights;        /* CTBB_SSM_* held                             */
    int32_t ffs;            /* 1 if built with a flying focal spot (in-plane and/or z) */
    double build_ms;        /* device time of the last build               */
    uint64_t n_pairs;       /* entry pairs (0 until a grouped iteration with
                               entry_pairs has built them)                 */
} ctbb_ssm_info;

/*
 * Build the stored system matrix on the device: per voxel column (i + nx*j),
 * entries (q, w) with q = row + Nrows*(channel + n_channels*view), sorted by q.
 * Chooses the flying-focal-spot model from geom->Phiffs / geom->Zffs like
 * main.cpp:103-109: in-plane (Phi), z (Z) or both, with the source offsets of
 * generate_ffs_offset (generate_system_matrix_ffs.cpp:242-290) as the
 * reference evaluates them (including its z deflection dr * tan(anode_angle)
 * with the angle in degrees passed to tan).
 * Replaces generate_system_matrix (src/generate_system_matrix.cpp:54-209) and
 * generate_system_matrix_ffs (src/generate_system_matrix_ffs.cpp:60-239);
 * the on-disk matrix.bin round trip (:212-303) becomes an HBM-resident matrix.
 * As in the reference's flow (load_raw before generate_system_matrix,
 * main.cpp:92, 101-109), geom must have passed ctbb_slice_tables: it sets
 * table_direction, whose sign moves the source along z from view to view
 * (generate_system_matrix.cpp:100). With table_direction 0, as
 * ctbb_configure_recon_params leaves it, the source stays at z = 0 and the
 * matrix models a circular scan.
 */
ctbb_status ctbb_gpu_generate_ssm(ctbb_ctx* ctx, const ctbb_geom_c* geom, int32_t weights,
                                  ctbb_ssm** out);
ctbb_status ctbb_gpu_ssm_info(const ctbb_ssm* ssm, ctbb_ssm_info* info);
/* Copy one column to host: nnz returned; idx/w may be NULL to query size. */
ctbb_status ctbb_gpu_ssm_column(const ctbb_ssm* ssm, uint64_t column, int32_t* idx, float* w,
                                uint64_t cap, uint64_t* nnz);
/*
 * Write / read the reference's matrix.bin layout: per column, a size_t count
 * then count x {int32 index, float32 value} (src/generate_system_matrix.cpp:212-303,
 * read back at src/icd_iteration.cpp:164-179).
 */
ctbb_status ctbb_gpu_ssm_export_reference(const ctbb_ssm* ssm, const char* path);
ctbb_status ctbb_gpu_ssm_import_reference(ctbb_ctx* ctx, const ctbb_geom_c* geom,
                                          const char* path, int32_t weights, ctbb_ssm** out);
void ctbb_gpu_ssm_free(ctbb_ssm* ssm);

/* ------------------------------------------------------------------------- */
/* ICD reconstruction                                                        */
/* ------------------------------------------------------------------------- */
enum {
    CTBB_ICD_SEQUENTIAL = 0, /* reference visiting order, FP64 state (parity mode) */
    CTBB_ICD_GROUPED = 1     /* many voxels in flight, FP32 error sinogram         */
};

typedef struct ctbb_icd_opts {
    int32_t mode;             /* CTBB_ICD_*                                       */
    int32_t weights;          /* grouped mode: CTBB_SSM_FP32 or CTBB_SSM_FP16     */
    int32_t refresh_every;    /* grouped: FP64 y - Ax refresh every K iterations (0: never) */
    int32_t warps_in_flight;  /* grouped: warps kept busy (0: coupling-bound default);
                                 capped at one cell rank of the visiting order      */
    int32_t lattice;          /* grouped: tile edge of the visiting order (0: derived from
                                 the warps in flight)                              */
    int32_t compute_cost;     /* evaluate the exact FP64 cost after each iteration
                                 (grouped mode: FP64 A x recomputed, e refreshed) */
    double stop_rel_change;   /* stop when |dcost|/cost < this, exact FP64 costs
                                 of consecutive iterations (0: fixed count)        */
    double relax;             /* grouped: step scale omega in (0, 2) (0: 1.0)     */
    int32_t priority;         /* grouped: visit only the priority subset built by
                                 ctbb_gpu_recon_set_priority (0: every voxel)     */
    int32_t warps_per_voxel;  /* grouped: 1 (0), 4 or 8 warps per voxel update; with
                                 4 or 8 the update's matrix entries stay in registers
                                 between gather and scatter                       */
    int32_t entries_per_lane; /* grouped, one warp per voxel: matrix entries each lane
                                 keeps in flight per round trip, 8 (0) or 16      */
    int32_t stage_column;     /* grouped, one warp per voxel: 0 reads the column's
                                 matrix entries from HBM for the gather and again
                                 for the scatter; 1 keeps them in a shared-memory
                                 stage between the two (4 updates per CTA), 2 the
                                 same with 8 updates per CTA and half the stage;
                                 3 runs each slice stack (up to 16 same-parity
                                 slices at one physical cell) as one CTA whose
                                 warps sweep the stack's data views in lockstep,
                                 so the sinogram sectors they share are fetched
                                 from HBM once; 4 and 5 (FP16 weights, entry
                                 pairs) run one update per CTA of 8 warps whose
                                 entry pairs the TMA engine copies into shared
                                 memory (one bulk copy per update, read by both
                                 gather and scatter), with one stage (4) or two
                                 (5: the next update's copy overlaps the current
                                 update); 6 is the one-stage form with the next
                                 item claimed (work queue, visiting order,
                                 column offsets) during the current update's
                                 penalty solve (a CTA holds two claimed items,
                                 so half the order's bound in flight);
                                 warps_in_flight counts 8 per update              */
    int32_t entry_pairs;      /* grouped, FP16 weights, one warp per voxel (streamed,
                                 stage_column 0; entries_per_lane then counts pairs)
                                 or 4 or 8 warps per voxel: 0
                                 reads the matrix as entry pairs ({sinogram index,
                                 two FP16 weights} for the two detector rows of a
                                 (view, channel): 4 bytes per entry, built once per
                                 matrix on first use and kept where pairs hold
                                 4/3 entries or more on average); -1 reads single
                                 entries (4-byte index + 2-byte weight)           */
    int32_t stack_align;      /* grouped, 4 or 8 warps per voxel: 1 starts each
                                 update's sweep of its view window at the data view
                                 where its slice stack's last member's window
                                 begins, wrapping around to the window start, so
                                 the stack's members (consecutive in the visiting
                                 order) read and update the sinogram sectors they
                                 share at about the same time; 0 sweeps each window
                                 from its start                                   */
    int32_t l2_hints;         /* grouped, 4 or 8 warps per voxel: 1 marks the matrix
                                 loads (read once per update) evict-first and the
                                 e gathers evict-last in L2; with stage_column 4/5
                                 1 marks the column's bulk copy evict-first; 0
                                 leaves them normal                               */
} ctbb_icd_opts;

/*
 * The grouped mode's penalised one-voxel update on caller-given inputs, for
 * verification: for each of n voxels, the surrogate numerator beta[i] and
 * denominator alpha[i] of icd_iteration.cpp:198-209, the voxel value
 * x9[9 i] and its 8 in-plane neighbours x9[9 i + 1 + l] in the order
 * {-nx-1, -nx, -nx+1, -1, +1, nx-1, nx, nx+1} of penalties.cpp:41-52 (NaN
 * marks a neighbour outside the volume), returns in step[i] the update
 * before the positivity clamp: the closed form of quadratic()
 * (penalties.cpp:61-85), or the root of edge_preserving()'s surrogate
 * equation (penalties.cpp:88-154), found by safeguarded Newton inside the
 * reference's bisection bracket. Host buffers; the call synchronises.
 */
ctbb_status ctbb_gpu_penalty_steps(ctbb_ctx* ctx, int32_t penalty, double lambda, double delta, uint64_t n,
                                   const double* alpha, const double* beta, const float* x9, double* step);

typedef struct ctbb_iter_stats {
    int32_t iterations;       /* iterations run by the call                       */
    int32_t reserved;
    double cost;              /* FP64 cost after the last iteration (if computed) */
    double rel_change;        /* |dcost|/cost of the last iteration               */
    double device_ms;         /* device time of the ICD kernels in the call       */
    double voxel_updates;     /* voxel updates performed                          */
    double entries;           /* SSM entries visited (sum of in-range nnz)        */
    double entries_scattered; /* grouped: entries of the updates that changed their
                                 voxel and so scattered into e (du != 0)          */
} ctbb_iter_stats;

/*
 * Device-resident reconstruction state for one volume: raw data y, the
 * current iterate x ([nz][ny][nx], rotating frame) and the error sinogram
 * e = y - Ax. slice_indices holds nz central view indices (load_raw).
 */
ctbb_status ctbb_gpu_recon_create(ctbb_ctx* ctx, const ctbb_geom_c* geom,
                                  const uint64_t* slice_indices, ctbb_recon** out);
void ctbb_gpu_recon_free(ctbb_recon* rc);
ctbb_status ctbb_gpu_recon_set_raw(ctbb_recon* rc, const float* raw_host);
ctbb_status ctbb_gpu_recon_set_raw_device(ctbb_recon* rc, const float* raw_dev);
/* Copy the recon's raw data y back to the host. */
ctbb_status ctbb_gpu_recon_get_raw(ctbb_recon* rc, float* raw_host);
/* Device pointer of the recon's raw buffer (for the GPU projector). */
float* ctbb_gpu_recon_raw_device(ctbb_recon* rc);
/* Initial image (host, float [nz][ny][nx]); NULL -> zeros. Resets e = y - Ax. */
ctbb_status ctbb_gpu_recon_set_volume(ctbb_recon* rc, const ctbb_ssm* ssm, const float* vol_host);
/* Same, choosing the starting sinogram estimate: CTBB_ESTIMATE_FORWARD
 * y_hat = A x0 (what ctbb_gpu_recon_set_volume does), or CTBB_ESTIMATE_ZERO
 * y_hat = 0 whatever x0 is, which is what the reference's icd_iteration does
 * for every start but a wFBP one (icd_iteration.cpp:47, 63): with an image
 * from initial_recon_path its first iteration measures the data against a
 * zero projection. ctbb_gpu_icd uses ZERO in sequential (parity) mode unless
 * geom->wfbp_initialize is set, and FORWARD in grouped mode. */
enum { CTBB_ESTIMATE_ZERO = 0, CTBB_ESTIMATE_FORWARD = 1 };
/* Multi-resolution start (no reference counterpart): the current image of
 * `coarse` (same scan, slices and field of view, half the in-plane voxel
 * count) upsampled 2x in-plane by bilinear interpolation becomes the image of
 * `fine`, and e = y - A x is recomputed in FP64, device to device. */
ctbb_status ctbb_gpu_recon_set_volume_upsampled(ctbb_recon* fine, const ctbb_ssm* fine_ssm, ctbb_recon* coarse);
ctbb_status ctbb_gpu_recon_set_volume_estimate(ctbb_recon* rc, const ctbb_ssm* ssm, const float* vol_host,
                                               int32_t estimate);
ctbb_status ctbb_gpu_recon_get_volume(ctbb_recon* rc, float* vol_host);
ctbb_status ctbb_gpu_recon_get_volume_f64(ctbb_recon* rc, double* vol_host);
/* Run n_iter ICD iterations. */
ctbb_status ctbb_gpu_recon_iterate(ctbb_recon* rc, const ctbb_ssm* ssm, const ctbb_icd_opts* opts,
                                   int32_t n_iter, ctbb_iter_stats* stats);
/* Sum over voxels inside the scanner FOV of the matrix entries whose sinogram
 * index lies inside the scan (the entries one ICD iteration visits). */
ctbb_status ctbb_gpu_recon_entries(ctbb_recon* rc, const ctbb_ssm* ssm, double* entries);
/* Recompute e = y - Ax with FP64 accumulation. */
ctbb_status ctbb_gpu_recon_refresh_residual(ctbb_recon* rc, const ctbb_ssm* ssm);
/* FP64 cost of the current iterate (quadratic: 1/2|e|^2 + lambda/4 sum w dx^2;
 * edge-preserving: |e|^2 + lambda/2 sum w rho(dx)). */
ctbb_status ctbb_gpu_recon_cost(ctbb_recon* rc, double* cost);

/*
 * Several independent reconstructions advanced together (no reference
 * counterpart: the reference reconstructs one scan per process). Each
 * iteration is one persistent launch that drains the merged work queue of
 * all scans, each scan's items spread in proportion to its size, replayed
 * from a CUDA graph captured on the context's stream. Up to 64 scans of one
 * context, each with its own matrix; opts->weights must be held by every
 * matrix. The scans keep their own state (ctbb_gpu_recon_* still apply).
 */
typedef struct ctbb_batch ctbb_batch;
ctbb_status ctbb_gpu_batch_create(ctbb_ctx* ctx, int32_t n, ctbb_recon* const* recons,
                                  const ctbb_ssm* const* ssms, ctbb_batch** out);
ctbb_status ctbb_gpu_batch_iterate(ctbb_batch* batch, const ctbb_icd_opts* opts, int32_t n_iter,
                                   ctbb_iter_stats* stats);
void ctbb_gpu_batch_free(ctbb_batch* batch);

/*
 * One-call drop-in for icd_iteration (src/icd_iteration.cpp:42-286): copies
 * raw and recon_volume (initial image) from the host, runs
 * geom->num_iterations iterations and writes the result back to recon_volume.
 */
ctbb_status ctbb_gpu_icd(ctbb_ctx* ctx, const ctbb_ssm* ssm, const ctbb_geom_c* geom,
                         const uint64_t* slice_indices, const float* raw, float* recon_volume,
                         const ctbb_icd_opts* opts, ctbb_iter_stats* stats);

/* ------------------------------------------------------------------------- */
/* Slice rotation                                                            */
/* ------------------------------------------------------------------------- */
enum { CTBB_ROTATE_FIXED2ROTATING = 1, CTBB_ROTATE_ROTATING2FIXED = -1 };

/*
 * Rotate every slice k by the tube angle of its central view with bilinear
 * interpolation and a zero border, host volume in place.
 * Replaces rotate_slices_rotating2fixed (src/rotate_slices.cpp:81-114),
 * rotate_slices_fixed2rotating (:48-79), rotate_slice (:116-154) and
 * interp2 (src/interp.h:41-76).
 */
ctbb_status ctbb_gpu_rotate(ctbb_ctx* ctx, const ctbb_geom_c* geom, const double* tube_angles_deg,
                            const uint64_t* slice_indices, float* vol_host, int32_t direction);
/* Same on device buffers (in and out must not alias). */
ctbb_status ctbb_gpu_rotate_device(ctbb_ctx* ctx, const ctbb_geom_c* geom,
                                   const double* tube_angles_deg, const uint64_t* slice_indices,
                                   const float* in_dev, float* out_dev, int32_t direction);

/*
 * ctbb_gpu_rotate_device without any device allocation. It has no
 * counterpart in the reference (whose rotation runs on the host).
 *
 * For callers that must not have a library call cudaMalloc/cudaFree: code
 * that carves all device memory out of its own pool at start-up, latency-
 * bound loops that cannot afford the allocator's implicit synchronisation,
 * or hosts that cap the process's device footprint. The only scratch the
 * rotation needs, the per-slice cos/sin table, is kept in a fixed device
 * array of 2 x 8192 doubles (128 KB), resident on each GPU from the
 * library's first use there until the process exits; volumes of more than 8192 slices are
 * rejected with CTBB_ERR_INVALID_ARG. Input and output stay caller-owned
 * device buffers and give the same result as ctbb_gpu_rotate_device.
 *
 * The first call on each device looks up the array's device address, so
 * make that first call before any stream capture starts. Every call
 * synchronises ctx's stream before it returns. The looked-up address is kept
 * for the life of the process: a cudaDeviceReset by the caller invalidates
 * it, and calls after such a reset are not supported. All calls share the
 * one array: calls whose work overlaps on the GPU (other host threads or
 * streams of the same device) race on it. Each call rewrites the entries it
 * uses, so nothing left by an earlier call leaks into a later one.
 */
ctbb_status ctbb_gpu_rotate_device_noalloc(ctbb_ctx* ctx, const ctbb_geom_c* geom,
                                           const double* tube_angles_deg,
                                           const uint64_t* slice_indices, const float* in_dev,
                                           float* out_dev, int32_t direction);

/*
 * Autotuner for grouped ICD (no reference counterpart). From the current
 * iterate, runs probe_iters iterations for each candidate (warps per voxel,
 * warps in flight, entries per lane, tile edge of the visiting order, column
 * schedule) and keeps the one with the
 * largest decrease of the FP64 cost per millisecond of device time. The
 * iterate and e are restored afterwards; *best = *base with those fields
 * set. Candidates: the lockstep stack kernel (stage_column 3) with 8
 * entries per lane; the shared-memory staged kernel (stage_column 1, 2);
 * one warp per voxel at 1/4, 1/2, 1 and 2 times the
 * coupling-bound default of warps in flight, with 8 or 16 entries per lane
 * in flight and the default tile edge for that concurrency (half of it too
 * at the default); 4 warps per voxel with four or eight updates per SM and
 * 8 warps per voxel with four (these read entry pairs with FP16 weights);
 * with FP16 weights, the bulk-staged kernels (stage_column 4, 5 and 6),
 * unless the matrix keeps no entry pairs (z flying focal spot).
 * Every launch keeps at most one cell rank of the visiting order (about
 * n / T^2 updates for tile edge T) in flight, so no two in-plane neighbours
 * of a slice are ever updated together; trials report the effective warps
 * in flight.
 */
#define CTBB_TUNE_MAX_TRIALS 32
typedef struct ctbb_tune_trial {
    int32_t warps_in_flight;
    int32_t warps_per_voxel;
    int32_t lattice;
    int32_t entries_per_lane;
    int32_t stage_column;
    int32_t entry_pairs;
    double device_ms;   /* ICD kernel time of the probe iterations */
    double cost;        /* FP64 cost after them                    */
    double score;       /* (start_cost - cost) / device_ms         */
} ctbb_tune_trial;
typedef struct ctbb_tune_report {
    int32_t n_trials;
    int32_t best;       /* index into trials */
    double start_cost;
    ctbb_tune_trial trials[CTBB_TUNE_MAX_TRIALS];
} ctbb_tune_report;
ctbb_status ctbb_gpu_recon_autotune(ctbb_recon* rc, const ctbb_ssm* ssm, const ctbb_icd_opts* base,
                                    int32_t probe_iters, ctbb_icd_opts* best, ctbb_tune_report* report);

/*
 * Learned warm start (no reference counterpart). A 3D residual CNN with 32
 * channels, `blocks` residual blocks and 3x3x3 kernels predicts, from an
 * early ICD iterate in the fixed frame, the correction to the converged
 * image. Training and inference run on the GPU (BF16 tensor-core
 * convolutions with FP32 accumulation, Adam on FP32 master weights).
 *
 * Parameter layout (flat FP32): W_in[27][32], b_in[32]; per block
 * W1[27][32][32] (tap, in, out), b1[32], W2[27][32][32], b2[32];
 * W_out[27][32], b_out[1]. Tap t = (dz+1)*9 + (dy+1)*3 + (dx+1).
 * Scaling: the network sees s_in * x and is trained on (x_conv - x) * s_out.
 * Volumes are device float arrays [nz][ny][nx] on the context's device.
 */
typedef struct ctbb_cnn ctbb_cnn;
ctbb_status ctbb_cnn_create(ctbb_ctx* ctx, int32_t blocks, uint64_t seed, ctbb_cnn** out);
void ctbb_cnn_free(ctbb_cnn* cnn);
/* Tensor-core path of the 32 -> 32 convolutions (forward and backward-data):
 * TCGEN05 = tcgen05.mma with a TMEM accumulator and TMA-staged operands;
 * MMA_SYNC (default) = the warp-level mma.sync kernel.
 * A tcgen05 wait that runs out makes the call return CTBB_ERR_TIMEOUT. */
enum { CTBB_CNN_ENGINE_MMA_SYNC = 0, CTBB_CNN_ENGINE_TCGEN05 = 1 };
ctbb_status ctbb_cnn_set_engine(ctbb_cnn* cnn, int32_t engine);
uint64_t ctbb_cnn_num_params(const ctbb_cnn* cnn);
ctbb_status ctbb_cnn_get_params(ctbb_cnn* cnn, float* params_host, uint64_t n);
ctbb_status ctbb_cnn_set_params(ctbb_cnn* cnn, const float* params_host, uint64_t n);
ctbb_status ctbb_cnn_set_scaling(ctbb_cnn* cnn, float s_in, float s_out);
ctbb_status ctbb_cnn_get_scaling(const ctbb_cnn* cnn, float* s_in, float* s_out);
/* Network output (predicted (x_conv - x) * s_out) for x_dev. */
ctbb_status ctbb_cnn_forward(ctbb_cnn* cnn, const float* x_dev, int32_t nx, int32_t ny, int32_t nz,
                             float* out_dev);
/* Adds d loss / d params to the gradient buffer, where loss =
 * sum w (out - (xc - x) s_out)^2 / sum w (weight_dev NULL: w = 1). */
ctbb_status ctbb_cnn_accumulate_gradient(ctbb_cnn* cnn, const float* x_dev, const float* xc_dev,
                                         const float* weight_dev, int32_t nx, int32_t ny, int32_t nz,
                                         double* loss);
ctbb_status ctbb_cnn_get_gradient(ctbb_cnn* cnn, float* grad_host, uint64_t n);
ctbb_status ctbb_cnn_zero_gradient(ctbb_cnn* cnn);
/* One Adam step on grad * grad_scale; clears the gradient buffer. */
ctbb_status ctbb_cnn_adam_step(ctbb_cnn* cnn, float lr, float beta1, float beta2, float eps, float grad_scale);

/* Apply the network to the current iterate: rotate to the fixed frame
 * (rotate_slices_rotating2fixed, rotate_slices.cpp:81-114), predict the
 * correction, rotate it back (rotate_slices_fixed2rotating, :48-79), add it
 * with the positivity clamp, recompute e = y - Ax in FP64, and keep
 * |step| per voxel as the priority map. tube_angles_deg: ct_data.tube_angles. */
ctbb_status ctbb_gpu_recon_warm_start(ctbb_recon* rc, const ctbb_ssm* ssm, ctbb_cnn* cnn,
                                      const double* tube_angles_deg);
/* Restrict priority passes (opts->priority = 1) to the `fraction` of voxels
 * with the largest warm-start step, kept in the visiting order of opts. */
ctbb_status ctbb_gpu_recon_set_priority(ctbb_recon* rc, const ctbb_icd_opts* opts, double fraction);

#ifdef __cplusplus
}
#endif

#endif /* CTBB_ICD_B200_H */
