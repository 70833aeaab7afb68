"""ctypes bindings of the C ABI declared in include/ctbb_icd_b200.h.

The shared library libctbb_icd_b200.so is built in-tree by
ctbb_icd_b200/build.py. Loading it needs no GPU; the GPU entry points return
CTBB_ERR_NO_DEVICE when none is present. There is no CPU fallback: every
compute entry point runs the CUDA kernels or fails.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libctbb_icd_b200.so")

CTBB_OK = 0
STATUS_NAMES = {
    0: "CTBB_OK", 1: "CTBB_ERR_INVALID_ARG", 2: "CTBB_ERR_CONFIG", 3: "CTBB_ERR_IO",
    4: "CTBB_ERR_RANGE", 5: "CTBB_ERR_CUDA", 6: "CTBB_ERR_NO_DEVICE", 7: "CTBB_ERR_OOM",
    8: "CTBB_ERR_TIMEOUT", 9: "CTBB_ERR_UNSUPPORTED", 10: "CTBB_ERR_FORMAT",
}
PENALTY_QUADRATIC, PENALTY_EDGE_PRESERVING = 0, 1
SSM_FP32, SSM_FP16, SSM_BOTH = 1, 2, 3
ICD_SEQUENTIAL, ICD_GROUPED = 0, 1
ROTATE_FIXED2ROTATING, ROTATE_ROTATING2FIXED = 1, -1
ESTIMATE_ZERO, ESTIMATE_FORWARD = 0, 1
CNN_ENGINE_MMA_SYNC, CNN_ENGINE_TCGEN05 = 0, 1


class CtbbError(RuntimeError):
    """A non-zero ctbb_status, carrying the library's message."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


_D, _U, _I = C.c_double, C.c_uint64, C.c_int32

# Field list of ctbb_geom_c: the numeric fields of recon_params
# (src/recon_structs.h:25-114 of the reference), in order.
GEOM_FIELDS = [
    ("acquisition_fov", _D), ("anode_angle", _D), ("axial_detector_spacing", _D),
    ("axial_focal_spot_shift", _D), ("center_channel_non_ffs", _D), ("center_row", _D),
    ("focal_spot_radius", _D), ("n_channels", _U), ("num_views_per_turn", _U),
    ("num_views_per_turn_without_ffs", _U), ("source_detector_distance", _D),
    ("transaxial_detector_spacing", _D), ("transaxial_focal_spot_shift", _D),
    ("fan_angle_increment", _D),
    ("penalty", _I), ("reserved0", _I), ("lambda_", _D), ("delta", _D), ("num_iterations", _U),
    ("Nrows", _U), ("first_view_angle", _D), ("num_z_ffs", _U), ("num_phi_ffs", _U),
    ("num_views", _U), ("table_feed_per_rotation", _D), ("tube_angle_increment", _D),
    ("z_end", _D), ("z_first_view", _D), ("z_good_slice", _D), ("z_matrix_start", _D),
    ("z_start", _D), ("table_direction", _I), ("reserved1", _I),
    ("fov_radius", _D), ("center_voxel_x", _D), ("center_voxel_y", _D), ("center_voxel_z", _D),
    ("dx", _D), ("dy", _D), ("dz", _D), ("nx", _U), ("ny", _U), ("nz", _U),
    ("FileType", _U), ("FileSubType", _U), ("RawOffset", _U), ("Readings", _U), ("Zffs", _U),
    ("Phiffs", _U), ("CollSlicewidth", _D), ("wfbp_initialize", _U),
    ("Nrows_projection", _U), ("views_per_slice", _U), ("voxel_size_x", _D),
    ("voxel_size_y", _D), ("voxel_size_z", _D), ("tube_z_increment", _D), ("beam_width", _D),
    ("beam_width_at_roi_edge", _D), ("num_views_for_system_matrix", _U), ("num_voxels_x", _U),
    ("num_voxels_y", _U), ("num_voxels_z", _U), ("slice_thickness", _D), ("recon_fov", _D),
]


class GeomC(C.Structure):
    _fields_ = GEOM_FIELDS

    def as_dict(self):
        out = {}
        for name, _ in GEOM_FIELDS:
            if name.startswith("reserved"):
                continue
            out["lambda" if name == "lambda_" else name] = getattr(self, name)
        return out


class PrmStrings(C.Structure):
    _fields_ = [
        ("initial_recon_path", C.c_char * 1024), ("matrix_path", C.c_char * 1024),
        ("output_dir", C.c_char * 1024), ("output_file", C.c_char * 1024),
        ("potential", C.c_char * 64), ("recon_path", C.c_char * 1024),
        ("sinogram_path", C.c_char * 1024), ("penalty", C.c_char * 64),
    ]


class PhantomSpec(C.Structure):
    _fields_ = [
        ("n_ellipsoids", _I), ("reserved", _I), ("seed", _U), ("ellipsoid_z_lo", _D),
        ("ellipsoid_z_hi", _D), ("i0_lo", _D), ("i0_hi", _D), ("clip_z_lo", _D), ("clip_z_hi", _D),
    ]


class SsmInfo(C.Structure):
    _fields_ = [
        ("n_columns", _U), ("n_views", _U), ("nnz", _U), ("max_col_nnz", _U),
        ("bytes_device", _U), ("weights", _I), ("ffs", _I), ("build_ms", _D), ("n_pairs", _U),
    ]


class IcdOpts(C.Structure):
    _fields_ = [
        ("mode", _I), ("weights", _I), ("refresh_every", _I), ("warps_in_flight", _I),
        ("lattice", _I), ("compute_cost", _I), ("stop_rel_change", _D), ("relax", _D),
        ("priority", _I), ("warps_per_voxel", _I), ("entries_per_lane", _I), ("stage_column", _I),
        ("entry_pairs", _I), ("stack_align", _I), ("l2_hints", _I),
    ]


class TuneTrial(C.Structure):
    _fields_ = [("warps_in_flight", _I), ("warps_per_voxel", _I), ("lattice", _I), ("entries_per_lane", _I),
                ("stage_column", _I), ("entry_pairs", _I), ("device_ms", _D), ("cost", _D), ("score", _D)]


class TuneReport(C.Structure):
    _fields_ = [("n_trials", _I), ("best", _I), ("start_cost", _D), ("trials", TuneTrial * 32)]


class IterStats(C.Structure):
    _fields_ = [
        ("iterations", _I), ("reserved", _I), ("cost", _D), ("rel_change", _D),
        ("device_ms", _D), ("voxel_updates", _D), ("entries", _D), ("entries_scattered", _D),
    ]


_P = C.c_void_p
_PD = C.POINTER(C.c_double)
_PF = C.POINTER(C.c_float)
_PU = C.POINTER(C.c_uint64)
_PI32 = C.POINTER(C.c_int32)
_PG = C.POINTER(GeomC)

# name -> (restype, argtypes). Every symbol declared in include/ctbb_icd_b200.h.
PROTOTYPES = {
    "ctbb_last_error": (C.c_char_p, []),
    "ctbb_status_str": (C.c_char_p, [_I]),
    "ctbb_configure_recon_params": (_I, [C.c_char_p, _PG, C.POINTER(PrmStrings)]),
    "ctbb_slice_tables": (_I, [_PG, _PD, _PD, _PD, _PU, _U]),
    "ctbb_read_raw": (_I, [C.c_char_p, _PG, _PF]),
    "ctbb_synth_raw_host": (_I, [_PG, C.POINTER(PhantomSpec), _PF, C.c_int]),
    "ctbb_write_raw_file": (_I, [C.c_char_p, _PG, _PF]),
    "ctbb_gpu_init": (_I, [C.c_int, _P, C.POINTER(_P)]),
    "ctbb_gpu_destroy": (None, [_P]),
    "ctbb_gpu_stream": (_P, [_P]),
    "ctbb_gpu_synchronize": (_I, [_P]),
    "ctbb_gpu_synth_raw": (_I, [_P, _PG, C.POINTER(PhantomSpec), _P]),
    "ctbb_gpu_generate_ssm": (_I, [_P, _PG, _I, C.POINTER(_P)]),
    "ctbb_gpu_ssm_info": (_I, [_P, C.POINTER(SsmInfo)]),
    "ctbb_gpu_ssm_column": (_I, [_P, _U, _PI32, _PF, _U, _PU]),
    "ctbb_gpu_ssm_export_reference": (_I, [_P, C.c_char_p]),
    "ctbb_gpu_ssm_import_reference": (_I, [_P, _PG, C.c_char_p, _I, C.POINTER(_P)]),
    "ctbb_gpu_ssm_free": (None, [_P]),
    "ctbb_gpu_recon_create": (_I, [_P, _PG, _PU, C.POINTER(_P)]),
    "ctbb_gpu_recon_free": (None, [_P]),
    "ctbb_gpu_recon_set_raw": (_I, [_P, _PF]),
    "ctbb_gpu_recon_set_raw_device": (_I, [_P, _P]),
    "ctbb_gpu_recon_raw_device": (_P, [_P]),
    "ctbb_gpu_recon_get_raw": (_I, [_P, _PF]),
    "ctbb_gpu_recon_set_volume": (_I, [_P, _P, _PF]),
    "ctbb_gpu_recon_get_volume": (_I, [_P, _PF]),
    "ctbb_gpu_recon_get_volume_f64": (_I, [_P, _PD]),
    "ctbb_gpu_recon_iterate": (_I, [_P, _P, C.POINTER(IcdOpts), _I, C.POINTER(IterStats)]),
    "ctbb_gpu_recon_entries": (_I, [_P, _P, _PD]),
    "ctbb_gpu_recon_refresh_residual": (_I, [_P, _P]),
    "ctbb_gpu_recon_cost": (_I, [_P, _PD]),
    "ctbb_gpu_batch_create": (_I, [_P, _I, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]),
    "ctbb_gpu_batch_iterate": (_I, [_P, C.POINTER(IcdOpts), _I, C.POINTER(IterStats)]),
    "ctbb_gpu_batch_free": (None, [_P]),
    "ctbb_gpu_icd": (_I, [_P, _P, _PG, _PU, _PF, _PF, C.POINTER(IcdOpts), C.POINTER(IterStats)]),
    "ctbb_gpu_rotate": (_I, [_P, _PG, _PD, _PU, _PF, _I]),
    "ctbb_gpu_rotate_device": (_I, [_P, _PG, _PD, _PU, _P, _P, _I]),
    "ctbb_gpu_rotate_device_noalloc": (_I, [_P, _PG, _PD, _PU, _P, _P, _I]),
    "ctbb_cnn_create": (_I, [_P, _I, _U, C.POINTER(_P)]),
    "ctbb_cnn_free": (None, [_P]),
    "ctbb_cnn_num_params": (_U, [_P]),
    "ctbb_cnn_get_params": (_I, [_P, _PF, _U]),
    "ctbb_cnn_set_params": (_I, [_P, _PF, _U]),
    "ctbb_cnn_set_scaling": (_I, [_P, C.c_float, C.c_float]),
    "ctbb_cnn_get_scaling": (_I, [_P, _PF, _PF]),
    "ctbb_cnn_forward": (_I, [_P, _P, _I, _I, _I, _P]),
    "ctbb_cnn_accumulate_gradient": (_I, [_P, _P, _P, _P, _I, _I, _I, _PD]),
    "ctbb_cnn_get_gradient": (_I, [_P, _PF, _U]),
    "ctbb_cnn_zero_gradient": (_I, [_P]),
    "ctbb_cnn_adam_step": (_I, [_P, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float]),
    "ctbb_gpu_recon_warm_start": (_I, [_P, _P, _P, _PD]),
    "ctbb_gpu_recon_autotune": (_I, [_P, _P, C.POINTER(IcdOpts), _I, C.POINTER(IcdOpts), C.POINTER(TuneReport)]),
    "ctbb_gpu_recon_set_priority": (_I, [_P, C.POINTER(IcdOpts), _D]),
    "ctbb_gpu_penalty_steps": (_I, [_P, _I, _D, _D, _U, _PD, _PD, _PF, _PD]),
    "ctbb_gpu_recon_set_volume_estimate": (_I, [_P, _P, _PF, _I]),
    "ctbb_cnn_set_engine": (_I, [_P, _I]),
    "ctbb_gpu_recon_set_volume_upsampled": (_I, [_P, _P, _P]),
}

_lib = None


def lib():
    """Load libctbb_icd_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(
                f"{LIB_PATH} is missing: build it with `python -m ctbb_icd_b200.build` "
                "(there is no CPU fallback)")
        handle = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(status: int) -> None:
    if status != CTBB_OK:
        msg = lib().ctbb_last_error().decode(errors="replace")
        raise CtbbError(status, msg or lib().ctbb_status_str(status).decode())


def ptr(arr, ctype):
    """ctypes pointer to a contiguous numpy array."""
    if arr is None:
        return None
    if not arr.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return arr.ctypes.data_as(C.POINTER(ctype))
