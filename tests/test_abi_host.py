"""C-ABI and host-side checks that need no GPU: every symbol of
include/ctbb_icd_b200.h is exported, the parameter-file checks and error
codes behave like the reference's exits, and GPU entry points fail loudly
without a device."""
import ctypes
import os
import re

import numpy as np
import pytest

import ctbb_icd_b200 as C
from ctbb_icd_b200 import workloads as W
from ctbb_icd_b200._lib import PROTOTYPES, lib
from conftest import ROOT, has_gpu

HEADER = os.path.join(ROOT, "include", "ctbb_icd_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ctbb_\w+)\s*\(", text)))


def test_header_declares_expected_entry_points():
    names = declared_functions()
    assert "ctbb_gpu_generate_ssm" in names and "ctbb_gpu_icd" in names and "ctbb_gpu_rotate" in names
    assert set(names) <= set(PROTOTYPES), set(names) - set(PROTOTYPES)


def test_library_exports_every_declared_symbol():
    L = lib()
    for name in declared_functions():
        assert hasattr(L, name), name
    # nm agrees (exported as C symbols, not mangled)
    import subprocess

    out = subprocess.run(["nm", "-D", "--defined-only", os.path.join(ROOT, "ctbb_icd_b200", "libctbb_icd_b200.so")],
                         capture_output=True, text=True).stdout
    exported = set(re.findall(r"\sT\s(ctbb_\w+)", out))
    assert set(declared_functions()) <= exported


def test_gpu_init_without_device_reports_no_device():
    if has_gpu():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    st = lib().ctbb_gpu_init(0, None, ctypes.byref(h))
    assert st == 6  # CTBB_ERR_NO_DEVICE
    assert lib().ctbb_last_error()


def _prm(tmp_path, drop=(), **over):
    w = W.workload("tiny")
    prm = w["prm"]
    prm.update(sinogram_path=str(tmp_path / "x.bin"), output_dir=str(tmp_path), output_file="o.img")
    prm.update(over)
    for k in drop:
        prm.pop(k, None)
    return W.write_prm(str(tmp_path / "p.prm"), prm)


def test_missing_required_field_is_config_error(tmp_path):
    with pytest.raises(C.CtbbError) as e:
        C.configure_recon_params(_prm(tmp_path, drop=("n_channels",)))
    assert e.value.status == 2 and "n_channels" in str(e.value)


def test_zero_is_missing_for_z_start(tmp_path):
    # setup.cpp:138 treats z_start == 0 as not set (quirk kept).
    with pytest.raises(C.CtbbError) as e:
        C.configure_recon_params(_prm(tmp_path, z_start=0.0))
    assert "z_start" in str(e.value)


def test_zero_allowed_fields_need_presence(tmp_path):
    with pytest.raises(C.CtbbError) as e:
        C.configure_recon_params(_prm(tmp_path, drop=("Zffs",)))
    assert "Zffs" in str(e.value)


def test_bad_penalty_rejected(tmp_path):
    with pytest.raises(C.CtbbError) as e:
        C.configure_recon_params(_prm(tmp_path, penalty="huber"))
    assert "penalty" in str(e.value)


def test_defaults_applied(tmp_path):
    rp = C.configure_recon_params(_prm(tmp_path, drop=("nx", "ny", "lambda", "delta", "recon_fov", "penalty")))
    g = rp.geom
    assert (g.nx, g.ny, g.lambda_, g.delta, g.recon_fov) == (512, 512, 0.3, 0.005, 25.0)
    assert rp.penalty == "quadratic" and g.penalty == C.PENALTY_QUADRATIC
    assert rp.matrix_path == os.path.join(str(tmp_path), "matrix.bin")


def test_missing_prm_file_is_io_error(tmp_path):
    with pytest.raises(C.CtbbError) as e:
        C.configure_recon_params(str(tmp_path / "nope.prm"))
    assert e.value.status == 3


def test_out_of_range_slices_are_range_error(tmp_path):
    # Two turns of the tiny scan cannot hold the requested slab (setup.cpp:359-377).
    rp = C.configure_recon_params(_prm(tmp_path, Readings=192))
    with pytest.raises(C.CtbbError) as e:
        C.slice_tables(rp)
    assert e.value.status == 4


def test_raw_file_round_trip(tmp_path):
    rp = C.configure_recon_params(_prm(tmp_path))
    raw = np.random.default_rng(1).random(rp.raw_shape, dtype=np.float32)
    C.write_raw_file(str(tmp_path / "x.bin"), rp, raw)
    data = C.load_raw(rp)
    assert np.array_equal(data.raw, raw)


def test_short_raw_file_is_io_error(tmp_path):
    rp = C.configure_recon_params(_prm(tmp_path))
    np.zeros(10, np.float32).tofile(str(tmp_path / "x.bin"))
    with pytest.raises(C.CtbbError) as e:
        C.load_raw(rp)
    assert e.value.status == 3


def test_sample_prm_fields_parse(tmp_path):
    # The reference's resources/sample_prm.yaml field set (paths rewritten);
    # it lacks fan_angle_increment, which setup.cpp:129 requires.
    text = """
sinogram_path: ./n_ffs_short_acr.ptr
output_dir:    ./
output_file:   n_ffs_short_acr.img
FileType:        0
FileSubType:     0
RawOffset:       0
Readings:        6148
acquisition_fov:                50.0
n_channels:                     736
num_views_per_turn_without_ffs: 1152
focal_spot_radius:              59.5
source_detector_distance:       108.56
anode_angle:                    7.0
axial_detector_spacing:         0.2189
axial_focal_spot_shift:         0.0375
center_channel_non_ffs:         366.25
center_row:                     7.5
transaxial_detector_spacing:    0.12858
transaxial_focal_spot_shift:    0.042698
table_feed_per_rotation:    1.92
Zffs:            0
Phiffs:          0
Nrows:           16
CollSlicewidth:  1.2
recon_fov:       25.0 # Diameter of
nx:              512
ny:              512
slice_thickness: 0.15
z_start:         -20.16
z_end:           -15.96
wfbp_initialize:        1
penalty:                edge-preserving
lambda:                 0.1
delta:                  0.005
system_memory_fraction: 0.75
num_iterations:         100
"""
    p = tmp_path / "sample.prm"
    p.write_text(text)
    with pytest.raises(C.CtbbError) as e:
        C.configure_recon_params(str(p))
    assert "fan_angle_increment" in str(e.value)
    p.write_text(text + "fan_angle_increment: 0.00118508\n")
    rp = C.configure_recon_params(str(p))
    assert rp.penalty == "edge-preserving" and rp.geom.num_views_for_system_matrix > 0


def _synth_noise_free(rp, ph, lo=0.0, hi=0.0):
    spec = W.phantom_spec(dict(ph, i0_lo=0.0, i0_hi=0.0))
    spec.clip_z_lo, spec.clip_z_hi = lo, hi
    raw = np.zeros(rp.raw_shape, np.float32)
    C.check(lib().ctbb_synth_raw_host(ctypes.byref(rp.geom), ctypes.byref(spec),
                                      raw.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 2))
    return raw.astype(np.float64)


def test_phantom_clip_is_additive_and_bounded(tmp_path):
    """Noise-free projector: cutting the phantom at a plane z = zm splits each
    line integral into its two parts; a clip holding the whole phantom
    changes nothing; a clip away from it gives zero."""
    _, rp = W.materialise("small_ffs", str(tmp_path), raw=False)
    C.slice_tables(rp)  # load_raw's data-view geometry (z of the first view, table direction)
    ph = W.WORKLOADS["small_ffs"]["phantom"]
    full = _synth_noise_free(rp, ph)
    assert np.array_equal(_synth_noise_free(rp, ph, -1e4, 1e4), full)
    zm = -5.5
    a = _synth_noise_free(rp, ph, -1e4, zm)
    b = _synth_noise_free(rp, ph, zm, 1e4)
    assert np.abs(a).max() > 0 and np.abs(b).max() > 0
    assert np.allclose(a + b, full, rtol=1e-5, atol=1e-5)
    assert np.abs(_synth_noise_free(rp, ph, 500.0, 600.0)).max() == 0.0
