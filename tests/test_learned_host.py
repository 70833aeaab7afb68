"""Host-side pieces of the learned warm start that need no GPU: masks, error
measure, workload shapes, the early-iterate protocol and the weights file."""
import numpy as np

from ctbb_icd_b200 import learned as L


class _Geom:
    num_voxels_x = num_voxels_y = 64
    center_voxel_x = center_voxel_y = 31.5
    voxel_size_x = voxel_size_y = 30.0 / 64
    acquisition_fov = 50.0


class _Rp:
    geom = _Geom()
    shape = (8, 64, 64)


def test_masks_and_interior():
    rp = _Rp()
    m = L.object_mask(rp, 13.0)
    assert m.shape == (64, 64) and m[32, 32] and not m[0, 0]
    # Disc area within a pixel ring of pi r^2.
    r_px = 13.0 / _Geom.voxel_size_x
    assert abs(m.sum() - np.pi * r_px ** 2) < 2 * np.pi * r_px
    assert L.fov_mask(rp).all()  # the 50 cm scanner FOV covers the 30 cm grid
    assert L.interior(16) == slice(2, 14) and L.interior(4) == slice(0, 4)


def test_rmse_hu():
    m = np.ones((4, 4), bool)
    x = np.zeros((3, 4, 4))
    ref = np.full((3, 4, 4), 10 * L.HU)
    assert abs(L.rmse_hu(x, ref, m) - 10.0) < 1e-12
    ref[0] = 0.0
    assert abs(L.rmse_hu(x, ref, m, slice(1, 3)) - 10.0) < 1e-12


def test_workload_shapes():
    assert L.workload_shape("cfg2") == (64, 512, 512)
    # the training grid (256 x 256 x 32 over cfg2's field of view) is the
    # half-size grid of the benchmark scan in-plane
    assert L.workload_shape(L.TRAIN_WORKLOAD) == (32, 256, 256)
    assert L.workload_shape(L.coarse_workload("cfg2")) == (64, 256, 256)


def test_committed_weights_and_protocol():
    d = np.load(L.WEIGHTS_PATH)
    from oracle import cnn_oracle as O

    assert d["params"].shape == (O.num_params(int(d["blocks"])),) and np.isfinite(d["params"]).all()
    assert int(d["n_early"]) == 3 and int(d["early_lattice"]) == 32
    # 2048 in-flight updates on the 256 x 256 x 32 training grid.
    shape = L.workload_shape(L.TRAIN_WORKLOAD)
    assert abs(float(d["early_density"]) * float(np.prod(shape)) - 2048) < 1e-6
    assert str(d["train_seeds"]) == "100:132"
    assert abs(float(d["s_in"]) - L.S_IN) < 1e-6 and abs(float(d["s_out"]) - L.S_OUT) < 1e-4
