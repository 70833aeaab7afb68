"""The rotation kernel's float-centre shortcut (ctbb_icd_b200/csrc/rotate.cu,
rotate_kernel<true>), checked on the CPU.

The reference computes the sample coordinate as (float)((double)xp + cvx)
with xp a float (rotate_slices.cpp:142-151). When the centre cvx is exactly a
float, the kernel computes the float sum xp + (float)cvx instead, which is
the correctly rounded exact sum; the two agree because the double sum of two
floats is exact unless one is below about 2^-29 of the other, and then the
float rounding returns the larger either way. numpy's float32 addition
rounds to nearest like the GPU's __fadd_rn.
"""
import numpy as np
import pytest


@pytest.mark.parametrize("cv", [255.5, 127.5, 63.5, 31.5, 5.5, 0.0, 7.0])
def test_float_sum_equals_reference_double_then_float(cv):
    rng = np.random.default_rng(int(cv * 2) + 1)
    assert float(np.float32(cv)) == cv
    n = 1 << 20
    # coordinates over a 512-voxel slice and beyond, plus values at a tie
    # with the centre and values far below its ulp
    xp = np.concatenate([
        rng.uniform(-600.0, 600.0, n),
        np.round(rng.uniform(-600.0, 600.0, n // 4)) + 0.5,
        rng.uniform(-1e-6, 1e-6, n // 8),
        rng.standard_normal(n // 8) * 2.0 ** -30,
        -cv + rng.uniform(-1e-3, 1e-3, n // 8),
    ]).astype(np.float32)
    ref = (xp.astype(np.float64) + cv).astype(np.float32)
    fast = xp + np.float32(cv)
    assert fast.dtype == np.float32
    assert np.array_equal(ref.view(np.int32), fast.view(np.int32))
