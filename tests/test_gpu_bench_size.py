"""GPU parity at the benchmark sizes, through the C ABI.

* cfg1 in full (736 channels x 16 rows, 3456 views, 128 x 128 x 16, quadratic
  penalty) and cfg2's scanner (736 x 64 rows, in-plane flying focal spot,
  2304 views/turn, edge-preserving penalty) on a central 64 x 64 x 4 slab:
  the stored system matrix against the reference program's own matrix.bin
  (every column's entry count and hash, a few columns entry by entry), the
  sequential-order ICD against the reference's iteration dumps 1-3 (bar:
  1e-5 relative) and the final de-rotated image
  (tests/golden/make_golden.py cfg1 cfg2_sub ran the reference program).
* the full cfg2 geometry (512 x 512, nvsm 2884) and its 7.5 cm central cut:
  sampled columns restricted to sampled views, bit for bit against the
  oracle's ray-driven builder evaluated only there (generate_system_matrix
  _ffs.cpp:104-222 restated in oracle/port.cpp).
"""
import os

import numpy as np
import pytest

import ctbb_icd_b200 as C
import oracle_util as O
from ctbb_icd_b200 import workloads as W

pytestmark = pytest.mark.gpu

ICD_REL_TOL = 1e-5  # per-iteration image agreement with the reference (FP64 iterates, stored as FP32)


@pytest.fixture(scope="module", params=["cfg1", "cfg2_sub"])
def bench_fixture(request, tmp_path_factory):
    d = str(tmp_path_factory.mktemp(request.param))
    z, prm_path = O.bench_size_fixture(request.param, d)
    rp = C.configure_recon_params(prm_path)
    data = C.load_raw(rp)
    return request.param, z, rp, data, d


def test_ssm_matches_reference_matrix_bin_at_bench_size(bench_fixture, ctx):
    name, z, rp, data, d = bench_fixture
    ssm = C.Ssm.generate(rp, ctx, C.SSM_FP32)
    ncol = int(rp.geom.nx * rp.geom.ny)
    path = os.path.join(d, "gpu_matrix.bin")
    ssm.export_reference(path)
    counts, hashes = O.column_hashes(path, ncol)
    os.remove(path)
    bad = np.nonzero((counts != z["col_counts"]) | (hashes != z["col_hashes"]))[0]
    assert bad.size == 0, (name, bad[:10], counts[bad[:3]], z["col_counts"][bad[:3]])
    for i, c in enumerate(z["sample_cols"]):
        idx, w = ssm.column(int(c))
        b, e = z["sample_ptr"][i], z["sample_ptr"][i + 1]
        assert np.array_equal(idx, z["sample_idx"][b:e]), (name, c)
        assert np.array_equal(w.view(np.int32), z["sample_w"][b:e].view(np.int32)), (name, c)
    ssm.free()


def test_sequential_icd_matches_reference_at_bench_size(bench_fixture, ctx):
    name, z, rp, data, d = bench_fixture
    ssm = C.Ssm.generate(rp, ctx, C.SSM_FP32)
    rc = C.Recon(rp, data.slice_indices, ctx)
    rc.set_raw(data.raw)
    rc.set_volume(ssm, None)
    opts = C.icd_opts(mode=C.ICD_SEQUENTIAL)
    for it in range(z["iterations_f32"].shape[0]):
        rc.iterate(ssm, 1, opts)
        x = rc.volume_f64()
        ref = z["iterations_f32"][it].astype(np.float64)
        rel = np.linalg.norm(x - ref) / np.linalg.norm(ref)
        assert rel < ICD_REL_TOL, (name, it + 1, rel)
        assert np.abs(x - ref).max() <= ICD_REL_TOL * np.abs(ref).max(), (name, it + 1)
    # the reference's final image: the last iterate de-rotated (rotate_slices.cpp:81-114)
    out = C.CtData(recon_volume=rc.volume_f64().astype(np.float32), tube_angles=data.tube_angles,
                   slice_indices=data.slice_indices)
    C.rotate_slices_rotating2fixed(rp, out, ctx)
    assert np.allclose(out.recon_volume, z["final"], rtol=1e-5, atol=1e-5 * np.abs(z["final"]).max())
    rc.free()
    ssm.free()


@pytest.mark.parametrize("name", ["cfg2", "cfg2_center"])
def test_ssm_full_geometry_sampled_columns_match_oracle(name, ctx, tmp_path):
    _, rp = W.materialise(name, str(tmp_path), raw=False)
    C.slice_tables(rp)  # load_raw's tables set table_direction: the source advances in z
    g = rp.geom
    assert g.table_direction == -1
    ssm = C.Ssm.generate(rp, ctx, C.SSM_FP32)
    nx, ncol = int(g.nx), int(g.nx * g.ny)
    nvsm = int(g.num_views_for_system_matrix)
    per_view = int(g.n_channels * g.Nrows_projection)
    rng = np.random.default_rng(2884)
    special = [0, nx - 1, ncol - nx, ncol - 1, nx // 2 + nx * (nx // 2), nx // 2 + nx * 3, 3 + nx * (nx // 2)]
    cols = np.unique(np.concatenate([special, rng.integers(0, ncol, 90)])).astype(np.int64)
    views = np.unique(np.concatenate([[0, 1, nvsm // 2, nvsm - 2, nvsm - 1],
                                      np.arange(rng.integers(0, 7), nvsm, 7)])).astype(np.int32)
    ref = O.port_ssm_subset(rp, cols, views)
    n_cmp = 0
    for c in cols:
        idx, w = O.restrict_views(*ssm.column(int(c)), views, per_view)
        ri, rw = ref[int(c)]
        assert np.array_equal(idx, ri), (name, c, idx.size, ri.size)
        assert np.array_equal(w.view(np.int32), rw.view(np.int32)), (name, c)
        n_cmp += idx.size
    assert n_cmp > 0
    ssm.free()
