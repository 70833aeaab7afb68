"""Pin the oracle (CPU restatement, oracle/port.cpp) and the host-side setup
code against outputs of the reference program itself (tests/golden/*.npz,
produced by make_golden.py from the reference sources). CPU only."""
import numpy as np

import oracle_util as O
from ctbb_icd_b200 import workloads as W


def test_port_ssm_matches_reference_matrix_bin(golden):
    m = O.port_ssm(golden.rp)
    assert m.nnz == golden.colptr[-1]
    assert np.array_equal(m.colptr, golden.colptr)
    assert np.array_equal(m.idx, golden.idx)
    # float weights bit for bit
    assert np.array_equal(m.w.view(np.int32), golden.w.view(np.int32))


def test_port_icd_matches_reference_iterations(golden):
    n = golden.iterations.shape[0] - 1
    dumps, _, _ = O.port_icd(golden.rp, golden.data.slice_indices, golden.raw, golden.csr(), n)
    for it in range(n):
        ref = golden.iterations[it + 1]
        rel = np.linalg.norm(dumps[it] - ref) / np.linalg.norm(ref)
        # Only the alpha/beta summation order differs (OpenMP reduction).
        assert rel < 1e-12, (it, rel)


def test_port_rotate_matches_reference_final_image(golden):
    last = golden.iterations[-1].astype(np.float32)
    out = O.port_rotate(golden.rp, golden.data.tube_angles, golden.data.slice_indices, last, -1)
    assert np.array_equal(out.view(np.int32), golden.final.view(np.int32))


def test_port_synth_reproduces_fixture_raw(golden):
    spec = W.phantom_spec({**W.WORKLOADS[golden.name]["phantom"],
                           **({} if "z_lo" in W.WORKLOADS[golden.name]["phantom"] else
                              {"z_lo": min(golden.rp.z_start, golden.rp.z_end),
                               "z_hi": max(golden.rp.z_start, golden.rp.z_end)})})
    raw = O.port_synth(golden.rp, spec)
    # Same libm on the same image: identical; elsewhere libm rounding may move a
    # Poisson draw by one count.
    assert np.abs(raw - golden.raw).max() < 2e-3
    assert np.mean(raw == golden.raw) > 0.999


def test_setup_derivations_match_reference(golden):
    fields, views, slices = O.parse_setup_dump(golden.setup_dump)
    g = golden.rp.geom
    for name, ref in fields.items():
        if name in ("penalty", "matrix_path"):
            continue
        key = "lambda_" if name == "lambda" else name
        mine = getattr(g, key)
        assert mine == ref, (name, mine, ref)
    assert golden.rp.penalty == fields["penalty"]
    assert np.array_equal(golden.data.tube_angles, views[:, 0])
    assert np.array_equal(golden.data.table_positions, views[:, 1])
    assert [int(s) for s in golden.data.slice_indices] == [s[1] for s in slices]
    assert np.array_equal(golden.data.slice_locations, np.array([s[0] for s in slices]))


def test_read_raw_matches_reference_layout(golden):
    # load_raw's double transpose is the identity on FileType 0 frames.
    assert np.array_equal(golden.data.raw, golden.raw)


def test_port_cost_decreases_over_reference_iterations(golden):
    costs = [O.port_cost(golden.rp, golden.data.slice_indices, golden.raw, golden.csr(), x)[0]
             for x in golden.iterations]
    assert all(b <= a * (1 + 1e-12) for a, b in zip(costs, costs[1:])), costs


def test_port_forward_is_linear(golden):
    rng = np.random.default_rng(0)
    m = golden.csr()
    x1 = rng.random(golden.rp.shape)
    x2 = rng.random(golden.rp.shape)
    f1 = O.port_forward(golden.rp, golden.data.slice_indices, m, x1)
    f2 = O.port_forward(golden.rp, golden.data.slice_indices, m, x2)
    f12 = O.port_forward(golden.rp, golden.data.slice_indices, m, 2 * x1 + 3 * x2)
    assert np.allclose(f12, 2 * f1 + 3 * f2, rtol=1e-12, atol=1e-12)


def test_port_ssm_subset_equals_full_build_restricted(tmp_path):
    """The column/view-restricted builder (used to check the full-size matrix
    on sampled columns) gives exactly the full builder's entries."""
    for name in ("tiny", "tiny_ffs", "small_ffs", "tiny_zphiffs"):
        _, rp = W.materialise(name, str(tmp_path / name), raw=False)
        full = O.port_ssm(rp)
        ncol = int(rp.geom.nx * rp.geom.ny)
        nvsm = int(rp.geom.num_views_for_system_matrix)
        per_view = int(rp.geom.n_channels * rp.geom.Nrows_projection)
        rng = np.random.default_rng(11)
        cols = np.unique(np.concatenate([[0, ncol - 1], rng.integers(0, ncol, 24)]))
        views = np.unique(np.concatenate([[0, nvsm - 1], rng.integers(0, nvsm, max(4, nvsm // 5))]))
        sub = O.port_ssm_subset(rp, cols, views)
        for c in cols:
            ri, rw = O.restrict_views(*full.column(int(c)), views, per_view)
            si, sw = sub[int(c)]
            assert np.array_equal(si, ri), (name, c)
            assert np.array_equal(sw.view(np.int32), rw.view(np.int32)), (name, c)
