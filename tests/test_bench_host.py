"""Host-side pieces of bench.py that run without a GPU: the traffic figures it
reads from the committed kernel profiles, the in-range entry count of the
CPU sample (the icd_iteration.cpp:205-207 window test), and the reference
arm: its rank rule and, on a reduced sample, its JSON line."""
import os
import sys
import types

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_every_bulk_kernel_the_autotuner_can_pick_has_a_traffic_figure():
    # stage_column 4/5 report icd_bulk_kernel, 6 icd_bulk_pipe_kernel
    for kernel in ("icd_bulk_kernel", "icd_bulk_pipe_kernel"):
        t = bench.read_traffic(kernel)
        assert t is not None and 1e11 < t < 1e13, (kernel, t)
    assert bench.read_traffic("no_such_kernel") is None


def test_sample_inrange_entries_matches_the_window_test():
    rng = np.random.default_rng(4)
    g = types.SimpleNamespace(n_channels=6, Nrows_projection=4, Readings=40, num_views_for_system_matrix=16)
    per_view = g.n_channels * g.Nrows_projection
    ncol = 5
    counts = rng.integers(0, 30, ncol)
    colptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    idx = np.concatenate([np.sort(rng.choice(g.num_views_for_system_matrix * per_view, c, replace=False))
                          for c in counts]).astype(np.int32)
    slice_indices = [0, 3, 20, 39]
    want = 0
    for si in slice_indices:
        start = (si - g.num_views_for_system_matrix // 2) * per_view
        for q in idx:
            want += 0 <= int(q) + start < g.Readings * per_view
    got = bench._sample_inrange_entries(g, slice_indices, colptr, idx)
    assert abs(got - want / (len(slice_indices) * ncol)) < 1e-12


def test_reference_arm_runs_on_rank_zero_only():
    args = types.SimpleNamespace(warmup=3, steps=2)
    assert bench.run_reference(args, rank=1, world=2) is None


@pytest.mark.slow
def test_reference_arm_line_keeps_the_contract(monkeypatch):
    """bench.py --impl reference on a reduced sample (16 x 16 x 4 voxels of
    the benchmark geometry): the reference program builds its own matrix,
    runs warm-up + timed iterations, and the line carries the contract's
    keys, a cpu_baseline describing the run and a host-only e2e."""
    from oracle import reference_run as R

    if not R.available():
        pytest.skip("reference program not built (oracle/Makefile ref)")
    monkeypatch.setattr(bench, "CPU_SAMPLE", dict(nx=16, nz=4, readings=3000))
    line = bench.run_reference(types.SimpleNamespace(warmup=3, steps=2), rank=0, world=1)
    assert line["impl"] == "reference" and "unavailable" not in line, line
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["metric"] == "voxel-updates/s" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["value"] == line["value"]
    assert line["cpu_baseline"]["cores"] >= 1 and "sample" in line["cpu_baseline"]
    assert line["e2e"] == {"value": line["value"], "unit": "voxel-updates/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["ssm_generation_s"] > 0
    assert "as shipped" in line["config"]["sample"]
