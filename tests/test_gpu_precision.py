"""Precision study of the grouped mode (the benchmark's config 3): matrix
weights in FP16 or FP32, FP32 error sinogram with an FP64 residual refresh
y - A x every K in {2, 5, 10} iterations, FP64 cost reductions.

Workload: cfg2's scanner (736 x 64 rows, in-plane flying focal spot, 2304
views/turn), voxel size and edge-preserving penalty on a central
64 x 64 x 4 slab over 3000 views, small enough for the FP64 CPU oracle. The
data are consistent with the slab: the oracle's FP64 forward projection of an
object that lies inside it (a water disc with four inserts, -100 .. +1000
HU), with Gaussian noise of Poisson variance at 1e5 photons per ray. (An
object extending past a 3.75 cm field of view would make this an interior
problem, whose minimiser is nearly flat along smooth image components:
images 12 HU apart then have costs equal to 1e-10.)
Reference optimum: the sequential-order FP64 mode (pinned to the reference
program's iterations at this geometry by test_gpu_bench_size.py) run until
it moves less than 0.01 HU over 100 iterations. Every cost below is the
oracle's FP64 cost (oracle/port.cpp port_cost, Appendix-B form of the
edge-preserving objective) of the image, with the reference's FP32 matrix.

Set CTBB_PRECISION_TABLE=<path> to write the table as JSON.
"""
import json
import os

import numpy as np
import pytest

import ctbb_icd_b200 as C
import oracle_util as O
from ctbb_icd_b200 import workloads as W

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

HU = 0.192 / 1000.0


def _slab_object(rp):
    """Water disc of radius 1.5 cm (mu 0.192 / cm) with four 0.3 cm inserts
    at -100, +100, +500 and +1000 HU, the same in every slice."""
    g = rp.geom
    nz, ny, nx = rp.shape
    xs = (np.arange(nx) - g.center_voxel_x) * g.voxel_size_x
    ys = (np.arange(ny) - g.center_voxel_y) * g.voxel_size_y
    X, Y = np.meshgrid(xs, ys)
    img = np.where(X ** 2 + Y ** 2 < 1.5 ** 2, 0.192, 0.0)
    for (cx, cy), hu in (((0.7, 0.0), -100.0), ((-0.7, 0.0), 100.0), ((0.0, 0.7), 500.0), ((0.0, -0.7), 1000.0)):
        img = np.where((X - cx) ** 2 + (Y - cy) ** 2 < 0.3 ** 2, 0.192 * (1.0 + hu / 1000.0), img)
    return np.broadcast_to(img, (nz, ny, nx)).astype(np.float64).copy()


@pytest.fixture(scope="module")
def study(ctx, tmp_path_factory):
    from oracle import reference_run as R

    d = str(tmp_path_factory.mktemp("precision"))
    w = W.workload("cfg2")
    prm = R.central_subvolume(dict(w["prm"], num_iterations=1), 64, 4, 3000, d)
    prm_path = R.write_prm(os.path.join(d, "p.prm"), prm)
    R.write_zero_raw(prm["sinogram_path"], prm["Readings"], prm["n_channels"], prm["Nrows"])
    rp = C.configure_recon_params(prm_path)
    data = C.load_raw(rp)
    ssm = C.Ssm.generate(rp, ctx, C.SSM_BOTH)
    csr = O.port_ssm(rp)
    x_true = _slab_object(rp)
    y = O.port_forward(rp, data.slice_indices, csr, x_true)
    # noise on the readings some voxel of the slab projects to (the others
    # would only add a constant to every cost)
    seen = O.port_forward(rp, data.slice_indices, csr, np.ones(rp.shape)) > 0
    rng = np.random.default_rng(5)
    y[seen] += rng.standard_normal(int(seen.sum())) / np.sqrt(1e5 * np.exp(-y[seen]))
    data.raw[...] = y.reshape(data.raw.shape).astype(np.float32)

    rc = C.Recon(rp, data.slice_indices, ctx)
    rc.set_raw(data.raw)
    rc.set_volume(ssm, None)
    prev, moved, n_seq = None, None, 0
    while n_seq < 3000:
        rc.iterate(ssm, 100, C.icd_opts(mode=C.ICD_SEQUENTIAL))
        n_seq += 100
        x = rc.volume_f64()
        if prev is not None:
            moved = np.abs(x - prev).max() / HU
            if moved < 0.01:
                break
        prev = x
    x_star = rc.volume_f64()
    rc.free()
    cost_star, _, _ = O.port_cost(rp, data.slice_indices, data.raw, csr, x_star)

    info = ssm.info()
    rows = []
    for weights, wname, wbytes in ((C.SSM_FP32, "fp32", 4), (C.SSM_FP16, "fp16", 2)):
        for K in (2, 5, 10):
            r = C.Recon(rp, data.slice_indices, ctx)
            r.set_raw(data.raw)
            r.set_volume(ssm, None)
            opts = C.icd_opts(mode=C.ICD_GROUPED, weights=weights, refresh_every=K)
            ms, it, ent, scat, last = 0.0, 0, 0.0, 0.0, None
            while it < 3000:
                st = r.iterate(ssm, 50, opts)
                ms += st.device_ms
                ent += st.entries
                scat += st.entries_scattered
                it += 50
                x = r.volume_f64()
                if last is not None and np.abs(x - last).max() / HU < 0.001:
                    break
                last = x
            x = r.volume_f64()
            r.free()
            cost, _, _ = O.port_cost(rp, data.slice_indices, data.raw, csr, x)
            b_iter = (4.0 * ent + 4.0 * scat) / it + (4 + wbytes) * float(info.nnz) + 8.0 * x.size
            rows.append(dict(weights=wname, refresh_every=K, iterations=it,
                             cost_rel_err=(cost - cost_star) / cost_star,
                             rmse_hu=float(np.sqrt(np.mean((x - x_star) ** 2)) / HU),
                             max_abs_hu=float(np.abs(x - x_star).max() / HU),
                             ssm_bytes=int(info.nnz * (4 + wbytes)),
                             ms_per_iteration=ms / it,
                             achieved_gbs=b_iter / (ms / it / 1e3) / 1e9))
    table = dict(workload="cfg2 scanner, central 64x64x4 slab, 3000 views, edge-preserving (delta 9.6e-4, "
                          "lambda 0.1), data of an object inside the slab (oracle FP64 projection + noise)", sequential_iterations=n_seq, sequential_last_move_hu=moved,
                 cost_star=cost_star, rows=rows)
    out = os.environ.get("CTBB_PRECISION_TABLE")
    if out:
        with open(out, "w") as f:
            json.dump(table, f, indent=1)
    print(json.dumps(table, indent=1))
    ssm.free()
    return table


def test_fp32_weights_reach_the_fp64_optimum(study):
    for r in study["rows"]:
        if r["weights"] == "fp32":
            assert abs(r["cost_rel_err"]) <= 1e-6, r
            assert r["rmse_hu"] <= 0.5, r


def test_fp16_weights_error_bound(study):
    """FP16 weights minimise the cost with every weight rounded (relative
    error <= 2^-11): the image they converge to stays within 0.5 HU RMSE of
    the FP64 optimum and its FP64 cost within 1e-5 relative."""
    for r in study["rows"]:
        if r["weights"] == "fp16":
            assert abs(r["cost_rel_err"]) <= 1e-5, r
            assert r["rmse_hu"] <= 0.5, r
