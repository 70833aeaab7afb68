"""GPU warm-start network: forward pass and parameter gradients of the CUDA
kernels (BF16 tensor-core convolutions, FP32 accumulation) against the FP64
CPU oracle, training through Adam, and the warm start inside ICD."""
import numpy as np
import pytest

import ctbb_icd_b200 as C
from ctbb_icd_b200 import learned as L
from oracle import cnn_oracle as O

pytestmark = pytest.mark.gpu

# BF16 activations and gradients (8-bit mantissa) with FP32 accumulation:
# bounds on the relative L2 error of the output and of each parameter
# tensor's gradient against the FP64 oracle.
FWD_TOL = 2e-2
GRAD_TOL = 5e-2


def _torch():
    import torch

    return torch


def _phantom(shape, seed):
    """Smooth positive volume in cm^-1 (water-like with blobs)."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    v = np.full(shape, 0.192)
    for _ in range(6):
        c = rng.uniform(0, 1, 3) * np.array(shape)
        r = rng.uniform(1.5, 4.0)
        d2 = ((z - c[0]) / 1.5) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2
        v += rng.uniform(-0.05, 0.1) * np.exp(-d2 / (r * r))
    return np.maximum(v + rng.normal(0, 0.004, shape), 0.0)


def _tensors(blocks):
    n_in = O.TAPS * O.C + O.C
    per = O.TAPS * O.C * O.C + O.C
    parts = [("W_in", 0, O.TAPS * O.C), ("b_in", O.TAPS * O.C, n_in)]
    o = n_in
    for i in range(2 * blocks):
        parts.append((f"W{i}", o, o + O.TAPS * O.C * O.C))
        parts.append((f"b{i}", o + O.TAPS * O.C * O.C, o + per))
        o += per
    parts.append(("W_out", o, o + O.TAPS * O.C))
    parts.append(("b_out", o + O.TAPS * O.C, o + O.TAPS * O.C + 1))
    return parts


@pytest.mark.parametrize("shape", [(5, 10, 20), (2, 8, 16), (3, 17, 33)])
def test_forward_matches_oracle(ctx, shape):
    torch = _torch()
    blocks = 2
    net = L.WarmStartNet(ctx, blocks)
    p = O.init_params(blocks, seed=7).astype(np.float32)
    net.set_params(p)
    x = _phantom(shape, 1).astype(np.float32)
    out = net.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    ref, _ = O.forward(p.astype(np.float64), x, blocks, s_in=L.S_IN)
    err = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    assert err < FWD_TOL, err
    net.free()


def test_gradient_matches_oracle(ctx):
    torch = _torch()
    blocks = 2
    shape = (5, 10, 20)
    net = L.WarmStartNet(ctx, blocks)
    p = O.init_params(blocks, seed=11).astype(np.float32)
    net.set_params(p)
    x = _phantom(shape, 2).astype(np.float32)
    xc = (x + 0.004 * np.sin(np.arange(x.size).reshape(shape) * 0.37)).astype(np.float32)
    w = (np.random.default_rng(3).uniform(0, 1, shape) > 0.2).astype(np.float32)
    tx, txc, tw = (torch.from_numpy(a).cuda() for a in (x, xc, w))
    net.zero_gradient()
    loss = net.accumulate_gradient(tx, txc, tw)
    g = net.gradient()
    ref_loss, ref_g, _ = O.loss_and_grad(p.astype(np.float64), x, xc, blocks, s_in=L.S_IN, s_out=L.S_OUT, w=w)
    assert abs(loss - ref_loss) <= 2 * FWD_TOL * ref_loss, (loss, ref_loss)
    for name, a, b in _tensors(blocks):
        gg, rr = g[a:b].astype(np.float64), ref_g[a:b]
        err = np.linalg.norm(gg - rr) / max(np.linalg.norm(rr), 1e-30)
        assert err < GRAD_TOL, (name, err)
    # Accumulation: a second call doubles the buffer.
    net.accumulate_gradient(tx, txc, tw)
    assert np.allclose(net.gradient(), 2 * g, rtol=1e-5, atol=1e-7)
    net.free()


def test_adam_training_reduces_loss(ctx):
    torch = _torch()
    net = L.WarmStartNet(ctx, 2, seed=5)
    shape = (4, 24, 40)
    pairs = []
    for s in range(3):
        x = _phantom(shape, 10 + s)
        # Target: half-way to a smoothed copy (early ICD iterates are rough).
        k = np.ones(3) / 3
        xs = x.copy()
        for ax in (1, 2):
            xs = np.apply_along_axis(lambda r: np.convolve(r, k, mode="same"), ax, xs)
        pairs.append((torch.from_numpy(x.astype(np.float32)).cuda(),
                      torch.from_numpy((x + 0.5 * (xs - x)).astype(np.float32)).cuda()))
    first = sum(net.accumulate_gradient(a, b) for a, b in pairs) / 3
    net.zero_gradient()
    for step in range(80):
        a, b = pairs[step % 3]
        net.accumulate_gradient(a, b)
        net.adam_step(2e-3)
    last = sum(net.accumulate_gradient(a, b) for a, b in pairs) / 3
    net.zero_gradient()
    assert last < 0.5 * first, (first, last)
    net.free()


def test_params_round_trip_and_save(ctx, tmp_path):
    net = L.WarmStartNet(ctx, 1, seed=9)
    p = net.params()
    assert p.size == O.num_params(1) == net.n_params
    q = (p * 0.5).astype(np.float32)
    net.set_params(q)
    assert np.array_equal(net.params(), q)
    path = str(tmp_path / "w.npz")
    net.save(path)
    net2 = L.WarmStartNet.load(ctx, path)
    assert np.array_equal(net2.params(), q) and net2.scaling() == net.scaling()
    with pytest.raises(C.CtbbError):
        net.set_params(q[:-1])
    net.free()
    net2.free()


def test_warm_start_with_zero_network_keeps_image(ctx):
    """All-zero network: the warm start leaves x unchanged and e = y - Ax
    refreshed; a priority pass then runs over the (all-zero) map's subset."""
    scan = L.make_scan(ctx, "small", seed=3)
    opts = C.icd_opts(mode=C.ICD_GROUPED, weights=C.SSM_FP32)
    scan.rc.iterate(scan.ssm, 2, opts)
    x0 = scan.rc.volume()
    net = L.WarmStartNet(ctx, 1)
    net.set_params(np.zeros(net.n_params, np.float32))
    scan.rc.warm_start(scan.ssm, net, scan.tables.tube_angles)
    assert np.array_equal(scan.rc.volume(), x0)
    c_ws = scan.rc.cost()
    scan.rc.refresh_residual(scan.ssm)
    assert abs(scan.rc.cost() - c_ws) <= 1e-9 * abs(c_ws)
    scan.rc.set_priority(0.25, opts)
    st = scan.rc.iterate(scan.ssm, 1, C.icd_opts(mode=C.ICD_GROUPED, weights=C.SSM_FP32, priority=True))
    assert st.iterations == 1
    net.free()


def test_warm_start_applies_rotated_correction(ctx):
    """A network whose output is a constant c adds c / s_out inside the
    rotated support; the priority subset then holds the moved voxels."""
    scan = L.make_scan(ctx, "small", seed=4)
    opts = C.icd_opts(mode=C.ICD_GROUPED, weights=C.SSM_FP32)
    scan.rc.iterate(scan.ssm, 2, opts)
    x0 = scan.rc.volume()
    net = L.WarmStartNet(ctx, 0)
    p = np.zeros(net.n_params, np.float32)
    p[-1] = 0.5  # b_out: constant output 0.5 -> +0.5 / s_out everywhere in the fixed frame
    net.set_params(p)
    scan.rc.warm_start(scan.ssm, net, scan.tables.tube_angles)
    x1 = scan.rc.volume()
    step = 0.5 / L.S_OUT
    # Voxels well inside the slice (away from the rotated frame's zero-filled
    # corners) receive the step up to float rounding.
    inner = L.fov_mask(scan.rp)
    nx = x0.shape[-1]
    yy, xx = np.mgrid[:nx, :nx]
    inner &= (xx - (nx - 1) / 2) ** 2 + (yy - (nx - 1) / 2) ** 2 < (0.4 * nx) ** 2
    d = (x1 - x0)[:, inner]
    assert np.allclose(d, step, rtol=1e-4, atol=1e-7), (d.min(), d.max(), step)
    scan.rc.set_priority(0.5, opts)
    st = scan.rc.iterate(scan.ssm, 1, C.icd_opts(mode=C.ICD_GROUPED, weights=C.SSM_FP32, priority=True))
    # The rotated frame's zero-filled border has no step, so the subset
    # leaves those voxels out.
    assert 0 < st.voxel_updates < x0.size
    net.free()


def test_autotune_leaves_iterate_and_picks_a_candidate(ctx):
    scan = L.make_scan(ctx, "cfg1_small", seed=2)
    opts = C.icd_opts(mode=C.ICD_GROUPED, weights=C.SSM_FP32)
    scan.rc.iterate(scan.ssm, 2, opts)
    scan.rc.refresh_residual(scan.ssm)
    x0, c0 = scan.rc.volume(), scan.rc.cost()
    best, trials = scan.rc.autotune(scan.ssm, opts, probe_iters=1)
    assert np.array_equal(scan.rc.volume(), x0)
    assert abs(scan.rc.cost() - c0) <= 1e-12 * abs(c0)
    chosen = [t for t in trials if t["best"]]
    assert len(chosen) == 1 and chosen[0]["score"] == max(t["score"] for t in trials)
    assert (best.warps_in_flight, best.warps_per_voxel, best.lattice, best.entries_per_lane) == (
        chosen[0]["warps_in_flight"], chosen[0]["warps_per_voxel"], chosen[0]["lattice"],
        chosen[0]["entries_per_lane"])
    assert {t["warps_per_voxel"] for t in trials} == {1, 4, 8}
    assert {t["entries_per_lane"] for t in trials} == {8, 16}
    assert {t["stage_column"] for t in trials} == {0, 1, 2, 3}
    assert best.entry_pairs == chosen[0]["entry_pairs"]
    # Every launch stays within the visiting order's concurrency bound.
    n = scan.rc.volume().size
    assert all(t["warps_in_flight"] // t["warps_per_voxel"] <= max(1, n // t["lattice"] ** 2) for t in trials)
    st = scan.rc.iterate(scan.ssm, 2, best)
    assert st.iterations == 2


@pytest.mark.parametrize("name", ["tiny_zffs", "small_ffs"])
def test_autotune_fp16_probes_bulk_kernels_only_with_entry_pairs(ctx, name):
    """With FP16 weights the tuner probes the bulk-staged kernels, which read
    entry pairs, only when the matrix keeps pairs: a z flying focal spot
    matrix whose rows do not pair up still tunes (over the other kernels)."""
    scan = L.make_scan(ctx, name, seed=3, weights=C.SSM_FP16)
    opts = C.icd_opts(mode=C.ICD_GROUPED, weights=C.SSM_FP16)
    scan.rc.iterate(scan.ssm, 1, opts)
    best, trials = scan.rc.autotune(scan.ssm, opts, probe_iters=1)
    stages = {t["stage_column"] for t in trials}
    if scan.ssm.info().n_pairs == 0:
        assert not stages & {4, 5, 6}, stages
    else:
        assert {4, 5, 6} <= stages, stages
    st = scan.rc.iterate(scan.ssm, 1, best)
    assert st.iterations == 1 and np.isfinite(scan.rc.volume()).all()
    scan.rc.free()
    scan.ssm.free()


def test_trained_warm_start_beats_plain_icd(ctx):
    """The committed network on a scan it was not trained on (seed 905 of the
    training geometry): after the warm start and the same number of full
    iterations (its early iterations included), the FP64 cost is below plain
    ICD's, and the image is closer to a much longer plain run's."""
    net = L.WarmStartNet.load(ctx)
    scan = L.make_scan(ctx, L.TRAIN_WORKLOAD, seed=905)
    opts = C.icd_opts(mode=C.ICD_GROUPED, weights=C.SSM_FP32)
    n = 12

    scan.rc.iterate(scan.ssm, n, opts)
    scan.rc.refresh_residual(scan.ssm)
    c_plain = scan.rc.cost()
    x_plain = scan.rc.volume()
    scan.rc.iterate(scan.ssm, 7 * n, opts)
    x_long = scan.rc.volume()

    scan.rc.set_volume(scan.ssm, None)
    scan.rc.iterate(scan.ssm, net.n_early, net.early_opts(scan.rc, opts))
    scan.rc.warm_start(scan.ssm, net, scan.tables.tube_angles)
    popts = C.icd_opts(mode=C.ICD_GROUPED, weights=C.SSM_FP32, priority=True)
    scan.rc.set_priority(0.2, popts)
    scan.rc.iterate(scan.ssm, 2, popts)
    scan.rc.iterate(scan.ssm, n - 3, opts)
    scan.rc.refresh_residual(scan.ssm)
    c_learned = scan.rc.cost()
    x_learned = scan.rc.volume()
    assert c_learned < c_plain, (c_learned, c_plain)
    assert scan.error_hu(x_learned, x_long) < scan.error_hu(x_plain, x_long)
    net.free()


@pytest.mark.parametrize("shape", [(3, 8, 16), (5, 37, 150), (2, 130, 257)])
def test_tcgen05_convolutions_match_mma_sync(ctx, shape):
    """The tcgen05 path (TMA-staged halo, 54 tcgen05.mma per 128-voxel line,
    TMEM accumulator) against the warp-level mma.sync kernel on ragged
    volumes (x extents that are not multiples of the 128-voxel tile, edges
    in every direction): same BF16 operands, FP32 accumulation in a different
    order, so outputs and gradients agree to BF16 rounding of the
    activations."""
    torch = _torch()
    net = L.WarmStartNet(ctx, 2, seed=3)
    x = torch.from_numpy(_phantom(shape, 11).astype(np.float32)).cuda()
    xc = (x + 0.002 * torch.randn_like(x)).contiguous()
    out = {}
    grads = {}
    for engine in (C.CNN_ENGINE_MMA_SYNC, C.CNN_ENGINE_TCGEN05):
        net.set_engine(engine)
        out[engine] = net.forward(x).cpu().numpy()
        net.zero_gradient()
        net.accumulate_gradient(x, xc)
        grads[engine] = net.gradient()
    a, b = out[C.CNN_ENGINE_MMA_SYNC], out[C.CNN_ENGINE_TCGEN05]
    assert np.isfinite(b).all()
    assert np.linalg.norm(a - b) <= 1e-2 * np.linalg.norm(a), np.linalg.norm(a - b) / np.linalg.norm(a)
    ga, gb = grads[C.CNN_ENGINE_MMA_SYNC], grads[C.CNN_ENGINE_TCGEN05]
    assert np.linalg.norm(ga - gb) <= 2e-2 * np.linalg.norm(ga), np.linalg.norm(ga - gb) / np.linalg.norm(ga)
    net.free()
