"""GPU parity: the CUDA path (through the C ABI) against the reference's own
outputs (golden fixtures) and the CPU oracle at larger sizes."""
import os

import numpy as np
import pytest

import ctbb_icd_b200 as C
import oracle_util as O
from ctbb_icd_b200 import workloads as W

pytestmark = pytest.mark.gpu

MU_W = 0.192
HU = MU_W / 1000.0  # cm^-1 per HU


@pytest.fixture(scope="module", params=["small", "small_ffs", "mid"])
def wl(request, tmp_path_factory):
    d = str(tmp_path_factory.mktemp(request.param))
    prm, rp = W.materialise(request.param, d)
    data = C.load_raw(rp)
    return request.param, rp, data, O.port_ssm(rp)


# ---------------------------------------------------------------- SSM ----
def test_ssm_matches_reference_matrix_bin(golden, ctx, tmp_path):
    ssm = C.Ssm.generate(golden.rp, ctx, C.SSM_BOTH)
    path = str(tmp_path / "matrix.bin")
    ssm.export_reference(path)
    m = O.read_matrix_bin(path, int(golden.rp.geom.nx * golden.rp.geom.ny))
    assert np.array_equal(m.colptr, golden.colptr)
    assert np.array_equal(m.idx, golden.idx)
    assert np.array_equal(m.w.view(np.int32), golden.w.view(np.int32))
    info = ssm.info()
    assert info.nnz == golden.colptr[-1]
    assert info.ffs == int(bool(golden.rp.geom.Phiffs or golden.rp.geom.Zffs))  # in-plane and/or z spot


def test_ssm_matches_port(wl, ctx):
    name, rp, data, ref = wl
    ssm = C.Ssm.generate(rp, ctx, C.SSM_FP32)
    assert ssm.info().nnz == ref.nnz
    ncol = int(rp.geom.nx * rp.geom.ny)
    for c in list(range(0, ncol, max(1, ncol // 97))) + [ncol - 1]:
        idx, w = ssm.column(c)
        ri, rw = ref.column(c)
        assert np.array_equal(idx, ri), (name, c)
        assert np.array_equal(w.view(np.int32), rw.view(np.int32)), (name, c)


def test_ssm_fp16_weights_are_rounded_fp32(ctx, golden):
    s32 = C.Ssm.generate(golden.rp, ctx, C.SSM_FP32)
    s16 = C.Ssm.generate(golden.rp, ctx, C.SSM_FP16)
    for c in (0, 37, 100):
        i32, w32 = s32.column(c)
        i16, w16 = s16.column(c)
        assert np.array_equal(i32, i16)
        assert np.array_equal(w16, w32.astype(np.float16).astype(np.float32))


def test_ssm_import_reference_round_trip(golden, ctx, tmp_path):
    path = str(tmp_path / "in.bin")
    with open(path, "wb") as f:
        for c in range(len(golden.colptr) - 1):
            b, e = golden.colptr[c], golden.colptr[c + 1]
            np.array([e - b], np.uint64).tofile(f)
            rec = np.empty((e - b, 2), np.int32)
            rec[:, 0] = golden.idx[b:e]
            rec[:, 1] = golden.w[b:e].view(np.int32)
            rec.tofile(f)
    ssm = C.Ssm.import_reference(golden.rp, path, ctx)
    out = str(tmp_path / "out.bin")
    ssm.export_reference(out)
    assert open(path, "rb").read() == open(out, "rb").read()


def test_ssm_import_rejects_corrupt_file(golden, ctx, tmp_path):
    path = str(tmp_path / "bad.bin")
    np.array([5], np.uint64).tofile(path)  # claims 5 entries, holds none
    with pytest.raises(C.CtbbError) as e:
        C.Ssm.import_reference(golden.rp, path, ctx)
    assert e.value.status == 10


# ----------------------------------------------------------- rotation ----
def test_rotate_matches_reference_final_image(golden, ctx):
    d = C.CtData(recon_volume=golden.iterations[-1].astype(np.float32), tube_angles=golden.data.tube_angles,
                 slice_indices=golden.data.slice_indices)
    C.rotate_slices_rotating2fixed(golden.rp, d, ctx)
    assert np.array_equal(d.recon_volume.view(np.int32), golden.final.view(np.int32))


def test_rotate_both_directions_match_port(wl, ctx):
    name, rp, data, _ = wl
    vol = np.random.default_rng(3).random(rp.shape, dtype=np.float32)
    for direction, fn in ((-1, C.rotate_slices_rotating2fixed), (1, C.rotate_slices_fixed2rotating)):
        d = C.CtData(recon_volume=vol.copy(), tube_angles=data.tube_angles, slice_indices=data.slice_indices)
        fn(rp, d, ctx)
        ref = O.port_rotate(rp, data.tube_angles, data.slice_indices, vol, direction)
        assert np.array_equal(d.recon_volume.view(np.int32), ref.view(np.int32)), (name, direction)


# ------------------------------------------------------ sequential ICD ----
def test_sequential_icd_matches_reference_iterations(golden, ctx):
    ssm = C.Ssm.generate(golden.rp, ctx, C.SSM_FP32)
    rc = C.Recon(golden.rp, golden.data.slice_indices, ctx)
    rc.set_raw(golden.raw)
    rc.set_volume(ssm, None)
    opts = C.icd_opts(mode=C.ICD_SEQUENTIAL)
    for it in range(golden.iterations.shape[0] - 1):
        rc.iterate(ssm, 1, opts)
        x = rc.volume_f64()
        ref = golden.iterations[it + 1]
        rel = np.linalg.norm(x - ref) / np.linalg.norm(ref)
        assert rel < 1e-5 and np.abs(x - ref).max() <= 1e-5 * np.abs(ref).max(), (it, rel)
        assert rel < 1e-12, (it, rel)  # only the alpha/beta summation order differs


def test_sequential_icd_matches_port(wl, ctx):
    name, rp, data, ref = wl
    ssm = C.Ssm.generate(rp, ctx, C.SSM_FP32)
    rc = C.Recon(rp, data.slice_indices, ctx)
    rc.set_raw(data.raw)
    rc.set_volume(ssm, None)
    dumps, _, _ = O.port_icd(rp, data.slice_indices, data.raw, ref, 3)
    for it in range(3):
        rc.iterate(ssm, 1, C.icd_opts(mode=C.ICD_SEQUENTIAL))
        x = rc.volume_f64()
        rel = np.linalg.norm(x - dumps[it]) / np.linalg.norm(dumps[it])
        assert rel < 1e-10, (name, it, rel)


def test_pipeline_stage_functions_reproduce_reference_output(golden, ctx):
    rp = C.configure_recon_params(golden.prm_path)
    data = C.load_raw(rp)
    C.initialize_recon_volume(rp, data)
    C.generate_system_matrix(rp, data, ctx)
    C.icd_iteration(rp, data, ctx)
    C.rotate_slices_rotating2fixed(rp, data, ctx)
    out = C.clean_up(rp, data)
    img = np.fromfile(out, np.float32).reshape(rp.shape)
    # FP64 iterates agree to ~1e-15; a float cast may flip one ulp.
    assert np.allclose(img, golden.final, rtol=1e-6, atol=1e-7)


# ------------------------------------------------ residual, cost, synth ----
def test_refresh_residual_and_cost_match_port(wl, ctx):
    name, rp, data, ref = wl
    ssm = C.Ssm.generate(rp, ctx, C.SSM_FP32)
    rng = np.random.default_rng(7)
    x0 = (0.2 * rng.random(rp.shape)).astype(np.float32)
    rc = C.Recon(rp, data.slice_indices, ctx)
    rc.set_raw(data.raw)
    rc.set_volume(ssm, x0)
    cost_ref, _, _ = O.port_cost(rp, data.slice_indices, data.raw, ref, x0.astype(np.float64))
    assert abs(rc.cost() - cost_ref) <= 1e-9 * abs(cost_ref), name
    # grouped representation: e = y - A x in FP32 after an FP64 refresh
    rc.iterate(ssm, 0, C.icd_opts(mode=C.ICD_GROUPED))
    rc.refresh_residual(ssm)
    assert abs(rc.cost() - cost_ref) <= 1e-5 * abs(cost_ref), name


def test_gpu_projector_matches_cpu(ctx, tmp_path):
    import ctypes

    prm, rp = W.materialise("small_ffs", str(tmp_path), raw=False)
    spec = W.phantom_spec("small_ffs")
    cpu = O.port_synth(rp, spec)
    sl = C.slice_tables(rp)
    rc = C.Recon(rp, sl.slice_indices, ctx)
    C.check(C.lib().ctbb_gpu_synth_raw(ctx.handle, ctypes.byref(rp.geom), ctypes.byref(spec),
                                       ctypes.c_void_p(rc.raw_device_ptr())))
    gpu = rc.raw()
    diff = np.abs(gpu - cpu)
    # libm rounding (exp/log/lgamma) can move a Poisson draw by one count in rare rays
    assert np.mean(diff == 0) > 0.99
    assert diff.max() < 0.05


# ------------------------------------------------------- grouped ICD ----
@pytest.fixture(scope="module")
def converged_cfg1_small(ctx, tmp_path_factory):
    """cfg1's scanner and quadratic penalty at 64 x 64 x 8: the converged
    plain sequential-order ICD image (30 iterations; iterations 20-60 agree
    to < 0.02 HU) and its FP64 cost."""
    prm, rp = W.materialise("cfg1_small", str(tmp_path_factory.mktemp("cfg1_small")))
    data = C.load_raw(rp)
    ssm = C.Ssm.generate(rp, ctx, C.SSM_BOTH)
    rc = C.Recon(rp, data.slice_indices, ctx)
    rc.set_raw(data.raw)
    rc.set_volume(ssm, None)
    rc.iterate(ssm, 30, C.icd_opts(mode=C.ICD_SEQUENTIAL))
    x_ref = rc.volume_f64()
    cost_ref = rc.cost()
    rc.free()
    return rp, data, ssm, x_ref, cost_ref


@pytest.mark.parametrize("weights,wpv,stage,pairs", [
    (C.SSM_FP32, 1, 0, 0), (C.SSM_FP16, 1, 0, 0), (C.SSM_FP16, 1, 0, -1), (C.SSM_FP32, 8, 0, 0), (C.SSM_FP16, 4, 0, 0),
    (C.SSM_FP16, 8, 0, 0), (C.SSM_FP16, 4, 0, -1), (C.SSM_FP16, 1, 1, 0), (C.SSM_FP32, 1, 2, 0),
    (C.SSM_FP16, 1, 3, 0), (C.SSM_FP32, 1, 3, 0), (C.SSM_FP16, 8, 4, 0), (C.SSM_FP16, 8, 5, 0),
    (C.SSM_FP16, 8, 6, 0)])
def test_grouped_icd_reaches_converged_cost(ctx, converged_cfg1_small, weights, wpv, stage, pairs):
    """FP16 with the streamed (one warp) or 4/8-warp kernels reads the
    matrix as entry pairs (pairs 0) or as single entries (pairs -1)."""
    rp, data, ssm, x_ref, cost_ref = converged_cfg1_small
    rc = C.Recon(rp, data.slice_indices, ctx)
    rc.set_raw(data.raw)
    rc.set_volume(ssm, None)
    costs = []
    for _ in range(6):
        rc.iterate(ssm, 5, C.icd_opts(mode=C.ICD_GROUPED, weights=weights, refresh_every=5, warps_per_voxel=wpv,
                                      stage_column=stage, entry_pairs=pairs))
        rc.refresh_residual(ssm)
        costs.append(rc.cost())
    x = rc.volume_f64()
    rmse_hu = np.sqrt(np.mean((x - x_ref) ** 2)) / HU
    assert all(b <= a * (1 + 1e-9) for a, b in zip(costs, costs[1:])), costs
    assert rmse_hu <= 0.5, rmse_hu
    assert abs(costs[-1] - cost_ref) <= 1e-6 * abs(cost_ref), (costs[-1], cost_ref)


@pytest.mark.parametrize("wpv", [4, 8])
def test_entry_pairs_match_single_entries(ctx, converged_cfg1_small, wpv):
    """One update in flight (the visiting order run one voxel at a time):
    the pair form of the FP16 matrix gives the same iterates as its single
    entries, up to the order of the FP32 partial sums (each thread sums a
    different share of the column)."""
    rp, data, ssm, _, _ = converged_cfg1_small
    out = {}
    for pairs in (0, -1):
        rc = C.Recon(rp, data.slice_indices, ctx)
        rc.set_raw(data.raw)
        rc.set_volume(ssm, None)
        rc.iterate(ssm, 2, C.icd_opts(mode=C.ICD_GROUPED, weights=C.SSM_FP16, warps_per_voxel=wpv,
                                      warps_in_flight=wpv, entry_pairs=pairs))
        out[pairs] = rc.volume_f64()
        rc.free()
    a, b = out[0], out[-1]
    assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b), np.linalg.norm(a - b) / np.linalg.norm(b)
    # runs of two detector rows make most pairs (a lone entry takes a pair too)
    info = ssm.info()
    assert info.nnz / 2 <= info.n_pairs <= 0.75 * info.nnz, (info.n_pairs, info.nnz)


@pytest.mark.parametrize("stage", [4, 5, 6])
@pytest.mark.parametrize("case", ["cfg1_small", "small_ffs"])
def test_bulk_staged_kernel_matches_cta_pairs(ctx, converged_cfg1_small, converged_small_ffs, case, stage):
    """One update in flight: the kernel whose entry pairs arrive in shared
    memory by bulk copy gives the iterates of the CTA kernel that loads the
    same pairs into registers, up to the order of the FP32 partial sums.
    cfg1_small's windows are longer than the shared-memory stage (3584
    pairs), so their tails take the streamed path as well."""
    rp, data, ssm, _, _ = converged_cfg1_small if case == "cfg1_small" else converged_small_ffs
    out = {}
    for st in (0, stage):
        rc = C.Recon(rp, data.slice_indices, ctx)
        rc.set_raw(data.raw)
        rc.set_volume(ssm, None)
        rc.iterate(ssm, 2, C.icd_opts(mode=C.ICD_GROUPED, weights=C.SSM_FP16, warps_per_voxel=8,
                                      warps_in_flight=8, stage_column=st))
        out[st] = rc.volume_f64()
        rc.free()
    a, b = out[stage], out[0]
    assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b), np.linalg.norm(a - b) / np.linalg.norm(b)


def test_batch_of_uneven_scans_converges(ctx, converged_cfg1_small, tmp_path):
    rp, data, ssm, x_ref, cost_ref = converged_cfg1_small
    scans = []
    for name in ("small", "small_ffs"):
        _, rpo = W.materialise(name, str(tmp_path / name))
        d = C.load_raw(rpo)
        s = C.Ssm.generate(rpo, ctx, C.SSM_BOTH)
        r = C.Recon(rpo, d.slice_indices, ctx)
        r.set_raw(d.raw)
        r.set_volume(s, None)
        scans.append((r, s, r.cost()))
    rc = C.Recon(rp, data.slice_indices, ctx)
    rc.set_raw(data.raw)
    rc.set_volume(ssm, None)
    batch = C.Batch([rc] + [r for r, _, _ in scans], [ssm] + [s for _, s, _ in scans], ctx)
    opts = C.icd_opts(mode=C.ICD_GROUPED, weights=C.SSM_FP32)
    total = int(np.prod(rp.shape)) + sum(int(np.prod(r.rp.shape)) for r, _, _ in scans)
    st = batch.iterate(15, opts)
    assert st.iterations == 15 and st.voxel_updates == 15 * total and st.device_ms > 0
    mid = []
    for r, s, _ in scans:
        r.refresh_residual(s)
        mid.append(r.cost())
    batch.iterate(15, opts)  # replays the captured iteration graph
    rc.refresh_residual(ssm)
    x = rc.volume_f64()
    rmse_hu = np.sqrt(np.mean((x - x_ref) ** 2)) / HU
    assert rmse_hu <= 0.5, rmse_hu
    assert abs(rc.cost() - cost_ref) <= 1e-6 * abs(cost_ref)
    for (r, s, c0), c15 in zip(scans, mid):
        r.refresh_residual(s)
        assert r.cost() < c15 < c0, (c0, c15, r.cost())
    batch.free()


@pytest.fixture(scope="module")
def converged_small_ffs(ctx, tmp_path_factory):
    """small_ffs (in-plane flying focal spot, edge-preserving penalty,
    32 x 32 x 6): the sequential-order ICD image run until it moves less than
    0.01 HU over 50 iterations, and its FP64 cost (the penalty is convex, so
    this optimum is the one any visiting order must reach)."""
    prm, rp = W.materialise("small_ffs", str(tmp_path_factory.mktemp("small_ffs_conv")))
    data = C.load_raw(rp)
    ssm = C.Ssm.generate(rp, ctx, C.SSM_BOTH)
    rc = C.Recon(rp, data.slice_indices, ctx)
    rc.set_raw(data.raw)
    rc.set_volume(ssm, None)
    prev, moved = None, None
    for _ in range(60):
        rc.iterate(ssm, 50, C.icd_opts(mode=C.ICD_SEQUENTIAL))
        x = rc.volume_f64()
        if prev is not None:
            moved = np.abs(x - prev).max() / HU
            if moved < 0.01:
                break
        prev = x
    assert moved is not None and moved < 0.01, moved
    x_ref, cost_ref = rc.volume_f64(), rc.cost()
    rc.free()
    return rp, data, ssm, x_ref, cost_ref


@pytest.mark.parametrize("weights,stage", [(C.SSM_FP32, 0), (C.SSM_FP16, 1), (C.SSM_FP16, 3), (C.SSM_FP16, 5),
                                           (C.SSM_FP16, 6)])
def test_grouped_edge_preserving_reaches_converged_cost(ctx, converged_small_ffs, weights, stage):
    rp, data, ssm, x_ref, cost_ref = converged_small_ffs
    rc = C.Recon(rp, data.slice_indices, ctx)
    rc.set_raw(data.raw)
    rc.set_volume(ssm, None)
    costs = []
    rmse_hu = None
    for _ in range(60):
        rc.iterate(ssm, 25, C.icd_opts(mode=C.ICD_GROUPED, weights=weights, refresh_every=5, stage_column=stage))
        rc.refresh_residual(ssm)
        costs.append(rc.cost())
        rmse_hu = np.sqrt(np.mean((rc.volume_f64() - x_ref) ** 2)) / HU
        if rmse_hu <= 0.1 and abs(costs[-1] - cost_ref) <= 1e-7 * abs(cost_ref):
            break
    assert all(b <= a * (1 + 1e-9) for a, b in zip(costs, costs[1:])), costs
    assert rmse_hu <= 0.5, rmse_hu
    assert abs(costs[-1] - cost_ref) <= 1e-6 * abs(cost_ref), (costs[-1], cost_ref)
    rc.free()


def test_initial_recon_path_start_matches_reference(golden, ctx, tmp_path):
    """A start from initial_recon_path (initialize_recon_volume.cpp:57-76)
    without wFBP: the reference keeps its sinogram estimate at zero
    (icd_iteration.cpp:47, 63); the parity mode does the same, and its first
    two iterations match the reference program's dumps."""
    from oracle import reference_run as R

    d = str(tmp_path)
    x0 = (golden.iterations[1] * 0.5).astype(np.float32)  # a non-zero start
    x0_path = os.path.join(d, "x0.img")
    x0.tofile(x0_path)
    text = open(golden.prm_path).read().replace(golden.dir, d)
    text = "\n".join(l for l in text.splitlines() if not l.startswith(("num_iterations", "initial_recon_path")))
    text += f"\nnum_iterations: 2\ninitial_recon_path: {x0_path}\n"
    prm_path = os.path.join(d, "start.prm")
    with open(prm_path, "w") as f:
        f.write(text)
    golden.raw.tofile(os.path.join(d, f"{golden.name}.bin"))
    rc_ref, stamps = R.run("O2", prm_path, d, threads=2)
    assert rc_ref == 0, stamps[-5:]

    rp = C.configure_recon_params(prm_path)
    data = C.load_raw(rp)
    C.initialize_recon_volume(rp, data)
    assert np.array_equal(data.recon_volume, x0)
    ssm = C.Ssm.generate(rp, ctx, C.SSM_FP32)
    rc = C.Recon(rp, data.slice_indices, ctx)
    rc.set_raw(data.raw)
    rc.set_volume(ssm, data.recon_volume, C.ESTIMATE_ZERO)
    for it in (1, 2):
        rc.iterate(ssm, 1, C.icd_opts(mode=C.ICD_SEQUENTIAL))
        ref = np.fromfile(os.path.join(d, "reconstructions", f"iteration{it}.rcn"), np.float64).reshape(rp.shape)
        x = rc.volume_f64()
        rel = np.linalg.norm(x - ref) / np.linalg.norm(ref)
        assert rel < 1e-12, (golden.name, it, rel)
    # The stage functions apply the same start in sequential mode.
    data2 = C.load_raw(rp)
    C.initialize_recon_volume(rp, data2)
    data2.system_matrix = ssm
    C.icd_iteration(rp, data2, ctx)
    assert np.allclose(data2.extra["volume_f64"], ref, rtol=1e-12, atol=1e-15)
    rc.free()


def test_stop_rel_change_uses_exact_cost(ctx, converged_cfg1_small):
    """The stopping rule compares exact FP64 costs (A x recomputed in FP64 in
    grouped mode): it stops once the relative change falls below the
    threshold, and the cost it reports is the oracle's FP64 cost of the image
    it returns."""
    rp, data, ssm, x_ref, cost_ref = converged_cfg1_small
    rc = C.Recon(rp, data.slice_indices, ctx)
    rc.set_raw(data.raw)
    rc.set_volume(ssm, None)
    st = rc.iterate(ssm, 200, C.icd_opts(mode=C.ICD_GROUPED, weights=C.SSM_FP32, stop_rel_change=1e-5))
    assert 1 < st.iterations < 200, st.iterations
    assert st.rel_change < 1e-5
    csr = O.Csr(*[np.asarray(a) for a in _ssm_arrays(ssm, rp)])
    oracle_cost, _, _ = O.port_cost(rp, data.slice_indices, data.raw, csr, rc.volume_f64())
    assert abs(st.cost - oracle_cost) <= 1e-9 * abs(oracle_cost), (st.cost, oracle_cost)
    rc.free()


def _ssm_arrays(ssm, rp):
    ncol = int(rp.geom.nx * rp.geom.ny)
    cols = [ssm.column(c) for c in range(ncol)]
    colptr = np.concatenate([[0], np.cumsum([c[0].size for c in cols])]).astype(np.int64)
    return colptr, np.concatenate([c[0] for c in cols]), np.concatenate([c[1] for c in cols])
