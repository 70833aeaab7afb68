"""Learned warm start for grouped ICD.

A small 3D residual CNN (libctbb_icd_b200: ctbb_cnn_*) is trained on pairs
(early ICD iterate, converged ICD iterate) that the GPU ICD itself produces on
seeded synthetic phantoms, both rotated to the fixed frame. At reconstruction
time the network's predicted correction is added to the early iterate
(ctbb_gpu_recon_warm_start), the voxels it moved most are revisited first
(priority passes over ctbb_gpu_recon_set_priority's subset), and plain grouped
ICD finishes the image. ICD from the initialize_recon_volume start remains the
fallback and the yardstick: every result is reported with its cost and its
RMSE in HU against the plain converged image.

Device memory for the training set and crops is held in torch tensors; all
arithmetic (ICD, rotation, the network's forward/backward passes and Adam)
runs in the library's CUDA kernels.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile
import time
from dataclasses import dataclass, field

import numpy as np

from . import workloads as W
from ._lib import check, lib, ptr

HU = W.MU_WATER / 1000.0  # one Hounsfield unit in cm^-1
DEFAULT_BLOCKS = 4
S_IN = 1.0 / W.MU_WATER          # network input: water -> 1
S_OUT = 10.0 / W.MU_WATER        # network target: 100 HU of correction -> 1
WEIGHTS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "warm_start.npz")


def _dev_ptr(t) -> C.c_void_p:
    import torch

    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
        raise TypeError("expected a contiguous float32 CUDA tensor")
    return C.c_void_p(t.data_ptr())


def _torch_sync():
    import torch

    torch.cuda.current_stream().synchronize()


class WarmStartNet:
    """Handle of the GPU network (ctbb_cnn_*). Volumes are [nz][ny][nx]
    float32 CUDA tensors."""

    def __init__(self, ctx, blocks: int = DEFAULT_BLOCKS, seed: int = 0):
        self.ctx = ctx
        self.blocks = int(blocks)
        h = C.c_void_p()
        check(lib().ctbb_cnn_create(ctx.handle, self.blocks, int(seed), C.byref(h)))
        self.handle = h
        self.set_scaling(S_IN, S_OUT)

    def set_engine(self, engine: int):
        """CNN_ENGINE_TCGEN05 or CNN_ENGINE_MMA_SYNC (default) for the 32 -> 32
        convolutions (ctbb_cnn_set_engine)."""
        check(lib().ctbb_cnn_set_engine(self.handle, int(engine)))

    @property
    def n_params(self) -> int:
        return int(lib().ctbb_cnn_num_params(self.handle))

    def params(self) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        check(lib().ctbb_cnn_get_params(self.handle, ptr(out, C.c_float), out.size))
        return out

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(lib().ctbb_cnn_set_params(self.handle, ptr(p, C.c_float), p.size))

    def set_scaling(self, s_in: float, s_out: float):
        check(lib().ctbb_cnn_set_scaling(self.handle, float(s_in), float(s_out)))

    def scaling(self):
        a, b = C.c_float(), C.c_float()
        check(lib().ctbb_cnn_get_scaling(self.handle, C.byref(a), C.byref(b)))
        return a.value, b.value

    def forward(self, x):
        import torch

        nz, ny, nx = x.shape
        out = torch.empty_like(x)
        _torch_sync()
        check(lib().ctbb_cnn_forward(self.handle, _dev_ptr(x), nx, ny, nz, _dev_ptr(out)))
        return out

    def accumulate_gradient(self, x, xc, weight=None) -> float:
        nz, ny, nx = x.shape
        loss = C.c_double()
        _torch_sync()
        check(lib().ctbb_cnn_accumulate_gradient(self.handle, _dev_ptr(x), _dev_ptr(xc),
                                                 None if weight is None else _dev_ptr(weight),
                                                 nx, ny, nz, C.byref(loss)))
        return loss.value

    def gradient(self) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        check(lib().ctbb_cnn_get_gradient(self.handle, ptr(out, C.c_float), out.size))
        return out

    def zero_gradient(self):
        check(lib().ctbb_cnn_zero_gradient(self.handle))

    def adam_step(self, lr: float, beta1=0.9, beta2=0.999, eps=1e-8, grad_scale=1.0):
        check(lib().ctbb_cnn_adam_step(self.handle, float(lr), float(beta1), float(beta2), float(eps),
                                       float(grad_scale)))

    # The network's input is the iterate after `n_early` grouped iterations
    # run with a fixed visiting-order tile edge and a fixed density of
    # concurrent updates (in-flight updates per voxel): the protocol its
    # training pairs were made with. early_opts() reproduces it on any volume.
    n_early = 3
    early_lattice = 32
    early_density = 2048.0 / (512 * 512 * 16)

    def early_opts(self, rc, base):
        import ctbb_icd_b200 as CB

        nvox = int(np.prod(rc.rp.shape))
        return CB.icd_opts(mode=base.mode, weights=base.weights, lattice=self.early_lattice,
                           warps_in_flight=max(32, int(round(self.early_density * nvox))))

    def save(self, path: str, **meta):
        s_in, s_out = self.scaling()
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        meta = dict(dict(n_early=self.n_early, early_lattice=self.early_lattice,
                         early_density=self.early_density), **meta)
        np.savez(path, params=self.params(), blocks=self.blocks, s_in=s_in, s_out=s_out,
                 **{k: np.asarray(v) for k, v in meta.items()})

    @classmethod
    def load(cls, ctx, path: str = WEIGHTS_PATH) -> "WarmStartNet":
        d = np.load(path)
        net = cls(ctx, int(d["blocks"]))
        net.set_params(d["params"])
        net.set_scaling(float(d["s_in"]), float(d["s_out"]))
        for k in ("n_early", "early_lattice"):
            if k in d:
                setattr(net, k, int(d[k]))
        if "early_density" in d:
            net.early_density = float(d["early_density"])
        return net

    def free(self):
        if getattr(self, "handle", None):
            lib().ctbb_cnn_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# --------------------------------------------------------------------------
# Scans and training pairs
# --------------------------------------------------------------------------
# Training geometry (the benchmark's config 5): cfg2's scanner, views, flying
# focal spot, phantom and penalty, reconstructed at 256 x 256 over cfg2's
# 30 cm field of view (1.17 mm voxels) with 32 slices of 0.6 mm, 3 turns.
# At inference the network runs on the same 256 x 256 grid: a full-size scan
# (512 x 512) gets its early iterations and the correction on a half-size
# grid of the same scan, and the corrected coarse image, upsampled 2x
# in-plane, becomes the start of the full-size ICD (warm_start_coarse).
TRAIN_WORKLOAD = "cfg2_train"
W.WORKLOADS[TRAIN_WORKLOAD] = dict(
    prm={**W.WORKLOADS["cfg2"]["prm"], "Readings": 3 * 2304,
         **W._recon(256, 30.0, 0.06, 32, -2.5, "edge-preserving", 0.1, 9.6e-4, 10)},
    phantom=dict(n_ellipsoids=40, seed=0, i0_lo=5e4, i0_hi=2e5),
)
# The 16-slice full-resolution slab of the earlier protocol (kept for
# comparison runs).
W.WORKLOADS["cfg2_slab"] = dict(
    prm={**W.WORKLOADS["cfg2"]["prm"], "Readings": 2 * 2304,
         **W._recon(512, 30.0, 0.06, 16, -2.0, "edge-preserving", 0.1, 9.6e-4, 10)},
    phantom=dict(n_ellipsoids=40, seed=0, i0_lo=5e4, i0_hi=2e5),
)


def coarse_workload(name: str) -> str:
    """Register (once) and return the half-resolution companion of a
    workload: same scan, slices and field of view, half the in-plane voxels."""
    cname = name + "_half"
    if cname not in W.WORKLOADS:
        w = W.workload(name)
        w["prm"]["nx"] = w["prm"]["nx"] // 2
        w["prm"]["ny"] = w["prm"]["ny"] // 2
        W.WORKLOADS[cname] = w
    return cname
# A phantom longer than the reconstructed slab makes the data inconsistent
# with the slab model: rays that leave the slab carry attenuation that ICD
# (the reference's and this one) can only place on in-slab voxels, and it
# lands in the grid-edge rows of the outer slices. Scans here cut the phantom
# to the slab (make_scan's clip); error figures also stay inside the object
# support (r < OBJECT_RADIUS_CM; the phantom reaches 12 cm) and skip
# EDGE_SLICES slices at each end.
OBJECT_RADIUS_CM = 13.0
EDGE_SLICES = 2


@dataclass
class Scan:
    rp: object
    tables: object
    rc: object
    ssm: object
    workdir: str
    fov_mask: np.ndarray = field(default=None)
    obj_mask: np.ndarray = field(default=None)

    def error_hu(self, x: np.ndarray, ref: np.ndarray) -> float:
        """RMSE in HU inside the object support on the interior slices."""
        return rmse_hu(x, ref, self.obj_mask, interior(x.shape[0]))


def fov_mask(rp) -> np.ndarray:
    """Voxels inside the scanner FOV (icd_iteration.cpp:181), per slice [ny][nx]."""
    g = rp.geom
    i = np.arange(int(g.num_voxels_x))
    j = np.arange(int(g.num_voxels_y))
    xx = (i[None, :] - g.center_voxel_x) * g.voxel_size_x
    yy = (j[:, None] - g.center_voxel_y) * g.voxel_size_y
    return (xx * xx + yy * yy) < (g.acquisition_fov / 2.0) ** 2


def workload_shape(name: str):
    """(nz, ny, nx) of a workload's reconstruction (host-side setup only)."""
    import ctbb_icd_b200 as CB

    w = W.workload(name)
    d = tempfile.mkdtemp(prefix="ctbb_shape_")
    w["prm"].update(sinogram_path=os.path.join(d, "raw.bin"), output_dir=d, output_file="out.img")
    return tuple(CB.configure_recon_params(W.write_prm(os.path.join(d, "s.prm"), w["prm"])).shape)


def make_scan(ctx, name: str, seed: int, ssm=None, weights=None, clip: bool = True, raw_from: "Scan" = None) -> Scan:
    """A workload's geometry with phantom seed `seed`: raw data from the GPU
    projector (phantom cut to the reconstructed slab unless clip=False), zero
    initial image. Reuses `ssm` when given (same geometry). With `raw_from`
    (a scan of the same acquisition on another grid) its raw frames are
    copied instead of projecting again."""
    import ctbb_icd_b200 as CB

    w = W.workload(name)
    w["phantom"]["seed"] = int(seed)
    prm = w["prm"]
    workdir = tempfile.mkdtemp(prefix="ctbb_scan_")
    prm.update(sinogram_path=os.path.join(workdir, "raw.bin"), output_dir=workdir, output_file="out.img")
    open(prm["sinogram_path"], "wb").close()
    rp = CB.configure_recon_params(W.write_prm(os.path.join(workdir, "scan.prm"), prm))
    tables = CB.slice_tables(rp)
    spec = W.phantom_spec(w["phantom"])
    spec.ellipsoid_z_lo = min(prm["z_start"], prm["z_end"])
    spec.ellipsoid_z_hi = max(prm["z_start"], prm["z_end"])
    if clip:
        spec.clip_z_lo, spec.clip_z_hi = W.slab_clip(rp, tables.slice_locations)
    rc = CB.Recon(rp, tables.slice_indices, ctx)
    if raw_from is not None:
        rc.set_raw_device(raw_from.rc.raw_device_ptr())
    else:
        check(lib().ctbb_gpu_synth_raw(ctx.handle, C.byref(rp.geom), C.byref(spec),
                                       C.c_void_p(rc.raw_device_ptr())))
    if ssm is None:
        ssm = CB.Ssm.generate(rp, ctx, weights if weights is not None else CB.SSM_FP32)
    rc.set_volume(ssm, None)
    return Scan(rp, tables, rc, ssm, workdir, fov_mask(rp), object_mask(rp))


def object_mask(rp, radius_cm: float = OBJECT_RADIUS_CM) -> np.ndarray:
    """In-plane disc [ny][nx] of radius `radius_cm` about the rotation axis."""
    g = rp.geom
    i = np.arange(int(g.num_voxels_x))
    j = np.arange(int(g.num_voxels_y))
    xx = (i[None, :] - g.center_voxel_x) * g.voxel_size_x
    yy = (j[:, None] - g.center_voxel_y) * g.voxel_size_y
    return (xx * xx + yy * yy) < radius_cm * radius_cm


def interior(nz: int, edge: int = EDGE_SLICES) -> slice:
    e = edge if nz > 2 * edge else 0
    return slice(e, nz - e)


def rmse_hu(x: np.ndarray, ref: np.ndarray, mask2d: np.ndarray, slices: slice | None = None) -> float:
    """RMSE in HU over mask2d on every slice (or the given slices)."""
    d = (np.asarray(x, np.float64) - np.asarray(ref, np.float64))
    if slices is not None:
        d = d[slices]
    d = d[:, mask2d]
    return float(np.sqrt(np.mean(d * d)) / HU)


def to_fixed(ctx, scan: Scan, vol: np.ndarray) -> np.ndarray:
    import ctbb_icd_b200 as CB

    out = np.ascontiguousarray(vol, dtype=np.float32).copy()
    check(lib().ctbb_gpu_rotate(ctx.handle, C.byref(scan.rp.geom), ptr(scan.tables.tube_angles, C.c_double),
                                ptr(scan.tables.slice_indices, C.c_uint64), ptr(out, C.c_float),
                                CB.ROTATE_ROTATING2FIXED))
    return out


def converge(scan: Scan, opts, max_iter: int = 400, rel: float = 1e-7, refresh_every: int = 10):
    """Plain grouped ICD until the FP64 cost changes by less than `rel` per
    iteration (cost after an FP64 residual refresh every `refresh_every`
    iterations). Returns the iterations run."""
    prev = None
    it = 0
    while it < max_iter:
        n = min(refresh_every, max_iter - it)
        scan.rc.iterate(scan.ssm, n, opts)
        it += n
        scan.rc.refresh_residual(scan.ssm)
        c = scan.rc.cost()
        if prev is not None and abs(prev - c) / abs(c) < rel * n:
            break
        prev = c
    return it


def make_pairs(ctx, seeds, n_early: int = 3, name: str = TRAIN_WORKLOAD, opts=None, max_iter: int = 400,
               log=print, early_opts=None):
    """(early iterate, converged iterate) pairs in the fixed frame, float32
    numpy [n][nz'][ny][nx] over the interior slices, plus the in-plane loss
    mask (object support) of the geometry."""
    import ctbb_icd_b200 as CB

    opts = opts or CB.icd_opts(mode=CB.ICD_GROUPED, weights=CB.SSM_FP32)
    ssm = None
    xs, xcs = [], []
    mask = None
    for s in seeds:
        t0 = time.time()
        scan = make_scan(ctx, name, s, ssm)
        ssm = scan.ssm
        scan.rc.iterate(ssm, n_early, early_opts(scan.rc) if early_opts else opts)
        x_early = scan.rc.volume()
        n = converge(scan, opts, max_iter=max_iter)
        xc = scan.rc.volume()
        sl = interior(xc.shape[0])
        xs.append(to_fixed(ctx, scan, x_early)[sl])
        xcs.append(to_fixed(ctx, scan, xc)[sl])
        mask = scan.obj_mask
        log(f"seed {s}: converged after {n + n_early} iterations, early->converged "
            f"{scan.error_hu(x_early, xc):.1f} HU ({time.time() - t0:.1f} s)")
        scan.rc.free()
    return np.stack(xs), np.stack(xcs), mask


def warm_start_coarse(fine: Scan, coarse: Scan, net: WarmStartNet, n_early: int, coarse_opts):
    """The learned start of a full-size scan: n_early grouped iterations from
    zero on the half-size grid of the same scan (the network's training
    grid), the network's correction there (ctbb_gpu_recon_warm_start), then
    that image upsampled 2x in-plane as the full-size iterate with
    e = y - A x refreshed in FP64 (ctbb_gpu_recon_set_volume_upsampled)."""
    coarse.rc.set_volume(coarse.ssm, None)
    coarse.rc.iterate(coarse.ssm, n_early, net.early_opts(coarse.rc, coarse_opts))
    coarse.rc.warm_start(coarse.ssm, net, coarse.tables.tube_angles)
    fine.rc.set_volume_upsampled(fine.ssm, coarse.rc)


def tuned_opts(ctx, name: str = TRAIN_WORKLOAD, n_early: int = 3, seed: int = 0, log=print):
    """Autotuned grouped-ICD options for a geometry, probed after n_early
    iterations of a seeded scan."""
    import ctbb_icd_b200 as CB

    scan = make_scan(ctx, name, seed)
    base = CB.icd_opts(mode=CB.ICD_GROUPED, weights=CB.SSM_FP32)
    scan.rc.iterate(scan.ssm, n_early, base)
    best, trials = scan.rc.autotune(scan.ssm, base, probe_iters=2)
    if log:
        log(f"autotune {name}: warps {best.warps_in_flight}, tile {best.lattice} "
            f"({len(trials)} trials)")
    scan.rc.free()
    return best, trials


def train(net: WarmStartNet, x_early: np.ndarray, x_conv: np.ndarray, mask2d: np.ndarray, steps: int = 1500,
          batch: int = 4, crop=(8, 128, 128), lr: float = 1e-3, lr_min: float = 1e-4, seed: int = 0,
          log=print, log_every: int = 100):
    """Adam on random crops of the training pairs (cosine learning-rate decay)."""
    import torch

    dev = torch.device("cuda", torch.cuda.current_device())
    X = torch.from_numpy(np.ascontiguousarray(x_early, np.float32)).to(dev)
    Y = torch.from_numpy(np.ascontiguousarray(x_conv, np.float32)).to(dev)
    M = torch.from_numpy(mask2d.astype(np.float32)).to(dev)
    n, nz, ny, nx = X.shape
    cz, cy, cx = min(crop[0], nz), min(crop[1], ny), min(crop[2], nx)
    g = np.random.default_rng(seed)
    hist = []
    for step in range(steps):
        loss = 0.0
        for _ in range(batch):
            i = int(g.integers(n))
            z = int(g.integers(nz - cz + 1))
            y = int(g.integers(ny - cy + 1))
            x = int(g.integers(nx - cx + 1))
            xb = X[i, z:z + cz, y:y + cy, x:x + cx].contiguous()
            yb = Y[i, z:z + cz, y:y + cy, x:x + cx].contiguous()
            mb = M[y:y + cy, x:x + cx].expand(cz, cy, cx).contiguous()
            if float(mb.sum()) == 0.0:
                mb = torch.ones_like(mb)
            loss += net.accumulate_gradient(xb, yb, mb)
        lr_t = lr_min + 0.5 * (lr - lr_min) * (1 + np.cos(np.pi * step / max(1, steps)))
        net.adam_step(lr_t, grad_scale=1.0 / batch)
        hist.append(loss / batch)
        if log and (step % log_every == 0 or step == steps - 1):
            log(f"step {step}: loss {np.mean(hist[-log_every:]):.5f} lr {lr_t:.2e}")
    return hist


def eval_loss(net: WarmStartNet, x_early: np.ndarray, x_conv: np.ndarray, mask2d: np.ndarray) -> float:
    """Mean weighted loss over whole volumes (the gradient buffer is cleared)."""
    import torch

    dev = torch.device("cuda", torch.cuda.current_device())
    M = torch.from_numpy(mask2d.astype(np.float32)).to(dev)
    tot = 0.0
    for xe, xc in zip(x_early, x_conv):
        xb = torch.from_numpy(np.ascontiguousarray(xe, np.float32)).to(dev)
        yb = torch.from_numpy(np.ascontiguousarray(xc, np.float32)).to(dev)
        tot += net.accumulate_gradient(xb, yb, M.expand(*xb.shape).contiguous())
    net.zero_gradient()
    return tot / len(x_early)


# --------------------------------------------------------------------------
# Time to <= tol HU: plain vs learned warm start
# --------------------------------------------------------------------------
def _timed(fn):
    import torch

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = fn()
    torch.cuda.synchronize()
    return r, time.perf_counter() - t0


def time_to_tolerance(scan: Scan, x_ref: np.ndarray, opts, tol_hu: float = 0.5, max_iter: int = 200,
                      net: WarmStartNet | None = None, n_early: int = 3, prio_fraction: float = 0.2,
                      prio_passes: int = 2, refresh_every: int = 10, coarse: Scan | None = None,
                      coarse_opts=None, tols=()):
    """Iterate from the zero start until RMSE(x, x_ref) <= tol_hu inside the
    object support on the interior slices (Scan.error_hu). With `net`, after
    n_early plain iterations the warm start is applied and `prio_passes`
    passes over the top `prio_fraction` voxels run before plain iterations
    resume; with `net` and `coarse` (the scan's half-size grid) the start is
    warm_start_coarse instead. Returns the wall time of the reconstruction
    work (RMSE checks excluded), the full iterations run, the trace and the
    time at which each tolerance in `tols` was first met."""
    import ctbb_icd_b200 as CB

    scan.rc.set_volume(scan.ssm, None)
    elapsed = 0.0
    trace = []
    it = 0
    first = {}

    def check_done(label):
        e = scan.error_hu(scan.rc.volume(), x_ref)
        trace.append((label, elapsed, e))
        for t in tols:
            if e <= t and t not in first:
                first[t] = elapsed
        return e <= tol_hu

    def result(reached):
        return {"seconds": elapsed, "iterations": it, "trace": trace, "reached": reached,
                "seconds_to": {str(t): first.get(t) for t in tols}}

    if net is not None and coarse is not None:
        _, dt = _timed(lambda: warm_start_coarse(scan, coarse, net, n_early, coarse_opts or opts))
        elapsed += dt
        if check_done(f"coarse x{n_early} + network + upsample"):
            return result(True)
    elif net is not None:
        eopts = net.early_opts(scan.rc, opts)
        _, dt = _timed(lambda: scan.rc.iterate(scan.ssm, n_early, eopts))
        elapsed += dt
        it += n_early
        check_done(f"plain x{n_early}")
        _, dt = _timed(lambda: scan.rc.warm_start(scan.ssm, net, scan.tables.tube_angles))
        elapsed += dt
        done = check_done("warm start")
        if not done and prio_passes > 0 and prio_fraction > 0:
            popts = CB.icd_opts(mode=opts.mode, weights=opts.weights, warps_in_flight=opts.warps_in_flight,
                                lattice=opts.lattice, relax=opts.relax, priority=True)
            _, dt = _timed(lambda: (scan.rc.set_priority(prio_fraction, popts),
                                    scan.rc.iterate(scan.ssm, prio_passes, popts)))
            elapsed += dt
            done = check_done(f"priority x{prio_passes} @ {prio_fraction}")
        if done:
            return result(True)
    while it < max_iter:
        refresh = refresh_every > 0 and it > 0 and it % refresh_every == 0

        def step():
            if refresh:
                scan.rc.refresh_residual(scan.ssm)
            return scan.rc.iterate(scan.ssm, 1, opts)

        _, dt = _timed(step)
        elapsed += dt
        it += 1
        if check_done(f"iter {it}"):
            return result(True)
    return result(False)
