"""B200-native reconstruction path for CTBB_ICD.

Python mirror of the reference program's stage functions (src/main.cpp:88-128):

    rp   = configure_recon_params(prm_path)          # setup.cpp:69
    data = load_raw(rp)                              # setup.cpp:245
    initialize_recon_volume(rp, data)                # initialize_recon_volume.cpp:51
    generate_system_matrix(rp, data)                 # generate_system_matrix[_ffs].cpp
    icd_iteration(rp, data)                          # icd_iteration.cpp:42
    rotate_slices_rotating2fixed(rp, data)           # rotate_slices.cpp:81
    clean_up(rp, data)                               # setup.cpp:422

Same argument meaning as the reference; errors raise CtbbError (the
reference printed a message and exited). All numerical work runs in the CUDA
kernels of libctbb_icd_b200.so; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from ._lib import (  # noqa: F401
    CNN_ENGINE_MMA_SYNC, CNN_ENGINE_TCGEN05, ESTIMATE_FORWARD, ESTIMATE_ZERO, ICD_GROUPED, ICD_SEQUENTIAL, PENALTY_EDGE_PRESERVING, PENALTY_QUADRATIC,
    ROTATE_FIXED2ROTATING, ROTATE_ROTATING2FIXED, SSM_BOTH, SSM_FP16, SSM_FP32, CtbbError,
    GeomC, IcdOpts, IterStats, PhantomSpec, PrmStrings, SsmInfo, check, lib, ptr,
)

__all__ = [
    "ReconParams", "CtData", "Context", "Ssm", "Recon", "CtbbError",
    "configure_recon_params", "load_raw", "initialize_recon_volume", "generate_system_matrix",
    "generate_system_matrix_ffs", "icd_iteration", "rotate_slices_rotating2fixed",
    "rotate_slices_fixed2rotating", "clean_up", "synth_raw_host", "write_raw_file",
    "slice_tables", "icd_opts", "WarmStartNet",
]


@dataclass
class ReconParams:
    """recon_params: numeric fields in `geom` (ctbb_geom_c), strings beside it."""

    geom: GeomC
    initial_recon_path: str = ""
    matrix_path: str = ""
    output_dir: str = ""
    output_file: str = ""
    potential: str = ""
    recon_path: str = ""
    sinogram_path: str = ""
    penalty: str = "quadratic"

    def __getattr__(self, name):
        geom = self.__dict__.get("geom")
        if geom is not None and name != "geom":
            key = "lambda_" if name == "lambda" else name
            return getattr(geom, key)
        raise AttributeError(name)

    @property
    def shape(self):
        g = self.geom
        return (int(g.num_voxels_z), int(g.num_voxels_y), int(g.num_voxels_x))

    @property
    def raw_shape(self):
        g = self.geom
        return (int(g.Readings), int(g.n_channels), int(g.Nrows_projection))


@dataclass
class CtData:
    """ct_data (recon_structs.h:116-125) as numpy arrays."""

    raw: np.ndarray | None = None             # float32 [Readings][n_channels][Nrows]
    recon_volume: np.ndarray | None = None    # float32 [nz][ny][nx]
    tube_angles: np.ndarray | None = None     # float64 degrees [Readings]
    table_positions: np.ndarray | None = None  # float64 cm [Readings]
    slice_locations: np.ndarray | None = None  # float64 cm [nz]
    slice_indices: np.ndarray | None = None    # uint64 [nz]
    system_matrix: "Ssm | None" = None         # device-resident SSM
    extra: dict = field(default_factory=dict)


def configure_recon_params(prm_path: str) -> ReconParams:
    """setup.cpp:69-243: parse, check required fields, apply defaults, derive."""
    g, s = GeomC(), PrmStrings()
    check(lib().ctbb_configure_recon_params(str(prm_path).encode(), C.byref(g), C.byref(s)))
    dec = lambda b: b.decode()  # noqa: E731
    return ReconParams(
        geom=g, initial_recon_path=dec(s.initial_recon_path), matrix_path=dec(s.matrix_path),
        output_dir=dec(s.output_dir), output_file=dec(s.output_file), potential=dec(s.potential),
        recon_path=dec(s.recon_path), sinogram_path=dec(s.sinogram_path), penalty=dec(s.penalty))


def slice_tables(rp: ReconParams, *, allow_bad_range: bool = False) -> CtData:
    """Tube angles, table positions and rotating-slice tables (setup.cpp:273-409)."""
    g = rp.geom
    n = int(g.Readings)
    ta = np.zeros(n, np.float64)
    tp = np.zeros(n, np.float64)
    cap = max(1, int(abs(g.z_end - g.z_start) / g.voxel_size_z) + 2)
    sl = np.zeros(cap, np.float64)
    si = np.zeros(cap, np.uint64)
    st = lib().ctbb_slice_tables(C.byref(g), ptr(ta, C.c_double), ptr(tp, C.c_double),
                                 ptr(sl, C.c_double), ptr(si, C.c_uint64), cap)
    if not (allow_bad_range and st == 4):
        check(st)
    nz = int(g.num_voxels_z)
    return CtData(tube_angles=ta, table_positions=tp, slice_locations=sl[:nz].copy(),
                  slice_indices=si[:nz].copy())


def load_raw(rp: ReconParams, *, raw: np.ndarray | None = None) -> CtData:
    """setup.cpp:245-420 for FileType 0; `raw` bypasses the file read."""
    data = slice_tables(rp)
    if raw is None:
        if not os.path.exists(rp.sinogram_path):
            raise CtbbError(3, f"Raw data file not found: {rp.sinogram_path}")
        raw = np.empty(rp.raw_shape, np.float32)
        check(lib().ctbb_read_raw(rp.sinogram_path.encode(), C.byref(rp.geom), ptr(raw, C.c_float)))
    data.raw = np.ascontiguousarray(raw, dtype=np.float32).reshape(rp.raw_shape)
    data.recon_volume = np.zeros(rp.shape, np.float32)
    return data


def initialize_recon_volume(rp: ReconParams, data: CtData) -> None:
    """initialize_recon_volume.cpp:51-184: zeros, or a float32 volume from
    initial_recon_path. The wFBP path needs the external ctbb_recon program,
    which is not part of this build."""
    if rp.initial_recon_path:
        if not os.path.exists(rp.initial_recon_path):
            raise CtbbError(3, "Specified initial reconstruction file not found")
        vol = np.fromfile(rp.initial_recon_path, np.float32)
        if vol.size < int(np.prod(rp.shape)):
            raise CtbbError(3, "Could not initialize reconstruction volume from given file")
        data.recon_volume = vol[: int(np.prod(rp.shape))].reshape(rp.shape).copy()
    elif int(rp.geom.wfbp_initialize) != 0:
        raise CtbbError(9, "wFBP initialisation needs the external ctbb_recon program")
    else:
        data.recon_volume = np.zeros(rp.shape, np.float32)


def synth_raw_host(rp: ReconParams, phantom: dict, n_threads: int = 1) -> np.ndarray:
    """Seeded synthetic raw frames on the CPU (stands in for ctbb_read)."""
    from .workloads import phantom_spec

    g = GeomC.from_buffer_copy(rp.geom)
    slice_tables(ReconParams(geom=g), allow_bad_range=True)  # sets z_first_view, table_direction
    spec = phantom_spec(phantom)
    raw = np.empty(rp.raw_shape, np.float32)
    check(lib().ctbb_synth_raw_host(C.byref(g), C.byref(spec), ptr(raw, C.c_float), int(n_threads)))
    return raw


def write_raw_file(path: str, rp: ReconParams, raw: np.ndarray) -> None:
    raw = np.ascontiguousarray(raw, dtype=np.float32)
    check(lib().ctbb_write_raw_file(str(path).encode(), C.byref(rp.geom), ptr(raw, C.c_float)))


# --------------------------------------------------------------------------
# GPU objects
# --------------------------------------------------------------------------
class Context:
    """One CUDA device + stream (ctbb_gpu_init)."""

    def __init__(self, device: int = 0, stream=None):
        h = C.c_void_p()
        check(lib().ctbb_gpu_init(int(device), stream, C.byref(h)))
        self.handle = h

    @property
    def stream(self) -> int:
        return lib().ctbb_gpu_stream(self.handle) or 0

    def synchronize(self):
        check(lib().ctbb_gpu_synchronize(self.handle))

    def close(self):
        if self.handle:
            lib().ctbb_gpu_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Context | None = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


class Ssm:
    """Device-resident stored system matrix."""

    def __init__(self, handle, ctx: Context):
        self.handle, self.ctx = handle, ctx

    @classmethod
    def generate(cls, rp: ReconParams, ctx: Context | None = None, weights: int = SSM_BOTH):
        ctx = ctx or default_context()
        h = C.c_void_p()
        check(lib().ctbb_gpu_generate_ssm(ctx.handle, C.byref(rp.geom), int(weights), C.byref(h)))
        return cls(h, ctx)

    @classmethod
    def import_reference(cls, rp: ReconParams, path: str, ctx: Context | None = None,
                         weights: int = SSM_BOTH):
        ctx = ctx or default_context()
        h = C.c_void_p()
        check(lib().ctbb_gpu_ssm_import_reference(ctx.handle, C.byref(rp.geom), str(path).encode(),
                                                  int(weights), C.byref(h)))
        return cls(h, ctx)

    def info(self) -> SsmInfo:
        i = SsmInfo()
        check(lib().ctbb_gpu_ssm_info(self.handle, C.byref(i)))
        return i

    def column(self, c: int):
        n = C.c_uint64()
        check(lib().ctbb_gpu_ssm_column(self.handle, int(c), None, None, 0, C.byref(n)))
        idx = np.empty(n.value, np.int32)
        w = np.empty(n.value, np.float32)
        check(lib().ctbb_gpu_ssm_column(self.handle, int(c), ptr(idx, C.c_int32), ptr(w, C.c_float),
                                        n.value, C.byref(n)))
        return idx, w

    def export_reference(self, path: str):
        check(lib().ctbb_gpu_ssm_export_reference(self.handle, str(path).encode()))

    def free(self):
        if self.handle:
            lib().ctbb_gpu_ssm_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def icd_opts(mode=ICD_GROUPED, weights=SSM_FP32, refresh_every=0, warps_in_flight=0, lattice=0,
             compute_cost=False, stop_rel_change=0.0, relax=0.0, priority=False,
             warps_per_voxel=1, entries_per_lane=0, stage_column=0, entry_pairs=0, stack_align=0,
             l2_hints=0) -> IcdOpts:
    o = IcdOpts()
    o.mode, o.weights, o.refresh_every = int(mode), int(weights), int(refresh_every)
    o.warps_in_flight, o.lattice = int(warps_in_flight), int(lattice)
    o.compute_cost, o.stop_rel_change = int(bool(compute_cost)), float(stop_rel_change)
    o.relax = float(relax)
    o.priority = int(bool(priority))
    o.warps_per_voxel = int(warps_per_voxel)
    o.entries_per_lane = int(entries_per_lane)
    o.stage_column = int(stage_column)
    o.entry_pairs = int(entry_pairs)
    o.stack_align = int(stack_align)
    o.l2_hints = int(l2_hints)
    return o


def penalty_steps(ctx: "Context", penalty: int, lam: float, delta: float, alpha: np.ndarray, beta: np.ndarray,
                  x9: np.ndarray) -> np.ndarray:
    """The grouped mode's penalised one-voxel update on given inputs
    (ctbb_gpu_penalty_steps): alpha, beta [n]; x9 [n, 9] = voxel value and
    its 8 in-plane neighbours (NaN: outside the volume)."""
    a = np.ascontiguousarray(alpha, np.float64)
    b = np.ascontiguousarray(beta, np.float64)
    x = np.ascontiguousarray(x9, np.float32).reshape(-1, 9)
    out = np.empty(a.size, np.float64)
    check(lib().ctbb_gpu_penalty_steps(ctx.handle, int(penalty), float(lam), float(delta), a.size,
                                       ptr(a, C.c_double), ptr(b, C.c_double), ptr(x, C.c_float),
                                       ptr(out, C.c_double)))
    return out


class Recon:
    """Device-resident ICD state (raw y, image x, error sinogram e)."""

    def __init__(self, rp: ReconParams, slice_indices: np.ndarray, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self.rp = rp
        self.slice_indices = np.ascontiguousarray(slice_indices, dtype=np.uint64)
        h = C.c_void_p()
        check(lib().ctbb_gpu_recon_create(self.ctx.handle, C.byref(rp.geom),
                                          ptr(self.slice_indices, C.c_uint64), C.byref(h)))
        self.handle = h

    def set_raw(self, raw: np.ndarray):
        raw = np.ascontiguousarray(raw, dtype=np.float32)
        check(lib().ctbb_gpu_recon_set_raw(self.handle, ptr(raw, C.c_float)))

    def set_raw_device(self, dev_ptr: int):
        check(lib().ctbb_gpu_recon_set_raw_device(self.handle, C.c_void_p(dev_ptr)))

    def raw(self) -> np.ndarray:
        out = np.empty(self.rp.raw_shape, np.float32)
        check(lib().ctbb_gpu_recon_get_raw(self.handle, ptr(out, C.c_float)))
        return out

    def raw_device_ptr(self) -> int:
        return lib().ctbb_gpu_recon_raw_device(self.handle) or 0

    def set_volume(self, ssm: Ssm, vol: np.ndarray | None = None, estimate: int = ESTIMATE_FORWARD):
        """Set the iterate (zeros if vol is None) and the sinogram estimate:
        ESTIMATE_FORWARD y_hat = A x, ESTIMATE_ZERO y_hat = 0 (the reference's
        start for every initial image but a wFBP one)."""
        v = None if vol is None else np.ascontiguousarray(vol, dtype=np.float32)
        check(lib().ctbb_gpu_recon_set_volume_estimate(self.handle, ssm.handle, ptr(v, C.c_float), int(estimate)))

    def set_volume_upsampled(self, ssm: Ssm, coarse: "Recon"):
        """Start from `coarse`'s image (half the in-plane size, same scan,
        slices and FOV) upsampled 2x in-plane; e = y - A x refreshed in FP64."""
        check(lib().ctbb_gpu_recon_set_volume_upsampled(self.handle, ssm.handle, coarse.handle))

    def volume(self) -> np.ndarray:
        out = np.empty(self.rp.shape, np.float32)
        check(lib().ctbb_gpu_recon_get_volume(self.handle, ptr(out, C.c_float)))
        return out

    def volume_f64(self) -> np.ndarray:
        out = np.empty(self.rp.shape, np.float64)
        check(lib().ctbb_gpu_recon_get_volume_f64(self.handle, ptr(out, C.c_double)))
        return out

    def iterate(self, ssm: Ssm, n_iter: int, opts: IcdOpts | None = None) -> IterStats:
        st = IterStats()
        o = opts or icd_opts()
        check(lib().ctbb_gpu_recon_iterate(self.handle, ssm.handle, C.byref(o), int(n_iter), C.byref(st)))
        return st

    def entries(self, ssm: Ssm) -> float:
        """In-range matrix entries one iteration visits (sum over voxels)."""
        e = C.c_double()
        check(lib().ctbb_gpu_recon_entries(self.handle, ssm.handle, C.byref(e)))
        return e.value

    def refresh_residual(self, ssm: Ssm):
        check(lib().ctbb_gpu_recon_refresh_residual(self.handle, ssm.handle))

    def cost(self) -> float:
        c = C.c_double()
        check(lib().ctbb_gpu_recon_cost(self.handle, C.byref(c)))
        return c.value

    def autotune(self, ssm: Ssm, opts: IcdOpts | None = None, probe_iters: int = 2):
        """Pick warps in flight and the visiting-order tile edge by measured
        cost decrease per device second (ctbb_gpu_recon_autotune). Returns
        (tuned opts, list of trial dicts); the iterate is left unchanged."""
        from ._lib import TuneReport

        best, rep = IcdOpts(), TuneReport()
        check(lib().ctbb_gpu_recon_autotune(self.handle, ssm.handle, C.byref(opts or icd_opts()),
                                            int(probe_iters), C.byref(best), C.byref(rep)))
        trials = [dict(warps_in_flight=t.warps_in_flight, warps_per_voxel=t.warps_per_voxel,
                       entries_per_lane=t.entries_per_lane, stage_column=t.stage_column,
                       entry_pairs=t.entry_pairs, lattice=t.lattice,
                       device_ms=t.device_ms,
                       cost=t.cost, score=t.score, best=(i == rep.best))
                  for i, t in enumerate(rep.trials[:rep.n_trials])]
        return best, trials

    def warm_start(self, ssm: Ssm, net, tube_angles: np.ndarray):
        """Add the network's predicted correction to the current iterate
        (fixed-frame prediction, rotated back), refresh e = y - Ax and keep the
        per-voxel step as the priority map (ctbb_gpu_recon_warm_start)."""
        ta = np.ascontiguousarray(tube_angles, dtype=np.float64)
        check(lib().ctbb_gpu_recon_warm_start(self.handle, ssm.handle, net.handle, ptr(ta, C.c_double)))

    def set_priority(self, fraction: float, opts: IcdOpts | None = None):
        """Priority passes (icd_opts(priority=True)) visit the `fraction` of
        voxels with the largest warm-start step."""
        o = opts or icd_opts()
        check(lib().ctbb_gpu_recon_set_priority(self.handle, C.byref(o), float(fraction)))

    def free(self):
        if self.handle:
            lib().ctbb_gpu_recon_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Batch:
    """Independent reconstructions advanced together by one persistent launch
    per iteration (ctbb_gpu_batch_*), replayed from a CUDA graph."""

    def __init__(self, recons: list, ssms: list, ctx: Context | None = None):
        self.ctx = ctx or recons[0].ctx
        self.recons, self.ssms = list(recons), list(ssms)
        rs = (C.c_void_p * len(recons))(*[r.handle.value for r in recons])
        ss = (C.c_void_p * len(ssms))(*[s.handle.value for s in ssms])
        h = C.c_void_p()
        check(lib().ctbb_gpu_batch_create(self.ctx.handle, len(recons), rs, ss, C.byref(h)))
        self.handle = h

    def iterate(self, n_iter: int, opts: IcdOpts | None = None) -> IterStats:
        st = IterStats()
        check(lib().ctbb_gpu_batch_iterate(self.handle, C.byref(opts or icd_opts()), int(n_iter), C.byref(st)))
        return st

    def free(self):
        if self.handle:
            lib().ctbb_gpu_batch_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# --------------------------------------------------------------------------
# Stage functions with the reference's names
# --------------------------------------------------------------------------
def generate_system_matrix(rp: ReconParams, data: CtData, ctx: Context | None = None,
                           weights: int = SSM_BOTH) -> Ssm:
    """generate_system_matrix.cpp:54 / generate_system_matrix_ffs.cpp:60 on the GPU.
    The in-plane FFS model is selected from rp.Phiffs, as main.cpp:103-109 does."""
    data.system_matrix = Ssm.generate(rp, ctx, weights)
    return data.system_matrix


generate_system_matrix_ffs = generate_system_matrix


def icd_iteration(rp: ReconParams, data: CtData, ctx: Context | None = None,
                  opts: IcdOpts | None = None, n_iter: int | None = None) -> IterStats:
    """icd_iteration.cpp:42-286: num_iterations ICD passes; data.recon_volume in/out."""
    if data.system_matrix is None:
        raise CtbbError(1, "generate_system_matrix must run before icd_iteration")
    ctx = ctx or data.system_matrix.ctx
    rc = Recon(rp, data.slice_indices, ctx)
    try:
        o = opts or icd_opts(mode=ICD_SEQUENTIAL)
        rc.set_raw(data.raw)
        # icd_iteration.cpp:47-63: in parity mode the estimate is zero unless
        # the start is a wFBP image (see ctbb_gpu_recon_set_volume_estimate).
        est = ESTIMATE_ZERO if (o.mode == ICD_SEQUENTIAL and not rp.geom.wfbp_initialize) else ESTIMATE_FORWARD
        rc.set_volume(data.system_matrix, data.recon_volume, est)
        st = rc.iterate(data.system_matrix, int(n_iter if n_iter is not None else rp.geom.num_iterations), o)
        data.recon_volume = rc.volume()
        data.extra["volume_f64"] = rc.volume_f64()
    finally:
        rc.free()
    return st


def _rotate(rp: ReconParams, data: CtData, direction: int, ctx: Context | None):
    ctx = ctx or default_context()
    vol = np.ascontiguousarray(data.recon_volume, dtype=np.float32).copy()
    check(lib().ctbb_gpu_rotate(ctx.handle, C.byref(rp.geom), ptr(data.tube_angles, C.c_double),
                                ptr(data.slice_indices, C.c_uint64), ptr(vol, C.c_float), int(direction)))
    data.recon_volume = vol


def rotate_slices_rotating2fixed(rp: ReconParams, data: CtData, ctx: Context | None = None):
    """rotate_slices.cpp:81-114 on the GPU."""
    _rotate(rp, data, ROTATE_ROTATING2FIXED, ctx)


def rotate_slices_fixed2rotating(rp: ReconParams, data: CtData, ctx: Context | None = None):
    """rotate_slices.cpp:48-79 on the GPU."""
    _rotate(rp, data, ROTATE_FIXED2ROTATING, ctx)


def clean_up(rp: ReconParams, data: CtData) -> str:
    """setup.cpp:422-438: write the float32 volume to output_dir/output_file."""
    name = rp.output_file or "reconstruction_final.img"
    path = os.path.join(rp.output_dir, name)
    np.ascontiguousarray(data.recon_volume, dtype=np.float32).tofile(path)
    if data.system_matrix is not None:
        data.system_matrix.free()
        data.system_matrix = None
    return path


from .learned import WarmStartNet  # noqa: E402
