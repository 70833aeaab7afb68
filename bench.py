#!/usr/bin/env python
"""Benchmark: voxel updates per second of grouped ICD on the full-size helical
workload (512 x 512 x 64 slices, 736 channels x 64 rows, in-plane flying
focal spot, 2304 views/turn, 4 turns, edge-preserving penalty).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one ICD iteration: every voxel of the volume updated once by the
persistent grouped-ICD kernel. Inputs (raw data, stored system matrix, image,
error sinogram) are resident in HBM before timing; the e2e figure repeats the
measurement through the reference-facing one-call API (ctbb_gpu_icd) with
host buffers, so host<->device copies are inside the timed region.

With N > 1 (torchrun) every rank reconstructs its own independent scan
(replicas, weak scaling, no data-path collective); `value` is the sum of all
ranks' voxel updates over the slowest rank's time.

--impl reference times the reference program (oracle/_ref/icd_ref_O2, the
CTBB_ICD sources built unmodified) on the host cores: its ICD iterations on a
bounded sample of the same geometry (see cpu_sample()).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "cfg2"
WORKLOAD_TEXT = ("grouped ICD, 512x512x64 @ 0.6 mm, 30 cm FOV, 736 ch x 64 rows, in-plane FFS, "
                 "2304 views/turn, 4 turns (9216 views), edge-preserving (delta 9.6e-4, lambda 0.1)")
HBM_FALLBACK_GBS = 6650.0


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


# --------------------------------------------------------------------------
# nvidia-smi clock sampling during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int, enabled: bool = True):
        self.gpu = gpu_index
        self.enabled = enabled
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        if not self.enabled:
            return
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for _, line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------------
# Our arm
# --------------------------------------------------------------------------
def setup_workload(ctx, workdir, seed, weights, name=WORKLOAD):
    import ctbb_icd_b200 as C
    from ctbb_icd_b200 import workloads as W

    w = W.workload(name)
    w["phantom"]["seed"] = seed
    prm = w["prm"]
    prm.update(sinogram_path=os.path.join(workdir, "raw.bin"), output_dir=workdir, output_file="out.img")
    open(prm["sinogram_path"], "wb").close()
    rp = C.configure_recon_params(W.write_prm(os.path.join(workdir, "bench.prm"), prm))
    tables = C.slice_tables(rp)
    spec = W.phantom_spec(w["phantom"])
    spec.ellipsoid_z_lo = min(prm["z_start"], prm["z_end"])
    spec.ellipsoid_z_hi = max(prm["z_start"], prm["z_end"])
    # Phantom cut to the reconstructed slab: data consistent with the model.
    spec.clip_z_lo, spec.clip_z_hi = W.slab_clip(rp, tables.slice_locations)
    rc = C.Recon(rp, tables.slice_indices, ctx)
    C.check(C.lib().ctbb_gpu_synth_raw(ctx.handle, ctypes.byref(rp.geom), ctypes.byref(spec),
                                       ctypes.c_void_p(rc.raw_device_ptr())))
    ssm = C.Ssm.generate(rp, ctx, weights)
    rc.set_volume(ssm, None)
    return rp, tables, rc, ssm


def run_ours(args, rank, world, dist):
    import torch

    import ctbb_icd_b200 as C

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    torch_stream = torch.cuda.Stream(device=local)
    if args.own_stream:
        ctx = C.Context(local)
        torch_stream = torch.cuda.ExternalStream(ctx.stream, device=local)
    else:
        ctx = C.Context(local, ctypes.c_void_p(torch_stream.cuda_stream))
    weights_fmt = C.SSM_FP16 if args.weights == "fp16" else C.SSM_FP32
    workdir = tempfile.mkdtemp(prefix="ctbb_bench_")
    t0 = time.time()
    rp, tables, rc, ssm = setup_workload(ctx, workdir, seed=rank, weights=C.SSM_BOTH if args.e2e else weights_fmt,
                                         name=args.workload)
    setup_s = time.time() - t0
    info = ssm.info()
    opts = C.icd_opts(mode=C.ICD_GROUPED, weights=weights_fmt, warps_in_flight=args.warps, lattice=args.lattice,
                      warps_per_voxel=args.wpv, entries_per_lane=args.epl)
    nvox = int(np.prod(rp.shape))
    tune = None
    if args.autotune:
        # Probe from an early iterate, as a user would before a long run.
        rc.iterate(ssm, 3, opts)
        opts, trials = rc.autotune(ssm, opts, probe_iters=2)
        tune = {"chosen": {"warps_per_voxel": opts.warps_per_voxel, "warps_in_flight": opts.warps_in_flight,
                           "entries_per_lane": opts.entries_per_lane, "lattice": opts.lattice},
                "trials": [[t["warps_per_voxel"], t["warps_in_flight"], t["entries_per_lane"], t["lattice"],
                            round(t["device_ms"], 1), round(t["score"], 1)] for t in trials],
                "trial_fields": ["warps_per_voxel", "warps_in_flight", "entries_per_lane", "lattice",
                                 "ms_2_iterations", "cost_decrease_per_ms"]}
        rc.set_volume(ssm, None)

    # Algorithmic bytes per iteration (one launch): e read + written once per
    # in-range entry (8 B), the SSM read once (index + weight), image r+w.
    rc.iterate(ssm, args.warmup, opts)
    st = rc.iterate(ssm, 1, opts)  # also yields the in-range entry count
    entries = rc.entries(ssm)
    w_bytes = 2 if weights_fmt == C.SSM_FP16 else 4
    b_iter = 8.0 * entries + (4 + w_bytes) * float(info.nnz) + 8.0 * nvox

    clocks = ClockSampler(local, enabled=args.clocks)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(torch_stream):
        start.record(torch_stream)
        st = rc.iterate(ssm, args.steps, opts)
        end.record(torch_stream)
    end.synchronize()
    torch.cuda.synchronize()
    elapsed_ms = start.elapsed_time(end)
    clocks.stop()
    kernel_ms_per_launch = st.device_ms / max(1, st.iterations)

    e2e = None
    if args.e2e:
        e2e = run_e2e(C, ctx, rp, tables, ssm, rc, opts, args, torch, torch_stream)

    from ctbb_icd_b200.replicas import max_over_ranks

    t_max = max_over_ranks(elapsed_ms, dist, device="cuda")
    if e2e and dist:
        e2e["seconds"] = max_over_ranks(e2e["seconds"], dist, device="cuda")
        e2e["value"] = world * e2e["updates"] / e2e["seconds"]
    out = None
    if rank == 0:
        peak, peak_kind = measured_peak()
        achieved = b_iter / (kernel_ms_per_launch / 1e3) / 1e9
        value = world * nvox * args.steps / (t_max / 1e3)
        kernel = "icd_grouped_kernel" if opts.warps_per_voxel <= 1 else "icd_cta_kernel"
        traffic = read_traffic(kernel)
        out = {
            "metric": "voxel-updates/s",
            "value": value,
            "unit": "voxel-updates/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": t_max / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded phantom: water + 6 inserts + 40 ellipsoids, Poisson noise, GPU projector)",
            "config": {
                "workload": WORKLOAD_TEXT if args.workload == WORKLOAD else args.workload,
                "weights": args.weights, "error_sinogram": "fp32", "voxels": nvox,
                "ssm_nnz": int(info.nnz), "ssm_bytes": int(info.bytes_device),
                "ssm_build_ms": round(info.build_ms, 2), "inrange_entries_per_iter": entries,
                "warps_in_flight": opts.warps_in_flight or "auto", "warps_per_voxel": max(1, opts.warps_per_voxel),
                "entries_per_lane": opts.entries_per_lane or 8,
                "lattice": opts.lattice or "auto", "autotune": tune,
                "l2": "inputs larger than L2 (e 1.74 GB, SSM > 20 GB)",
                "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                "setup_s": round(setup_s, 1),
            },
            "roofline": {
                "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "kernel": kernel,
                "algorithmic_bytes_per_launch": b_iter,
                "kernel_ms_per_launch": kernel_ms_per_launch, "peak_source": peak_kind,
            },
            "gpu_launches": int(args.steps),
            "clocks": clocks.summary(),
        }
        if e2e:
            out["e2e"] = {"value": e2e["value"], "unit": "voxel-updates/s",
                          "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"]}
            out["gpu_launches"] += e2e["launches"]
        if args.cpu_baseline and world == 1:
            cb = cpu_sample(ctx, iterations=3)
            out["cpu_baseline"] = {k: cb.get(k) for k in ("value", "unit", "cores", "kind", "sample")}
    rc.free()
    ssm.free()
    ctx.close()
    return out


def run_e2e(C, ctx, rp, tables, ssm, rc, opts, args, torch, torch_stream):
    """The same metric through ctbb_gpu_icd (the icd_iteration drop-in) with
    pinned host buffers: per step one call that uploads the raw data and the
    zero initial image, runs the workload's iteration count and returns the
    image (what a caller of icd_iteration does)."""
    raw = torch.empty(rp.raw_shape, dtype=torch.float32).pin_memory()
    C.check(C.lib().ctbb_gpu_recon_get_raw(rc.handle, C.ptr(raw.numpy(), ctypes.c_float)))
    vol = torch.zeros(rp.shape, dtype=torch.float32).pin_memory()
    g = C.GeomC.from_buffer_copy(rp.geom)
    g.num_iterations = args.e2e_iters
    si = np.ascontiguousarray(tables.slice_indices, np.uint64)
    st = C.IterStats()

    def one():
        C.check(C.lib().ctbb_gpu_icd(ctx.handle, ssm.handle, ctypes.byref(g), C.ptr(si, ctypes.c_uint64),
                                     C.ptr(raw.numpy(), ctypes.c_float), C.ptr(vol.numpy(), ctypes.c_float),
                                     ctypes.byref(opts), ctypes.byref(st)))

    def reset():
        vol.zero_()

    reset()
    one()  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        reset()
        one()
    torch.cuda.synchronize()
    secs = time.perf_counter() - t0
    nvox = int(np.prod(rp.shape))
    # Kernel launches per call: residual init, f64->f32 image and residual
    # conversion (2), e2e_iters ICD iterations, entry count (first call only).
    launches_per = 3 + args.e2e_iters
    return {"value": nvox * args.e2e_iters * args.e2e_steps / secs, "seconds": secs,
            "updates": nvox * args.e2e_iters * args.e2e_steps,
            "h2d": int(raw.numel() * 4 + vol.numel() * 4), "d2h": int(vol.numel() * 4),
            "launches": launches_per * args.e2e_steps}


def read_traffic(kernel: str = "icd_grouped_kernel"):
    """DRAM bytes per launch of the ICD kernel from the committed ncu summary
    of that kernel on this workload."""
    p = os.path.join(ROOT, "profiles", f"{kernel.replace('_kernel', '')}_cfg2.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# --------------------------------------------------------------------------
# Reference arm / CPU baseline
# --------------------------------------------------------------------------
CPU_SAMPLE = dict(nx=64, nz=16, readings=3200)


def _sample_prm(nx, nz, readings):
    """Benchmark geometry restricted to an nx x nx x nz central sub-volume at
    the same voxel size, over `readings` views, with a z-range the scan covers."""
    import ctbb_icd_b200 as C
    from ctbb_icd_b200 import workloads as W

    w = W.workload(WORKLOAD)
    prm = w["prm"]
    dx = prm["recon_fov"] / prm["nx"]
    prm.update(nx=nx, ny=nx, recon_fov=dx * nx, Readings=readings)
    d = tempfile.mkdtemp(prefix="ctbb_ref_")
    prm.update(sinogram_path=os.path.join(d, "raw.bin"), output_dir=d, output_file="ref.img",
               matrix_path=os.path.join(d, "matrix.bin"))
    open(prm["sinogram_path"], "wb").close()
    # Allowed window of setup.cpp:359-371 for this geometry; centre the slab in it.
    rp = C.configure_recon_params(W.write_prm(os.path.join(d, "ref.prm"), dict(prm, z_start=-1.0, z_end=-1.1)))
    g = rp.geom
    tzi, vz = g.tube_z_increment, g.voxel_size_z
    zf = (float(readings) / float(g.num_views_per_turn)) * g.table_feed_per_rotation / 10.0
    half = np.ceil(0.5 * g.beam_width_at_roi_edge / vz) * vz
    lo, hi = zf - (readings - 1) * tzi + half, zf - half
    mid = 0.5 * (lo + hi)
    z_start = mid + 0.5 * nz * vz
    prm.update(z_start=z_start, z_end=z_start - (nz + 0.5) * vz)
    return w, prm, d


def cpu_sample(ctx=None, iterations=3, threads=None):
    """Time the reference program's ICD iterations on a bounded sample of the
    benchmark geometry: same scanner, views per turn, flying focal spot,
    voxel size (0.586 mm) and slice thickness, but a 64 x 64 x 16 central
    sub-volume (3.75 cm FOV) and the 3200 views around it. The matrix.bin it
    reads is exported from the GPU builder, which reproduces the reference's
    generate_system_matrix_ffs bit for bit (tests/test_gpu_parity.py); the
    reference's own generator would take minutes single-threaded here.

    The reference's time per voxel grows with the matrix entries it visits,
    and the small FOV shortens the system-matrix window (num_views_for_system
    _matrix follows the FOV radius), so the rate is also reported normalised
    to the full workload's entries per voxel (`value`)."""
    import ctbb_icd_b200 as C
    from ctbb_icd_b200 import workloads as W

    binary = os.path.join(ROOT, "oracle", "_ref", "icd_ref_O2")
    if not os.path.exists(binary):
        return {"value": None, "unit": "voxel-updates/s", "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref/icd_ref_O2 is not built"}
    s = CPU_SAMPLE
    w, prm, d = _sample_prm(s["nx"], s["nz"], s["readings"])
    prm["num_iterations"] = iterations
    prm_path = W.write_prm(os.path.join(d, "ref.prm"), prm)
    own_ctx = ctx is None
    if own_ctx:
        ctx = C.Context(0)
    rp = C.configure_recon_params(prm_path)
    tables = C.slice_tables(rp)
    spec = W.phantom_spec(w["phantom"])
    spec.ellipsoid_z_lo, spec.ellipsoid_z_hi = prm["z_end"], prm["z_start"]
    rc = C.Recon(rp, tables.slice_indices, ctx)
    C.check(C.lib().ctbb_gpu_synth_raw(ctx.handle, ctypes.byref(rp.geom), ctypes.byref(spec),
                                       ctypes.c_void_p(rc.raw_device_ptr())))
    C.write_raw_file(prm["sinogram_path"], rp, rc.raw())
    ssm = C.Ssm.generate(rp, ctx, C.SSM_FP32)
    ssm.export_reference(prm["matrix_path"])
    nvox = s["nx"] * s["nx"] * s["nz"]
    sample_entries = rc.entries(ssm) / nvox
    rc.free()
    ssm.free()
    full_entries = workload_entries_per_voxel(ctx)
    if own_ctx:
        ctx.close()
    ncpu = os.cpu_count() or 1
    threads = threads or min(ncpu, 11)  # the reference hard-codes 11 OpenMP threads (icd_iteration.cpp:40)
    env = dict(os.environ, OMP_THREAD_LIMIT=str(threads))
    os.makedirs(os.path.join(d, "reconstructions"), exist_ok=True)
    stamps = []
    p = subprocess.Popen([binary, prm_path], cwd=d, env=env, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                         text=True, bufsize=1)
    for line in p.stdout:
        if line.startswith("Iteration #") or line.startswith("Rotating ICD slices"):
            stamps.append(time.perf_counter())
    p.wait()
    subprocess.run(["rm", "-rf", d])
    if p.returncode != 0 or len(stamps) < 2:
        return {"value": None, "unit": "voxel-updates/s", "cores": threads, "kind": "reference",
                "sample": f"reference run failed (exit {p.returncode})"}
    per_iter = np.diff(stamps)
    raw_rate = nvox / float(np.median(per_iter))
    value = raw_rate * sample_entries / full_entries
    return {"value": value, "unit": "voxel-updates/s", "cores": threads, "kind": "reference",
            "sample": (f"reference icd_iteration (-O2 build of the unmodified sources, OpenMP {threads} threads "
                       f"of {ncpu} cores) on a {s['nx']}x{s['nx']}x{s['nz']} central sub-volume of the benchmark "
                       f"geometry, {s['readings']} views; median of {len(per_iter)} iterations "
                       f"{float(np.median(per_iter)):.3f} s = {raw_rate:.4g} vu/s at {sample_entries:.0f} entries/voxel, "
                       f"scaled to the workload's {full_entries:.0f} entries/voxel"),
            "seconds_per_iteration": [float(t) for t in per_iter], "raw_rate": raw_rate,
            "entries_per_voxel_sample": sample_entries, "entries_per_voxel_workload": full_entries}


_FULL_ENTRIES = {}


def workload_entries_per_voxel(ctx):
    """In-range matrix entries per voxel of the full benchmark workload."""
    if "v" not in _FULL_ENTRIES:
        import ctbb_icd_b200 as C
        from ctbb_icd_b200 import workloads as W

        w = W.workload(WORKLOAD)
        d = tempfile.mkdtemp(prefix="ctbb_ent_")
        prm = dict(w["prm"], sinogram_path=os.path.join(d, "r.bin"), output_dir=d, output_file="o.img")
        rp = C.configure_recon_params(W.write_prm(os.path.join(d, "w.prm"), prm))
        tables = C.slice_tables(rp)
        ssm = C.Ssm.generate(rp, ctx, C.SSM_FP16)
        rc = C.Recon(rp, tables.slice_indices, ctx)
        _FULL_ENTRIES["v"] = rc.entries(ssm) / float(np.prod(rp.shape))
        rc.free()
        ssm.free()
        subprocess.run(["rm", "-rf", d])
    return _FULL_ENTRIES["v"]


def run_reference(args, rank, world):
    if rank != 0:
        return None
    r = cpu_sample(iterations=args.warmup + args.steps)
    if not r.get("value"):
        return {"impl": "reference", "unavailable": r.get("sample", "reference run failed")}
    times = r["seconds_per_iteration"][-args.steps:]
    scale = r["entries_per_voxel_sample"] / r["entries_per_voxel_workload"]
    nvox = CPU_SAMPLE["nx"] ** 2 * CPU_SAMPLE["nz"]
    v = nvox * len(times) / float(np.sum(times)) * scale
    cb = dict(r, value=v)
    return {
        "impl": "reference", "metric": "voxel-updates/s", "value": v, "unit": "voxel-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * float(np.mean(times)) / scale,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": "reference CPU ICD, bounded sample of the grouped-ICD "
                                                    "benchmark geometry", "sample": cb["sample"]},
        "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": v, "unit": "voxel-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--weights", choices=["fp16", "fp32"], default="fp16")
    ap.add_argument("--workload", default=WORKLOAD,
                    help="workload name from ctbb_icd_b200.workloads (the benchmark is cfg2)")
    ap.add_argument("--warps", type=int, default=0, help="warps in flight (0: auto)")
    ap.add_argument("--lattice", type=int, default=0)
    ap.add_argument("--wpv", type=int, default=1, help="warps per voxel update: 1, 4 or 8")
    ap.add_argument("--epl", type=int, default=0, help="entries per lane in flight: 8 or 16 (0: 8)")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="skip the library's autotuner (warps per voxel, warps in flight, tile edge) and use "
                         "--wpv/--warps/--lattice as given")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--e2e-iters", type=int, default=10, help="ICD iterations per drop-in call")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-clocks", dest="clocks", action="store_false", help="skip nvidia-smi clock sampling")
    ap.add_argument("--own-stream", action="store_true", help="run on the library's own stream")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = tdist
    try:
        if args.impl == "reference":
            out = run_reference(args, rank, world)
        else:
            out = run_ours(args, rank, world, dist)
        if rank == 0 and out is not None:
            print(json.dumps(out), flush=True)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
