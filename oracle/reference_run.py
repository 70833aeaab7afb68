"""Runs the CTBB_ICD reference program (oracle/_ref/icd_ref*, built from the
reference's own sources by oracle/Makefile) on a parameter file, with raw
frames from the oracle's CPU projector and every derived geometry value taken
from the reference's own setup code (oracle/_ref/ref_setup_dump).

TEST INFRASTRUCTURE / CPU BASELINE ONLY: used by tests/golden/make_golden.py,
tests/ and bench.py's reference arm and CPU-baseline leg. Nothing here loads
the product library (libctbb_icd_b200.so); the only compiled code it runs is
the reference program and the oracle's restatement.
"""
from __future__ import annotations

import os
import re
import subprocess
import time

import numpy as np

from .port_binding import port, ptr

ORACLE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(ORACLE, "_ref")
BINARIES = {
    "shipped": os.path.join(REF_DIR, "icd_ref"),       # as shipped: -g, OMP_N_THREADS 11
    "O2": os.path.join(REF_DIR, "icd_ref_O2"),         # -O2, OMP_N_THREADS 11
    "cores": os.path.join(REF_DIR, "icd_ref_cores"),   # -O2, OMP_N_THREADS = processor count
}
SETUP_DUMP = os.path.join(REF_DIR, "ref_setup_dump")


def available() -> bool:
    return all(os.path.exists(p) for p in list(BINARIES.values()) + [SETUP_DUMP])


# ------------------------------------------------------------------ files ----
def prm_text(prm: dict) -> str:
    from ctbb_icd_b200.workloads import prm_text as text

    return text(prm)


def write_prm(path: str, prm: dict) -> str:
    with open(path, "w") as f:
        f.write(prm_text(prm))
    return path


def write_zero_raw(path: str, readings: int, n_channels: int, n_rows: int) -> None:
    """A FileType 0 raw file of the right size reading as zeros (sparse)."""
    with open(path, "wb") as f:
        f.truncate(int(readings) * int(n_channels) * int(n_rows) * 4)


def write_raw(path: str, raw: np.ndarray) -> None:
    """FileType 0 frames: float32 [view][channel][row], no header (RawOffset 0)."""
    np.ascontiguousarray(raw, np.float32).tofile(path)


def write_matrix_bin(path: str, colptr, idx, w) -> None:
    """The reference's matrix.bin layout (generate_system_matrix.cpp:212-303):
    per column a size_t count, then count x {int32 index, float32 weight}."""
    with open(path, "wb") as f:
        for c in range(len(colptr) - 1):
            b, e = int(colptr[c]), int(colptr[c + 1])
            np.array([e - b], np.uint64).tofile(f)
            rec = np.empty((e - b, 2), np.int32)
            rec[:, 0] = idx[b:e]
            rec[:, 1] = np.asarray(w[b:e], np.float32).view(np.int32)
            rec.tofile(f)


# --------------------------------------------------------------- geometry ----
def setup_dump(prm_path: str):
    """(fields, views [Readings x (tube angle deg, table position cm)],
    slices [(location, index)]) from the reference's configure_recon_params
    and load_raw. Raises RuntimeError with the reference's message when it
    rejects the file (for example an invalid z range)."""
    r = subprocess.run([SETUP_DUMP, prm_path], capture_output=True, text=True)
    if r.returncode != 0 or "===DUMP===" not in r.stdout:
        raise RuntimeError(r.stdout[-2000:] + r.stderr[-1000:])
    fields, views, slices = {}, [], []
    for line in r.stdout.split("===DUMP===", 1)[1].strip().splitlines():
        parts = line.split()
        if parts[0] == "view":
            views.append((float(parts[2]), float(parts[3])))
        elif parts[0] == "slice":
            slices.append((float(parts[2]), int(parts[3])))
        elif parts[0] in ("penalty", "matrix_path"):
            fields[parts[0]] = parts[1] if len(parts) > 1 else ""
        else:
            v = parts[1]
            fields[parts[0]] = float(v) if any(ch in v for ch in ".en") or v.startswith("-") else int(v)
    return fields, np.array(views), slices


def allowed_z_range(prm: dict, workdir: str):
    """The reconstructable z window the reference reports (setup.cpp:359-377)
    for this scan: asked with an out-of-range slab, it prints the window."""
    probe = dict(prm, z_start=1000.0, z_end=999.0)
    path = write_prm(os.path.join(workdir, "probe.prm"), probe)
    write_zero_raw(probe["sinogram_path"], prm["Readings"], prm["n_channels"], prm["Nrows"])
    r = subprocess.run([SETUP_DUMP, path], capture_output=True, text=True)
    m = re.search(r"Allowed reconstruction range is: (\S+) : (\S+)", r.stdout)
    if not m:
        raise RuntimeError("no allowed range reported: " + r.stdout[-1000:])
    return float(m.group(1)), float(m.group(2))


def geometry(fields: dict):
    """ctbb_geom_c (ctypes) filled from the reference's own derived values."""
    from ctbb_icd_b200._lib import GEOM_FIELDS, GeomC

    import ctypes as C

    g = GeomC()
    for name, typ in GEOM_FIELDS:
        key = "lambda" if name == "lambda_" else name
        if key in fields and key != "penalty":
            v = fields[key]
            setattr(g, name, float(v) if typ is C.c_double else int(round(float(v))))
    g.penalty = 1 if fields.get("penalty") == "edge-preserving" else 0
    return g


def central_subvolume(prm: dict, nx: int, nz: int, readings: int, workdir: str) -> dict:
    """`prm` restricted to an nx x nx x nz central sub-volume at the same voxel
    size, over `readings` views, with the slab centred in the window the
    reference allows (paths under `workdir`)."""
    p = dict(prm)
    dx = p["recon_fov"] / p["nx"]
    p.update(nx=nx, ny=nx, recon_fov=dx * nx, Readings=readings,
             sinogram_path=os.path.join(workdir, "raw.bin"), output_dir=workdir, output_file="ref.img")
    lo, hi = allowed_z_range(p, workdir)
    vz = p["slice_thickness"]
    mid = 0.5 * (lo + hi)
    z_start = mid + 0.5 * nz * vz
    p.update(z_start=z_start, z_end=z_start - (nz + 0.5) * vz)
    return p


# ----------------------------------------------------------------- oracle ----
def synth_raw(g, phantom: dict) -> np.ndarray:
    """Seeded synthetic frames from the oracle's CPU projector (phantom.h)."""
    import ctypes as C

    from ctbb_icd_b200.workloads import phantom_spec

    spec = phantom_spec(phantom)
    raw = np.empty((int(g.Readings), int(g.n_channels), int(g.Nrows_projection)), np.float32)
    port().port_synth(C.byref(g), C.byref(spec), ptr(raw, C.c_float))
    return raw


def oracle_matrix(g):
    """(colptr, idx, w) from the oracle's ray-driven builder, which reproduces
    the reference's matrix.bin bit for bit (tests/test_oracle_pin.py)."""
    import ctypes as C

    L = port()
    h = L.port_ssm_build(C.byref(g))
    try:
        nnz = L.port_ssm_nnz(h)
        ncol = int(g.num_voxels_x * g.num_voxels_y)
        colptr = np.empty(ncol + 1, np.int64)
        idx = np.empty(nnz, np.int32)
        w = np.empty(nnz, np.float32)
        L.port_ssm_copy(h, ptr(colptr, C.c_int64), ptr(idx, C.c_int32), ptr(w, C.c_float))
    finally:
        L.port_ssm_free(h)
    return colptr, idx, w


# -------------------------------------------------------------------- run ----
def run(kind: str, prm_path: str, workdir: str, threads: int | None = None, timeout: float = 3600):
    """Run one reference build on a parameter file; returns (returncode,
    [(seconds since start, stdout line)]). `threads` caps OpenMP through
    OMP_THREAD_LIMIT (the builds' own thread counts are 11 or the processor
    count)."""
    env = dict(os.environ)
    if threads:
        env["OMP_THREAD_LIMIT"] = str(int(threads))
    os.makedirs(os.path.join(workdir, "reconstructions"), exist_ok=True)
    t0 = time.perf_counter()
    stamps = []
    p = subprocess.Popen([BINARIES[kind], prm_path], cwd=workdir, env=env, stdout=subprocess.PIPE,
                         stderr=subprocess.STDOUT, text=True, bufsize=1)
    try:
        for line in p.stdout:
            stamps.append((time.perf_counter() - t0, line.rstrip("\n")))
        p.wait(timeout=timeout)
    except subprocess.TimeoutExpired:
        p.kill()
        p.wait()
    return p.returncode, stamps


def stage_times(stamps):
    """Wall seconds of the stages, from the reference's own stdout markers:
    system-matrix generation ("Generating system matrix" to the first
    "Iteration #" line, when the matrix was generated), each ICD iteration
    (between consecutive "Iteration #" lines, the last one ending at
    "Rotating ICD slices"), and the de-rotation."""
    t_ssm = next((t for t, l in stamps if l.startswith("Generating system matrix")), None)
    its = [t for t, l in stamps if l.startswith("Iteration #")]
    t_rot = next((t for t, l in stamps if l.startswith("Rotating ICD slices")), None)
    t_end = stamps[-1][0] if stamps else None
    ends = its[1:] + ([t_rot] if t_rot is not None else [])
    return {
        "ssm_s": (its[0] - t_ssm) if (t_ssm is not None and its) else None,
        "iteration_s": [b - a for a, b in zip(its, ends)],
        "rotate_s": (t_end - t_rot) if t_rot is not None else None,
    }
