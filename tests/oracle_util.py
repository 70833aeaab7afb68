"""Test-side access to the oracle: the CPU restatement (oracle/port.cpp) and
the reference program's file formats. Imported only by tests/, bench.py's
CPU-baseline leg and __graft_entry__.smoke()."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "icd_ref_O2")
REF_BIN_SHIPPED = os.path.join(ROOT, "oracle", "_ref", "icd_ref")
REF_BIN_CORES = os.path.join(ROOT, "oracle", "_ref", "icd_ref_cores")
REF_SETUP_DUMP = os.path.join(ROOT, "oracle", "_ref", "ref_setup_dump")

from oracle.port_binding import PORT_LIB, port  # noqa: E402
from oracle.port_binding import ptr as _p  # noqa: E402


class Csr:
    """Column-major sparse matrix (colptr, idx, w) like the reference SSM."""

    def __init__(self, colptr, idx, w):
        self.colptr, self.idx, self.w = colptr, idx, w

    def column(self, c):
        b, e = self.colptr[c], self.colptr[c + 1]
        return self.idx[b:e], self.w[b:e]

    @property
    def nnz(self):
        return int(self.colptr[-1])


def port_ssm(rp) -> Csr:
    L = port()
    h = L.port_ssm_build(C.byref(rp.geom))
    try:
        nnz = L.port_ssm_nnz(h)
        ncol = int(rp.geom.num_voxels_x * rp.geom.num_voxels_y)
        colptr = np.empty(ncol + 1, np.int64)
        idx = np.empty(nnz, np.int32)
        w = np.empty(nnz, np.float32)
        L.port_ssm_copy(h, _p(colptr, C.c_int64), _p(idx, C.c_int32), _p(w, C.c_float))
    finally:
        L.port_ssm_free(h)
    return Csr(colptr, idx, w)


def port_ssm_subset(rp, cols, views):
    """Entries of the given columns restricted to the given SSM views (the
    oracle's ray-driven builder evaluated only where it reaches them).
    Returns {column: (idx int32, w float32)} in the reference's entry order."""
    L = port()
    cols = np.ascontiguousarray(cols, np.int64)
    views = np.ascontiguousarray(np.sort(np.asarray(views)), np.int32)
    counts = np.zeros(len(cols) * len(views), np.uint32)
    cap = 1 << 16
    while True:
        idx = np.empty(cap, np.int32)
        w = np.empty(cap, np.float32)
        n = int(L.port_ssm_subset(C.byref(rp.geom), len(cols), _p(cols, C.c_int64), len(views),
                                  _p(views, C.c_int32), counts.ctypes.data_as(C.POINTER(C.c_uint32)),
                                  _p(idx, C.c_int32), _p(w, C.c_float), cap))
        if n <= cap:
            break
        cap = n
    out, pos = {}, 0
    per_col = counts.reshape(len(cols), len(views)).sum(axis=1)
    for c, m in zip(cols, per_col):
        out[int(c)] = (idx[pos:pos + m].copy(), w[pos:pos + m].copy())
        pos += int(m)
    return out


def restrict_views(idx, w, views, n_per_view):
    """Entries of a column whose matrix view (q // (n_channels * Nrows)) is in `views`."""
    keep = np.isin(idx // n_per_view, np.asarray(views))
    return idx[keep], w[keep]


def port_icd(rp, slice_indices, raw, ssm: Csr, n_iter, x0=None, est0=None):
    """Sequential ICD on the CPU; returns (dumps[n_iter, nz, ny, nx] FP64, x, est)."""
    L = port()
    shape = rp.shape
    x = np.zeros(int(np.prod(shape)), np.float64) if x0 is None else np.array(x0, np.float64).ravel().copy()
    est = np.zeros(raw.size, np.float64) if est0 is None else np.array(est0, np.float64).ravel().copy()
    dumps = np.zeros((n_iter, x.size), np.float64)
    si = np.ascontiguousarray(slice_indices, np.uint64)
    raw = np.ascontiguousarray(raw, np.float32)
    L.port_icd(C.byref(rp.geom), _p(si, C.c_uint64), _p(raw, C.c_float), _p(ssm.colptr, C.c_int64),
               _p(ssm.idx, C.c_int32), _p(ssm.w, C.c_float), _p(x, C.c_double), _p(est, C.c_double),
               int(n_iter), _p(dumps, C.c_double))
    return dumps.reshape((n_iter,) + shape), x.reshape(shape), est


def port_rotate(rp, tube_angles, slice_indices, vol, direction):
    out = np.ascontiguousarray(vol, np.float32).copy()
    ta = np.ascontiguousarray(tube_angles, np.float64)
    si = np.ascontiguousarray(slice_indices, np.uint64)
    port().port_rotate(C.byref(rp.geom), _p(ta, C.c_double), _p(si, C.c_uint64), _p(out, C.c_float), int(direction))
    return out


def port_forward(rp, slice_indices, ssm: Csr, x):
    out = np.empty(int(rp.geom.Readings * rp.geom.n_channels * rp.geom.Nrows_projection), np.float64)
    si = np.ascontiguousarray(slice_indices, np.uint64)
    xx = np.ascontiguousarray(x, np.float64)
    port().port_forward(C.byref(rp.geom), _p(si, C.c_uint64), _p(ssm.colptr, C.c_int64), _p(ssm.idx, C.c_int32),
                        _p(ssm.w, C.c_float), _p(xx, C.c_double), _p(out, C.c_double))
    return out


def port_cost(rp, slice_indices, raw, ssm: Csr, x):
    si = np.ascontiguousarray(slice_indices, np.uint64)
    xx = np.ascontiguousarray(x, np.float64)
    raw = np.ascontiguousarray(raw, np.float32)
    d, p = C.c_double(), C.c_double()
    tot = port().port_cost(C.byref(rp.geom), _p(si, C.c_uint64), _p(raw, C.c_float), _p(ssm.colptr, C.c_int64),
                           _p(ssm.idx, C.c_int32), _p(ssm.w, C.c_float), _p(xx, C.c_double), C.byref(d), C.byref(p))
    return tot, d.value, p.value


def port_synth(rp, spec):
    from ctbb_icd_b200 import GeomC, slice_tables, ReconParams

    g = GeomC.from_buffer_copy(rp.geom)
    slice_tables(ReconParams(geom=g), allow_bad_range=True)
    raw = np.empty(rp.raw_shape, np.float32)
    port().port_synth(C.byref(g), C.byref(spec), _p(raw, C.c_float))
    return raw


def read_matrix_bin(path, ncol) -> Csr:
    """The reference's matrix.bin: per column size_t n, then n x {int32, float32}."""
    buf = np.fromfile(path, np.uint8)
    colptr = np.zeros(ncol + 1, np.int64)
    idx_parts, w_parts = [], []
    pos = 0
    for c in range(ncol):
        n = int(buf[pos:pos + 8].view(np.uint64)[0])
        pos += 8
        rec = buf[pos:pos + 8 * n].view(np.int32).reshape(n, 2)
        idx_parts.append(rec[:, 0].copy())
        w_parts.append(rec[:, 1].copy().view(np.float32))
        pos += 8 * n
        colptr[c + 1] = colptr[c] + n
    if pos != buf.size:
        raise ValueError(f"{path}: {buf.size - pos} trailing bytes")
    idx = np.concatenate(idx_parts) if idx_parts else np.zeros(0, np.int32)
    w = np.concatenate(w_parts) if w_parts else np.zeros(0, np.float32)
    return Csr(colptr, idx, w)


def parse_setup_dump(text: str):
    """Output of oracle/_ref/ref_setup_dump -> (fields dict, views, slices)."""
    body = (text.split("===DUMP===", 1)[1] if "===DUMP===" in text else text).strip().splitlines()
    fields, views, slices = {}, [], []
    for line in body:
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


def run_reference(prm_path, workdir, binary=REF_BIN, threads=None, timeout=3600):
    """Run the reference program; returns its stdout text."""
    env = dict(os.environ)
    env["OMP_THREAD_LIMIT"] = str(threads or os.cpu_count() or 1)
    os.makedirs(os.path.join(workdir, "reconstructions"), exist_ok=True)
    r = subprocess.run([binary, prm_path], cwd=workdir, env=env, capture_output=True, text=True,
                       timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"reference exited {r.returncode}: {r.stdout[-2000:]}")
    return r.stdout


def column_hashes(path, ncol):
    """Per column of a matrix.bin: (entry count, 64-bit BLAKE2b of the
    column's count and records)."""
    import hashlib

    buf = np.fromfile(path, np.uint8)
    counts = np.zeros(ncol, np.int64)
    hashes = np.zeros(ncol, np.uint64)
    pos = 0
    for c in range(ncol):
        n = int(buf[pos:pos + 8].view(np.uint64)[0])
        end = pos + 8 + 8 * n
        counts[c] = n
        hashes[c] = np.frombuffer(hashlib.blake2b(buf[pos:end].tobytes(), digest_size=8).digest(), np.uint64)[0]
        pos = end
    if pos != buf.size:
        raise ValueError(f"{path}: {buf.size - pos} trailing bytes")
    return counts, hashes


def raw_hash(raw):
    import hashlib

    return hashlib.blake2b(np.ascontiguousarray(raw, np.float32).tobytes(), digest_size=16).hexdigest()


def bench_size_fixture(name, directory):
    """Materialise a benchmark-size golden fixture (make_golden.py cfg1 /
    cfg2_sub) in `directory`: the parameter file, and the raw frames
    regenerated with the oracle projector on the reference's own geometry
    (checked against the fixture's hash). Returns (npz, prm_path)."""
    import ast

    from oracle import reference_run as R

    z = np.load(os.path.join(ROOT, "tests", "golden", f"{name}.npz"))
    text = str(z["prm"]).replace("@DIR@", directory)
    prm_path = os.path.join(directory, f"{name}.prm")
    with open(prm_path, "w") as f:
        f.write(text)
    kv = dict(line.split(": ", 1) for line in text.splitlines() if ": " in line and not line.startswith("#"))
    R.write_zero_raw(kv["sinogram_path"], int(kv["Readings"]), int(kv["n_channels"]), int(kv["Nrows"]))
    fields, _, _ = R.setup_dump(prm_path)
    raw = R.synth_raw(R.geometry(fields), ast.literal_eval(str(z["phantom"])))
    if raw_hash(raw) != str(z["raw_hash"]):
        raise AssertionError(f"{name}: regenerated raw frames differ from the fixture's")
    R.write_raw(kv["sinogram_path"], raw)
    os.makedirs(os.path.join(directory, "reconstructions"), exist_ok=True)
    return z, prm_path


def port_penalty_steps(penalty, lam, delta, alpha, beta, x9):
    """The reference's one-voxel penalised update (penalties.cpp:61-154) on
    given inputs; x9 [n, 9] = voxel and 8 neighbours (NaN: outside)."""
    a = np.ascontiguousarray(alpha, np.float64)
    b = np.ascontiguousarray(beta, np.float64)
    x = np.ascontiguousarray(x9, np.float32).reshape(-1, 9)
    out = np.empty(a.size, np.float64)
    port().port_penalty_steps(int(penalty), float(lam), float(delta), a.size, _p(a, C.c_double), _p(b, C.c_double),
                              _p(x, C.c_float), _p(out, C.c_double))
    return out

