"""Generate the golden fixtures in tests/golden/ by running the CTBB_ICD
reference program itself (oracle/_ref/icd_ref_O2, built from the reference
sources by oracle/Makefile) and its setup stage (oracle/_ref/ref_setup_dump).

    python tests/golden/make_golden.py            # tiny, tiny_ffs
    python tests/golden/make_golden.py cfg1 cfg2_sub   # benchmark-size fixtures

For each workload the fixture holds: the parameter file, the raw frames fed
to the reference (FileType 0, from the seeded CPU projector), the
reference's matrix.bin (as colptr/idx/w), its FP64 iteration dumps
iteration{1..N}.rcn, the final de-rotated float image, and the full-precision
recon_params / view / slice tables printed by ref_setup_dump.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle_util as O  # noqa: E402
import ctbb_icd_b200 as C  # noqa: E402
from ctbb_icd_b200 import workloads as W  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def make(name: str) -> str:
    with tempfile.TemporaryDirectory() as d:
        prm_path, rp = W.materialise(name, d)
        stdout = O.run_reference(prm_path, d, binary=O.REF_BIN, threads=4)
        import subprocess

        dump = subprocess.run([O.REF_SETUP_DUMP, prm_path], capture_output=True, text=True, check=True).stdout
        ncol = int(rp.geom.num_voxels_x * rp.geom.num_voxels_y)
        m = O.read_matrix_bin(os.path.join(d, "matrix.bin"), ncol)
        n_iter = int(rp.geom.num_iterations)
        shape = rp.shape
        iters = np.stack([np.fromfile(os.path.join(d, "reconstructions", f"iteration{n}.rcn"), np.float64)
                          .reshape(shape) for n in range(n_iter + 1)])
        final = np.fromfile(os.path.join(d, rp.output_file), np.float32).reshape(shape)
        raw = np.fromfile(rp.sinogram_path, np.float32).reshape(rp.raw_shape)
        prm_text = open(prm_path).read().replace(d, "@DIR@")
        path = os.path.join(OUT, f"{name}.npz")
        np.savez_compressed(
            path, prm=np.array(prm_text), raw=raw, colptr=m.colptr, idx=m.idx, w=m.w, iterations=iters,
            final=final, setup_dump=np.array(dump.split("===DUMP===", 1)[1]),
            ref_stdout_tail=np.array(stdout[-4000:]))
    return path


# ----------------------------------------------------------------------------
# Benchmark-size fixtures. The reference's matrix.bin (1.25 GB at cfg1) and the
# raw frames are too large to commit, so these fixtures hold per-column hashes
# of matrix.bin, a few full columns, the parameter file, the phantom and a hash
# of the raw frames; the tests regenerate the frames with the oracle projector
# (reference_run.synth_raw) and compare hashes.
# ----------------------------------------------------------------------------
def bench_size_prm(name, d):
    """(prm dict, phantom dict) of a benchmark-size fixture, paths under d."""
    from oracle import reference_run as R

    if name == "cfg1":
        w = W.workload("cfg1")
        prm = dict(w["prm"], num_iterations=3, sinogram_path=os.path.join(d, "raw.bin"), output_dir=d,
                   output_file="ref.img")
    elif name == "cfg2_sub":
        # cfg2's scanner (736 x 64 rows, in-plane FFS, 2304 views/turn), voxel
        # size and edge-preserving penalty on a central 64 x 64 x 4 slab.
        w = W.workload("cfg2")
        prm = R.central_subvolume(dict(w["prm"], num_iterations=3), 64, 4, 3000, d)
    else:
        raise KeyError(name)
    ph = dict(w["phantom"], z_lo=min(prm["z_start"], prm["z_end"]), z_hi=max(prm["z_start"], prm["z_end"]))
    return prm, ph


def make_bench_size(name: str, threads: int = 8) -> str:
    from oracle import reference_run as R

    with tempfile.TemporaryDirectory() as d:
        prm, ph = bench_size_prm(name, d)
        prm_path = R.write_prm(os.path.join(d, f"{name}.prm"), prm)
        R.write_zero_raw(prm["sinogram_path"], prm["Readings"], prm["n_channels"], prm["Nrows"])
        fields, views, slices = R.setup_dump(prm_path)
        g = R.geometry(fields)
        raw = R.synth_raw(g, ph)
        R.write_raw(prm["sinogram_path"], raw)
        rc, stamps = R.run("O2", prm_path, d, threads=threads)
        if rc != 0:
            raise RuntimeError("\n".join(l for _, l in stamps[-20:]))
        ncol = int(g.num_voxels_x * g.num_voxels_y)
        counts, hashes = O.column_hashes(os.path.join(d, "matrix.bin"), ncol)
        m = O.read_matrix_bin(os.path.join(d, "matrix.bin"), ncol)
        nx = int(g.num_voxels_x)
        sample = np.array(sorted({0, ncol - 1, nx // 2 + nx * (nx // 2), nx // 4 + nx * (nx // 3)}), np.int64)
        s_ptr = np.concatenate([[0], np.cumsum([m.colptr[c + 1] - m.colptr[c] for c in sample])]).astype(np.int64)
        s_idx = np.concatenate([m.column(int(c))[0] for c in sample])
        s_w = np.concatenate([m.column(int(c))[1] for c in sample])
        shape = (int(g.num_voxels_z), int(g.num_voxels_y), int(g.num_voxels_x))
        n_iter = int(prm["num_iterations"])
        iters = np.stack([np.fromfile(os.path.join(d, "reconstructions", f"iteration{n}.rcn"), np.float64)
                          .reshape(shape) for n in range(1, n_iter + 1)]).astype(np.float32)
        final = np.fromfile(os.path.join(d, prm["output_file"]), np.float32).reshape(shape)
        t = R.stage_times(stamps)
        path = os.path.join(OUT, f"{name}.npz")
        np.savez_compressed(
            path, prm=np.array(R.prm_text(prm).replace(d, "@DIR@")), phantom=np.array(repr(ph)),
            raw_hash=np.array(O.raw_hash(raw)), col_counts=counts, col_hashes=hashes,
            sample_cols=sample, sample_ptr=s_ptr, sample_idx=s_idx, sample_w=s_w,
            iterations_f32=iters, final=final,
            ref_times=np.array(repr({k: v for k, v in t.items()})),
            ref_stdout_tail=np.array("\n".join(l for _, l in stamps[-40:])))
    return path


if __name__ == "__main__":
    names = sys.argv[1:] or ["tiny", "tiny_ffs"]
    for n in names:
        p = make_bench_size(n) if n in ("cfg1", "cfg2_sub") else make(n)
        print(p, os.path.getsize(p))
