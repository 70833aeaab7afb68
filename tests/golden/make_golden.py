"""Generate the golden fixtures in tests/golden/ by running the CTBB_ICD
reference program itself (oracle/_ref/icd_ref_O2, built from the reference
sources by oracle/Makefile) and its setup stage (oracle/_ref/ref_setup_dump).

    python tests/golden/make_golden.py            # tiny, tiny_ffs

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


if __name__ == "__main__":
    names = sys.argv[1:] or ["tiny", "tiny_ffs"]
    for n in names:
        p = make(n)
        print(p, os.path.getsize(p))
