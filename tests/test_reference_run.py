"""The reference-run path (oracle/reference_run.py: geometry from the
reference's own setup code, frames from the oracle projector, the reference
program itself) reproduces the golden fixture bit for bit. CPU only."""
import os

import numpy as np
import pytest

import oracle_util as O
from ctbb_icd_b200 import workloads as W
from oracle import reference_run as R

pytestmark = pytest.mark.skipif(not R.available(), reason="reference program not built (oracle/Makefile ref)")


def test_reference_run_reproduces_tiny_fixture(tmp_path):
    z = np.load(os.path.join(O.ROOT, "tests", "golden", "tiny.npz"))
    d = str(tmp_path)
    prm_path = os.path.join(d, "tiny.prm")
    with open(prm_path, "w") as f:
        f.write(str(z["prm"]).replace("@DIR@", d))
    prm = W.workload("tiny")["prm"]
    R.write_zero_raw(os.path.join(d, "tiny.bin"), prm["Readings"], prm["n_channels"], prm["Nrows"])
    fields, views, slices = R.setup_dump(prm_path)
    g = R.geometry(fields)
    ph = dict(W.WORKLOADS["tiny"]["phantom"], z_lo=min(prm["z_start"], prm["z_end"]),
              z_hi=max(prm["z_start"], prm["z_end"]))
    raw = R.synth_raw(g, ph)
    assert np.array_equal(raw.view(np.int32), z["raw"].view(np.int32))
    R.write_raw(os.path.join(d, "tiny.bin"), raw)
    rc, stamps = R.run("O2", prm_path, d, threads=2)
    assert rc == 0, stamps[-5:]
    t = R.stage_times(stamps)
    assert t["ssm_s"] is not None and len(t["iteration_s"]) == int(prm["num_iterations"])
    m = O.read_matrix_bin(os.path.join(d, "matrix.bin"), int(g.num_voxels_x * g.num_voxels_y))
    assert np.array_equal(m.idx, z["idx"]) and np.array_equal(m.w.view(np.int32), z["w"].view(np.int32))
    # the oracle's matrix, written in the reference's format, is the same file
    colptr, idx, w = R.oracle_matrix(g)
    R.write_matrix_bin(os.path.join(d, "port.bin"), colptr, idx, w)
    assert open(os.path.join(d, "port.bin"), "rb").read() == open(os.path.join(d, "matrix.bin"), "rb").read()
