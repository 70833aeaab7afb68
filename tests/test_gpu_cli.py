"""ctbb_icd end to end on the reference's own golden runs: the per-iteration
images it writes and the final image against the reference program's."""
import os
import subprocess

import numpy as np
import pytest

from ctbb_icd_b200 import build as B

pytestmark = pytest.mark.gpu


def test_cli_sequential_matches_reference_program(golden):
    r = subprocess.run([B.CLI, "--sequential", golden.prm_path], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    n = golden.rp.geom.num_iterations
    shape = golden.rp.shape
    for it in range(0, n + 1):
        x = np.fromfile(os.path.join(golden.dir, "reconstructions", f"iteration{it}.rcn"), np.float64)
        ref = golden.iterations[it].ravel()
        assert np.linalg.norm(x - ref) <= 1e-12 * np.linalg.norm(ref), it
    out = np.fromfile(os.path.join(golden.dir, golden.rp.output_file), np.float32).reshape(shape)
    assert np.allclose(out, golden.final, rtol=1e-6, atol=1e-9)


def test_cli_grouped_runs(golden):
    r = subprocess.run([B.CLI, "-v", "--timing", golden.prm_path], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    out = np.fromfile(os.path.join(golden.dir, golden.rp.output_file), np.float32)
    assert out.size == int(np.prod(golden.rp.shape)) and np.isfinite(out).all()
