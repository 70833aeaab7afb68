"""The reference's wFBP start, pinned against the oracle. CPU only.

With wfbp_initialize set, icd_iteration.cpp:63-116 forward-projects the
initial image into its FP64 sinogram estimate before the first iteration,
re-aligning each slice's central view to the first view of its flying
focal spot stack (:90-94). The wFBP image itself comes from an external
program, but initialize_recon_volume.cpp:57-76 loads initial_recon_path
first when it is given and then runs no external program, so the
reference program runs this path here on a chosen image. The oracle's
forward projection (port_forward) followed by its sequential ICD from that
estimate reproduces the reference's first two iterations.

The GPU side of the chain: ctbb_gpu_icd and icd_iteration start from
e = y - A x0 when wfbp_initialize is set (CTBB_ESTIMATE_FORWARD), and the
GPU's FP64 forward projection matches port_forward
(tests/test_gpu_parity.py::test_refresh_residual_and_cost_match_port).
"""
import os

import numpy as np
import pytest

import ctbb_icd_b200 as C
import oracle_util as O
from oracle import reference_run as R

pytestmark = pytest.mark.skipif(not R.available(), reason="reference program not built (oracle/Makefile ref)")


@pytest.mark.parametrize("name", ["tiny", "tiny_ffs"])
def test_wfbp_start_forward_projection_matches_oracle(name, tmp_path):
    from conftest import Golden

    g0 = Golden(name, tmp_path / "golden")
    d = str(tmp_path)
    os.makedirs(os.path.join(d, "reconstructions"), exist_ok=True)
    x0 = (g0.iterations[1] * 0.5).astype(np.float32)  # a non-zero start
    x0_path = os.path.join(d, "x0.img")
    x0.tofile(x0_path)
    text = open(g0.prm_path).read().replace(g0.dir, d)
    text = "\n".join(l for l in text.splitlines()
                     if not l.startswith(("num_iterations", "initial_recon_path", "wfbp_initialize")))
    text += f"\nnum_iterations: 2\ninitial_recon_path: {x0_path}\nwfbp_initialize: 1\n"
    prm_path = os.path.join(d, "start.prm")
    with open(prm_path, "w") as f:
        f.write(text)
    g0.raw.tofile(os.path.join(d, f"{name}.bin"))
    rc_ref, stamps = R.run("O2", prm_path, d, threads=2)
    assert rc_ref == 0, stamps[-5:]

    rp = C.configure_recon_params(prm_path)
    assert rp.geom.wfbp_initialize == 1
    data = C.load_raw(rp)
    ssm = g0.csr()
    est0 = O.port_forward(rp, data.slice_indices, ssm, x0.astype(np.float64))
    dumps, _, _ = O.port_icd(rp, data.slice_indices, data.raw, ssm, 2, x0=x0, est0=est0)
    for it in (1, 2):
        ref = np.fromfile(os.path.join(d, "reconstructions", f"iteration{it}.rcn"), np.float64).reshape(rp.shape)
        rel = np.linalg.norm(dumps[it - 1] - ref) / np.linalg.norm(ref)
        assert rel < 1e-12, (name, it, rel)
    # The forward-projected start differs from the zero-estimate start.
    zero_dumps, _, _ = O.port_icd(rp, data.slice_indices, data.raw, ssm, 1, x0=x0)
    ref1 = np.fromfile(os.path.join(d, "reconstructions", "iteration1.rcn"), np.float64).reshape(rp.shape)
    assert np.linalg.norm(zero_dumps[0] - ref1) > 1e-6 * np.linalg.norm(ref1)
