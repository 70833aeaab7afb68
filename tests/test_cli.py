"""The ctbb_icd command-line program (the reference's main.cpp flow): usage,
the empty parameter file, and the reference's error exit on a bad parameter
file. None of these reach the GPU."""
import os
import subprocess

from ctbb_icd_b200 import build as B
from ctbb_icd_b200 import workloads as W


def _run(*args):
    assert os.path.exists(B.CLI), "ctbb_icd is built by python -m ctbb_icd_b200.build"
    return subprocess.run([B.CLI, *args], capture_output=True, text=True, timeout=60)


def test_usage():
    r = _run()
    assert r.returncode == 0 and "usage: ctbb_icd [options] input_prm_file" in r.stdout


def test_empty_prm_lists_every_parameter_key():
    r = _run("--empty-prm")
    assert r.returncode == 0
    keys = {ln.split(":")[0].strip() for ln in r.stdout.splitlines() if ln and not ln.startswith("#") and ":" in ln}
    for name in ("tiny_ffs", "cfg2"):
        prm = W.workload(name)["prm"]
        missing = {k for k in prm if k not in keys}
        assert not missing, missing


def test_bad_parameter_file_exits_like_the_reference(tmp_path):
    p = tmp_path / "bad.prm"
    p.write_text("nx: 64\n")
    r = _run(str(p))
    assert r.returncode == 1
    assert "configure_recon_params failed" in r.stdout and "sinogram_path" in r.stdout
