import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: longer-running test")


def _ensure_built():
    from ctbb_icd_b200 import build as B

    if not os.path.exists(B.LIB):
        B.build()
    port = os.path.join(ROOT, "oracle", "_ref", "liboracle_port.so")
    if not os.path.exists(port):
        B.build_oracle()


_ensure_built()


class Golden:
    """One golden fixture produced by the reference program (make_golden.py)."""

    def __init__(self, name, tmpdir):
        import ctbb_icd_b200 as C

        z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
        self.name = name
        self.dir = str(tmpdir)
        os.makedirs(os.path.join(self.dir, "reconstructions"), exist_ok=True)
        self.prm_path = os.path.join(self.dir, f"{name}.prm")
        with open(self.prm_path, "w") as f:
            f.write(str(z["prm"]).replace("@DIR@", self.dir))
        self.raw = z["raw"]
        self.raw.tofile(os.path.join(self.dir, f"{name}.bin"))
        self.colptr, self.idx, self.w = z["colptr"], z["idx"], z["w"]
        self.iterations = z["iterations"]
        self.final = z["final"]
        self.setup_dump = str(z["setup_dump"])
        self.rp = C.configure_recon_params(self.prm_path)
        self.data = C.load_raw(self.rp)

    def csr(self):
        from oracle_util import Csr

        return Csr(self.colptr, self.idx, self.w)


@pytest.fixture(scope="session", params=["tiny", "tiny_ffs", "tiny_zffs", "tiny_zphiffs"])
def golden(request, tmp_path_factory):
    return Golden(request.param, tmp_path_factory.mktemp(request.param))


def has_gpu():
    try:
        import ctypes

        from ctbb_icd_b200._lib import lib

        h = ctypes.c_void_p()
        st = lib().ctbb_gpu_init(0, None, ctypes.byref(h))
        if st == 0:
            lib().ctbb_gpu_destroy(h)
            return True
    except Exception:
        pass
    return False


@pytest.fixture(scope="session")
def ctx():
    import ctbb_icd_b200 as C

    if not has_gpu():
        pytest.fail("GPU test needs a CUDA device (the CUDA path has no CPU fallback)")
    c = C.Context(0)
    yield c
    c.close()
