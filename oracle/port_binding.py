"""ctypes binding of the oracle's CPU restatement (oracle/_ref/liboracle_port.so,
built from oracle/port.cpp by `make -C oracle port`).

TEST INFRASTRUCTURE / CPU BASELINE ONLY: loaded by tests/, bench.py's
reference arm and CPU-baseline leg, and __graft_entry__.smoke() as the
checker. It needs only the ctypes struct definitions of the C ABI header
(ctbb_icd_b200._lib, pure Python); it never loads the product library."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

ORACLE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(ORACLE, "_ref", "liboracle_port.so")

_port = None


def port():
    """The loaded oracle library, built on first use if missing."""
    global _port
    if _port is None:
        from ctbb_icd_b200._lib import GeomC, PhantomSpec

        if not os.path.exists(PORT_LIB):
            subprocess.run(["make", "-s", "-C", ORACLE, "port"], check=True)
        L = C.CDLL(PORT_LIB)
        PG = C.POINTER(GeomC)
        PD, PF, PU, PI, PI64 = (C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_uint64),
                                C.POINTER(C.c_int32), C.POINTER(C.c_int64))
        L.port_ssm_build.restype = C.c_void_p
        L.port_ssm_build.argtypes = [PG]
        L.port_ssm_nnz.restype = C.c_uint64
        L.port_ssm_nnz.argtypes = [C.c_void_p]
        L.port_ssm_copy.argtypes = [C.c_void_p, PI64, PI, PF]
        L.port_ssm_free.argtypes = [C.c_void_p]
        L.port_ssm_subset.restype = C.c_uint64
        L.port_ssm_subset.argtypes = [PG, C.c_int, PI64, C.c_int, PI, C.POINTER(C.c_uint32), PI, PF, C.c_uint64]
        L.port_icd.argtypes = [PG, PU, PF, PI64, PI, PF, PD, PD, C.c_int, PD]
        L.port_rotate.argtypes = [PG, PD, PU, PF, C.c_int]
        L.port_forward.argtypes = [PG, PU, PI64, PI, PF, PD, PD]
        L.port_cost.restype = C.c_double
        L.port_cost.argtypes = [PG, PU, PF, PI64, PI, PF, PD, PD, PD]
        L.port_synth.argtypes = [PG, C.POINTER(PhantomSpec), PF]
        L.port_penalty_steps.argtypes = [C.c_int, C.c_double, C.c_double, C.c_uint64, PD, PD, PF, PD]
        _port = L
    return _port


def ptr(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))
