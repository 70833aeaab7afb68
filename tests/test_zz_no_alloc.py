"""The allocation-free rotation entry point, ctbb_gpu_rotate_device_noalloc.

It exists for callers that cannot let the library allocate device memory
(fixed up-front memory pools, allocation-free real-time loops). This file is
collected last so a run that stops at the first failure has already run every
other test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import ctbb_icd_b200 as C
from ctbb_icd_b200 import workloads as W
from ctbb_icd_b200._lib import lib

pytestmark = pytest.mark.gpu


def _rotate(fn_name, ctx, rp, tables, d_in, d_out, direction):
    fn = getattr(lib(), fn_name)
    return fn(ctx.handle, ctypes.byref(rp.geom), C.ptr(tables.tube_angles, ctypes.c_double),
              C.ptr(tables.slice_indices, ctypes.c_uint64), ctypes.c_void_p(d_in.data_ptr()),
              ctypes.c_void_p(d_out.data_ptr()), int(direction))


def test_noalloc_rotation_matches_allocating_entry_point(ctx, tmp_path):
    import torch

    _, rp = W.materialise("mid", str(tmp_path), raw=False)
    tables = C.slice_tables(rp)
    rng = np.random.default_rng(11)
    for call, direction in enumerate((C.ROTATE_ROTATING2FIXED, C.ROTATE_FIXED2ROTATING)):
        vol = torch.from_numpy(rng.random(rp.shape, dtype=np.float32)).cuda()
        ref = torch.empty_like(vol)
        out = torch.full_like(vol, float("nan"))
        torch.cuda.synchronize()
        C.check(_rotate("ctbb_gpu_rotate_device", ctx, rp, tables, vol, ref, direction))
        C.check(_rotate("ctbb_gpu_rotate_device_noalloc", ctx, rp, tables, vol, out, direction))
        torch.cuda.synchronize()
        a, b = ref.cpu().numpy(), out.cpu().numpy()
        # Same kernel and inputs: bit-identical, like the rotation parity tests.
        assert np.array_equal(a.view(np.int32), b.view(np.int32)), f"call {call}"


def test_noalloc_rotation_rejects_too_many_slices(ctx, tmp_path):
    import torch

    _, rp = W.materialise("tiny", str(tmp_path), raw=False)
    tables = C.slice_tables(rp)
    g = C.GeomC.from_buffer_copy(rp.geom)
    g.num_voxels_z = 8193
    d = torch.zeros(16, device="cuda")
    fn = lib().ctbb_gpu_rotate_device_noalloc
    st = fn(ctx.handle, ctypes.byref(g), C.ptr(tables.tube_angles, ctypes.c_double),
            C.ptr(tables.slice_indices, ctypes.c_uint64), ctypes.c_void_p(d.data_ptr()),
            ctypes.c_void_p(d.data_ptr() + 4), -1)
    assert st == 1 and b"8192" in lib().ctbb_last_error()


def _fill_device_memory():
    """cudaMalloc the device until allocations of 256 bytes fail; returns the
    pointers (to be freed with _release)."""
    from cuda.bindings import runtime as rt

    ptrs = []
    err, free, _ = rt.cudaMemGetInfo()
    assert err == rt.cudaError_t.cudaSuccess
    size = int(free)
    while size >= 256:
        err, p = rt.cudaMalloc(size)
        if err == rt.cudaError_t.cudaSuccess:
            ptrs.append(p)
        else:
            size //= 2
    rt.cudaGetLastError()  # the failed cudaMalloc calls leave no sticky error; clear the last one
    return ptrs


def _release(ptrs):
    from cuda.bindings import runtime as rt

    for p in ptrs:
        rt.cudaFree(p)


def test_noalloc_rotation_runs_with_no_device_memory_left(ctx, tmp_path):
    """With every byte of device memory taken, the allocation-free entry point
    still rotates (bit-identical to before), while the allocating one, the
    positive control, fails with CTBB_ERR_OOM: an allocation inside the
    no-alloc path would fail the same way."""
    import torch

    _, rp = W.materialise("mid", str(tmp_path), raw=False)
    tables = C.slice_tables(rp)
    vol = torch.from_numpy(np.random.default_rng(5).random(rp.shape, dtype=np.float32)).cuda()
    ref = torch.empty_like(vol)
    out = torch.full_like(vol, float("nan"))
    out2 = torch.full_like(vol, float("nan"))
    d = C.ROTATE_ROTATING2FIXED
    C.check(_rotate("ctbb_gpu_rotate_device", ctx, rp, tables, vol, ref, d))
    C.check(_rotate("ctbb_gpu_rotate_device_noalloc", ctx, rp, tables, vol, out, d))  # device set-up done
    torch.cuda.synchronize()
    filler = _fill_device_memory()
    try:
        st_noalloc = _rotate("ctbb_gpu_rotate_device_noalloc", ctx, rp, tables, vol, out2, d)
        st_alloc = _rotate("ctbb_gpu_rotate_device", ctx, rp, tables, vol, out, d)
    finally:
        _release(filler)
    assert st_noalloc == 0, lib().ctbb_last_error()
    assert st_alloc == 7, (st_alloc, lib().ctbb_last_error())  # CTBB_ERR_OOM
    torch.cuda.synchronize()
    a, b = ref.cpu().numpy(), out2.cpu().numpy()
    assert np.array_equal(a.view(np.int32), b.view(np.int32))
