"""Allocation-free backprojection: ufob_backproject_run_static() through the C
ABI must give the result of ufob_backproject_run() for the same properties,
and the FP64 oracle's, without allocating device memory.

It exists for callers that cannot call cudaMalloc (memory-pool hosts,
streaming acquisition); its only scratch is a fixed device
array shared by all calls, so two calls in a row with different geometry
check that each call rewrites what it reads.  This file is collected last."""
import ctypes

import numpy as np
import pytest
import torch

import oracle
import ufob

pytestmark = pytest.mark.gpu

TOL = 1e-5  # the relative L2 bound the backprojection tests use


def _props(**kw):
    p = ufob.BPProps()
    ufob.lib().ufob_bp_props_init(ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _run_static(props, sino, width, dtype=ufob.F32, layout=ufob.ROWS):
    L = ufob.lib()
    fn = L.ufob_backproject_run_static
    fn.argtypes = [ctypes.POINTER(ufob.BPProps), ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_uint32,
                   ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_void_p,
                   ctypes.c_void_p]
    fn.restype = ctypes.c_int
    nz, h, pitch = sino.shape
    ow = props.roi_width or width
    oh = props.roi_height or width
    out = torch.empty((nz, oh, ow), dtype=torch.float32, device="cuda")
    st = fn(ctypes.byref(props), sino.data_ptr(), dtype, layout, width, h, nz, pitch, pitch * h, out.data_ptr(),
            torch.cuda.current_stream().cuda_stream)
    return st, out


def _run_handle(props, sino, width, dtype=ufob.F32, layout=ufob.ROWS):
    L = ufob.lib()
    h = ctypes.c_void_p()
    ufob.check(L.ufob_backproject_create(ctypes.byref(props), ctypes.byref(h)))
    try:
        nz, rows, pitch = sino.shape
        ow = props.roi_width or width
        oh = props.roi_height or width
        out = torch.empty((nz, oh, ow), dtype=torch.float32, device="cuda")
        ufob.check(L.ufob_backproject_run(h, sino.data_ptr(), dtype, layout, width, rows, nz, pitch, pitch * rows,
                                          out.data_ptr(), torch.cuda.current_stream().cuda_stream))
        return out
    finally:
        L.ufob_backproject_destroy(h)


def _rel(a, b):
    return ((a.double() - b.double()).norm() / b.double().norm()).item()


def test_static_matches_allocating_entry_point_twice(cuda):
    rng = np.random.default_rng(42)
    # call 1: stack of 6 slices, 360 rows, 256 bins, axis and angle offset set
    s1 = torch.from_numpy(rng.standard_normal((6, 360, 256)).astype(np.float32)).cuda()
    p1 = _props(axis_pos=127.25, angle_offset=0.2)
    st, got1 = _run_static(p1, s1, 256)
    assert st == ufob.OK, ufob.lib().ufob_last_error()
    ref1 = _run_handle(p1, s1, 256)
    # call 2: different geometry and fewer rows, so stale table entries would show
    s2 = torch.from_numpy(rng.standard_normal((2, 100, 128)).astype(np.float32)).cuda()
    p2 = _props(num_projections=150, offset=30, angle_step=0.02, roi_x=8, roi_width=96, roi_height=80)
    st, got2 = _run_static(p2, s2, 128)
    assert st == ufob.OK, ufob.lib().ufob_last_error()
    ref2 = _run_handle(p2, s2, 128)
    torch.cuda.synchronize()
    assert _rel(got1, ref1) < TOL
    assert _rel(got2, ref2) < TOL
    # and the FP64 oracle of the reference's backproject task on the same rows
    o1 = oracle.backproject(s1[0].cpu().numpy(), axis_pos=127.25, angle_offset=0.2)
    assert oracle.rel_l2(got1[0].cpu().numpy(), o1) < TOL
    o2 = oracle.backproject(s2[1].cpu().numpy(), num_projections=150, offset=30, angle_step=0.02, roi_x=8,
                            roi_width=96, roi_height=80)
    assert oracle.rel_l2(got2[1].cpu().numpy(), o2) < TOL


def test_static_allocates_nothing(cuda):
    """Neither the engine's allocation counter nor the device's free memory moves across calls
    (after the first call on the device, which loads the module and looks up the table)."""
    L = ufob.lib()
    L.ufob_device_alloc_count.restype = ctypes.c_uint64
    rng = np.random.default_rng(5)
    s = torch.from_numpy(rng.standard_normal((3, 720, 384)).astype(np.float32)).cuda()
    p = _props(axis_pos=190.5)
    st, warm = _run_static(p, s, 384)
    assert st == ufob.OK, ufob.lib().ufob_last_error()
    out = torch.empty_like(warm)
    torch.cuda.synchronize()
    allocs, free = L.ufob_device_alloc_count(), torch.cuda.mem_get_info()[0]
    fn = L.ufob_backproject_run_static
    for _ in range(2):
        st = fn(ctypes.byref(p), s.data_ptr(), ufob.F32, ufob.ROWS, 384, 720, 3, 384, 384 * 720, out.data_ptr(),
                torch.cuda.current_stream().cuda_stream)
        assert st == ufob.OK, ufob.lib().ufob_last_error()
    torch.cuda.synchronize()
    assert L.ufob_device_alloc_count() == allocs
    assert torch.cuda.mem_get_info()[0] == free
    assert torch.equal(out, warm)


def test_static_single_sinogram(cuda):
    """One sinogram of 512 bins x 1536 rows: the allocating entry point splits it into angle groups
    (partial images summed), the static one runs it whole; equal within round-off."""
    rng = np.random.default_rng(11)
    s = torch.from_numpy(rng.standard_normal((1, 1536, 512)).astype(np.float32)).cuda()
    p = _props(axis_pos=255.5)
    st, got = _run_static(p, s, 512)
    assert st == ufob.OK, ufob.lib().ufob_last_error()
    ref = _run_handle(p, s, 512)
    assert _rel(got, ref) < TOL
    assert oracle.rel_l2(got[0].cpu().numpy(), oracle.backproject(s[0].cpu().numpy(), axis_pos=255.5)) < TOL


def test_static_pairs_form(cuda):
    rng = np.random.default_rng(7)
    raw = torch.from_numpy(rng.standard_normal((4, 200, 128)).astype(np.float32)).cuda()
    pairs = ufob.FilterTask().process(raw, dtype=ufob.F16, layout=ufob.PAIRS)
    p = _props(compensated=1)
    st, got = _run_static(p, pairs, 128, ufob.F16, ufob.PAIRS)
    assert st == ufob.OK, ufob.lib().ufob_last_error()
    ref = _run_handle(p, pairs, 128, ufob.F16, ufob.PAIRS)
    assert _rel(got, ref) < TOL


def test_static_rejects_sizes_beyond_the_table(cuda):
    sino = torch.zeros((1, 8, 64), dtype=torch.float32, device="cuda")
    L = ufob.lib()
    fn = L.ufob_backproject_run_static
    fn.argtypes = [ctypes.POINTER(ufob.BPProps), ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_uint32,
                   ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_void_p,
                   ctypes.c_void_p]
    out = torch.empty((1, 64, 64), device="cuda")
    p = _props()
    st = fn(ctypes.byref(p), sino.data_ptr(), ufob.F32, ufob.ROWS, 64, 32769, 1, 64, 0, out.data_ptr(), None)
    assert st == ufob.ERR_UNSUPPORTED
    assert b"static angle table" in L.ufob_last_error()
