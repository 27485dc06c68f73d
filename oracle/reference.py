"""The reference itself, run on the CPU (TEST INFRASTRUCTURE ONLY).

``_ref/libufo_ref.so`` (built by ``make -f ref.mk`` from the reference sources)
holds the reference's own ``filter``, ``backproject`` and ``general-backproject``
task code (src/ufo-filter-task.c, src/ufo-backproject-task.c,
src/ufo-general-backproject-task.c with src/common/ufo-scarray.c,
ufo-ctgeometry.c, ufo-conebeam.c) and its OpenCL kernels
(src/kernels/backproject.cl, filter.cl, fft.cl, forwardproject.cl, ffc.cl,
conebeam.cl) compiled for the CPU against small GLib/OpenCL/ufo-core shims.  The FFT library the
reference calls (vendored oclfft or clFFT) is replaced by an FP64 FFT.  The
kernels ``general-backproject`` generates at run time from
src/kernels/templates/general_bp_*.in, and the ``lamino-backproject`` kernels
its build writes with src/kernels/tools/make_burst_kernels.py (run here the way
src/kernels/meson.build:59-83 runs it), are compiled for the CPU when the tasks
ask for them (refshim/ref_clc_jit.cpp), which needs the reference tree
(``UFO_FILTERS_SOURCE``) and g++.  ``lamino-backproject`` (src/ufo-lamino-
backproject-task.c, src/lamino-roi.c) and ``stacked-backproject``
(src/ufo-stacked-backproject-task.c; src/kernels/stacked-backproject.cl, whose
work-groups run as OpenMP teams) are in the library too.

Used to pin the FP64 oracle (oracle.py) and to generate the golden fixtures
under tests/golden/, and as the reference arm of the CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libufo_ref.so")
REF_SOURCE = os.environ.get("UFO_FILTERS_SOURCE", "/root/reference")
_LIB = None

FILTERS = ["ramp", "ramp-fromreal", "butterworth", "faris-byer", "hamming", "bh3"]


def available():
    return os.path.exists(LIB_PATH)


def build():
    """Build _ref/ from the reference sources (needs them on this machine)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "-f", "ref.mk"])


def lib():
    global _LIB
    if _LIB is None:
        if not available():
            raise RuntimeError("reference CPU build missing: run `make -C oracle -f ref.mk` where the reference "
                               "sources are present")
        L = ctypes.CDLL(LIB_PATH)
        vp, u, i, f, d = ctypes.c_void_p, ctypes.c_uint, ctypes.c_int, ctypes.c_float, ctypes.c_double
        L.ref_filter_run.argtypes = [i, f, f, f, f, f, u, u, vp, vp, vp, ctypes.c_char_p, i]
        L.ref_filter_run.restype = i
        L.ref_backproject_run.argtypes = [vp, u, u, vp, ctypes.c_size_t, u, u, d, d, d, i, u, u, u, u,
                                          ctypes.POINTER(u), ctypes.POINTER(u), ctypes.c_char_p, i]
        L.ref_backproject_run.restype = i
        L.ref_fft_spread.argtypes = [vp, vp, i, i, i]
        L.ref_fft_pack.argtypes = [vp, vp, i, i, i, f]
        L.refshim_fft.argtypes = [vp, ctypes.c_size_t, ctypes.c_size_t, i]
        L.ref_forwardproject.argtypes = [vp, i, i, f, f, vp]
        L.ref_flat_correct.argtypes = [vp, vp, vp, vp, i, i, i, i, i, f, f]
        L.ref_weight_projection.argtypes = [vp, vp, i, i, f, f, f, f, f, f]
        L.ref_gbp_new.restype = vp
        L.ref_gbp_set.argtypes = [vp, ctypes.c_char_p, vp, u, ctypes.c_char_p]
        L.ref_gbp_set.restype = i
        L.ref_gbp_run.argtypes = [vp, vp, u, u, u, vp, ctypes.c_size_t, ctypes.POINTER(u), ctypes.c_char_p, i]
        L.ref_gbp_run.restype = i
        L.ref_lamino_new.restype = vp
        L.ref_lamino_set.argtypes = [vp, ctypes.c_char_p, vp, u, ctypes.c_char_p]
        L.ref_lamino_set.restype = i
        L.ref_lamino_run.argtypes = [vp, vp, u, u, u, vp, ctypes.c_size_t, ctypes.POINTER(u), ctypes.c_char_p, i]
        L.ref_lamino_run.restype = i
        L.ref_stacked_new.restype = vp
        L.ref_stacked_set.argtypes = [vp, ctypes.c_char_p, d, ctypes.c_char_p]
        L.ref_stacked_set.restype = i
        L.ref_stacked_run.argtypes = [vp, vp, u, u, u, vp, ctypes.c_size_t, ctypes.POINTER(u), ctypes.c_char_p, i]
        L.ref_stacked_run.restype = i
        L.refshim_set_dirs.argtypes = [ctypes.c_char_p] * 3
        L.refshim_set_device_limits.argtypes = [ctypes.c_ulong] * 3
        L.refshim_set_dirs(os.path.join(REF_SOURCE, "src", "kernels").encode(),
                           os.path.join(HERE, "refshim").encode(), os.path.join(HERE, "_ref", "jit").encode())
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def filter_coefficients(nfft, filter="ramp-fromreal", cutoff=0.5, order=4.0, tau=0.1, theta=1.0, scale=1.0):
    """The coefficient vector the reference's filter task builds (2*nfft floats)."""
    coeff = np.zeros(2 * nfft, dtype=np.float32)
    err = ctypes.create_string_buffer(512)
    ftype = FILTERS.index(filter) if isinstance(filter, str) else int(filter)
    rc = lib().ref_filter_run(ftype, cutoff, order, tau, theta, scale, 2 * nfft, 1, None, None, _p(coeff), err, 512)
    if rc:
        raise ValueError(err.value.decode())
    return coeff


def fft_filter_ifft(sino, size_x=0, crop_width=0, **filter_props):
    """``fft ! filter ! ifft`` through the reference's kernels and filter task
    (FP32 data, FP64 transforms)."""
    sino = np.ascontiguousarray(sino, dtype=np.float32)
    shape = sino.shape
    W = shape[-1]
    rows = int(np.prod(shape[:-1]))
    nfft = size_x if size_x else W
    crop = crop_width if crop_width else nfft
    L = lib()
    spec = np.zeros((rows, 2 * nfft), dtype=np.float32)
    L.ref_fft_spread(_p(spec), _p(sino), W, rows, nfft)
    L.refshim_fft(_p(spec), nfft, rows, 1)
    filt = np.zeros_like(spec)
    err = ctypes.create_string_buffer(512)
    ftype = filter_props.get("filter", "ramp-fromreal")
    ftype = FILTERS.index(ftype) if isinstance(ftype, str) else int(ftype)
    rc = L.ref_filter_run(ftype, filter_props.get("cutoff", 0.5), filter_props.get("order", 4.0),
                          filter_props.get("tau", 0.1), filter_props.get("theta", 1.0), filter_props.get("scale", 1.0),
                          2 * nfft, rows, _p(spec), _p(filt), None, err, 512)
    if rc:
        raise ValueError(err.value.decode())
    L.refshim_fft(_p(filt), nfft, rows, 0)
    out = np.zeros((rows, crop), dtype=np.float32)
    L.ref_fft_pack(_p(filt), _p(out), crop, rows, nfft, np.float32(1.0 / nfft))
    return out.reshape(shape[:-1] + (crop,))


def backproject(sino, num_projections=0, offset=0, axis_pos=-1.0, angle_step=-1.0, angle_offset=0.0,
                mode="texture", roi_x=0, roi_y=0, roi_width=0, roi_height=0):
    """The reference's backproject task (backproject.cl on the CPU, exact linear weights)."""
    sino = np.ascontiguousarray(sino, dtype=np.float32)
    P, W = sino.shape
    ow = roi_width if roi_width else W
    oh = roi_height if roi_height else W
    out = np.zeros(ow * oh, dtype=np.float32)
    rw, rh = ctypes.c_uint(), ctypes.c_uint()
    err = ctypes.create_string_buffer(512)
    rc = lib().ref_backproject_run(_p(sino), W, P, _p(out), out.size, num_projections, offset, axis_pos, angle_step,
                                   angle_offset, 0 if mode == "nearest" else 1, roi_x, roi_y, roi_width, roi_height,
                                   ctypes.byref(rw), ctypes.byref(rh), err, 512)
    if rc:
        raise ValueError(err.value.decode())
    return out[:rw.value * rh.value].reshape(rh.value, rw.value)


def fbp(sino, axis_pos=-1.0, size_x=0, crop_width=0, filter_props=None, **bp_props):
    filt = fft_filter_ifft(sino, size_x=size_x, crop_width=crop_width, **(filter_props or {}))
    return backproject(filt, axis_pos=axis_pos, **bp_props)


def forwardproject(slice_img, n_angles, axis_pos, angle_step):
    img = np.ascontiguousarray(slice_img, dtype=np.float32)
    W = img.shape[-1]
    out = np.zeros((n_angles, W), dtype=np.float32)
    lib().ref_forwardproject(_p(img), W, n_angles, axis_pos, angle_step, _p(out))
    return out


def flat_field_correct(data, dark, flat, absorption_correct=False, fix_nan_and_inf=False, sinogram_input=False,
                       dark_scale=1.0, flat_scale=1.0):
    """src/kernels/ffc.cl on each frame [H, W] of data [..., H, W]."""
    data = np.ascontiguousarray(data, dtype=np.float32)
    dark = np.ascontiguousarray(dark, dtype=np.float32)
    flat = np.ascontiguousarray(flat, dtype=np.float32)
    H, W = data.shape[-2:]
    frames = data.reshape(-1, H, W)
    out = np.empty_like(frames)
    for i in range(frames.shape[0]):
        fr = np.ascontiguousarray(frames[i])
        lib().ref_flat_correct(_p(out[i]), _p(fr), _p(dark), _p(flat), W, H, int(sinogram_input),
                               int(absorption_correct), int(fix_nan_and_inf), float(dark_scale), float(flat_scale))
    return out.reshape(data.shape)


def weight_projection(proj, cx, cz, sd, od, mr, cs):
    """src/kernels/conebeam.cl on one projection [H, W] with the task's FP32 kernel arguments."""
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    H, W = proj.shape
    out = np.empty_like(proj)
    lib().ref_weight_projection(_p(proj), _p(out), W, H, float(cx), float(cz), float(sd), float(od), float(mr),
                                float(cs))
    return out


GBP_ENUMS = ("parameter", "compute-type", "result-type", "store-type", "addressing-mode")
GBP_STORE_DTYPES = {"half": np.float16, "float": np.float32, "double": np.float64, "uchar": np.uint8,
                    "ushort": np.uint16, "uint": np.uint32}


def general_backproject(proj, props, max_alloc_slices=0):
    """The reference's ``general-backproject`` task over projections ``proj``
    [n, height, width] with ``props`` = {reference property name: value}
    (scalars, sequences for the array properties, value nicks for the
    enumerations).  The task generates its OpenCL kernel (make_kernel), which
    runs on the CPU with the exact-weight linear sampler.  ``max_alloc_slices``
    > 0 reports a device allocation limit of that many slices so that the task
    splits its volume into chunks.  Returns the volume [slices, y, x] in the
    store type."""
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    n, h, w = proj.shape
    L = lib()
    t = L.ref_gbp_new()
    props = dict(props)
    props.setdefault("num-projections", n)
    store = props.get("store-type", "float")
    for name, value in props.items():
        if name in GBP_ENUMS:
            rc = L.ref_gbp_set(t, name.encode(), None, 0, str(value).encode())
        else:
            arr = np.atleast_1d(np.asarray(value, dtype=np.float64))
            rc = L.ref_gbp_set(t, name.encode(), _p(arr), arr.size, None)
        if rc:
            raise ValueError("general-backproject: unknown property or value %s=%r" % (name, value))
    dims = (ctypes.c_uint * 4)()
    err = ctypes.create_string_buffer(512)
    # first pass: requisition only (volume dimensions)
    probe = L.ref_gbp_new()
    for name, value in props.items():
        if name in GBP_ENUMS:
            L.ref_gbp_set(probe, name.encode(), None, 0, str(value).encode())
        else:
            arr = np.atleast_1d(np.asarray(value, dtype=np.float64))
            L.ref_gbp_set(probe, name.encode(), _p(arr), arr.size, None)
    rc = L.ref_gbp_run(probe, _p(proj), w, h, min(n, 1), None, 0, dims, err, 512)
    if rc < 0:
        raise ValueError(err.value.decode())
    nx, ny, nz, bpp = dims[0], dims[1], dims[2], dims[3]
    slice_bytes = nx * ny * bpp
    L.refshim_set_device_limits(64 << 30, slice_bytes * max_alloc_slices if max_alloc_slices else 4 << 30, 256)
    try:
        out = np.zeros((nz, ny, nx), dtype=GBP_STORE_DTYPES[store])
        rc = L.ref_gbp_run(t, _p(proj), w, h, n, _p(out), out.nbytes, dims, err, 512)
    finally:
        L.refshim_set_device_limits(64 << 30, 4 << 30, 256)
    if rc < 0:
        raise ValueError(err.value.decode())
    return out


LAMINO_KERNELS = ("z", "lamino", "center", "roll")
LAMINO_ENUMS = ("parameter", "addressing-mode")


def _lamino_kernel_files():
    """Write {z,lamino,center,roll}_kernel.cl with the reference's generator, with the bursts
    its build passes (src/kernels/meson.build:66-70)."""
    jit = os.path.join(HERE, "_ref", "jit")
    os.makedirs(jit, exist_ok=True)
    tools = os.path.join(REF_SOURCE, "src", "kernels", "tools", "make_burst_kernels.py")
    for name in LAMINO_KERNELS:
        path = os.path.join(jit, name + "_kernel.cl")
        if not os.path.exists(path):
            tmpl = os.path.join(REF_SOURCE, "src", "kernels", "templates", name + "_template.in")
            src = subprocess.check_output(["python3", tools, tmpl, "1", "2", "4", "8", "16"], text=True)
            with open(path + ".tmp", "w") as f:
                f.write(src)
            os.replace(path + ".tmp", path)


def lamino_backproject(proj, props):
    """The reference's ``lamino-backproject`` task over projections [n, height, width] with
    ``props`` = {reference property name: value}; returns the FP32 volume [z, y, x]."""
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    n, h, w = proj.shape
    _lamino_kernel_files()
    L = lib()
    t = L.ref_lamino_new()
    props = dict(props)
    props.setdefault("num-projections", n)
    for name, value in props.items():
        if name in LAMINO_ENUMS:
            rc = L.ref_lamino_set(t, name.encode(), None, 0, str(value).encode())
        else:
            arr = np.atleast_1d(np.asarray(value, dtype=np.float64))
            rc = L.ref_lamino_set(t, name.encode(), _p(arr), arr.size, None)
        if rc:
            raise ValueError("lamino-backproject: unknown property or value %s=%r" % (name, value))
    dims = (ctypes.c_uint * 4)()
    err = ctypes.create_string_buffer(512)
    rc = L.ref_lamino_run(t, _p(proj), w, h, 0, None, 0, dims, err, 512)
    if rc < 0:
        raise ValueError(err.value.decode())
    out = np.zeros((dims[2], dims[1], dims[0]), dtype=np.float32)
    t = L.ref_lamino_new()
    for name, value in props.items():
        if name in LAMINO_ENUMS:
            L.ref_lamino_set(t, name.encode(), None, 0, str(value).encode())
        else:
            arr = np.atleast_1d(np.asarray(value, dtype=np.float64))
            L.ref_lamino_set(t, name.encode(), _p(arr), arr.size, None)
    rc = L.ref_lamino_run(t, _p(proj), w, h, n, _p(out), out.size, dims, err, 512)
    if rc < 0:
        raise ValueError(err.value.decode())
    return out


def stacked_backproject(sino, props):
    """The reference's ``stacked-backproject`` task on a stack [z, projections, width] with
    ``props`` = {reference property name: value} ("precision-mode" by nick); returns the FP32
    volume [z, roi height, roi width] (slices past the last full group of 2 or 4, which the task
    leaves unwritten, stay zero)."""
    sino = np.ascontiguousarray(sino, dtype=np.float32)
    z, rows, w = sino.shape
    L = lib()

    def task():
        t = L.ref_stacked_new()
        for name, value in props.items():
            if name == "precision-mode":
                rc = L.ref_stacked_set(t, name.encode(), 0.0, str(value).encode())
            else:
                rc = L.ref_stacked_set(t, name.encode(), float(value), None)
            if rc:
                raise ValueError("stacked-backproject: unknown property or value %s=%r" % (name, value))
        return t

    dims = (ctypes.c_uint * 4)()
    err = ctypes.create_string_buffer(512)
    if L.ref_stacked_run(task(), _p(sino), w, rows, z, None, 0, dims, err, 512) < 0:
        raise ValueError(err.value.decode())
    out = np.zeros((dims[2], dims[1], dims[0]), dtype=np.float32)
    if L.ref_stacked_run(task(), _p(sino), w, rows, z, _p(out), out.size, dims, err, 512) < 0:
        raise ValueError(err.value.decode())
    return out
