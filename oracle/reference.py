"""The reference itself, run on the CPU (TEST INFRASTRUCTURE ONLY).

``_ref/libufo_ref.so`` (built by ``make -f ref.mk`` from the reference sources)
holds the reference's own ``filter`` and ``backproject`` task code
(src/ufo-filter-task.c, src/ufo-backproject-task.c) and its OpenCL kernels
(src/kernels/backproject.cl, filter.cl, fft.cl, forwardproject.cl, ffc.cl,
conebeam.cl) compiled for the CPU against small GLib/OpenCL/ufo-core shims.  The FFT library the
reference calls (vendored oclfft or clFFT) is replaced by an FP64 FFT.

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
