"""CPU oracle for the filtered-backprojection path (TEST INFRASTRUCTURE ONLY).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this module, and only as the checker.  The engine under
``ufo-filters_b200/`` never calls it.

It restates in NumPy/FP64 what the reference ufo-filters tasks compute:

* ``filter_coefficients`` -- src/ufo-filter-task.c:162-336 (ramp, ramp-fromreal,
  butterworth, faris-byer, hamming, bh3; mirroring; ramp-fromreal's FFT).
* ``fft_filter_ifft`` -- the ``fft ! filter ! ifft`` chain:
  src/ufo-fft-task.c:123-196,293-336 (spread/zero-pad to size-x),
  src/kernels/filter.cl:20-29 (element-wise multiply of the interleaved floats),
  src/ufo-ifft-task.c:111-177,287-311 (backward FFT, real part, crop, 1/N).
* ``backproject`` -- src/ufo-backproject-task.c:96-150,174-267 and
  src/kernels/backproject.cl:24-94 (via the C oracle).
* ``general_backproject`` -- src/ufo-general-backproject-task.c (via the C oracle).
* ``stacked_backproject`` -- src/ufo-stacked-backproject-task.c,
  src/kernels/stacked-backproject.cl (three precision modes).
* ``lamino_backproject`` -- src/ufo-lamino-backproject-task.c and the kernels
  generated from src/kernels/templates/*_template.in.
* ``flat_field_correct`` -- src/kernels/ffc.cl:20-50 with the task's arguments
  (src/ufo-flat-field-correct-task.c:120-170), in FP32.
* ``transpose_projections`` -- src/ufo-transpose-projections-task.c:60-120.
* ``cone_weight_params`` / ``cone_beam_weight`` --
  src/ufo-cone-beam-projection-weight-task.c:113-151 and
  src/kernels/conebeam.cl:20-36, in FP32.

The heavy loops live in ``ufob_oracle.c`` (built into ``liboracle.so`` by the
Makefile next to this file).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

FILTERS = ["ramp", "ramp-fromreal", "butterworth", "faris-byer", "hamming", "bh3"]

INTERP_EXACT, INTERP_TEX8, INTERP_NEAREST = 0, 1, 2
ADDR_CLAMP, ADDR_CLAMP_TO_EDGE = 0, 1

# geometry table columns (must match ufob_oracle.c)
GEOM_COLS = [
    "axis-angle-z", "axis-angle-x", "axis-angle-y",
    "volume-angle-x", "volume-angle-y", "volume-angle-z",
    "detector-angle-x", "detector-angle-y", "detector-angle-z",
    "center-position-x", "center-position-z",
    "source-position-x", "source-position-y", "source-position-z",
    "detector-position-x", "detector-position-y", "detector-position-z",
]
F_WITH_AXIS, F_WITH_VOLUME, F_PERPENDICULAR = 1, 2, 4
F_SHIFTED_DETECTOR, F_SHIFTED_SOURCE, F_PARALLEL = 8, 16, 32


def lib():
    """Load (building on first use) the C oracle."""
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        src = os.path.join(HERE, "ufob_oracle.c")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])
        _LIB = ctypes.CDLL(path)
        d, i, pf, pd = ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p
        _LIB.oracle_bp_parallel.argtypes = [pf, i, i, i, pd, pd, i, d, i, i, i, i, i, pd]
        _LIB.oracle_gbp.argtypes = [pf, i, i, i, pd, i, i, pd, d, d, d, d, d, i, i, i, d, i, i, pd]
        _LIB.oracle_gbp_project_point.argtypes = [pd, i, d, d, d, pd, pd]
        _LIB.oracle_gbp_project_point.restype = d
        _LIB.oracle_forwardproject.argtypes = [pf, i, i, d, d, pd]
        _LIB.oracle_ellipse_sinogram.argtypes = [pd, i, i, i, pd, d, d, pd]
        _LIB.oracle_ellipse_image.argtypes = [pd, i, i, d, d, i, pd]
    return _LIB


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


# --------------------------------------------------------------------------- filter

def _mirror(f, width):
    """src/ufo-filter-task.c:162-169"""
    for k in range(width // 2 + 2, width, 2):
        f[k] = f[width - k]
        f[k + 1] = f[width - k + 1]


def _padding_value(x):
    """src/ufo-filter-task.c:242-252"""
    padding, result = 2 * x, 1
    while result < padding:
        result *= 2
    return result


def filter_coefficients(nfft, filter="ramp-fromreal", cutoff=0.5, order=4.0, tau=0.1, theta=1.0,
                        scale=1.0):
    """Interleaved float coefficients (length 2*nfft) that the ``filter`` task
    multiplies into the complex spectrum, restated from
    src/ufo-filter-task.c:162-336.  ``width`` there is the interleaved float
    width 2*nfft.  Values are computed in double and stored as float, as in the
    reference; ramp-fromreal's FFT is taken here in FP64."""
    width = 2 * nfft
    if width & (width - 1):
        raise ValueError("Invalid filter input width %u, must be a power of two" % width)
    f = np.zeros(width, dtype=np.float32)
    f[0] = f[1] = np.float32(0.5 / width)
    ftype = FILTERS.index(filter) if isinstance(filter, str) else int(filter)
    f64 = lambda v: np.float32(v)  # noqa: E731  (double -> gfloat store)
    scale = float(np.float32(scale))
    cutoff = float(np.float32(cutoff))
    order = float(np.float32(order))
    tau = float(np.float32(tau))
    theta = float(np.float32(theta))
    if ftype == 0:  # ramp :171-182
        step = 2.0 / width
        for k in range(1, width // 4 + 1):
            f[2 * k] = f64(k * step * scale)
            f[2 * k + 1] = f[2 * k]
    elif ftype == 1:  # ramp-fromreal :184-195
        f[0] = f[1] = f64(0.25 * scale)
        for k in range(1, width // 4 + 1):
            f[2 * k] = f64(-scale / (k * k * math.pi * math.pi)) if k % 2 else 0.0
            f[2 * k + 1] = f[2 * k]
    elif ftype == 2:  # butterworth :197-209
        step = 2.0 / width
        for k in range(0, width // 4 + 1):
            fr = k * step
            f[2 * k] = f64(fr / (1.0 + math.pow(fr / cutoff, 2.0 * order)) * scale)
            f[2 * k + 1] = f[2 * k]
    elif ftype == 3:  # faris-byer :254-276
        pi_squared_tau = math.pi * math.pi * tau
        sin_theta_2 = -math.sin(theta) / 2
        padding = _padding_value(width)
        f[0] = 0
        for x in range(1, width // 2 + 1):
            if x % 2 != 0:
                f[x] = f64(1 / (pi_squared_tau * x))
        for i in range(width // 2 + 1, width):
            x = width + 1 - i
            if x % 2 != 0:
                f[padding - width - i - 1] = f64(sin_theta_2 / (x * x * pi_squared_tau))
    elif ftype == 4:  # hamming :211-224
        step = 2.0 / width
        for k in range(0, width // 4 + 1):
            fr = k * step
            f[2 * k] = f64(fr * (0.54 + 0.46 * math.cos(math.pi * fr / cutoff)) * scale) if fr < cutoff else 0
            f[2 * k + 1] = f[2 * k]
    elif ftype == 5:  # bh3 :226-240
        step = 2.0 / width
        a0, a1, a2 = 0.42, 0.5, 0.08
        for k in range(1, width // 4 + 1):
            fr = k * step
            f[2 * k] = f64(fr * (a0 + a1 * math.cos(fr * math.pi) + a2 * math.cos(2.0 * fr * math.pi)) * scale)
            f[2 * k + 1] = f[2 * k]
    else:
        raise ValueError("unknown filter %r" % (filter,))
    _mirror(f, width)
    out = f.astype(np.float64)
    if ftype == 1:  # :317-334 forward FFT of the interleaved (h, h) pairs, in place
        z = np.fft.fft(out[0::2] + 1j * out[1::2])
        out = np.empty(width, dtype=np.float64)
        out[0::2] = z.real
        out[1::2] = z.imag
    return out


def fft_sizes(width, size_x=0, crop_width=0):
    """(nfft, out_width) of ``fft dimensions=1 [size-x] ! filter ! ifft [crop-width]``:
    src/ufo-fft-task.c:123-196 (auto-zeropadding is effectively FALSE) and
    src/ufo-ifft-task.c:111-177 (crop-width defaults to the full FFT width)."""
    if size_x and size_x < width:
        raise ValueError("Specified size must be greater than or equal to input size")
    nfft = size_x if size_x else width
    if crop_width and crop_width > nfft:
        raise ValueError("Cropped size must be less than or equal to input size")
    return nfft, (crop_width if crop_width else nfft)


def fft_filter_ifft(sino, size_x=0, crop_width=0, **filter_props):
    """FP64 ``fft ! filter ! ifft`` over the last axis of ``sino``."""
    sino = np.asarray(sino, dtype=np.float64)
    width = sino.shape[-1]
    nfft, out_w = fft_sizes(width, size_x, crop_width)
    coeff = filter_coefficients(nfft, **filter_props)
    X = np.fft.fft(sino, n=nfft, axis=-1)
    Y = X.real * coeff[0::2] + 1j * (X.imag * coeff[1::2])
    y = np.fft.ifft(Y, axis=-1).real
    return y[..., :out_w]


# --------------------------------------------------------------------------- backproject

def bp_luts(n_projections, angle_step=0.0, angle_offset=0.0):
    """src/ufo-backproject-task.c:174-196,245-251: FP64 sin/cos LUTs."""
    step = angle_step if angle_step > 0.0 else math.pi / n_projections
    ang = angle_offset + np.arange(n_projections, dtype=np.float64) * step
    return np.sin(ang), np.cos(ang)


def backproject(sino, num_projections=0, offset=0, axis_pos=-1.0, angle_step=-1.0, angle_offset=0.0,
                mode="texture", roi_x=0, roi_y=0, roi_width=0, roi_height=0, interp=INTERP_EXACT,
                luts_fp32=False):
    """``backproject`` of one sinogram [P, W] or a stack [Z, P, W] -> FP64 slices."""
    sino = np.ascontiguousarray(sino, dtype=np.float32)
    squeeze = sino.ndim == 2
    if squeeze:
        sino = sino[None]
    nz, P, W = sino.shape
    n_proj = num_projections if num_projections else P
    if P > n_proj:
        raise ValueError("Total number of projections (%u) must be greater than or equal to "
                         "sinogram height (%u)" % (n_proj, P))
    if offset + P > n_proj:
        raise ValueError("offset + sinogram height exceeds num-projections")
    rw = roi_width if roi_width else W
    rh = roi_height if roi_height else W
    axis = axis_pos if axis_pos > 0.0 else float(np.float32(W) / np.float32(2.0))
    s, c = bp_luts(n_proj, angle_step if angle_step > 0 else 0.0, angle_offset)
    if luts_fp32:
        s = s.astype(np.float32).astype(np.float64)
        c = c.astype(np.float32).astype(np.float64)
    if mode == "nearest":
        interp = INTERP_NEAREST
    out = np.zeros((nz, rh, rw), dtype=np.float64)
    lib().oracle_bp_parallel(_p(sino), W, P, nz, _p(s), _p(c), offset, float(np.float32(axis)),
                             roi_x, roi_y, rw, rh, interp, _p(out))
    return out[0] if squeeze else out


def stacked_backproject(sino, precision_mode="single", num_projections=0, offset=0, axis_pos=-1.0, angle_step=-1.0,
                        angle_offset=0.0, roi_x=0, roi_y=0, roi_width=0, roi_height=0):
    """``stacked-backproject`` (src/ufo-stacked-backproject-task.c:200-430,
    src/kernels/stacked-backproject.cl) of a stack [Z, P, W] -> FP64 slices.
    Orientation h = bx cos - by sin + axis (:77); "single" and "half" sample
    linearly with exact weights and zero outside ("half" after rounding the
    sinograms to FP16); "int8" quantises with the global min/max, samples the
    nearest texel floor(h) clamped to the edge, sums integers and dequantises as
    uninterleave_uint (:360-380), in FP32 like the kernels."""
    sino = np.ascontiguousarray(sino, dtype=np.float32)
    nz, P, W = sino.shape
    n_proj = num_projections if num_projections else P
    if P > n_proj or offset + P > n_proj:
        raise ValueError("sinogram height exceeds num-projections")
    rw = roi_width if roi_width else W
    rh = roi_height if roi_height else W
    axis = axis_pos if axis_pos > 0.0 else float(np.float32(W) / np.float32(2.0))
    s, c = bp_luts(n_proj, angle_step if angle_step > 0 else 0.0, angle_offset)
    if precision_mode in ("single", "half"):
        src = sino if precision_mode == "single" else sino.astype(np.float16).astype(np.float32)
        out = np.zeros((nz, rh, rw), dtype=np.float64)
        ms = np.ascontiguousarray(-s)
        lib().oracle_bp_parallel(_p(np.ascontiguousarray(src)), W, P, nz, _p(ms), _p(c), offset,
                                 float(np.float32(axis)), roi_x, roi_y, rw, rh, INTERP_EXACT, _p(out))
        return out
    if precision_mode != "int8":
        raise ValueError("precision_mode must be int8, half or single")
    f32 = np.float32
    mn, mx = f32(sino.min()), f32(sino.max())
    scale = f32(f32(255.0) / (mx - mn))
    q = np.minimum(np.trunc((sino - mn) * scale), 255).astype(np.int64)
    s32 = s[offset:offset + P].astype(np.float32).astype(np.float64)
    c32 = c[offset:offset + P].astype(np.float32).astype(np.float64)
    ax = float(np.float32(axis))
    bx = (np.arange(rw) + roi_x) - ax + 0.5
    by = (np.arange(rh) + roi_y) - ax + 0.5
    sums = np.zeros((nz, rh, rw), dtype=np.int64)
    for p in range(P):
        h = bx[None, :] * c32[p] - by[:, None] * s32[p] + ax
        i = np.clip(np.floor(h).astype(np.int64), 0, W - 1)
        sums += q[:, p, :][:, i]
    dq = f32((mx - mn) / f32(255.0))
    v = (sums.astype(np.float32) * dq + mn).astype(np.float32)
    return ((v * f32(math.pi)) / f32(P)).astype(np.float64)


def fbp(sino, axis_pos=-1.0, size_x=0, crop_width=0, filter_props=None, **bp_props):
    """FP64 ``fft ! filter ! ifft ! backproject``."""
    filtered = fft_filter_ifft(sino, size_x=size_x, crop_width=crop_width, **(filter_props or {}))
    return backproject(filtered.astype(np.float32), axis_pos=axis_pos, **bp_props)


# --------------------------------------------------------------------------- general backproject

def _almost_zero(values):
    return all(abs(v) < 1e-7 for v in values)


def gbp_flags(geom, parameter="z"):
    """Geometry-class flags, src/ufo-general-backproject-task.c:1294-1320."""
    g = {k: list(np.atleast_1d(v)) for k, v in geom.items()}
    is_axis = parameter in ("axis-angle-x", "axis-angle-y", "axis-angle-z")
    is_vol = parameter.startswith("volume-angle")
    is_det_rot = parameter.startswith("detector-angle")
    is_det_pos = parameter.startswith("detector-position")
    flags = 0
    if is_axis or not (_almost_zero(g["axis-angle-x"]) and _almost_zero(g["axis-angle-y"])):
        flags |= F_WITH_AXIS
    if is_vol or not (_almost_zero(g["volume-angle-x"]) and _almost_zero(g["volume-angle-y"])
                      and _almost_zero(g["volume-angle-z"])):
        flags |= F_WITH_VOLUME
    if not (_almost_zero(g["detector-position-x"]) and _almost_zero(g["detector-position-z"])):
        flags |= F_SHIFTED_DETECTOR
    if not (_almost_zero(g["source-position-x"]) and _almost_zero(g["source-position-z"])):
        flags |= F_SHIFTED_SOURCE
    if (not is_det_rot and not is_det_pos and _almost_zero(g["detector-angle-x"])
            and _almost_zero(g["detector-angle-y"]) and _almost_zero(g["detector-angle-z"])):
        flags |= F_PERPENDICULAR
    if all(math.isinf(v) for v in g["source-position-y"]):
        flags |= F_PARALLEL
    return flags


GBP_DEFAULTS = {
    "axis-angle-x": 0.0, "axis-angle-y": 0.0,
    "volume-angle-x": 0.0, "volume-angle-y": 0.0, "volume-angle-z": 0.0,
    "detector-angle-x": 0.0, "detector-angle-y": 0.0, "detector-angle-z": 0.0,
    "center-position-x": 0.0, "center-position-z": 0.0,
    "source-position-x": 0.0, "source-position-y": -math.inf, "source-position-z": 0.0,
    "detector-position-x": 0.0, "detector-position-y": 0.0, "detector-position-z": 0.0,
}


def gbp_geometry_table(num_projections, overall_angle=2 * math.pi, **geom):
    """[n_proj, 17] FP64 table; scalars broadcast (ufo-scarray.c:95-108); the
    tomographic angles default to i / n * overall-angle (:1435-1446)."""
    n = num_projections
    table = np.zeros((n, len(GEOM_COLS)), dtype=np.float64)
    for j, name in enumerate(GEOM_COLS):
        if name == "axis-angle-z":
            v = geom.get(name)
            if v is None or np.size(v) != n:
                v = np.arange(n, dtype=np.float64) / n * overall_angle
        else:
            v = geom.get(name, GBP_DEFAULTS[name])
            if np.size(v) not in (1, n):
                raise ValueError("%s must have 1 or num-projections values" % name)
        table[:, j] = np.broadcast_to(np.asarray(v, dtype=np.float64).reshape(-1), (n,))
    return table


def _region(reg, length):
    """compute_slice_region (:280-291): (start, step) or (-(length/2), 1)."""
    if reg is not None and reg[2]:
        return float(reg[0]), float(reg[2])
    return -float(np.float32(length) / np.float32(2)), 1.0


def _region_size(reg):
    return int(math.ceil((reg[1] - reg[0]) / reg[2]))


def general_backproject(proj, num_projections, region=(0.0, 0.0, 0.0), x_region=(0.0, 0.0, 0.0),
                        y_region=(0.0, 0.0, 0.0), z=0.0, parameter="z", overall_angle=2 * math.pi,
                        addressing_mode="clamp", interp=INTERP_EXACT, **geom):
    """FP64 ``general-backproject`` of projections [n_proj, H, W] -> volume [nz, ny, nx]."""
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    n, H, W = proj.shape
    if n != num_projections:
        raise ValueError("need num-projections projections")
    nx = W if not x_region[2] else _region_size(x_region)
    ny = W if not y_region[2] else _region_size(y_region)
    x0, dx = _region(x_region if x_region[2] else None, nx)
    y0, dy = _region(y_region if y_region[2] else None, ny)
    if abs(region[2]) < 1e-7:
        start, stop, step = 0.0, 1.0, 1.0
    else:
        start, stop, step = region
    nz = int(math.ceil((stop - start) / step))
    slice_values = start + np.arange(nz, dtype=np.float64) * step
    table = gbp_geometry_table(n, overall_angle, **geom)
    flags = gbp_flags({k: geom.get(k, GBP_DEFAULTS.get(k, 0.0)) for k in GEOM_COLS if k != "axis-angle-z"},
                      parameter)
    param_col = -1 if parameter == "z" else GEOM_COLS.index(parameter)
    norm = abs(overall_angle) / n
    addr = {"clamp": ADDR_CLAMP, "clamp_to_edge": ADDR_CLAMP_TO_EDGE, "none": ADDR_CLAMP_TO_EDGE}[addressing_mode]
    out = np.zeros((nz, ny, nx), dtype=np.float64)
    lib().oracle_gbp(_p(proj), W, H, n, _p(table), flags, param_col, _p(slice_values), float(z),
                     x0, dx, y0, dy, nx, ny, nz, norm, interp, addr, _p(out))
    return out


def _bilinear(img, u, v, addressing_mode="clamp"):
    """Linear sample of img [H, W] at unnormalised (u, v), texel centres at +1/2;
    outside the image 0 ("clamp") or the edge texel ("clamp_to_edge", "none")."""
    H, W = img.shape
    x, y = u - 0.5, v - 0.5
    i0, j0 = np.floor(x).astype(np.int64), np.floor(y).astype(np.int64)
    a, b = x - i0, y - j0

    def fetch(i, j):
        if addressing_mode == "clamp":
            ok = (i >= 0) & (i < W) & (j >= 0) & (j < H)
            return np.where(ok, img[np.clip(j, 0, H - 1), np.clip(i, 0, W - 1)], 0.0)
        return img[np.clip(j, 0, H - 1), np.clip(i, 0, W - 1)]
    return ((1 - a) * (1 - b) * fetch(i0, j0) + a * (1 - b) * fetch(i0 + 1, j0) + (1 - a) * b * fetch(i0, j0 + 1)
            + a * b * fetch(i0 + 1, j0 + 1))


def lamino_backproject(proj, num_projections, x_region, y_region, region, z=0.0, projection_offset=(0, 0),
                       center=(0.0, 0.0), overall_angle=math.pi, tomo_angle=None, lamino_angle=0.0, roll_angle=0.0,
                       parameter="z", addressing_mode="clamp"):
    """``lamino-backproject`` of projections [n, H, W] -> FP64 volume [nz, ny, nx].

    src/ufo-lamino-backproject-task.c:239-256 (sizes), :280-360 (the FP32
    scalars, formed here the same way) and the generated kernels
    (src/kernels/templates/{z,center,lamino,roll}_template.in, definitions.in:
    rotate() updates pixel.x before it enters pixel.y, as written there)."""
    f32 = np.float32
    proj = np.asarray(proj, dtype=np.float64)
    n = num_projections
    if proj.shape[0] != n:
        raise ValueError("need num-projections projections")
    size = lambda r: 0 if r[2] == 0 else max(0, int((r[1] - r[0] - 1) / r[2]) + 1)  # C integer division
    nx, ny = size([int(t) for t in x_region]), size([int(t) for t in y_region])
    reg = [f32(t) for t in region]
    nz = int(math.ceil(f32((reg[1] - reg[0]) / reg[2])))
    norm = float(f32(abs(float(f32(overall_angle))) / n))
    xs, x0 = float(int(x_region[2])), float(int(x_region[0]))
    ys, y0 = float(int(y_region[2])), float(int(y_region[0]))
    px_off, py_off = int(projection_offset[0]), int(projection_offset[1])
    if parameter == "x-center":
        xc0, xcs = float(f32(reg[0] - f32(px_off))), float(reg[2])
    else:
        xc0 = float(f32(f32(center[0]) - f32(px_off)))
        xcs = xc0
    yc = float(f32(f32(center[1]) - f32(py_off)))
    ix, iy = np.meshgrid(np.arange(nx, dtype=np.float64), np.arange(ny, dtype=np.float64))
    vx, vy = ix * xs + x0, iy * ys + y0
    out = np.zeros((nz, ny, nx))
    ov = f32(overall_angle)
    for k in range(nz):
        vz = float(f32(f32(k) * reg[2] + reg[0])) if parameter == "z" else float(f32(z))
        la = f32(lamino_angle)
        sL, cL = float(f32(math.sin(la))), float(f32(math.cos(la)))
        ra = f32(-f32(roll_angle))
        sR, cR = float(f32(math.sin(ra))), float(f32(math.cos(ra)))
        xcc = xc0
        if parameter == "x-center":
            xcc = float(f32(f32(k) * f32(xcs) + f32(xc0)))
        elif parameter == "lamino-angle":
            a = f32(f32(k) * reg[2] + reg[0])
            sL, cL = float(f32(math.sin(a))), float(f32(math.cos(a)))
        elif parameter == "roll-angle":
            a = f32(f32(k) * -reg[2] - reg[0])
            sR, cR = float(f32(math.sin(a))), float(f32(math.cos(a)))
        acc = np.zeros((ny, nx))
        for p in range(n):
            t = f32(tomo_angle) if tomo_angle is not None else f32(f32(ov * f32(p)) / f32(n))
            sn, cs = float(f32(math.sin(t))), float(f32(math.cos(t)))
            px = vx * cs + vy * sn + xcc
            py = (vx * cL) * sn + (-vy * cL) * cs + (vz * sL + yc)
            a1, b1 = px - xc0, py - yc
            a2 = a1 * cR + b1 * sR
            b2 = -a2 * sR + b1 * cR
            acc += _bilinear(proj[p], a2 + xc0, b2 + yc, addressing_mode)
        out[k] = acc * norm
    return out


def _to_half(x):
    return np.asarray(x, dtype=np.float64).astype(np.float16).astype(np.float64)


def general_backproject_store(proj, num_projections, store_type="float", gray_map_min=0.0, gray_map_max=0.0,
                              burst=8, **kw):
    """``general-backproject`` with the reference's store-type accumulation: the
    generated kernel adds norm * (sum over one burst of projections) into the
    volume in the store type once per burst (general_bp_body.in,
    make_type_conversion :705-719): integer types clamp the gray-mapped value,
    truncate and wrap; half rounds to half at every addition."""
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    n = num_projections
    overall = kw.get("overall_angle", 2 * math.pi)
    norm = abs(overall) / n
    geom = dict(kw)
    tomo = geom.pop("axis-angle-z", None)
    if tomo is None or np.size(tomo) != n:
        tomo = np.arange(n, dtype=np.float64) / n * overall
    arrays = {k: v for k, v in geom.items() if k in GEOM_COLS and np.size(v) == n and n > 1}
    acc = None
    maxv = {"uchar": 255.0, "ushort": 65535.0, "uint": 4294967295.0}.get(store_type)
    mod = {"uchar": 256, "ushort": 65536, "uint": 2 ** 32}.get(store_type)
    for b0 in range(0, n, burst):
        b1 = min(n, b0 + burst)
        sub = dict(geom)
        for k, v in arrays.items():
            sub[k] = np.asarray(v)[b0:b1]
        sub["axis-angle-z"] = np.asarray(tomo)[b0:b1]
        sub["overall_angle"] = overall
        part = general_backproject(proj[b0:b1], b1 - b0, **sub) / (abs(overall) / (b1 - b0))  # burst sum
        contrib = norm * part
        if acc is None:
            acc = np.zeros_like(contrib)
        if store_type == "float":
            acc = (acc.astype(np.float32) + contrib.astype(np.float32)).astype(np.float64)
        elif store_type == "double":
            acc = acc + contrib
        elif store_type == "half":
            acc = _to_half(_to_half(acc) + _to_half(contrib))
        else:
            gs = maxv / (gray_map_max - gray_map_min)
            gv = np.clip(gs * (contrib - gray_map_min), 0.0, maxv)
            acc = np.mod(acc + np.trunc(gv), mod)
    return acc


def forwardproject(slice_img, n_angles, axis_pos, angle_step):
    img = np.ascontiguousarray(slice_img, dtype=np.float32)
    W = img.shape[-1]
    out = np.zeros((n_angles, W), dtype=np.float64)
    lib().oracle_forwardproject(_p(img), W, n_angles, float(axis_pos), float(angle_step), _p(out))
    return out


# --------------------------------------------------------------------------- preprocessing

def flat_field_correct(data, dark, flat, absorption_correct=False, fix_nan_and_inf=False, sinogram_input=False,
                       dark_scale=1.0, flat_scale=1.0):
    """src/kernels/ffc.cl:31-47 in FP32, one rounding per operation: dark/flat
    [H, W] broadcast over frames [..., H, W] (one row [W] with sinogram-input,
    where the kernel indexes them by the column alone, :33)."""
    f32 = np.float32
    d = np.asarray(data, dtype=f32)
    dark, flat = np.asarray(dark, dtype=f32), np.asarray(flat, dtype=f32)
    if sinogram_input:
        dark, flat = dark.reshape(-1), flat.reshape(-1)
    cd = dark * f32(dark_scale)
    cf = flat * f32(flat_scale)
    with np.errstate(all="ignore"):
        if absorption_correct:
            r = np.log((cf - cd) / (d - cd))
        else:
            r = (d - cd) / (cf - cd)
    r = r.astype(f32)
    if fix_nan_and_inf:  # :42-44
        r = np.where(np.isfinite(r), r, f32(0.0))
    return r


def transpose_projections(proj):
    """Projections [N, H, W] -> sinograms [H, N, W] (row y of projection p is row
    p of sinogram y, src/ufo-transpose-projections-task.c:76-97)."""
    return np.ascontiguousarray(np.transpose(np.asarray(proj, dtype=np.float32), (1, 0, 2)))


def _scarray_value(values, index):
    """ufo_scarray_get_double (src/common/ufo-scarray.c:118-127): one value
    broadcasts, else the value at `index` (which must exist)."""
    v = np.atleast_1d(np.asarray(values, dtype=np.float64))
    if v.size == 1:
        return float(v[0])
    if index >= v.size:
        raise IndexError("scalar array has %d values, index %d" % (v.size, index))
    return float(v[index])


def cone_weight_params(index, center_position_x, center_position_z, source_distance, detector_distance,
                       axis_angle_x=0.0):
    """FP32 kernel arguments of projection `index`
    (src/ufo-cone-beam-projection-weight-task.c:128-139): center, source
    distance, overall distance, magnification reciprocal, cos of the axis angle."""
    f32 = np.float32
    cs = f32(math.cos(_scarray_value(axis_angle_x, index)))
    cx = f32(_scarray_value(center_position_x, index))
    cz = f32(_scarray_value(center_position_z, index))
    sd = f32(_scarray_value(source_distance, index))
    dd = f32(_scarray_value(detector_distance, index))
    od = f32(sd + dd)
    mr = f32(sd / od)
    if cs > f32(0.9999999):
        od = sd
    return cx, cz, sd, od, mr, cs


def cone_beam_weight(proj, first=0, **props):
    """src/kernels/conebeam.cl:20-36 for projections [n, H, W] (indices first ..
    first+n-1) in FP32; props are the task's array properties."""
    f32 = np.float32
    p3 = np.asarray(proj, dtype=f32)
    squeeze = p3.ndim == 2
    if squeeze:
        p3 = p3[None]
    n, H, W = p3.shape
    out = np.empty_like(p3)
    kw = {k.replace("-", "_"): v for k, v in props.items()}
    idx = np.arange(W, dtype=f32)
    idy = np.arange(H, dtype=f32)[:, None]
    for i in range(n):
        cx, cz, sd, od, mr, cs = cone_weight_params(first + i, **kw)
        x = ((idx - cx) + f32(0.5)) * mr
        y = ((idy - cz) + f32(0.5)) * mr
        den = np.sqrt((od * od + x * x) + y * y)
        out[i] = ((p3[i] * sd) * cs) / den
    return out[0] if squeeze else out


# --------------------------------------------------------------------------- phantoms

def random_ellipses(seed, n=10, semi=(0.05, 0.4), density=(-0.5, 1.0)):
    """Rows (cx, cy, a, b, phi, rho): centres uniform in the unit disc, semi-axes
    uniform in ``semi``, angles uniform in [0, pi), densities uniform in ``density``."""
    rng = np.random.default_rng(seed)
    r = np.sqrt(rng.uniform(0, 1, n))
    t = rng.uniform(0, 2 * math.pi, n)
    ell = np.stack([r * np.cos(t), r * np.sin(t), rng.uniform(*semi, n), rng.uniform(*semi, n),
                    rng.uniform(0, math.pi, n), rng.uniform(*density, n)], axis=1)
    return np.ascontiguousarray(ell, dtype=np.float64)


def random_ellipsoids(seed, n=50, semi=(0.05, 0.4), density=(-0.5, 1.0)):
    """Rows (cx, cy, cz, a, b, c, phi, rho): centres uniform in the unit ball,
    semi-axes uniform in ``semi``, rotation about z uniform in [0, pi),
    densities uniform in ``density``."""
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    v *= rng.uniform(0, 1, (n, 1)) ** (1.0 / 3.0)
    ell = np.concatenate([v, rng.uniform(*semi, (n, 3)), rng.uniform(0, math.pi, (n, 1)),
                          rng.uniform(*density, (n, 1))], axis=1)
    return np.ascontiguousarray(ell, dtype=np.float64)


def ellipsoid_slice_ellipses(ell3, z, nz, scale):
    """Ellipses (cx, cy, a, b, phi, rho) that slice z of an nz-slice stack cuts
    from the ellipsoids (slice centre height (z + 0.5 - nz/2) / scale)."""
    zu = (z + 0.5 - 0.5 * nz) / scale
    rows = []
    for q in ell3:
        dz = (zu - q[2]) / q[5]
        if dz * dz < 1.0:
            f = math.sqrt(1.0 - dz * dz)
            rows.append([q[0], q[1], q[3] * f, q[4] * f, q[6], q[7]])
    return np.ascontiguousarray(np.array(rows, dtype=np.float64).reshape(-1, 6))


def ellipse_sinogram(ell, width, angles, axis=None, scale=None):
    """Analytic parallel-beam sinogram [P, width] in pixel-length units."""
    axis = width / 2.0 if axis is None else axis
    scale = width / 2.0 if scale is None else scale
    angles = np.ascontiguousarray(angles, dtype=np.float64)
    out = np.zeros((len(angles), width), dtype=np.float64)
    lib().oracle_ellipse_sinogram(_p(ell), len(ell), width, len(angles), _p(angles), float(axis), float(scale),
                                  _p(out))
    return out


def ellipse_image(ell, n, axis=None, scale=None, ss=4):
    axis = n / 2.0 if axis is None else axis
    scale = n / 2.0 if scale is None else scale
    out = np.zeros((n, n), dtype=np.float64)
    lib().oracle_ellipse_image(_p(ell), len(ell), n, float(axis), float(scale), ss, _p(out))
    return out


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


# --------------------------------------------------------------------------- CNN (sparse-view correction)

def conv3x3_nhwc(x, w, bias=None, relu=False):
    """FP64 3x3 convolution, zero padding: x [N,H,W,Cin], w [Cout,9,Cin] with tap
    t = 3*(dy+1) + (dx+1) -> [N,H,W,Cout]."""
    x = np.asarray(x, dtype=np.float64)
    w = np.asarray(w, dtype=np.float64)
    N, H, W, C = x.shape
    xp = np.zeros((N, H + 2, W + 2, C))
    xp[:, 1:-1, 1:-1] = x
    out = np.zeros((N, H, W, w.shape[0]))
    for t in range(9):
        dy, dx = t // 3 - 1, t % 3 - 1
        out += np.einsum("nhwc,oc->nhwo", xp[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W], w[:, t])
    if bias is not None:
        out += np.asarray(bias, dtype=np.float64)
    if relu:
        out = np.maximum(out, 0.0)
    return out


def conv3x3_wgrad_nhwc(x, dz):
    """dW[co][t][ci] = sum_p dz[p][co] * x[p + off(t)][ci] (FP64)."""
    x = np.asarray(x, dtype=np.float64)
    dz = np.asarray(dz, dtype=np.float64)
    N, H, W, C = x.shape
    xp = np.zeros((N, H + 2, W + 2, C))
    xp[:, 1:-1, 1:-1] = x
    dw = np.zeros((dz.shape[-1], 9, C))
    for t in range(9):
        dy, dx = t // 3 - 1, t % 3 - 1
        dw[:, t] = np.einsum("nhwo,nhwc->oc", dz, xp[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W])
    return dw


def conv3x3_dgrad_weights(w):
    """Weights of the data-gradient convolution: [Cin][9][Cout], taps flipped."""
    w = np.asarray(w)
    return np.ascontiguousarray(w[:, ::-1, :].transpose(2, 1, 0))


def bf16_round(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


# Layer table of the sparse-view correction network: (Cin, Cout, relu) for
# enc1..enc4, dec3, dec2, dec1, out.  Must match cnn_net.cu.
CNN_LAYERS = [(16, 32, 1), (32, 64, 1), (64, 128, 1), (128, 256, 1),
              (256, 128, 1), (128, 64, 1), (64, 32, 1), (32, 16, 0)]


def cnn_num_params():
    return sum(co * 9 * ci + co for ci, co, _ in CNN_LAYERS)


def cnn_unpack(params):
    """Flat FP32 parameter vector -> [(w [Cout,9,Cin], b [Cout])]."""
    out, off = [], 0
    for ci, co, _ in CNN_LAYERS:
        n = co * 9 * ci
        w = np.asarray(params[off:off + n], dtype=np.float64).reshape(co, 9, ci)
        off += n
        b = np.asarray(params[off:off + co], dtype=np.float64)
        off += co
        out.append((w, b))
    return out


def cnn_pack(layers):
    return np.concatenate([np.concatenate([w.ravel(), b.ravel()]) for w, b in layers])


CNN_S = 4  # space-to-depth factor of the network input/output


def _unshuffle(img):
    """[B, 4H, 4W] -> [B, H, W, 16], channel 4*dy + dx."""
    B, H4, W4 = img.shape
    x = np.zeros((B, H4 // CNN_S, W4 // CNN_S, CNN_S * CNN_S))
    for dy in range(CNN_S):
        for dx in range(CNN_S):
            x[..., CNN_S * dy + dx] = img[:, dy::CNN_S, dx::CNN_S]
    return x


def _shuffle(o):
    """[B, H, W, 16] -> [B, 4H, 4W]."""
    B, H, W, _ = o.shape
    img = np.zeros((B, CNN_S * H, CNN_S * W))
    for dy in range(CNN_S):
        for dx in range(CNN_S):
            img[:, dy::CNN_S, dx::CNN_S] = o[..., CNN_S * dy + dx]
    return img


def _pool(x):
    return 0.25 * (x[:, 0::2, 0::2] + x[:, 0::2, 1::2] + x[:, 1::2, 0::2] + x[:, 1::2, 1::2])


def _pool_grad(d):
    return 0.25 * np.repeat(np.repeat(d, 2, axis=1), 2, axis=2)


def _up(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def _up_grad(d):
    return d[:, 0::2, 0::2] + d[:, 0::2, 1::2] + d[:, 1::2, 0::2] + d[:, 1::2, 1::2]


def cnn_forward(params, fbp, scale=1.0, bf16=False, keep=False):
    """Forward pass of the correction network (restated from cnn_net.cu's
    layer list): returns fbp + scale * shuffle(o[..., :4]).  With ``bf16`` the
    weights and every stored activation are rounded to BF16 where the CUDA
    engine stores BF16 (accumulation stays exact)."""
    r = bf16_round if bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    fbp = np.asarray(fbp, dtype=np.float64)
    L = [(r(w), b) for w, b in cnn_unpack(params)]
    a = {}
    a["x0"] = r(_unshuffle(np.asarray(fbp, dtype=np.float32) * np.float32(1.0 / scale)))
    a["e1"] = r(conv3x3_nhwc(a["x0"], *L[0], relu=True))
    a["p1"] = r(_pool(a["e1"]))
    a["e2"] = r(conv3x3_nhwc(a["p1"], *L[1], relu=True))
    a["p2"] = r(_pool(a["e2"]))
    a["e3"] = r(conv3x3_nhwc(a["p2"], *L[2], relu=True))
    a["p3"] = r(_pool(a["e3"]))
    a["e4"] = r(conv3x3_nhwc(a["p3"], *L[3], relu=True))
    a["d3"] = r(conv3x3_nhwc(a["e4"], *L[4], relu=True))
    a["u3"] = r(_up(a["d3"]) + a["e3"])
    a["d2"] = r(conv3x3_nhwc(a["u3"], *L[5], relu=True))
    a["u2"] = r(_up(a["d2"]) + a["e2"])
    a["d1"] = r(conv3x3_nhwc(a["u2"], *L[6], relu=True))
    a["u1"] = r(_up(a["d1"]) + a["e1"])
    a["o"] = conv3x3_nhwc(a["u1"], *L[7])
    pred = fbp + scale * _shuffle(a["o"])
    return (pred, a, L) if keep else pred


def cnn_loss_and_grads(params, fbp, target, scale=1.0, bf16=False):
    """MSE loss and its gradient with respect to the flat parameter vector
    (FP64 backward of ``cnn_forward``; with ``bf16`` the per-layer output
    gradients are rounded to BF16 where the CUDA engine rounds them)."""
    r = bf16_round if bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    pred, a, L = cnn_forward(params, fbp, scale, bf16, keep=True)
    target = np.asarray(target, dtype=np.float64)
    n = pred.size
    diff = pred - target
    loss = float(np.mean(diff * diff))
    dpred = 2.0 * diff / n
    grads = [None] * 8

    def layer(i, x, y, dy, want_dx=True):
        dz = r(dy * (y > 0)) if CNN_LAYERS[i][2] else r(dy)
        grads[i] = (conv3x3_wgrad_nhwc(x, dz), dz.sum(axis=(0, 1, 2)))
        if want_dx:
            return conv3x3_nhwc(dz, conv3x3_dgrad_weights(L[i][0]))
        return None

    dzo = r(_unshuffle(scale * dpred))
    grads[7] = (conv3x3_wgrad_nhwc(a["u1"], dzo), dzo.sum(axis=(0, 1, 2)))
    du1 = conv3x3_nhwc(dzo, conv3x3_dgrad_weights(L[7][0]))
    g_e1 = du1.copy()
    du2 = layer(6, a["u2"], a["d1"], _up_grad(du1))
    g_e2 = du2.copy()
    du3 = layer(5, a["u3"], a["d2"], _up_grad(du2))
    g_e3 = du3.copy()
    de4 = layer(4, a["e4"], a["d3"], _up_grad(du3))
    dp3 = layer(3, a["p3"], a["e4"], de4)
    g_e3 = g_e3 + _pool_grad(dp3)
    dp2 = layer(2, a["p2"], a["e3"], g_e3)
    g_e2 = g_e2 + _pool_grad(dp2)
    dp1 = layer(1, a["p1"], a["e2"], g_e2)
    g_e1 = g_e1 + _pool_grad(dp1)
    layer(0, a["x0"], a["e1"], g_e1, want_dx=False)
    return loss, cnn_pack(grads)


def cnn_init(seed):
    """He-initialised parameters (the engine initialises its own; this is for
    CPU-side checks)."""
    rng = np.random.default_rng(seed)
    layers = []
    for i, (ci, co, _) in enumerate(CNN_LAYERS):
        w = rng.normal(0.0, math.sqrt(2.0 / (9.0 * ci)), size=(co, 9, ci))
        b = rng.normal(0.0, 0.05, size=co)
        layers.append((w, b))
    return cnn_pack(layers).astype(np.float32)
