"""Python binding of the B200 FBP engine (ctypes over ``include/ufob.h``).

The task classes mirror the ufo-filters tasks they replace: they are created by
name (``get_task("filter")``, like ``Ufo.PluginManager().get_task``), take the
reference's properties through ``task.props.<name>`` (dashes become
underscores, as in PyGObject) and run on device tensors.  Device memory is held
in torch CUDA tensors; every computation happens in the engine's own CUDA
kernels inside ``libufob.so``.  There is no CPU path: if the library or a
usable sm_100 GPU is missing, the calls raise.
"""
from __future__ import annotations

import ctypes
import math
import os

__all__ = ["lib", "UfobError", "get_task", "FilterTask", "BackprojectTask", "FBP", "GeneralBackprojectTask",
           "Batch", "FlatFieldCorrectTask", "ConeBeamProjectionWeightTask", "TransposeProjectionsTask", "StackedBackprojectTask",
           "LaminoBackprojectTask", "F32", "F16", "BF16", "F64", "U8", "U16", "U32", "ROWS", "PAIRS", "QUADS"]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libufob.so")

OK, ERR_INVALID, ERR_SETUP, ERR_REQUISITION, ERR_CUDA, ERR_NOMEM, ERR_TIMEOUT, ERR_UNSUPPORTED = range(8)
F32, F16, BF16, F64, U8, U16, U32 = range(7)
ROWS, PAIRS, QUADS = 0, 1, 2
FILTERS = ["ramp", "ramp-fromreal", "butterworth", "faris-byer", "hamming", "bh3"]
DTYPES = {"f32": F32, "float": F32, "f16": F16, "half": F16, "bf16": BF16, "f64": F64, "double": F64,
          "u8": U8, "uchar": U8, "u16": U16, "ushort": U16, "u32": U32, "uint": U32}

_lib = None


class UfobError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s (status %d)" % (message, status))
        self.status = status


class FilterProps(ctypes.Structure):
    _fields_ = [("filter", ctypes.c_int), ("cutoff", ctypes.c_float), ("order", ctypes.c_float),
                ("tau", ctypes.c_float), ("theta", ctypes.c_float), ("scale", ctypes.c_float),
                ("size_x", ctypes.c_uint32), ("crop_width", ctypes.c_uint32)]


class BPProps(ctypes.Structure):
    _fields_ = [("num_projections", ctypes.c_uint32), ("offset", ctypes.c_uint32), ("axis_pos", ctypes.c_double),
                ("angle_step", ctypes.c_double), ("angle_offset", ctypes.c_double), ("mode", ctypes.c_int),
                ("roi_x", ctypes.c_uint32), ("roi_y", ctypes.c_uint32), ("roi_width", ctypes.c_uint32),
                ("roi_height", ctypes.c_uint32), ("compensated", ctypes.c_int), ("tile", ctypes.c_int),
                ("half_sums", ctypes.c_int), ("angle_groups", ctypes.c_int)]


class Job(ctypes.Structure):
    _fields_ = [("d_sino", ctypes.c_void_p), ("d_out", ctypes.c_void_p), ("width", ctypes.c_uint32),
                ("height", ctypes.c_uint32), ("axis_pos", ctypes.c_double), ("angle_step", ctypes.c_double),
                ("angle_offset", ctypes.c_double)]


class FFCProps(ctypes.Structure):
    _fields_ = [("fix_nan_and_inf", ctypes.c_int), ("absorption_correct", ctypes.c_int),
                ("sinogram_input", ctypes.c_int), ("dark_scale", ctypes.c_float), ("flat_scale", ctypes.c_float)]


class Preprocess(ctypes.Structure):
    _fields_ = [("ffc", ctypes.POINTER(FFCProps)), ("d_dark", ctypes.c_void_p), ("d_flat", ctypes.c_void_p),
                ("cone", ctypes.c_void_p)]


def lib():
    """Load libufob.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libufob.so not found at %s: build it with `python ufo-filters_b200/build.py`" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        vp, u32, u64, d, i, cs = (ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_double, ctypes.c_int,
                                  ctypes.c_char_p)
        pu32 = ctypes.POINTER(ctypes.c_uint32)
        sig = {
            "ufob_last_error": ([], cs),
            "ufob_status_string": ([i], cs),
            "ufob_device_check": ([ctypes.POINTER(i), ctypes.POINTER(i), ctypes.POINTER(i)], i),
            "ufob_device_status": ([], i),
            "ufob_filter_props_init": ([ctypes.POINTER(FilterProps)], None),
            "ufob_filter_create": ([ctypes.POINTER(FilterProps), ctypes.POINTER(vp)], i),
            "ufob_filter_set_property": ([vp, cs, d], i),
            "ufob_filter_set_property_string": ([vp, cs, cs], i),
            "ufob_filter_get_requisition": ([vp, u32, u32, pu32, pu32], i),
            "ufob_filter_run": ([vp, vp, u32, u32, u32, vp, i, i, u32, vp], i),
            "ufob_filter_run_quads": ([vp, vp, u32, u32, u32, u32, vp, u32, vp], i),
            "ufob_filter_coefficients": ([vp, u32, vp, u32], i),
            "ufob_filter_apply_spectrum": ([vp, vp, vp, u32, u32, vp], i),
            "ufob_filter_destroy": ([vp], None),
            "ufob_bp_props_init": ([ctypes.POINTER(BPProps)], None),
            "ufob_backproject_create": ([ctypes.POINTER(BPProps), ctypes.POINTER(vp)], i),
            "ufob_backproject_set_property": ([vp, cs, d], i),
            "ufob_backproject_set_property_string": ([vp, cs, cs], i),
            "ufob_backproject_get_requisition": ([vp, u32, u32, pu32, pu32], i),
            "ufob_backproject_run": ([vp, vp, i, i, u32, u32, u32, u32, u64, vp, vp], i),
            "ufob_backproject_destroy": ([vp], None),
            "ufob_backproject_run_static": ([ctypes.POINTER(BPProps), vp, i, i, u32, u32, u32, u32, u64, vp, vp], i),
            "ufob_fbp_create": ([ctypes.POINTER(FilterProps), ctypes.POINTER(BPProps), i, ctypes.POINTER(vp)], i),
            "ufob_fbp_run": ([vp, vp, u32, u32, u32, vp, vp], i),
            "ufob_fbp_run_host": ([vp, vp, u32, u32, u32, vp, u32], i),
            "ufob_fbp_get_requisition": ([vp, u32, u32, pu32, pu32], i),
            "ufob_fbp_destroy": ([vp], None),
            "ufob_fbp_set_timing": ([vp, i], i),
            "ufob_fbp_kernel_times": ([vp, ctypes.POINTER(d), pu32, ctypes.POINTER(d), pu32], i),
            "ufob_gbp_create": ([ctypes.POINTER(vp)], i),
            "ufob_gbp_set_property": ([vp, cs, d], i),
            "ufob_gbp_set_property_string": ([vp, cs, cs], i),
            "ufob_gbp_set_array": ([vp, cs, vp, u32], i),
            "ufob_gbp_setup": ([vp], i),
            "ufob_gbp_get_requisition": ([vp, u32, u32, pu32, pu32, pu32], i),
            "ufob_gbp_run": ([vp, vp, u32, u32, vp, vp], i),
            "ufob_gbp_process": ([vp, vp, u32, u32, vp], i),
            "ufob_gbp_generate": ([vp, vp, u32, vp], i),
            "ufob_gbp_destroy": ([vp], None),
            "ufob_batch_create": ([ctypes.POINTER(FilterProps), i, ctypes.POINTER(vp)], i),
            "ufob_batch_run": ([vp, ctypes.POINTER(Job), u32, vp], i),
            "ufob_batch_destroy": ([vp], None),
            "ufob_batch_variant": ([vp], i),
            "ufob_batch_variants": ([], i),
            "ufob_batch_set_variant": ([vp, i], i),
            "ufob_phantom_sinogram": ([vp, u32, u32, u32, d, d, d, vp, vp], i),
            "ufob_phantom_stack": ([vp, u32, u32, u32, u32, d, d, d, vp, vp], i),
            "ufob_launch_count": ([], ctypes.c_uint64),
            "ufob_device_alloc_count": ([], ctypes.c_uint64),
            "ufob_forwardproject": ([vp, u32, u32, d, d, vp, vp], i),
            "ufob_phantom_images": ([vp, vp, u32, u32, d, d, i, vp, vp], i),
            "ufob_measure_peaks": ([ctypes.POINTER(d), ctypes.POINTER(d)], i),
            "ufob_cnn_create": ([u64, ctypes.c_float, ctypes.POINTER(vp)], i),
            "ufob_cnn_destroy": ([vp], None),
            "ufob_cnn_forward": ([vp, vp, vp, i, i, i, vp], i),
            "ufob_cnn_forward_nhwc": ([vp, vp, vp, i, i, i, vp], i),
            "ufob_cnn_train_step": ([vp, vp, vp, i, i, i, ctypes.c_float, ctypes.POINTER(d), vp], i),
            "ufob_cnn_num_params": ([], u64),
            "ufob_cnn_get_state": ([vp, i, vp, u64], i),
            "ufob_cnn_set_state": ([vp, i, vp, u64], i),
            "ufob_cnn_get_step": ([vp], ctypes.c_int64),
            "ufob_cnn_set_step": ([vp, ctypes.c_int64], i),
            "ufob_conv3x3_forward": ([vp, vp, vp, vp, vp, vp, i, i, i, i, i, i, vp], i),
            "ufob_conv3x3_wgrad": ([vp, vp, vp, i, i, i, i, i, vp], i),
            "ufob_stacked_bp_create": ([ctypes.POINTER(vp)], i),
            "ufob_stacked_bp_set_property": ([vp, cs, d], i),
            "ufob_stacked_bp_set_property_string": ([vp, cs, cs], i),
            "ufob_stacked_bp_get_requisition": ([vp, u32, u32, pu32, pu32], i),
            "ufob_stacked_bp_run": ([vp, vp, u32, u32, u32, vp, vp], i),
            "ufob_stacked_bp_destroy": ([vp], None),
            "ufob_lamino_create": ([ctypes.POINTER(vp)], i),
            "ufob_lamino_set_property": ([vp, cs, d], i),
            "ufob_lamino_set_property_string": ([vp, cs, cs], i),
            "ufob_lamino_set_array": ([vp, cs, vp, u32], i),
            "ufob_lamino_setup": ([vp], i),
            "ufob_lamino_get_requisition": ([vp, pu32, pu32, pu32], i),
            "ufob_lamino_run": ([vp, vp, u32, u32, vp, vp], i),
            "ufob_lamino_process": ([vp, vp, u32, u32, vp], i),
            "ufob_lamino_generate": ([vp, vp, vp], i),
            "ufob_lamino_destroy": ([vp], None),
            "ufob_ffc_props_init": ([ctypes.POINTER(FFCProps)], None),
            "ufob_ffc_set_property": ([ctypes.POINTER(FFCProps), cs, d], i),
            "ufob_flat_field_correct": ([ctypes.POINTER(FFCProps), vp, vp, vp, u32, u32, u32, vp, vp], i),
            "ufob_cone_weight_create": ([ctypes.POINTER(vp)], i),
            "ufob_cone_weight_set_array": ([vp, cs, vp, u32], i),
            "ufob_cone_weight_set_property": ([vp, cs, d], i),
            "ufob_cone_weight_run": ([vp, vp, u32, u32, u32, vp, vp], i),
            "ufob_cone_weight_set_count": ([vp, u32], i),
            "ufob_cone_weight_get_count": ([vp], u32),
            "ufob_cone_weight_destroy": ([vp], None),
            "ufob_transpose_projections": ([vp, u32, u32, u32, vp, u32, u32, vp], i),
            "ufob_filter_run_projections": ([vp, ctypes.POINTER(Preprocess), vp, u32, u32, u32, u32, i, u32, u32, vp, i,
                                             i, u32, vp], i),
            "ufob_fbp_run_projections": ([vp, ctypes.POINTER(Preprocess), vp, u32, u32, u32, u32, u32, vp, vp], i),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def check(status):
    if status != OK:
        raise UfobError(status, lib().ufob_last_error().decode())
    return status


def _ptr(t):
    """Device pointer of a CUDA tensor (or an int address)."""
    if t is None:
        return None
    if isinstance(t, int):
        return t
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    return t.data_ptr()


def _stream(stream):
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return stream if isinstance(stream, int) else stream.cuda_stream


class _Props:
    """Attribute-style property access: props.axis_pos = 255.5 -> set_property('axis-pos', 255.5)."""

    def __init__(self, task):
        object.__setattr__(self, "_task", task)

    def __setattr__(self, name, value):
        self._task.set_property(name.replace("_", "-"), value)

    def __getattr__(self, name):
        return self._task.get_property(name.replace("_", "-"))


class _Task:
    _set_num = None
    _set_str = None

    def __init__(self):
        self.props = _Props(self)
        self._values = {}

    def set_property(self, name, value):
        if isinstance(value, str):
            check(self._set_str(self._h, name.encode(), value.encode()))
        else:
            check(self._set_num(self._h, name.encode(), float(value)))
        self._values[name] = value

    def get_property(self, name):
        if name in self._values:
            return self._values[name]
        raise AttributeError(name)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._destroy(h)
            self._h = None


class FilterTask(_Task):
    """Fused ``fft ! filter ! ifft`` (ramp filter along detector rows).

    Properties: filter, cutoff, order, tau, theta, scale (filter task),
    size-x (fft task), crop-width (ifft task)."""

    def __init__(self, **props):
        super().__init__()
        L = lib()
        h = ctypes.c_void_p()
        check(L.ufob_filter_create(None, ctypes.byref(h)))
        self._h = h
        self._set_num, self._set_str, self._destroy = (L.ufob_filter_set_property, L.ufob_filter_set_property_string,
                                                       L.ufob_filter_destroy)
        for k, v in props.items():
            self.set_property(k.replace("_", "-"), v)

    def get_requisition(self, width, height):
        w, h = ctypes.c_uint32(), ctypes.c_uint32()
        check(lib().ufob_filter_get_requisition(self._h, width, height, ctypes.byref(w), ctypes.byref(h)))
        return w.value, h.value

    def coefficients(self, width):
        import numpy as np
        w, _ = self.get_requisition(width, 1)
        n = 2 * (self.get_property("size-x") if self._values.get("size-x") else width)
        out = np.zeros(n, dtype=np.float32)
        check(lib().ufob_filter_coefficients(self._h, width, out.ctypes.data, n))
        return out

    def process(self, sino, dtype=F32, layout=ROWS, out=None, stream=None):
        """Filter the rows of a float32 CUDA tensor [..., H, W]; returns [..., H, crop]
        (or [..., H, pair_pitch] int32 pairs for layout=PAIRS, or for a stack
        [Z, H, W] with layout=QUADS the [ceil(Z/4), H, crop+1, 4] int32 slice-quad cells)."""
        import torch
        if sino.dtype != torch.float32 or not sino.is_cuda:
            raise ValueError("sinogram must be a float32 CUDA tensor")
        sino = sino.contiguous()
        W = sino.shape[-1]
        rows = sino.numel() // W
        cw, _ = self.get_requisition(W, 1)
        dt = DTYPES.get(dtype, dtype) if isinstance(dtype, str) else dtype
        if layout == QUADS:
            if dt != F16:
                raise ValueError("the QUADS layout is F16 only")
            s3 = sino if sino.dim() == 3 else sino.reshape(-1, *sino.shape[-2:])
            Z, H = s3.shape[0], s3.shape[1]
            shape = ((Z + 3) // 4, H, cw + 1, 4)
            out = torch.empty(shape, dtype=torch.int32, device=sino.device) if out is None else out
            check(lib().ufob_filter_run_quads(self._h, _ptr(s3), W, H, Z, W, _ptr(out), cw + 1, _stream(stream)))
            return out
        if layout == PAIRS:
            pitch = (cw + 1 + 3) // 4 * 4
            shape = tuple(sino.shape[:-1]) + (pitch,)
            out = torch.empty(shape, dtype=torch.int32, device=sino.device) if out is None else out
        else:
            pitch = cw
            tdt = {F32: torch.float32, F16: torch.float16, BF16: torch.bfloat16}[dt]
            shape = tuple(sino.shape[:-1]) + (cw,)
            out = torch.empty(shape, dtype=tdt, device=sino.device) if out is None else out
        check(lib().ufob_filter_run(self._h, _ptr(sino), W, rows, W, _ptr(out), dt, layout, pitch, _stream(stream)))
        return out

    def process_projections(self, proj, ffc=None, dark=None, flat=None, cone=None, sinograms=True, first_row=0,
                            n_rows=0, dtype=F32, layout=ROWS, out=None, stream=None):
        """Filter projections [N, H, W] (float32 CUDA) after flat-field correction
        (`ffc` a FlatFieldCorrectTask with its dark/flat frames) and/or the cone-beam
        weight (`cone` a ConeBeamProjectionWeightTask), fused into the filter's loads.
        sinograms=True: returns the sinograms [n_rows, N, crop] of detector rows
        first_row.. (QUADS: their slice-quad cells); False: rows in projection order
        [N, n_rows, crop]."""
        import torch
        if proj.dtype != torch.float32 or not proj.is_cuda or proj.dim() != 3:
            raise ValueError("projections must be a [N, H, W] float32 CUDA tensor")
        proj = proj.contiguous()
        N, H, W = proj.shape
        rows = n_rows or H - first_row
        cw, _ = self.get_requisition(W, 1)
        dt = DTYPES.get(dtype, dtype) if isinstance(dtype, str) else dtype
        pre, keep = _preprocess(ffc, dark, flat, cone)
        lead = (rows, N) if sinograms else (N, rows)
        if layout == QUADS:
            pitch = cw + 1
            shape = ((rows + 3) // 4, N, pitch, 4)
            tdt = torch.int32
        elif layout == PAIRS:
            pitch = (cw + 1 + 3) // 4 * 4
            shape, tdt = lead + (pitch,), torch.int32
        else:
            pitch = cw
            shape, tdt = lead + (cw,), {F32: torch.float32, F16: torch.float16, BF16: torch.bfloat16}[dt]
        out = torch.empty(shape, dtype=tdt, device=proj.device) if out is None else out
        check(lib().ufob_filter_run_projections(self._h, pre, _ptr(proj), W, H, N, W, int(sinograms), first_row,
                                                rows, _ptr(out), dt, layout, pitch, _stream(stream)))
        del keep
        return out

    def apply_spectrum(self, spec, stream=None):
        """The reference ``filter`` task alone on complex-interleaved rows [..., 2*N]."""
        import torch
        spec = spec.contiguous()
        out = torch.empty_like(spec)
        w2 = spec.shape[-1]
        check(lib().ufob_filter_apply_spectrum(self._h, _ptr(spec), _ptr(out), w2, spec.numel() // w2,
                                               _stream(stream)))
        return out


class BackprojectTask(_Task):
    """Parallel-beam ``backproject``.

    Properties: num-projections, offset, axis-pos, angle-step, angle-offset,
    mode (nearest|texture), roi-x, roi-y, roi-width, roi-height; engine
    extensions: compensated, tile."""

    def __init__(self, **props):
        super().__init__()
        L = lib()
        h = ctypes.c_void_p()
        check(L.ufob_backproject_create(None, ctypes.byref(h)))
        self._h = h
        self._set_num, self._set_str, self._destroy = (L.ufob_backproject_set_property,
                                                       L.ufob_backproject_set_property_string,
                                                       L.ufob_backproject_destroy)
        for k, v in props.items():
            self.set_property(k.replace("_", "-"), v)

    def get_requisition(self, width, height):
        w, h = ctypes.c_uint32(), ctypes.c_uint32()
        check(lib().ufob_backproject_get_requisition(self._h, width, height, ctypes.byref(w), ctypes.byref(h)))
        return w.value, h.value

    def process(self, sino, dtype=F32, layout=ROWS, width=None, out=None, stream=None, nslices=None):
        """Backproject [H, W] or [Z, H, W] float32 sinograms (or F16/BF16 pairs
        from FilterTask.process(layout=PAIRS), then pass ``width``)."""
        import torch
        if layout == QUADS:
            # [G, H, cells, 4] cells from FilterTask.process(layout=QUADS); pass width and nslices
            q = sino.contiguous()
            G, H, cells = q.shape[0], q.shape[1], q.shape[2]
            if width is None:
                raise ValueError("pass width= for the QUADS layout")
            Z = nslices or 4 * G
            ow, oh = self.get_requisition(width, H)
            out = torch.empty((Z, oh, ow), dtype=torch.float32, device=q.device) if out is None else out
            check(lib().ufob_backproject_run(self._h, _ptr(q), F16, QUADS, width, H, Z, cells, cells * H, _ptr(out),
                                             _stream(stream)))
            return out
        squeeze = sino.dim() == 2
        s3 = sino.unsqueeze(0) if squeeze else sino
        s3 = s3.contiguous()
        Z, H, pitch = s3.shape
        W = pitch if layout == ROWS else width
        if W is None:
            raise ValueError("pass width= for the pair layout")
        ow, oh = self.get_requisition(W, H)
        out = torch.empty((Z, oh, ow), dtype=torch.float32, device=s3.device) if out is None else out
        check(lib().ufob_backproject_run(self._h, _ptr(s3), dtype, layout, W, H, Z, pitch, pitch * H, _ptr(out),
                                         _stream(stream)))
        return out[0] if squeeze else out


class FBP:
    """``fft ! filter ! ifft ! backproject`` for a sinogram stack, one call.

    storage: filtered-sinogram storage type (F32, F16 or BF16)."""

    def __init__(self, filter_props=None, bp_props=None, storage=F32):
        L = lib()
        fp = FilterProps()
        L.ufob_filter_props_init(ctypes.byref(fp))
        for k, v in (filter_props or {}).items():
            k = k.replace("-", "_")
            if k == "filter" and isinstance(v, str):
                v = FILTERS.index(v)
            setattr(fp, k, v)
        bpp = BPProps()
        L.ufob_bp_props_init(ctypes.byref(bpp))
        for k, v in (bp_props or {}).items():
            k = k.replace("-", "_")
            if k == "mode" and isinstance(v, str):
                v = {"nearest": 0, "texture": 1}[v]
            setattr(bpp, k, v)
        h = ctypes.c_void_p()
        check(L.ufob_fbp_create(ctypes.byref(fp), ctypes.byref(bpp), DTYPES.get(storage, storage)
                                if isinstance(storage, str) else storage, ctypes.byref(h)))
        self._h = h
        self._destroy = L.ufob_fbp_destroy

    def get_requisition(self, width, height):
        w, h = ctypes.c_uint32(), ctypes.c_uint32()
        check(lib().ufob_fbp_get_requisition(self._h, width, height, ctypes.byref(w), ctypes.byref(h)))
        return w.value, h.value

    def process(self, sino, out=None, stream=None):
        import torch
        squeeze = sino.dim() == 2
        s3 = (sino.unsqueeze(0) if squeeze else sino).contiguous()
        Z, H, W = s3.shape
        ow, oh = self.get_requisition(W, H)
        out = torch.empty((Z, oh, ow), dtype=torch.float32, device=s3.device) if out is None else out
        check(lib().ufob_fbp_run(self._h, _ptr(s3), W, H, Z, _ptr(out), _stream(stream)))
        return out[0] if squeeze else out

    def process_projections(self, proj, ffc=None, dark=None, flat=None, first_row=0, n_rows=0, out=None,
                            stream=None):
        """``flat-field-correct ! transpose-projections ! fft ! filter ! ifft !
        backproject`` from projections [N, H, W] (float32 CUDA): one slice per
        detector row first_row .. first_row + n_rows - 1, [n_rows, roi_h, roi_w]."""
        import torch
        proj = proj.contiguous()
        N, H, W = proj.shape
        rows = n_rows or H - first_row
        ow, oh = self.get_requisition(W, N)
        out = torch.empty((rows, oh, ow), dtype=torch.float32, device=proj.device) if out is None else out
        pre, keep = _preprocess(ffc, dark, flat, None)
        check(lib().ufob_fbp_run_projections(self._h, pre, _ptr(proj), W, H, N, first_row, rows, _ptr(out),
                                             _stream(stream)))
        del keep
        return out

    def set_timing(self, enable=True):
        check(lib().ufob_fbp_set_timing(self._h, int(enable)))

    def kernel_times(self):
        """{'filter': (ms, launches), 'backproject': (ms, launches)} since set_timing()."""
        fm, bm = ctypes.c_double(), ctypes.c_double()
        fl, bl = ctypes.c_uint32(), ctypes.c_uint32()
        check(lib().ufob_fbp_kernel_times(self._h, ctypes.byref(fm), ctypes.byref(fl), ctypes.byref(bm),
                                          ctypes.byref(bl)))
        return {"filter": (fm.value, fl.value), "backproject": (bm.value, bl.value)}

    def process_host(self, sino, out=None, slices_per_chunk=32):
        """Host tensors/arrays in, host out; copies overlap compute inside the engine."""
        import torch
        Z, H, W = sino.shape
        ow, oh = self.get_requisition(W, H)
        if out is None:
            out = torch.empty((Z, oh, ow), dtype=torch.float32)
        check(lib().ufob_fbp_run_host(self._h, sino.data_ptr(), W, H, Z, out.data_ptr(), slices_per_chunk))
        return out

    def __del__(self):
        # the destroy function is bound at creation: module globals may be gone at interpreter exit
        h, fn = getattr(self, "_h", None), getattr(self, "_destroy", None)
        if h and fn:
            fn(h)
            self._h = None


class GeneralBackprojectTask(_Task):
    """``general-backproject``: parallel, cone and laminography volumes."""

    def __init__(self, **props):
        super().__init__()
        L = lib()
        h = ctypes.c_void_p()
        check(L.ufob_gbp_create(ctypes.byref(h)))
        self._h = h
        self._set_num, self._set_str, self._destroy = (L.ufob_gbp_set_property, L.ufob_gbp_set_property_string,
                                                       L.ufob_gbp_destroy)
        for k, v in props.items():
            self.set_property(k.replace("_", "-"), v)

    def set_property(self, name, value):
        if isinstance(value, (list, tuple)) or hasattr(value, "__len__") and not isinstance(value, str):
            import numpy as np
            arr = np.ascontiguousarray(value, dtype=np.float64).reshape(-1)
            check(lib().ufob_gbp_set_array(self._h, name.encode(), arr.ctypes.data, arr.size))
            self._values[name] = arr
        else:
            super().set_property(name, value)

    def setup(self):
        check(lib().ufob_gbp_setup(self._h))

    def get_requisition(self, width, height):
        w, h, n = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        check(lib().ufob_gbp_get_requisition(self._h, width, height, ctypes.byref(w), ctypes.byref(h),
                                             ctypes.byref(n)))
        return w.value, h.value, n.value

    def process(self, proj, out=None, stream=None, dtype=None):
        import torch
        proj = proj.contiguous()
        n, H, W = proj.shape
        self.setup()
        ow, oh, ns = self.get_requisition(W, H)
        st = self._values.get("store-type", "float")
        tdt = {"half": torch.float16, "float": torch.float32, "double": torch.float64, "uchar": torch.uint8,
               "ushort": torch.uint16, "uint": torch.uint32}[st]
        out = torch.empty((ns, oh, ow), dtype=tdt, device=proj.device) if out is None else out
        check(lib().ufob_gbp_run(self._h, _ptr(proj), W, H, _ptr(out), _stream(stream)))
        return out


class Batch:
    """Uneven batch of parallel-beam FBP jobs in one persistent launch."""

    def __init__(self, filter_props=None, storage=F32):
        L = lib()
        fp = FilterProps()
        L.ufob_filter_props_init(ctypes.byref(fp))
        for k, v in (filter_props or {}).items():
            setattr(fp, k.replace("-", "_"), v)
        h = ctypes.c_void_p()
        check(L.ufob_batch_create(ctypes.byref(fp), storage, ctypes.byref(h)))
        self._h = h
        self._destroy = L.ufob_batch_destroy

    def run(self, jobs, stream=None):
        arr = (Job * len(jobs))()
        for i, j in enumerate(jobs):
            arr[i] = Job(_ptr(j["sino"]), _ptr(j["out"]), j["sino"].shape[-1], j["sino"].shape[-2],
                         j.get("axis_pos", -1.0), j.get("angle_step", -1.0), j.get("angle_offset", 0.0))
        check(lib().ufob_batch_run(self._h, arr, len(jobs), _stream(stream)))

    def variant(self):
        return int(lib().ufob_batch_variant(self._h))

    @staticmethod
    def variants():
        """Number of tile-shape variants of the batch backprojector."""
        return int(lib().ufob_batch_variants())

    def set_variant(self, v):
        """Pin tile-shape variant v (0 .. variants()-1) instead of autotuning; -1 autotunes."""
        check(lib().ufob_batch_set_variant(self._h, int(v)))

    def __del__(self):
        h, fn = getattr(self, "_h", None), getattr(self, "_destroy", None)
        if h and fn:
            fn(h)
            self._h = None


class StackedBackprojectTask(_Task):
    """``stacked-backproject``: a stack of sinograms [Z, P, W] -> [Z, roi_h, roi_w]
    with the task's orientation (h = bx cos - by sin + axis).

    Properties: num-projections, offset, axis-pos, angle-step, angle-offset,
    roi-x/y/width/height and precision-mode ("int8", "half", "single")."""

    def __init__(self, **props):
        super().__init__()
        L = lib()
        h = ctypes.c_void_p()
        check(L.ufob_stacked_bp_create(ctypes.byref(h)))
        self._h = h
        self._set_num, self._set_str, self._destroy = (L.ufob_stacked_bp_set_property,
                                                       L.ufob_stacked_bp_set_property_string,
                                                       L.ufob_stacked_bp_destroy)
        for k, v in props.items():
            self.set_property(k.replace("_", "-"), v)

    def get_requisition(self, width, height):
        w, h = ctypes.c_uint32(), ctypes.c_uint32()
        check(lib().ufob_stacked_bp_get_requisition(self._h, width, height, ctypes.byref(w), ctypes.byref(h)))
        return w.value, h.value

    def process(self, sino, out=None, stream=None):
        import torch
        if sino.dtype != torch.float32 or not sino.is_cuda:
            raise ValueError("sinograms must be a float32 CUDA tensor")
        squeeze = sino.dim() == 2
        s3 = (sino.unsqueeze(0) if squeeze else sino).contiguous()
        Z, H, W = s3.shape
        ow, oh = self.get_requisition(W, H)
        out = torch.empty((Z, oh, ow), dtype=torch.float32, device=s3.device) if out is None else out
        check(lib().ufob_stacked_bp_run(self._h, _ptr(s3), W, H, Z, _ptr(out), _stream(stream)))
        return out[0] if squeeze else out


class LaminoBackprojectTask(_Task):
    """``lamino-backproject`` (a reductor).  Array properties x-region, y-region
    (integers from, to, step), region (the swept parameter's from, to, step),
    projection-offset, center; numbers z, num-projections, overall-angle,
    tomo-angle, lamino-angle, roll-angle; strings parameter ("z", "x-center",
    "lamino-angle", "roll-angle") and addressing-mode."""

    ARRAYS = ("x-region", "y-region", "region", "projection-offset", "center")

    def __init__(self, **props):
        super().__init__()
        L = lib()
        h = ctypes.c_void_p()
        check(L.ufob_lamino_create(ctypes.byref(h)))
        self._h = h
        self._set_num, self._set_str, self._destroy = (L.ufob_lamino_set_property, L.ufob_lamino_set_property_string,
                                                       L.ufob_lamino_destroy)
        for k, v in props.items():
            self.set_property(k.replace("_", "-"), v)

    def set_property(self, name, value):
        if name in self.ARRAYS:
            import numpy as np
            arr = np.ascontiguousarray(value, dtype=np.float64).reshape(-1)
            check(lib().ufob_lamino_set_array(self._h, name.encode(), arr.ctypes.data, arr.size))
            self._values[name] = tuple(arr)
        else:
            super().set_property(name, value)

    def setup(self):
        check(lib().ufob_lamino_setup(self._h))

    def get_requisition(self):
        x, y, z = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        check(lib().ufob_lamino_get_requisition(self._h, ctypes.byref(x), ctypes.byref(y), ctypes.byref(z)))
        return x.value, y.value, z.value

    def process(self, proj, out=None, stream=None):
        """All projections [n, H, W] (float32 CUDA) -> volume [nz, ny, nx]."""
        import torch
        proj = proj.contiguous()
        _, H, W = proj.shape
        self.setup()
        nx, ny, nz = self.get_requisition()
        out = torch.empty((nz, ny, nx), dtype=torch.float32, device=proj.device) if out is None else out
        check(lib().ufob_lamino_run(self._h, _ptr(proj), W, H, _ptr(out), _stream(stream)))
        return out

    def push(self, projection, stream=None):
        """The task's process(): one projection [H, W]."""
        H, W = projection.shape
        check(lib().ufob_lamino_process(self._h, _ptr(projection.contiguous()), W, H, _stream(stream)))

    def generate(self, out=None, stream=None):
        import torch
        nx, ny, nz = self.get_requisition()
        out = torch.empty((nz, ny, nx), dtype=torch.float32, device="cuda") if out is None else out
        check(lib().ufob_lamino_generate(self._h, _ptr(out), _stream(stream)))
        return out


def _preprocess(ffc, dark, flat, cone):
    """ctypes Preprocess for the fused filter entry points (None when empty) and
    the objects it points into, to be kept alive over the call."""
    if ffc is None and cone is None:
        return None, ()
    pre = Preprocess()
    keep = [pre]
    if ffc is not None:
        if dark is None or flat is None:
            raise ValueError("flat-field correction needs dark and flat")
        dark, flat = dark.contiguous(), flat.contiguous()
        pre.ffc = ctypes.pointer(ffc._p)
        pre.d_dark, pre.d_flat = _ptr(dark), _ptr(flat)
        keep += [dark, flat, ffc]
    if cone is not None:
        pre.cone = cone._h
        keep.append(cone)
    return ctypes.byref(pre), keep


class FlatFieldCorrectTask:
    """``flat-field-correct``: (data - dark*ds) / (flat*fs - dark*ds), or with
    absorption-correct the log of the inverse ratio.

    Properties: fix-nan-and-inf, absorption-correct, sinogram-input,
    dark-scale, flat-scale (reference defaults)."""

    def __init__(self, **props):
        self._p = FFCProps()
        lib().ufob_ffc_props_init(ctypes.byref(self._p))
        self._values = {}
        for k, v in props.items():
            self.set_property(k.replace("_", "-"), v)

    def set_property(self, name, value):
        check(lib().ufob_ffc_set_property(ctypes.byref(self._p), name.encode(), float(value)))
        self._values[name] = value

    def get_property(self, name):
        f = {"fix-nan-and-inf": "fix_nan_and_inf", "absorption-correct": "absorption_correct",
             "sinogram-input": "sinogram_input", "dark-scale": "dark_scale", "flat-scale": "flat_scale"}[name]
        v = getattr(self._p, f)
        return bool(v) if isinstance(v, int) else v

    def process(self, data, dark, flat, out=None, stream=None):
        """data [..., H, W] float32 CUDA; dark/flat [H, W] (or [W] with sinogram-input)."""
        import torch
        data, dark, flat = data.contiguous(), dark.contiguous(), flat.contiguous()
        W = data.shape[-1]
        H = data.shape[-2] if data.dim() >= 2 else 1
        n = data.numel() // (W * H)
        want = (W,) if self._p.sinogram_input else (H, W)
        if tuple(dark.shape) != want or tuple(flat.shape) != want:
            raise UfobError(ERR_REQUISITION, "flat-field-correct inputs must have the same size")
        out = torch.empty_like(data) if out is None else out
        check(lib().ufob_flat_field_correct(ctypes.byref(self._p), _ptr(data), _ptr(dark), _ptr(flat), W, H, n,
                                            _ptr(out), _stream(stream)))
        return out


class ConeBeamProjectionWeightTask(_Task):
    """``cone-beam-projection-weight``.  Array properties center-position-x/z,
    source-distance, detector-distance (required) and axis-angle-x (default 0);
    one value broadcasts, else projection i uses value i.  Counts the
    projections it has weighted, like the task's process()."""

    def __init__(self, **props):
        super().__init__()
        L = lib()
        h = ctypes.c_void_p()
        check(L.ufob_cone_weight_create(ctypes.byref(h)))
        self._h = h
        self._destroy = L.ufob_cone_weight_destroy
        for k, v in props.items():
            self.set_property(k.replace("_", "-"), v)

    def set_property(self, name, value):
        import numpy as np
        arr = np.ascontiguousarray(np.atleast_1d(np.asarray(value, dtype=np.float64)).reshape(-1))
        check(lib().ufob_cone_weight_set_array(self._h, name.encode(), arr.ctypes.data, arr.size))
        self._values[name] = value

    @property
    def count(self):
        return int(lib().ufob_cone_weight_get_count(self._h))

    @count.setter
    def count(self, value):
        check(lib().ufob_cone_weight_set_count(self._h, int(value)))

    def process(self, proj, out=None, stream=None):
        """proj [H, W] (one projection) or [n, H, W], float32 CUDA."""
        import torch
        proj = proj.contiguous()
        p3 = proj.unsqueeze(0) if proj.dim() == 2 else proj
        n, H, W = p3.shape
        out = torch.empty_like(proj) if out is None else out
        check(lib().ufob_cone_weight_run(self._h, _ptr(p3), W, H, n, _ptr(out), _stream(stream)))
        return out


class TransposeProjectionsTask:
    """``transpose-projections`` (a reductor): process() takes projections
    [H, W] (or [n, H, W]) one after another, generate() then returns the
    sinograms [num_projections, W] one per call (None at the end).  The
    sinogram stack lives on the device; `sinograms` is all of it [H, N, W]."""

    def __init__(self, num_projections=0, **props):
        self.num_projections = int(props.get("num-projections", num_projections))
        self.sinograms = None
        self._next = 0
        self._gen = 0

    def set_property(self, name, value):
        if name.replace("_", "-") != "num-projections":
            raise UfobError(ERR_INVALID, "transpose-projections: no property named '%s'" % name)
        self.num_projections = int(value)

    def get_requisition(self, width, height):
        return width, self.num_projections

    def process(self, proj, stream=None):
        """Returns False once num_projections projections were taken (as the task does)."""
        import torch
        p3 = (proj.unsqueeze(0) if proj.dim() == 2 else proj).contiguous()
        n, H, W = p3.shape
        if self.sinograms is None:
            if self.num_projections <= 0:
                raise UfobError(ERR_SETUP, "transpose-projections: num-projections not set")
            self.sinograms = torch.zeros((H, self.num_projections, W), dtype=torch.float32, device=p3.device)
        if self._next >= self.num_projections:
            return False
        n = min(n, self.num_projections - self._next)
        check(lib().ufob_transpose_projections(_ptr(p3), W, H, n, _ptr(self.sinograms), self.num_projections,
                                               self._next, _stream(stream)))
        self._next += n
        return True

    def generate(self):
        if self.sinograms is None or self._gen >= self.sinograms.shape[0]:
            return None
        self._gen += 1
        return self.sinograms[self._gen - 1]


def get_task(name, **props):
    """Create a task by its ufo-filters name."""
    table = {"filter": FilterTask, "backproject": BackprojectTask, "general-backproject": GeneralBackprojectTask,
             "flat-field-correct": FlatFieldCorrectTask, "cone-beam-projection-weight": ConeBeamProjectionWeightTask,
             "transpose-projections": TransposeProjectionsTask, "stacked-backproject": StackedBackprojectTask,
             "lamino-backproject": LaminoBackprojectTask}
    if name not in table:
        raise KeyError("no task named %r (available: %s)" % (name, ", ".join(sorted(table))))
    return table[name](**props)


def device_status():
    check(lib().ufob_device_status())


def phantom_sinogram(ellipses, width, n_angles, angle_step=None, axis=None, scale=None, out=None, stream=None):
    """Analytic ellipse sinogram [n_angles, width] computed on the device."""
    import numpy as np
    import torch
    ell = np.ascontiguousarray(ellipses, dtype=np.float64)
    step = math.pi / n_angles if angle_step is None else angle_step
    axis = width / 2.0 if axis is None else axis
    scale = width / 2.0 if scale is None else scale
    out = torch.empty((n_angles, width), dtype=torch.float32, device="cuda") if out is None else out
    check(lib().ufob_phantom_sinogram(ell.ctypes.data, len(ell), width, n_angles, step, axis, scale, _ptr(out),
                                      _stream(stream)))
    return out


def phantom_stack(ellipsoids, width, n_angles, nslices, angle_step=None, axis=None, scale=None, out=None,
                  stream=None):
    """Analytic ellipsoid sinogram stack [nslices, n_angles, width] computed on the device."""
    import numpy as np
    import torch
    ell = np.ascontiguousarray(ellipsoids, dtype=np.float64)
    step = math.pi / n_angles if angle_step is None else angle_step
    axis = width / 2.0 if axis is None else axis
    scale = width / 2.0 if scale is None else scale
    out = torch.empty((nslices, n_angles, width), dtype=torch.float32, device="cuda") if out is None else out
    check(lib().ufob_phantom_stack(ell.ctypes.data, len(ell), width, n_angles, nslices, step, axis, scale,
                                   _ptr(out), _stream(stream)))
    return out


def launch_count():
    return int(lib().ufob_launch_count())


def device_alloc_count():
    """Device allocations (cudaMalloc) the engine has made in this process so far."""
    return int(lib().ufob_device_alloc_count())


def measure_peaks():
    """(shared-memory GB/s, FP32 TFLOP/s) sustained by this device."""
    a, b = ctypes.c_double(), ctypes.c_double()
    check(lib().ufob_measure_peaks(ctypes.byref(a), ctypes.byref(b)))
    return a.value, b.value


def forwardproject(slice_img, n_angles, axis_pos=None, angle_step=None, out=None, stream=None):
    """Ray-marching forward projection of a [W, W] CUDA tensor into [n_angles, W]."""
    import torch
    W = slice_img.shape[-1]
    axis_pos = W / 2.0 if axis_pos is None else axis_pos
    angle_step = math.pi / n_angles if angle_step is None else angle_step
    img = slice_img.contiguous()
    out = torch.empty((n_angles, W), dtype=torch.float32, device=img.device) if out is None else out
    check(lib().ufob_forwardproject(_ptr(img), W, n_angles, axis_pos, angle_step, _ptr(out), _stream(stream)))
    return out


def phantom_images(ellipse_lists, N, axis=None, scale=None, supersample=4, stream=None):
    """Rasterise a list of ellipse arrays into a [len(lists), N, N] CUDA tensor."""
    import numpy as np
    import torch
    offs = np.zeros(len(ellipse_lists) + 1, dtype=np.uint32)
    for i, e in enumerate(ellipse_lists):
        offs[i + 1] = offs[i] + len(e)
    ell = np.ascontiguousarray(np.concatenate([np.asarray(e, dtype=np.float64).reshape(-1, 6)
                                               for e in ellipse_lists]), dtype=np.float64)
    axis = N / 2.0 if axis is None else axis
    scale = N / 2.0 if scale is None else scale
    out = torch.empty((len(ellipse_lists), N, N), dtype=torch.float32, device="cuda")
    check(lib().ufob_phantom_images(ell.ctypes.data, offs.ctypes.data, len(ellipse_lists), N, axis, scale,
                                    supersample, _ptr(out), _stream(stream)))
    return out
