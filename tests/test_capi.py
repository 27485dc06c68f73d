"""Host-side checks of the C ABI that need no GPU: the library loads, exports
every function include/ufob.h declares, and enforces the reference tasks'
property ranges and requisition rules (src/ufo-filter-task.c:290-300,
src/ufo-fft-task.c:139-145, src/ufo-ifft-task.c:132-137,
src/ufo-backproject-task.c:224-244)."""
import ctypes
import os
import re

import pytest

import ufob

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "ufob.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ufob_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = ufob.lib()
    names = declared_functions()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    ufob.lib()
    for n in declared_functions():
        assert getattr(ufob.lib(), n).argtypes is not None or n in (), n


def _filter(**props):
    return ufob.FilterTask(**props)


def test_filter_defaults_and_requisition():
    f = _filter()
    assert f.get_requisition(512, 100) == (512, 100)
    f.props.size_x = 1024
    assert f.get_requisition(512, 100) == (1024, 100)  # ifft crop-width defaults to the FFT width
    f.props.crop_width = 512
    assert f.get_requisition(512, 100) == (512, 100)


def test_filter_rejects_non_power_of_two():
    f = _filter()
    with pytest.raises(ufob.UfobError) as e:
        f.get_requisition(1536, 10)
    assert e.value.status == ufob.ERR_REQUISITION
    assert "power of two" in str(e.value)
    f.props.size_x = 2048
    assert f.get_requisition(1536, 10) == (2048, 10)


def test_filter_size_smaller_than_input_fails():
    f = _filter(size_x=256)
    with pytest.raises(ufob.UfobError) as e:
        f.get_requisition(512, 1)
    assert "greater than or equal" in str(e.value)


def test_filter_crop_larger_than_fft_fails():
    f = _filter(crop_width=1024)
    with pytest.raises(ufob.UfobError):
        f.get_requisition(512, 1)


@pytest.mark.parametrize("name,value", [("cutoff", 1.5), ("cutoff", -0.1), ("order", 1.0), ("order", 33.0),
                                        ("size-x", 40000), ("crop-width", 40000), ("filter", 9)])
def test_filter_property_ranges(name, value):
    f = _filter()
    with pytest.raises(ufob.UfobError) as e:
        f.set_property(name, value)
    assert e.value.status == ufob.ERR_INVALID


def test_filter_enum_by_nick():
    f = _filter()
    for nick in ufob.FILTERS:
        f.props.filter = nick
    with pytest.raises(ufob.UfobError):
        f.props.filter = "shepp-logan"
    with pytest.raises(ufob.UfobError):
        f.set_property("no-such-property", 1)


def test_backproject_requisition_defaults():
    bp = ufob.BackprojectTask()
    assert bp.get_requisition(512, 360) == (512, 512)  # roi defaults to width x width
    bp.props.roi_width = 100
    bp.props.roi_height = 50
    assert bp.get_requisition(512, 360) == (100, 50)


def test_backproject_height_exceeds_num_projections():
    bp = ufob.BackprojectTask(num_projections=100)
    with pytest.raises(ufob.UfobError) as e:
        bp.get_requisition(64, 180)
    assert e.value.status == ufob.ERR_REQUISITION
    assert "must be greater than or equal to sinogram height" in str(e.value)


def test_backproject_offset_beyond_table():
    bp = ufob.BackprojectTask(num_projections=100, offset=50)
    assert bp.get_requisition(64, 50) == (64, 64)
    with pytest.raises(ufob.UfobError):
        bp.get_requisition(64, 51)


@pytest.mark.parametrize("name,value", [("axis-pos", -2.0), ("axis-pos", 40000.0), ("num-projections", 40000),
                                        ("angle-offset", -1.0), ("mode", 5)])
def test_backproject_property_ranges(name, value):
    bp = ufob.BackprojectTask()
    with pytest.raises(ufob.UfobError):
        bp.set_property(name, value)


def test_backproject_mode_nick():
    bp = ufob.BackprojectTask()
    bp.props.mode = "nearest"
    bp.props.mode = "texture"
    with pytest.raises(ufob.UfobError):
        bp.props.mode = "linear"


def test_run_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = ufob.lib()
    st = L.ufob_device_check(None, None, None)
    assert st == ufob.ERR_CUDA
    assert L.ufob_last_error()


def test_status_strings():
    L = ufob.lib()
    for s in range(8):
        assert L.ufob_status_string(s)


def test_batch_variant_pinning_range():
    """Tile variants can be pinned from 0 to variants()-1, or -1 for the autotuner."""
    b = ufob.Batch()
    n = ufob.Batch.variants()
    assert n == 8
    b.set_variant(n - 1)
    b.set_variant(-1)
    with pytest.raises(ufob.UfobError):
        b.set_variant(n)
    with pytest.raises(ufob.UfobError):
        b.set_variant(-2)

