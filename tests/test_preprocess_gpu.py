"""Preprocessing tasks on the GPU against the oracle: flat-field-correct,
transpose-projections and cone-beam-projection-weight on their own, and fused
into the filter stage (raw projections -> filtered sinograms in one kernel) and
into the whole parallel-beam reconstruction.

Reference: src/kernels/ffc.cl:20-50, src/ufo-flat-field-correct-task.c:120-170,
src/ufo-transpose-projections-task.c:60-120,
src/ufo-cone-beam-projection-weight-task.c:113-151, src/kernels/conebeam.cl:20-36.
Tolerances: the element-wise steps are FP32 with the kernels' operation order
and IEEE division/square root, so results are bit-exact except for the log of
absorption correction (a few ulp); filtered outputs are compared to the FP64
oracle within 1e-5 relative L2 (FP32 storage) and 1e-3 (FP16 storage)."""
import math

import numpy as np
import pytest
import torch

import oracle
import ufob

pytestmark = pytest.mark.gpu


def _frames(seed, n, H, W):
    rng = np.random.default_rng(seed)
    dark = rng.uniform(90, 110, (H, W)).astype(np.float32)
    flat = (dark + rng.uniform(800, 1200, (H, W))).astype(np.float32)
    data = (dark + rng.uniform(50, 1000, (n, H, W))).astype(np.float32)
    return data, dark, flat


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


FFC_CASES = [dict(), dict(absorption_correct=1), dict(absorption_correct=1, fix_nan_and_inf=1),
             dict(dark_scale=0.5, flat_scale=1.5), dict(fix_nan_and_inf=1, dark_scale=2.0)]


@pytest.mark.parametrize("props", FFC_CASES)
@pytest.mark.parametrize("W", [64, 37])  # vector and scalar paths
def test_flat_field_correct_matches_oracle(cuda, props, W):
    data, dark, flat = _frames(3, 3, 11, W)
    data[0, 0, :4] = dark[0, :4]  # zero transmission: inf / NaN cases
    task = ufob.FlatFieldCorrectTask(**props)
    got = task.process(_t(data), _t(dark), _t(flat)).cpu().numpy()
    ref = oracle.flat_field_correct(data, dark, flat, **props)
    if props.get("absorption_correct"):
        fin = np.isfinite(ref)
        np.testing.assert_array_equal(np.isfinite(got), fin)
        np.testing.assert_allclose(got[fin], ref[fin], rtol=4e-7, atol=1e-7)
    else:
        np.testing.assert_array_equal(got, ref)


def test_flat_field_correct_sinogram_input(cuda):
    data, dark, flat = _frames(4, 1, 9, 40)
    task = ufob.FlatFieldCorrectTask(sinogram_input=True)
    got = task.process(_t(data[0]), _t(dark[0]), _t(flat[0])).cpu().numpy()
    np.testing.assert_array_equal(got, oracle.flat_field_correct(data[0], dark[0], flat[0], sinogram_input=True))
    with pytest.raises(ufob.UfobError):  # frame-sized dark with sinogram-input
        task.process(_t(data[0]), _t(dark), _t(flat))


CONE = dict(center_position_x=30.5, center_position_z=9.25, source_distance=500.0, detector_distance=120.0)


@pytest.mark.parametrize("axis_angle", [0.0, 0.35])
@pytest.mark.parametrize("W", [64, 61])
def test_cone_weight_matches_oracle(cuda, axis_angle, W):
    rng = np.random.default_rng(5)
    proj = rng.standard_normal((4, 20, W)).astype(np.float32)
    props = dict(CONE, axis_angle_x=axis_angle)
    w = ufob.ConeBeamProjectionWeightTask(**props)
    got = w.process(_t(proj)).cpu().numpy()
    np.testing.assert_array_equal(got, oracle.cone_beam_weight(proj, **props))
    assert w.count == 4


def test_cone_weight_per_projection_arrays_and_count(cuda):
    rng = np.random.default_rng(6)
    proj = rng.standard_normal((5, 8, 32)).astype(np.float32)
    props = dict(center_position_x=list(rng.uniform(14, 18, 5)), center_position_z=4.0,
                 source_distance=list(rng.uniform(200, 400, 5)), detector_distance=60.0,
                 axis_angle_x=list(rng.uniform(0, 0.5, 5)))
    ref = oracle.cone_beam_weight(proj, **props)
    w = ufob.ConeBeamProjectionWeightTask(**props)
    a = w.process(_t(proj[:2])).cpu().numpy()  # projections 0, 1
    x = _t(proj[2:])
    w.process(x, out=x)  # in place, projections 2..4
    np.testing.assert_array_equal(a, ref[:2])
    np.testing.assert_array_equal(x.cpu().numpy(), ref[2:])
    assert w.count == 5
    with pytest.raises(ufob.UfobError):  # projection 5 has no value
        w.process(_t(proj[:1]))
    with pytest.raises(ufob.UfobError):  # unset properties
        ufob.ConeBeamProjectionWeightTask(source_distance=1.0).process(_t(proj))


def test_transpose_projections_task(cuda):
    rng = np.random.default_rng(7)
    N, H, W = 7, 5, 36
    proj = rng.standard_normal((N + 2, H, W)).astype(np.float32)
    t = ufob.TransposeProjectionsTask(num_projections=N)
    assert t.process(_t(proj[0]))        # one projection at a time,
    assert t.process(_t(proj[1:4]))      # or several
    assert t.process(_t(proj[4:]))       # more than num-projections: the rest is dropped
    assert not t.process(_t(proj[0]))
    np.testing.assert_array_equal(t.sinograms.cpu().numpy(), oracle.transpose_projections(proj[:N]))
    rows = []
    while (s := t.generate()) is not None:
        rows.append(s.cpu().numpy())
    assert len(rows) == H
    np.testing.assert_array_equal(np.stack(rows), oracle.transpose_projections(proj[:N]))


def test_transpose_scalar_path(cuda):
    proj = np.arange(3 * 4 * 7, dtype=np.float32).reshape(3, 4, 7)
    t = ufob.TransposeProjectionsTask(num_projections=3)
    t.process(_t(proj))
    np.testing.assert_array_equal(t.sinograms.cpu().numpy(), oracle.transpose_projections(proj))


@pytest.mark.parametrize("props", [dict(), dict(absorption_correct=1, fix_nan_and_inf=1)])
def test_filter_fused_ffc_transpose(cuda, props):
    """flat-field-correct ! transpose-projections ! fft ! filter ! ifft in one kernel."""
    N, H, W = 40, 9, 128
    data, dark, flat = _frames(8, N, H, W)
    ffc = ufob.FlatFieldCorrectTask(**props)
    f = ufob.FilterTask()
    got = f.process_projections(_t(data), ffc=ffc, dark=_t(dark), flat=_t(flat)).cpu().numpy()
    corrected = oracle.flat_field_correct(data, dark, flat, **props)
    ref = oracle.fft_filter_ifft(oracle.transpose_projections(corrected))
    assert got.shape == (H, N, W)
    assert oracle.rel_l2(got, ref) < 1e-5
    # the unfused engine path gives the same bits: same element-wise ops, same filter
    sinos = oracle.transpose_projections(ffc.process(_t(data), _t(dark), _t(flat)).cpu().numpy())
    np.testing.assert_array_equal(got, f.process(_t(sinos)).cpu().numpy())
    # a sub-range of detector rows
    sub = f.process_projections(_t(data), ffc=ffc, dark=_t(dark), flat=_t(flat), first_row=3, n_rows=4).cpu().numpy()
    np.testing.assert_array_equal(sub, got[3:7])


def test_filter_fused_quads(cuda):
    N, H, W = 60, 6, 64
    data, dark, flat = _frames(9, N, H, W)
    ffc = ufob.FlatFieldCorrectTask(absorption_correct=1)
    f = ufob.FilterTask()
    q = f.process_projections(_t(data), ffc=ffc, dark=_t(dark), flat=_t(flat), dtype=ufob.F16, layout=ufob.QUADS)
    sinos = oracle.transpose_projections(ffc.process(_t(data), _t(dark), _t(flat)).cpu().numpy())
    ref = f.process(_t(sinos), dtype=ufob.F16, layout=ufob.QUADS)
    assert q.shape == ref.shape == ((H + 3) // 4, N, W + 1, 4)
    assert torch.equal(q, ref)


def test_filter_fused_cone_weight_projection_order(cuda):
    """cone-beam-projection-weight ! fft ! filter ! ifft (the FDK order) in one kernel."""
    rng = np.random.default_rng(10)
    N, H, W = 6, 10, 64
    proj = rng.standard_normal((N, H, W)).astype(np.float32)
    props = dict(center_position_x=31.5, center_position_z=4.5, source_distance=list(rng.uniform(300, 400, N)),
                 detector_distance=80.0)
    cone = ufob.ConeBeamProjectionWeightTask(**props)
    f = ufob.FilterTask()
    got = f.process_projections(_t(proj), cone=cone, sinograms=False).cpu().numpy()
    assert cone.count == N
    ref = oracle.fft_filter_ifft(oracle.cone_beam_weight(proj, **props))
    assert got.shape == (N, H, W)
    assert oracle.rel_l2(got, ref) < 1e-5
    cone.count = 0
    weighted = cone.process(_t(proj))
    np.testing.assert_array_equal(got, f.process(weighted).cpu().numpy())


def test_fdk_chain_matches_oracle(cuda):
    """cone-beam-projection-weight ! fft ! filter ! ifft ! general-backproject (cone)."""
    rng = np.random.default_rng(11)
    N, H, W = 48, 24, 64
    proj = rng.uniform(0, 1, (N, H, W)).astype(np.float32)
    sd, dd = 150.0, 50.0
    cone = ufob.ConeBeamProjectionWeightTask(center_position_x=W / 2, center_position_z=H / 2, source_distance=sd,
                                             detector_distance=dd)
    filt = ufob.FilterTask().process_projections(_t(proj), cone=cone, sinograms=False)
    geom = {"source-position-y": -sd, "detector-position-y": dd, "center-position-x": W / 2,
            "center-position-z": H / 2}
    g = ufob.GeneralBackprojectTask(num_projections=N, region=(-4.0, 4.0, 1.0), **geom)
    got = g.process(filt).cpu().numpy()
    wref = oracle.cone_beam_weight(proj, center_position_x=W / 2, center_position_z=H / 2, source_distance=sd,
                                   detector_distance=dd)
    fref = oracle.fft_filter_ifft(wref).astype(np.float32)
    ref = oracle.general_backproject(fref, N, region=(-4.0, 4.0, 1.0), **geom)
    assert oracle.rel_l2(got, ref) < 1e-4


@pytest.mark.parametrize("storage,tol", [(ufob.F32, 1e-4), (ufob.F16, 1e-3)])
def test_fbp_from_raw_projections(cuda, storage, tol):
    """flat-field-correct ! transpose-projections ! fft ! filter ! ifft ! backproject."""
    N, H, W = 120, 10, 128
    rng = np.random.default_rng(12)
    ang = np.arange(N) * math.pi / N
    sinos = np.stack([oracle.ellipse_sinogram(oracle.random_ellipses(50 + y), W, ang) for y in range(H)])
    trans = np.exp(-0.02 * sinos).transpose(1, 0, 2)  # projections [N, H, W] of the transmission
    dark = rng.uniform(95, 105, (H, W)).astype(np.float32)
    flat = (dark + 1000).astype(np.float32)
    data = (dark + (flat - dark) * trans).astype(np.float32)
    ffc = ufob.FlatFieldCorrectTask(absorption_correct=1)
    fbp = ufob.FBP(storage=storage)
    got = fbp.process_projections(_t(data), ffc=ffc, dark=_t(dark), flat=_t(flat)).cpu().numpy()
    ref = oracle.fbp(oracle.transpose_projections(oracle.flat_field_correct(data, dark, flat,
                                                                            absorption_correct=True)))
    assert got.shape == (H, W, W)
    assert oracle.rel_l2(got, ref) < tol
    sub = fbp.process_projections(_t(data), ffc=ffc, dark=_t(dark), flat=_t(flat), first_row=2, n_rows=5).cpu().numpy()
    if storage == ufob.F32:
        np.testing.assert_array_equal(sub, got[2:7])
    else:  # the FP16 filter pairs slices (2g, 2g+1) in one complex FFT: other partners, other round-off
        assert oracle.rel_l2(sub, got[2:7]) < 1e-4


def test_fused_sinogram_input_rows(cuda):
    """sinogram-input: one dark/flat row for every row, applied in projection order."""
    Z, P, W = 3, 50, 64
    rng = np.random.default_rng(13)
    dark = rng.uniform(90, 110, W).astype(np.float32)
    flat = (dark + 1000).astype(np.float32)
    data = (dark + rng.uniform(50, 1000, (Z, P, W))).astype(np.float32)
    ffc = ufob.FlatFieldCorrectTask(sinogram_input=True, absorption_correct=True)
    got = ufob.FilterTask().process_projections(_t(data), ffc=ffc, dark=_t(dark), flat=_t(flat),
                                                sinograms=False).cpu().numpy()
    ref = oracle.fft_filter_ifft(oracle.flat_field_correct(data, dark, flat, sinogram_input=True,
                                                           absorption_correct=True))
    assert got.shape == (Z, P, W)
    assert oracle.rel_l2(got, ref) < 1e-5


def test_fused_cone_weight_row_subrange(cuda):
    """Detector rows first_row.. of each projection: the weight uses their absolute row."""
    rng = np.random.default_rng(14)
    N, H, W = 4, 16, 64
    proj = rng.standard_normal((N, H, W)).astype(np.float32)
    props = dict(center_position_x=30.0, center_position_z=7.5, source_distance=250.0, detector_distance=90.0,
                 axis_angle_x=0.2)
    cone = ufob.ConeBeamProjectionWeightTask(**props)
    got = ufob.FilterTask().process_projections(_t(proj), cone=cone, sinograms=False, first_row=5,
                                                n_rows=6).cpu().numpy()
    ref = oracle.fft_filter_ifft(oracle.cone_beam_weight(proj, **props)[:, 5:11])
    assert got.shape == (N, 6, W)
    assert oracle.rel_l2(got, ref) < 1e-5


@pytest.mark.parametrize("dtype,layout", [(ufob.F16, ufob.PAIRS), (ufob.BF16, ufob.PAIRS), (ufob.BF16, ufob.ROWS),
                                          (ufob.F16, ufob.ROWS)])
def test_fused_16bit_outputs_equal_unfused(cuda, dtype, layout):
    N, H, W = 30, 5, 128
    data, dark, flat = _frames(15, N, H, W)
    ffc = ufob.FlatFieldCorrectTask(absorption_correct=1)
    f = ufob.FilterTask()
    got = f.process_projections(_t(data), ffc=ffc, dark=_t(dark), flat=_t(flat), dtype=dtype, layout=layout)
    sinos = oracle.transpose_projections(ffc.process(_t(data), _t(dark), _t(flat)).cpu().numpy())
    ref = f.process(_t(sinos), dtype=dtype, layout=layout)
    assert got.shape == ref.shape
    assert torch.equal(got, ref)


def test_fused_rejections(cuda):
    f = ufob.FilterTask()
    data, dark, flat = _frames(16, 4, 3, 64)
    ffc = ufob.FlatFieldCorrectTask()
    with pytest.raises(ufob.UfobError):  # QUADS holds sinograms only
        f.process_projections(_t(data), ffc=ffc, dark=_t(dark), flat=_t(flat), sinograms=False, dtype=ufob.F16,
                              layout=ufob.QUADS)
    with pytest.raises(ufob.UfobError):  # rows past the projection height
        f.process_projections(_t(data), ffc=ffc, dark=_t(dark), flat=_t(flat), first_row=2, n_rows=2)
    with pytest.raises(ValueError):
        f.process_projections(_t(data), ffc=ffc)  # dark and flat missing


def test_volume_sharded_single_rank_on_gpu(cuda):
    """reconstruct_volume_sharded with the engine's own filter and general backprojector (one
    process: the exchange is the identity) equals the direct FDK chain."""
    from ufob import dist as udist
    rng = np.random.default_rng(17)
    N, H, W = 24, 16, 64
    proj = rng.uniform(0, 1, (N, H, W)).astype(np.float32)
    geom = {"source-position-y": -150.0, "detector-position-y": 50.0, "center-position-x": W / 2,
            "center-position-z": H / 2}
    cone = dict(center_position_x=W / 2, center_position_z=H / 2, source_distance=150.0, detector_distance=50.0)
    f = ufob.FilterTask()
    filt = lambda p: f.process_projections(p, cone=ufob.ConeBeamProjectionWeightTask(**cone), sinograms=False)
    bp = lambda allp, reg: ufob.GeneralBackprojectTask(num_projections=N, region=reg, **geom).process(allp)
    z0, z1, vol = udist.reconstruct_volume_sharded(udist.Ctx(), _t(proj), N, (-4.0, 4.0, 1.0), filt, bp)
    ref = bp(filt(_t(proj)), (-4.0, 4.0, 1.0))
    assert (z0, z1) == (0, 8)
    assert torch.equal(vol, ref)


def test_engine_matches_reference_kernel_fixtures(cuda):
    """The engine's flat-field correction and cone-beam weight against the outputs of the
    reference's own ffc.cl / conebeam.cl (compiled for the CPU, tests/golden/reference_pre.npz)."""
    import os
    from test_oracle_pinned_pre import CONE_CASES, FFC_CASES
    G = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_pre.npz"))
    for i, c in enumerate(FFC_CASES):
        props = {k: int(v) if isinstance(v, bool) else v for k, v in c.items()}
        got = ufob.FlatFieldCorrectTask(**props).process(_t(G["ffc_data"]), _t(G["ffc_dark"]),
                                                         _t(G["ffc_flat"])).cpu().numpy()
        ref = G["ffc_%d" % i]
        fin = np.isfinite(ref)
        np.testing.assert_array_equal(np.isfinite(got), fin)
        np.testing.assert_allclose(got[fin], ref[fin], rtol=3e-7, atol=1e-7)
    for i, c in enumerate(CONE_CASES):
        got = ufob.ConeBeamProjectionWeightTask(**c).process(_t(G["cone_input"])).cpu().numpy()
        np.testing.assert_allclose(got, G["cone_%d" % i], rtol=3e-7, atol=1e-7)
