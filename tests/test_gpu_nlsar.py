"""Parity of the CUDA NL-SAR path with the oracle, through the C ABI.

Tolerances (FP32 against the FP64 oracle): reflectivity and coherence within
1e-4 relative, phase within 1e-3 rad.  They are asserted on every pixel whose
FP64 result is well conditioned: no weight of the selected combination within
1e-3 LUT-index units of a boundary where the weight changes, no weighted
intensity variance within 1e-4 of zero relative to the squared mean (where the
reference's alpha formula divides by a vanishing variance), and, in ENL-argmax
mode, a bias-reduced ENL margin above 1e-4 between the best and second-best
combination.  Coherence and phase are asserted where, in addition, the
weighted complex mean cancels by at most a factor 20 (sum w|C01| over
|sum w C01|): FP32 rounding of that sum scales with the factor, for the
reference's own FP32 kernels as for these.  On the remaining pixels one LUT
bin or one selection may flip between any two FP32 implementations; at least
99% of all pixels must still meet the tolerance.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import despeckcl_b200 as dcl  # noqa: E402
from despeckcl_b200 import synthetic  # noqa: E402
from nlsar_parity import KAPPA_MAX, PHASE_TOL, REL_TOL, check_crops, check_parity, run_gpu, wrapped  # noqa: E402,F401

SWS, PATCHES, SCALES = 21, [3, 5, 7], [1, 3]


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()


@pytest.mark.parametrize("mode", ["reference", "argmax_enl"])
@pytest.mark.parametrize("shape,seed", [((48, 64), 1), ((33, 70), 2), ((96, 96), 3)])
def test_nlsar_matches_fp64_oracle(oracle, train_stats, shape, seed, mode):
    a1, a2, ph = synthetic.insar_scene(*shape, seed)
    m = 0 if mode == "reference" else 1
    o = oracle.nlsar_insar(a1, a2, ph, SWS, PATCHES, SCALES, train_stats, select_mode=m, use_double=True, diag=True)
    g = run_gpu(a1, a2, ph, train_stats, mode, selection=True)
    check_parity(g, o[:3], o[3], mode)
    # the per-pixel selection agrees wherever the ENL margin is clear and no
    # weight of any combination sits within 1e-3 index units of a LUT edge
    d = o[3]
    clear = ((d.enl_margin > 1e-4) & (d.var_cond > 1e-4) & (d.bin_margin_all > 1e-3)
             if mode == "argmax_enl" else np.ones(shape, bool))
    assert np.array_equal(g[3][clear], d.sel[clear])
    assert (g[3] == d.sel).mean() >= 0.995


@pytest.mark.parametrize("mode", ["reference", "argmax_enl"])
def test_nlsar_matches_fp32_oracle(oracle, train_stats, mode):
    a1, a2, ph = synthetic.insar_scene(64, 80, 4)
    m = 0 if mode == "reference" else 1
    o32 = oracle.nlsar_insar(a1, a2, ph, SWS, PATCHES, SCALES, train_stats, select_mode=m)
    o64 = oracle.nlsar_insar(a1, a2, ph, SWS, PATCHES, SCALES, train_stats, select_mode=m, use_double=True,
                             diag=True)
    g = run_gpu(a1, a2, ph, train_stats, mode)
    check_parity(g, o32, o64[3], mode)


@pytest.mark.parametrize("shape", [(1, 1), (1, 7), (5, 3), (17, 2)])
def test_nlsar_degenerate_shapes(oracle, train_stats, shape):
    a1, a2, ph = synthetic.insar_scene(max(shape[0], 2), max(shape[1], 2), 9)
    a1, a2, ph = (x[:shape[0], :shape[1]].copy() for x in (a1, a2, ph))
    o = oracle.nlsar_insar(a1, a2, ph, SWS, PATCHES, SCALES, train_stats, use_double=True, diag=True)
    g = run_gpu(a1, a2, ph, train_stats, "reference")
    check_parity(g, o[:3], o[3], "reference", min_all=0.0, min_stable=0.0)


@pytest.mark.parametrize("seed", range(8))
def test_random_small_shapes(oracle, train_stats, seed):
    # heights and widths drawn from 1..40 (tiles cut by the scene edge, the
    # virtual last row and column inside the first tile), both selection modes
    rng = np.random.default_rng(1000 + seed)
    H, W = int(rng.integers(1, 41)), int(rng.integers(1, 41))
    a1, a2, ph = synthetic.insar_scene(max(H, 2), max(W, 2), 200 + seed)
    a1, a2, ph = (x[:H, :W].copy() for x in (a1, a2, ph))
    mode = ("reference", "argmax_enl")[seed % 2]
    o = oracle.nlsar_insar(a1, a2, ph, SWS, PATCHES, SCALES, train_stats, select_mode=seed % 2, use_double=True,
                           diag=True)
    o32 = oracle.nlsar_insar(a1, a2, ph, SWS, PATCHES, SCALES, train_stats, select_mode=seed % 2)
    # on a few dozen pixels one flipped bin is a few percent: the bar for all
    # pixels is what the FP32 oracle (the reference's arithmetic) reaches,
    # less two pixels
    with np.errstate(divide="ignore", invalid="ignore"):
        ok32 = ((np.abs(o32[0] - o[0]) <= 1e-4 * np.abs(o[0])) &
                (np.abs(o32[2] - o[2]) <= 1e-4 * np.maximum(np.abs(o[2]), 1e-3)) &
                (wrapped(o32[1] - o[1]) <= 1e-3))
    g = run_gpu(a1, a2, ph, train_stats, mode)
    check_parity(g, o[:3], o[3], mode, min_all=max(0.0, ok32.mean() - 2.0 / (H * W)), min_stable=0.0)


def test_nlsar_example_parameters(oracle):
    # the reference example's settings (examples/insar_test.py:43-56):
    # patches {3,5,7,9,11}, scales {1,3,5}, training on a 25x25 area
    P, S = [3, 5, 7, 9, 11], [1, 3, 5]
    t1, t2, tp = synthetic.training_area(25, seed=3)
    stats = oracle.training_insar(t1, t2, tp, P, S)
    a1, a2, ph = synthetic.insar_scene(40, 52, 5)
    for mode, m in (("reference", 0), ("argmax_enl", 1)):
        o = oracle.nlsar_insar(a1, a2, ph, 21, P, S, stats, select_mode=m, use_double=True, diag=True)
        g = run_gpu(a1, a2, ph, stats, mode, patches=P, scales=S)
        # a 25x25 training area gives coarse LUTs (a few pairs for the largest
        # patches), so more pixels sit near a bin edge
        check_parity(g, o[:3], o[3], mode, min_all=0.97)


def test_reference_mode_with_extra_stats_key(oracle, train_stats):
    # a statistics key outside patch_sizes x scale_sizes sorts last: the
    # reference then filters every pixel with the first combination's weights
    # and alpha 0 (nlsar_filter_sub_image.cpp:418-422, 537-545)
    stats = dict(train_stats)
    stats[(9, 3)] = train_stats[(7, 3)]
    a1, a2, ph = synthetic.insar_scene(40, 40, 6)
    o = oracle.nlsar_insar(a1, a2, ph, SWS, PATCHES, SCALES, stats, use_double=True, diag=True)
    g = run_gpu(a1, a2, ph, stats, "reference", selection=True)
    check_parity(g, o[:3], o[3], "reference")
    assert (g[3] == 0).all()


def test_covariance_path_matches_oracle(oracle, train_stats):
    a1, a2, ph = synthetic.insar_scene(40, 56, 8)
    cov8 = oracle.covmat_create(a1, a2, ph)
    # a generic (non-InSAR) covariance: perturb the imaginary diagonal and the
    # lower off-diagonal so that all 8 planes carry independent data
    rng = np.random.default_rng(0)
    cov8[1] = rng.normal(0, 0.1, cov8[1].shape)
    cov8[4] *= 1.01
    for mode, m in (("reference", 0), ("argmax_enl", 1)):
        o = oracle.nlsar_covmat(cov8, SWS, PATCHES, SCALES, train_stats, select_mode=m, use_double=True)
        cplx = (cov8[0::2] + 1j * cov8[1::2]).reshape(2, 2, 40, 56)
        g = dcl.nlsar(cplx, SWS, PATCHES, SCALES, train_stats, select_mode=mode)
        gi = np.empty_like(o)
        gi[0::2] = g.real.reshape(4, 40, 56)
        gi[1::2] = g.imag.reshape(4, 40, 56)
        # each element within 1e-4 of its own magnitude, or of 1e-2 of the
        # pixel's larger diagonal where it is much smaller than that (noise on
        # the imaginary diagonal, near-zero off-diagonals): FP32 rounding of a
        # weighted sum scales with the magnitudes summed; no scale is zero
        diag_mag = np.maximum(np.abs(o[0]), np.abs(o[6]))
        scale = np.maximum(np.abs(o), 1e-2 * diag_mag[None])
        assert (scale > 0).all()
        err = np.abs(gi - o) / scale
        assert np.isfinite(err).all()
        assert (err <= 1e-4).mean() >= 0.99, err.max()


def test_specialised_and_generic_kernels_agree(tmp_path, train_stats):
    # the compile-time specialised kernel serves (21, {3,5,7}); the generic
    # kernel (forced through DESPECKCL_B200_GENERIC=1 in a child process)
    # must give the same result up to FP32 summation order
    import os
    import pickle
    import subprocess
    import sys

    a1, a2, ph = synthetic.insar_scene(64, 96, 30)
    fast = run_gpu(a1, a2, ph, train_stats, "argmax_enl")
    f = tmp_path / "in.pkl"
    stats = {k: (v.lut_size, v.dissims_min, v.dissims_max, v.quantilles, v.chi2cdf_inv)
             for k, v in train_stats.items()}
    pickle.dump((a1, a2, ph, stats), open(f, "wb"))
    code = (
        "import pickle,sys,numpy as np; sys.path.insert(0, %r); import despeckcl_b200 as d; "
        "a1,a2,ph,st=pickle.load(open(%r,'rb')); "
        "st={k: d.Stats(*v) for k,v in st.items()}; "
        "r=d.nlsar_insar(a1,a2,ph,21,[3,5,7],[1,3],st,select_mode='argmax_enl'); "
        "pickle.dump(r, open(%r,'wb'))" % (os.path.dirname(os.path.dirname(os.path.abspath(__file__))), str(f),
                                          str(tmp_path / "out.pkl")))
    env = dict(os.environ, DESPECKCL_B200_GENERIC="1")
    subprocess.run([sys.executable, "-c", code], env=env, check=True)
    gen = pickle.load(open(tmp_path / "out.pkl", "rb"))
    e = np.abs(fast[0] - gen[0]) / gen[0]
    assert (e <= 1e-4).mean() >= 0.99
    assert (wrapped(fast[1] - gen[1]) <= 1e-3).mean() >= 0.99


@pytest.mark.parametrize("P,S,mode", [
    ([3, 5, 7], [1, 3], "argmax_enl"),
    ([3, 5, 7], [1, 3], "reference"),
    ([3, 5, 7, 9, 11], [1, 3, 5], "argmax_enl"),   # two pass shapes, staged for patch 11
])
def test_covariance_specialised_and_generic_kernels_agree(tmp_path, oracle, train_stats, P, S, mode):
    # 8-plane covariance input: the specialised kernel (32 x 24 tiles) against
    # the generic one, forced in a child process, up to FP32 summation order
    import os
    import pickle
    import subprocess
    import sys

    a1, a2, ph = synthetic.insar_scene(75, 90, 31)
    cov8 = oracle.covmat_create(a1, a2, ph).astype(np.float32)
    rng = np.random.default_rng(5)
    cov8[1] = rng.normal(0, 0.1, cov8[1].shape)
    cov8[7] = rng.normal(0, 0.1, cov8[7].shape)
    cov8[4] *= 1.02
    cplx = (cov8[0::2] + 1j * cov8[1::2]).reshape(2, 2, 75, 90)
    st_obj = train_stats
    if P != PATCHES or S != SCALES:
        t1, t2, tp = synthetic.training_area(64, seed=3)
        st_obj = dcl.nlsar_train_insar(t1, t2, tp, P, S)
    fast = dcl.nlsar(cplx, SWS, P, S, st_obj, select_mode=mode)
    f = tmp_path / "in.pkl"
    stats = {k: (v.lut_size, v.dissims_min, v.dissims_max, v.quantilles, v.chi2cdf_inv)
             for k, v in st_obj.items()}
    pickle.dump((cplx, stats), open(f, "wb"))
    code = (
        "import pickle,sys,numpy as np; sys.path.insert(0, %r); import despeckcl_b200 as d; "
        "c,st=pickle.load(open(%r,'rb')); "
        "st={k: d.Stats(*v) for k,v in st.items()}; "
        "r=d.nlsar(c,21,%r,%r,st,select_mode=%r); "
        "pickle.dump(r, open(%r,'wb'))" % (os.path.dirname(os.path.dirname(os.path.abspath(__file__))), str(f),
                                          P, S, mode, str(tmp_path / "out.pkl")))
    env = dict(os.environ, DESPECKCL_B200_GENERIC="1")
    subprocess.run([sys.executable, "-c", code], env=env, check=True)
    gen = pickle.load(open(tmp_path / "out.pkl", "rb"))
    scale = np.maximum(np.abs(gen), np.abs(gen[0, 0]).real[None, None] * 1e-2)
    err = np.abs(fast - gen) / scale
    assert (err <= 1e-4).mean() >= 0.99, err.max()


@pytest.mark.parametrize("P,S,mode", [
    ([3, 5, 7, 9, 11], [1, 3, 5], "argmax_enl"),
    ([3, 5, 7, 9, 11], [1, 3, 5], "reference"),
    ([9], [1, 3], "argmax_enl"),
    ([9, 11], [1, 3], "argmax_enl"),
])
def test_example_settings_specialised_and_generic_kernels_agree(tmp_path, P, S, mode):
    # the reference example's settings (patches 3..11, scales 1..5): passes of
    # {3,5,7} and {9,11} at each scale, staged for patch 11, in the
    # specialised kernel; reference selection runs patch 11 at scale 5 alone.
    # Patch 9 alone and passes of {9,11} alone take the other instantiations
    # of those sizes.  The generic kernel, forced in a child process, must
    # agree up to FP32 summation order.
    import os
    import pickle
    import subprocess
    import sys

    t1, t2, tp = synthetic.training_area(64, seed=3)
    stats = dcl.nlsar_train_insar(t1, t2, tp, P, S)
    a1, a2, ph = synthetic.insar_scene(70, 90, 32)
    fast = run_gpu(a1, a2, ph, stats, mode, patches=P, scales=S)
    f = tmp_path / "in.pkl"
    st = {k: (v.lut_size, v.dissims_min, v.dissims_max, v.quantilles, v.chi2cdf_inv) for k, v in stats.items()}
    pickle.dump((a1, a2, ph, st), open(f, "wb"))
    code = (
        "import pickle,sys,numpy as np; sys.path.insert(0, %r); import despeckcl_b200 as d; "
        "a1,a2,ph,st=pickle.load(open(%r,'rb')); "
        "st={k: d.Stats(*v) for k,v in st.items()}; "
        "r=d.nlsar_insar(a1,a2,ph,21,%r,%r,st,select_mode=%r); "
        "pickle.dump(r, open(%r,'wb'))" % (os.path.dirname(os.path.dirname(os.path.abspath(__file__))), str(f),
                                          P, S, mode, str(tmp_path / "out.pkl")))
    env = dict(os.environ, DESPECKCL_B200_GENERIC="1")
    subprocess.run([sys.executable, "-c", code], env=env, check=True)
    gen = pickle.load(open(tmp_path / "out.pkl", "rb"))
    e = np.abs(fast[0] - gen[0]) / gen[0]
    assert (e <= 1e-4).mean() >= 0.99
    assert (wrapped(fast[1] - gen[1]) <= 1e-3).mean() >= 0.99


def test_host_entry_point_equals_device_entry_point(train_stats):
    a1, a2, ph = synthetic.insar_scene(70, 90, 10)
    host = dcl.nlsar_insar(a1, a2, ph, SWS, PATCHES, SCALES, train_stats, select_mode="argmax_enl")
    dev = run_gpu(a1, a2, ph, train_stats, "argmax_enl")
    for h, d in zip(host, dev):
        np.testing.assert_array_equal(h, d)


@pytest.mark.parametrize("shape,mode,bands", [((1061, 97), "argmax_enl", 4), ((520, 64), "reference", 2),
                                              ((777, 41), "argmax_enl", 25), ((1700, 1500), "argmax_enl", None)])
def test_banded_host_entry_point_equals_device_entry_point(train_stats, monkeypatch, shape, mode, bands):
    # the host entry point filters scenes of many waves of tiles in row bands
    # whose copies overlap the filtering (1700 x 1500: two bands by itself;
    # the smaller scenes are cut by DESPECKCL_B200_BANDS); results must equal
    # one launch's
    if bands is not None:
        monkeypatch.setenv("DESPECKCL_B200_BANDS", str(bands))
    a1, a2, ph = synthetic.insar_scene(*shape, 21)
    host = dcl.nlsar_insar(a1, a2, ph, SWS, PATCHES, SCALES, train_stats, select_mode=mode)
    dev = run_gpu(a1, a2, ph, train_stats, mode)
    for h, d in zip(host, dev):
        np.testing.assert_array_equal(h, d)


@pytest.mark.parametrize("shape,bands", [((530, 70), 2), ((1045, 45), 5)])
def test_banded_covariance_host_entry_point_equals_device_entry_point(oracle, train_stats, monkeypatch, shape, bands):
    import ctypes

    import despeckcl_b200.api as api

    monkeypatch.setenv("DESPECKCL_B200_BANDS", str(bands))
    H, W = shape
    a1, a2, ph = synthetic.insar_scene(H, W, 22)
    cov8 = np.ascontiguousarray(oracle.covmat_create(a1, a2, ph), dtype=np.float32)
    cov8[1] = np.random.default_rng(1).normal(0, 0.1, cov8[1].shape)
    L = api.lib()
    pk, pp, npn = api._ints(PATCHES)
    sk, sp, nsn = api._ints(SCALES)
    arr, n, keep = api._entries(train_stats)
    host = np.empty_like(cov8)
    api._check(L.dcl_nlsar_covmat(api._fp(cov8), api._fp(host), H, W, 2, SWS, pp, npn, sp, nsn, arr, n,
                                  ctypes.c_float(15.0), ctypes.c_float(49.0), 1))
    din = torch.from_numpy(cov8).cuda()
    dout = torch.empty_like(din)
    api._check(L.dcl_nlsar_covmat_device(ctypes.c_void_p(din.data_ptr()), ctypes.c_void_p(dout.data_ptr()), H, W, 2,
                                         SWS, pp, npn, sp, nsn, arr, n, ctypes.c_float(15.0), ctypes.c_float(49.0), 1,
                                         None))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(host, dout.cpu().numpy())


def test_shift_invariance_is_bit_exact(train_stats):
    # each output pixel depends only on its overlap-radius neighbourhood, so a
    # crop filtered alone reproduces the interior of the full scene exactly
    a1, a2, ph = synthetic.insar_scene(200, 260, 12)
    full = run_gpu(a1, a2, ph, train_stats, "argmax_enl")
    y0, x0, h, w = 37, 61, 90, 120
    crop = run_gpu(*(x[y0:y0 + h, x0:x0 + w].copy() for x in (a1, a2, ph)), train_stats, "argmax_enl")
    ov = 14
    for f, c in zip(full, crop):
        np.testing.assert_array_equal(c[ov:h - ov - 1, ov:w - ov - 1],
                                      f[y0 + ov:y0 + h - ov - 1, x0 + ov:x0 + w - ov - 1])


def test_batched_launch_equals_single_scenes(train_stats):
    shapes = [(64, 96), (130, 70), (33, 200)]
    scenes = [synthetic.insar_scene(h, w, 20 + i) for i, (h, w) in enumerate(shapes)]
    tens = [tuple(torch.from_numpy(x).cuda() for x in s) for s in scenes]
    outs = dcl.nlsar_insar_batch_device(tens, SWS, PATCHES, SCALES, train_stats, select_mode="argmax_enl")
    torch.cuda.synchronize()
    for s, o in zip(scenes, outs):
        single = run_gpu(*s, train_stats, "argmax_enl")
        for a, b in zip(o, single):
            np.testing.assert_array_equal(a.cpu().numpy(), b)


def test_constant_scene_is_a_fixed_point(train_stats):
    a = np.full((64, 64), 2.0, np.float32)
    z = np.full((64, 64), 0.5, np.float32)
    ref, ph, coh = run_gpu(a, a, z, train_stats, "argmax_enl")
    np.testing.assert_allclose(ref, 4.0, rtol=1e-5)
    np.testing.assert_allclose(ph, 0.5, atol=1e-5)
    np.testing.assert_allclose(coh, 1.0, rtol=1e-5)


@pytest.mark.parametrize("mode", ["reference", "argmax_enl"])
def test_config1_scene(oracle, train_stats, mode):
    # the 512 x 512 scene of the first benchmark configuration, seed 1, in
    # both selection modes (the benchmark runs the ENL argmax)
    a1, a2, ph = synthetic.insar_scene(512, 512, 1)
    m = 0 if mode == "reference" else 1
    o = oracle.nlsar_insar(a1, a2, ph, SWS, PATCHES, SCALES, train_stats, select_mode=m, use_double=True,
                           diag=True)
    g = run_gpu(a1, a2, ph, train_stats, mode, selection=True)
    frac_ok, frac_stable = check_parity(g, o[:3], o[3], mode)
    d = o[3]
    clear = ((d.enl_margin > 1e-4) & (d.var_cond > 1e-4) & (d.bin_margin_all > 1e-3)
             if m == 1 else np.ones(a1.shape, bool))
    assert np.array_equal(g[3][clear], d.sel[clear])
    assert (g[3] == d.sel).mean() >= 0.995
    print(f"config-1 {mode}: {frac_ok:.5f} within tolerance, {frac_stable:.3f} well conditioned")


def test_config2_scene_crops_argmax(oracle, train_stats):
    # the 4096 x 4096 scene of the headline benchmark (seed 1), ENL argmax:
    # the GPU filters the whole scene, the FP64 oracle six 96 x 96 crops
    a1, a2, ph = synthetic.insar_scene(4096, 4096, 1)
    sel = torch.zeros((4096, 4096), dtype=torch.int32, device="cuda")
    t = [torch.from_numpy(x).cuda() for x in (a1, a2, ph)]
    out = dcl.nlsar_insar_device(*t, SWS, PATCHES, SCALES, train_stats, select_mode="argmax_enl", selection=sel)
    torch.cuda.synchronize()
    g = [x.cpu().numpy() for x in out]
    frac_ok, frac_stable = check_crops(oracle, train_stats, (a1, a2, ph), g, sel.cpu().numpy(), "argmax_enl",
                                       ncrops=6, seed=2)
    print(f"config-2 crops: {frac_ok:.5f} within tolerance, {frac_stable:.3f} well conditioned")


def test_boxcar_matches_oracle(oracle):
    a1, a2, ph = synthetic.insar_scene(300, 530, 13)
    # w <= 15 runs the radius-specialised kernel, w = 17 the generic one
    for w in (1, 3, 5, 7, 15, 17):
        o = oracle.boxcar(a1, a2, ph, w)
        g = dcl.boxcar(a1, a2, ph, w)
        np.testing.assert_allclose(g[0], o[0], rtol=1e-5)
        np.testing.assert_array_less(wrapped(g[1] - o[1]), 1e-4)
        np.testing.assert_allclose(g[2], o[2], rtol=1e-4, atol=1e-6)


def test_boxcar_plane_alignment(oracle):
    # rows a multiple of 4 long, planes at 16-byte boundaries (the host entry
    # point's buffers) and one float past them (device views into a larger
    # buffer): same bits, and the oracle's values within tolerance
    H, W = 300, 528
    a1, a2, ph = synthetic.insar_scene(H, W, 14)
    n = H * W
    flat = torch.empty(3 * n + 4, dtype=torch.float32, device="cuda")
    for w in (1, 3, 7, 9, 15):
        o = oracle.boxcar(a1, a2, ph, w)
        g = dcl.boxcar(a1, a2, ph, w)
        np.testing.assert_allclose(g[0], o[0], rtol=1e-5)
        np.testing.assert_array_less(wrapped(g[1] - o[1]), 1e-4)
        np.testing.assert_allclose(g[2], o[2], rtol=1e-4, atol=1e-6)
        planes = []
        for i, a in enumerate((a1, a2, ph)):
            v = flat[1 + i * n:1 + (i + 1) * n].view(H, W)
            v.copy_(torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)))
            assert v.data_ptr() % 16 != 0
            planes.append(v)
        d = dcl.boxcar_device(*planes, w)
        torch.cuda.synchronize()
        for x, y in zip(g, d):
            np.testing.assert_array_equal(x, y.cpu().numpy())


def test_training_matches_oracle(oracle):
    t1, t2, tp = synthetic.training_area(128, seed=7)
    mine = dcl.nlsar_train_insar(t1, t2, tp, PATCHES, SCALES)
    ref = oracle.training_insar(t1, t2, tp, PATCHES, SCALES)
    assert sorted(mine.keys()) == sorted(ref.keys())
    for k in ref:
        a, b = mine[k], ref[k]
        n = 128 - k[1] + 1
        npatch = (-(-n // k[0])) ** 2
        npairs = npatch * (npatch - 1) // 2
        assert a.lut_size == 256
        assert a.dissims_min == pytest.approx(b.dissims_min, rel=1e-5)
        assert a.dissims_max == pytest.approx(b.dissims_max, rel=1e-5)
        assert np.abs(a.quantilles - b.quantilles).max() <= 5.0 / npairs + 1e-7
        np.testing.assert_array_equal(a.chi2cdf_inv, b.chi2cdf_inv)


def test_prepared_batch_graph_autotune_equal_single_scenes(train_stats):
    # a prepared batch (eager, CUDA-graph replay, either kernel instantiation
    # the autotuner may pick) reproduces the single-scene results bit for bit
    shapes = [(70, 40), (129, 257), (32, 33), (300, 90)]
    scenes = [synthetic.insar_scene(h, w, 50 + i) for i, (h, w) in enumerate(shapes)]
    tens = [tuple(torch.from_numpy(x).cuda() for x in s) for s in scenes]
    singles = [run_gpu(*s, train_stats, "argmax_enl") for s in scenes]
    for graph in (False, True):
        b = dcl.NlsarBatch(tens, SWS, PATCHES, SCALES, train_stats, select_mode="argmax_enl", graph=graph,
                           autotune=True)
        assert b.variant in (0, 1)
        for _ in range(2):
            outs = b.run()
            torch.cuda.synchronize()
            for o, ref in zip(outs, singles):
                for a, r in zip(o, ref):
                    np.testing.assert_array_equal(a.cpu().numpy(), r)
        b.close()


def test_kernel_instantiations_agree_bitwise(train_stats):
    # the 2- and 4-pixel-per-thread instantiations on 32 x 32 tiles and the
    # 32 x 16-tile one sum in the same per-pixel order, so they agree exactly
    a1, a2, ph = synthetic.insar_scene(77, 99, 60)
    tens = [tuple(torch.from_numpy(x).cuda() for x in (a1, a2, ph))]
    res = []
    for v in (0, 1, 2):
        b = dcl.NlsarBatch(tens, SWS, PATCHES, SCALES, train_stats, graph=False, autotune=False, variant=v)
        assert b.variant == v
        res.append([o.cpu().numpy() for o in b.run()[0]])
        b.close()
    for other in res[1:]:
        for a, r in zip(res[0], other):
            np.testing.assert_array_equal(a, r)


def _polsar_scene(H, W, seed, homogeneous=False):
    """A single-look 3-channel (PolSAR) covariance image [18][H][W]: per
    region a random Hermitian positive-definite covariance, speckled as
    k = L x with x ~ CN(0, I) and the pixel covariance k k^H."""
    rng = np.random.default_rng(seed)
    cov = np.zeros((3, 3, H, W), np.complex128)

    def region_L():
        z = rng.normal(size=(3, 5)) + 1j * rng.normal(size=(3, 5))
        return np.linalg.cholesky(z @ z.conj().T / 5)

    L0 = region_L()
    labels = np.zeros((H, W), np.int32)
    Ls = [L0]
    if not homogeneous:
        for _ in range(6):
            y0, x0 = rng.integers(0, H), rng.integers(0, W)
            labels[y0:y0 + H // 3, x0:x0 + W // 3] = len(Ls)
            Ls.append(region_L())
    x = (rng.normal(size=(3, H, W)) + 1j * rng.normal(size=(3, H, W))) / np.sqrt(2)
    k = np.zeros((3, H, W), np.complex128)
    for i, L in enumerate(Ls):
        m = labels == i
        k[:, m] = L @ x[:, m]
    cov = k[:, None] * k[None, :].conj()
    planes = np.empty((18, H, W), np.float32)
    planes[0::2] = cov.real.reshape(9, H, W)
    planes[1::2] = cov.imag.reshape(9, H, W)
    return planes, cov.astype(np.complex64)


def test_training_3x3_matches_oracle(oracle):
    planes, cplx = _polsar_scene(40, 44, 40, homogeneous=True)
    mine = dcl.nlsar_train(cplx, [3, 5], [1, 3])
    ref = oracle.training_covmat(planes, [3, 5], [1, 3])
    assert sorted(mine.keys()) == sorted(ref.keys())
    for k in ref:
        a, b = mine[k], ref[k]
        n = 40 - k[1] + 1
        npatch = (-(-n // k[0])) * (-(-(44 - k[1] + 1) // k[0]))
        npairs = npatch * (npatch - 1) // 2
        assert a.dissims_min == pytest.approx(b.dissims_min, rel=1e-4, abs=1e-4)
        assert a.dissims_max == pytest.approx(b.dissims_max, rel=1e-4)
        assert np.abs(a.quantilles - b.quantilles).max() <= 5.0 / npairs + 1e-7
        np.testing.assert_array_equal(a.chi2cdf_inv, b.chi2cdf_inv)


@pytest.mark.parametrize("mode", ["reference", "argmax_enl"])
@pytest.mark.parametrize("sws,patches", [(SWS, PATCHES), (15, [3, 5]), (SWS, [3, 5, 7, 9, 11])])
def test_covariance_3x3_path_matches_oracle(oracle, mode, sws, patches):
    # search 21 with patches {3,5,7} runs the specialised 3x3 kernel, with
    # patches 3..11 its two-pass-shape instantiation staged for patch 11,
    # search 15 with {3,5} the generic one
    tp, _ = _polsar_scene(40, 40, 41, homogeneous=True)
    stats = oracle.training_covmat(tp, sorted(set(patches) | {3, 5, 7}), [1, 3])
    planes, cplx = _polsar_scene(44, 60, 42)
    m = 0 if mode == "reference" else 1
    o = oracle.nlsar_covmat(planes, sws, patches, SCALES, stats, select_mode=m, use_double=True)
    o32 = oracle.nlsar_covmat(planes, sws, patches, SCALES, stats, select_mode=m)
    g = dcl.nlsar(cplx, sws, patches, SCALES, stats, select_mode=mode)
    gi = np.empty_like(o)
    gi[0::2] = g.real.reshape(9, 44, 60)
    gi[1::2] = g.imag.reshape(9, 44, 60)
    # errors relative to the element, floored at 1% of the geometric mean of
    # the two diagonal intensities of its row and column
    diag = o[[0, 8, 16]]
    scale = np.empty_like(o)
    for r in range(3):
        for c in range(3):
            floor = 1e-2 * np.sqrt(np.abs(diag[r] * diag[c]))
            for part in (0, 1):
                scale[2 * (r * 3 + c) + part] = np.maximum(np.abs(o[2 * (r * 3 + c) + part]), floor)
    with np.errstate(divide="ignore", invalid="ignore"):
        err = np.abs(gi - o) / scale
        err32 = np.abs(o32 - o) / scale
    # single-look 3x3 covariances are near-singular at scale 1, so LUT bins
    # and selections flip between any two FP32 implementations on about 1%
    # of the pixels: the CUDA path must stay as close to the FP64 oracle as
    # the FP32 oracle (the reference's own FP32 arithmetic) does
    for e_tol, planes_sel in ((1e-3, slice(None)), (1e-4, [0, 8, 16])):
        ok_g = (err[planes_sel] <= e_tol).mean()
        ok_32 = (err32[planes_sel] <= e_tol).mean()
        assert ok_g >= min(0.99, ok_32 - 0.005), (e_tol, ok_g, ok_32)
        assert ok_g >= 0.98


@pytest.mark.parametrize("shape,sws,patches,scales,bands", [
    ((37, 29), 11, [3, 5], [1], None),          # generic kernel, one band
    ((150, 47), 11, [3, 5], [1, 3], 5),         # generic kernel, host call in 5 row bands
    ((170, 53), 21, [3, 5, 7], [1, 3], 4),      # specialised kernel, 4 bands
    ((60, 44), 21, [3, 5, 7, 9, 11], [1, 3, 5], None),  # patches up to 11: two pass shapes
])
def test_covariance_3x3_device_entry_point_equals_host(oracle, monkeypatch, shape, sws, patches, scales, bands):
    if bands is not None:
        monkeypatch.setenv("DESPECKCL_B200_BANDS", str(bands))
    H, W = shape
    tp, _ = _polsar_scene(40, 40, 43, homogeneous=True)
    stats = oracle.training_covmat(tp, sorted(set(patches) | {3, 5, 7}), sorted(set(scales) | {1, 3}))
    planes, cplx = _polsar_scene(H, W, 44)
    host = dcl.nlsar(cplx, sws, patches, scales, stats, select_mode="argmax_enl")
    hi = np.empty_like(planes)
    hi[0::2] = host.real.reshape(9, H, W)
    hi[1::2] = host.imag.reshape(9, H, W)
    t = torch.from_numpy(planes).cuda()
    out = torch.empty_like(t)
    import ctypes

    import despeckcl_b200.api as api
    pk, pp, npn = api._ints(patches)
    sk, sp, nsn = api._ints(scales)
    arr, n, keep = api._entries(stats)
    api._check(dcl.lib().dcl_nlsar_covmat_device(api._dptr(t), api._dptr(out), H, W, 3, sws, pp, npn, sp, nsn, arr,
                                                 n, ctypes.c_float(15.0), ctypes.c_float(49.0), 1,
                                                 api._stream(None)))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), hi)
