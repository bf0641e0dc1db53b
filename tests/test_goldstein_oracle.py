"""The Goldstein oracle pinned against the reference's known answers and its
own kernels, and the host-side argument checks of dcl_goldstein.

Reference tests restated (paths relative to the reference project root):
  src/compute/goldstein/cl_wrappers/goldstein_patch_ft_test.cpp:38-130
      a constant patch transforms to a Dirac of height p^2 (forward FFT
      unnormalised), and forward + backward is the identity (1/p^2 backward)
  src/compute/goldstein/cl_wrappers/patches_pack_test.cpp:36-86 and
  patches_packing_test.cpp:35-107
      pack(unpack(x)) = x: the overlap weights form a partition of unity
Both are visible end to end: with alpha = 0 the weighting is 1 and the filter
returns raw + raw (the pack kernel adds onto the raw interferogram,
goldstein_filter_sub_image.cpp:130-176), so ampl = a1 + a2 and phase = phi; a
constant interferogram z0 gives ampl = |z0| (1 + (p^2 |z0|)^alpha).
Where the reference tree is present, its own .cl kernels run on the CPU
(oracle/_ref) and must agree with the restatement.
"""
import ctypes

import numpy as np
import pytest

from despeckcl_b200 import synthetic


def wrapped(d):
    return np.abs(np.angle(np.exp(1j * d)))


@pytest.mark.parametrize("use_double", [True, False])
@pytest.mark.parametrize("alpha", [0.5, 0.8])
def test_constant_interferogram_closed_form(oracle, use_double, alpha):
    H, W = 70, 90
    a1 = np.full((H, W), 1.3, np.float32)
    a2 = np.full((H, W), 0.7, np.float32)
    phi = np.full((H, W), 0.4, np.float32)
    ref, ph = oracle.goldstein(a1, a2, phi, 32, 4, alpha, use_double)
    z0 = 0.5 * (1.3 + 0.7)
    want = z0 * (1 + (32 * 32 * z0) ** alpha)
    np.testing.assert_allclose(ref, want, rtol=1e-5)
    assert wrapped(ph - 0.4).max() < 1e-5


@pytest.mark.parametrize("shape", [(48, 48), (100, 73), (257, 300)])
def test_alpha_zero_returns_raw_plus_raw(oracle, shape):
    a1, a2, phi = synthetic.insar_scene(*shape, 11)
    ref, ph = oracle.goldstein(a1, a2, phi, 32, 4, 0.0, True)
    np.testing.assert_allclose(ref, a1 + a2, rtol=1e-6, atol=1e-7)
    assert wrapped(ph - phi).max() < 1e-5


# (61, 40) and (85, 85) with overlap 4, and (64, 200) with overlap 7, are
# scenes for which the reference's tile iterator adds a second tile row and/or
# column that only the clamped last row / column sees
@pytest.mark.parametrize("shape,ov,alpha", [((48, 48), 4, 0.5), ((100, 73), 4, 0.5), ((257, 300), 4, 0.7),
                                            ((90, 130), 2, 0.5), ((64, 200), 7, 0.3), ((61, 40), 4, 0.5),
                                            ((85, 85), 4, 0.5)])
def test_restatement_matches_reference_kernels(oracle, shape, ov, alpha):
    a1, a2, phi = synthetic.insar_scene(*shape, 5)
    got = oracle.ref_goldstein(a1, a2, phi, 32, ov, alpha)
    if got is None:
        pytest.skip("reference source tree absent: kernels not built")
    rr, pr, cr = got
    rd, pd = oracle.goldstein(a1, a2, phi, 32, ov, alpha, True)
    scale = np.abs(rd).mean()
    assert (np.abs(rr - rd) <= 1e-4 * np.maximum(np.abs(rd), 0.05 * scale)).all()
    strong = rd > 0.05 * scale
    assert wrapped(pr - pd)[strong].max() < 1e-3
    assert (cr == 0).all()  # coherence untouched


def test_float_restatement_tracks_double(oracle):
    a1, a2, phi = synthetic.insar_scene(200, 160, 9)
    rf, pf = oracle.goldstein(a1, a2, phi, 32, 4, 0.5, False)
    rd, pd = oracle.goldstein(a1, a2, phi, 32, 4, 0.5, True)
    scale = np.abs(rd).mean()
    assert (np.abs(rf - rd) <= 1e-4 * np.maximum(np.abs(rd), 0.05 * scale)).all()


def test_tile_side_follows_round_up(oracle):
    L = oracle.lib()
    # round_up(n, m) = n - n % m + m: a multiple is still raised by m
    assert L.oracle_goldstein_tile_side(40, 40, 32, 4) == 72   # 48 -> 72
    assert L.oracle_goldstein_tile_side(100, 73, 32, 4) == 120
    assert L.oracle_goldstein_tile_side(16, 16, 32, 4) == 48


@pytest.mark.parametrize("p,ov,code", [(16, 2, -5), (64, 4, -5), (32, 8, -1), (32, -1, -1)])
def test_goldstein_argument_checks_on_the_host(p, ov, code):
    import despeckcl_b200 as dcl

    a = np.ones((40, 40), np.float32)
    with pytest.raises(dcl.DespeckclError) as e:
        dcl.goldstein(a, a, a, p, ov, 0.5)
    assert e.value.code == code
