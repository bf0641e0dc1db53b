"""The oracle pinned against the reference's own known-answer tests and, where
they compile here, against the reference's own translation units.

Reference test files (paths relative to the reference project root) restated:
  src/compute/nlsar/sim_measures_test.cpp:29-108
  src/compute/nlsar/stats_test.cpp:32-98
  src/compute/nlsar/best_params_test.cpp:30-62
  src/compute/nlsar/cl_wrappers/compute_alphas_test.cpp:35-126
  src/compute/nlsar/cl_wrappers/compute_enls_nobias_test.cpp:32-69
  src/compute/nlsar/cl_wrappers/covmat_create_test.cpp:37-178
  src/compute/nlsar/cl_wrappers/covmat_decompose_test.cpp:36-109
  src/compute/nlsar/cl_wrappers/covmat_rescale_test.cpp:35-87
  src/compute/nlsar/cl_wrappers/covmat_spatial_avg_test.cpp:37-165
  src/compute/nlsar/cl_wrappers/compute_nl_statistics_test.cpp:33-107
  src/compute/nlsar/cl_wrappers/weighted_means_test.cpp:32-92
  src/data/tile_test.cpp, src/data/tile_iterator.cpp
"""
import ctypes

import numpy as np
import pytest


def test_det_2x2_and_similarity_of_identical_pixels(oracle):
    # det of identity is 1 -> similarity between identical pixels is 0
    assert oracle.lib().oracle_pixel_similarity_2x2(1, 0, 0, 1, 1, 0, 0, 1) == pytest.approx(0.0, abs=1e-6)
    # a singular pixel next to a regular one: log(0) -> +inf dissimilarity
    s = oracle.lib().oracle_pixel_similarity_2x2(1, 1, 0, 1, 1, 0, 0, 1)
    assert np.isinf(s) and s > 0
    # two singular pixels: -inf + inf -> NaN -> 0 (sim_measures.h:61-63)
    assert oracle.lib().oracle_pixel_similarity_2x2(1, 1, 0, 1, 1, 1, 0, 1) == 0.0


def test_similarity_matches_reference_translation_unit(oracle):
    ref = oracle.ref_pieces()
    if ref is None:
        pytest.skip("reference source tree absent: pieces not built")
    rng = np.random.default_rng(3)
    for _ in range(2000):
        a = rng.gamma(2.0, 2.0, 2)
        b = rng.gamma(2.0, 2.0, 2)
        ga, gb = rng.uniform(0, 1, 2)
        pa, pb = rng.uniform(-np.pi, np.pi, 2)
        args = [a[0] ** 2, ga * a[0] * a[1] * np.cos(pa), ga * a[0] * a[1] * np.sin(pa), a[1] ** 2,
                b[0] ** 2, gb * b[0] * b[1] * np.cos(pb), gb * b[0] * b[1] * np.sin(pb), b[1] ** 2]
        args = [float(np.float32(x)) for x in args]
        assert oracle.lib().oracle_pixel_similarity_2x2(*args) == ref.ref_pixel_similarity_2x2(*args)


@pytest.mark.parametrize("m,det", [
    # the six Hermitian 3x3 cases of sim_measures_test.cpp:40-72, as
    # (a00, a11, a22, re a10, im a10, re a20, im a20, re a21, im a21)
    ((3, 2, 1, 0, 0, 0, 0, 0, 0), 6.0),
    ((2, 3, 1, 4, -3, 1, -2, 1, -1), -8.0),
    ((3, 2, 1, 0, -3, 2, 1, 0, 0), -13.0),
    ((3, 5, 1, 0, -3, 2, 1, 1, -1), -43.0),
    ((4, 5, 3, 0, -1, 2, 1, 1, -1), 18.0),
    ((5, 5, 5, 0, 4, -4, 0, 0, 4), 13.0),
])
def test_det_3x3_reference_cases(oracle, m, det):
    ref = oracle.ref_pieces()
    if ref is None:
        pytest.skip("reference source tree absent: pieces not built")
    arr = (ctypes.c_float * 9)(*m)
    assert ref.ref_det_covmat_3x3(arr) == pytest.approx(det, abs=1e-5)


def test_chi2_inverse_matches_scipy(oracle):
    sps = pytest.importorskip("scipy.stats")
    ys = np.arange(255) / 256.0
    mine = np.array([oracle.chi2_inv(y, 49) for y in ys], np.float32)
    ref = sps.chi2.ppf(ys, 49).astype(np.float32)
    np.testing.assert_array_equal(mine, ref)
    assert oracle.chi2_inv(0.5, 49) == pytest.approx(48.33497, rel=1e-6)


def test_stats_quantile_error_uniform(oracle):
    # stats_test.cpp:32-46: dissims 0..10000, L=1000 -> max LUT step 1/L
    st = oracle.stats_from_dissims(np.arange(10001, dtype=np.float32), 1000)
    assert np.max(np.diff(st.quantilles)) == pytest.approx(1.0 / 1000, abs=1e-6)
    assert st.chi2cdf_inv[-1] == 100000


def test_stats_quantile_error_kinked(oracle):
    # stats_test.cpp:48-65: second part of the range doubled -> max step 2/L
    d = np.arange(10001, dtype=np.float32)
    d[4000:] = 2 * np.arange(4000, 10001)
    st = oracle.stats_from_dissims(d, 1000)
    assert np.max(np.diff(st.quantilles)) == pytest.approx(2.0 / 1000, abs=1e-6)


def test_stats_quantiles_match_empirical_cdf(oracle):
    # stats_test.cpp:67-98 with gamma(2,2) samples
    rng = np.random.default_rng(0)
    d = np.sort(rng.gamma(2.0, 2.0, 10000).astype(np.float32))
    L = 1000
    st = oracle.stats_from_dissims(d, L)
    err = np.max(np.diff(st.quantilles))
    idx = np.minimum(((d - st.dissims_min) / (st.dissims_max - st.dissims_min) * L).astype(np.int64), L - 1)
    q = np.arange(d.size, dtype=np.float32) / d.size
    assert np.all(q - st.quantilles[idx] <= err)


def test_alpha_single_values(oracle):
    # compute_alphas_test.cpp:35-80: I=0, var=2 -> alpha 1
    var = (ctypes.c_float * 2)(2.0, 2.0)
    inl = (ctypes.c_float * 2)(0.0, 0.0)
    assert oracle.lib().oracle_alpha(var, inl, 2) == 1.0
    # range check (:82-126): alpha in [0, 1] for var >= I^2 >= 0 inputs
    rng = np.random.default_rng(1)
    for _ in range(500):
        i0, i1 = rng.uniform(0, 3, 2)
        v = (ctypes.c_float * 2)(*(np.array([i0, i1]) ** 2 * rng.uniform(1, 4, 2)))
        a = oracle.lib().oracle_alpha(v, (ctypes.c_float * 2)(i0, i1), 2)
        assert 0.0 <= a <= 1.0


def test_enl_nobias_single_value(oracle):
    # compute_enls_nobias_test.cpp:32-69: enl 1, alpha 0.5, wsum 2 -> 4/3
    assert oracle.lib().oracle_enl_nobias(1.0, 0.5, 2.0) == pytest.approx(1.333333333, rel=1e-6)


def test_covmat_create_determinant_and_structure(oracle):
    # covmat_create_test.cpp: single-look covariance is singular, Hermitian
    rng = np.random.default_rng(2)
    a1 = rng.gamma(2, 2, (10, 10)).astype(np.float32)
    a2 = rng.gamma(2, 2, (10, 10)).astype(np.float32)
    ph = rng.uniform(-np.pi, np.pi, (10, 10)).astype(np.float32)
    c = oracle.covmat_create(a1, a2, ph)
    det = c[0] * c[6] - (c[2] ** 2 + c[3] ** 2)
    assert np.max(np.abs(det) / (c[0] * c[6])) < 1e-5
    np.testing.assert_array_equal(c[4], c[2])
    np.testing.assert_array_equal(c[5], -c[3])
    assert np.all(c[1] == 0) and np.all(c[7] == 0)


def test_covmat_decompose_round_trip(oracle, train_stats):
    # covmat_decompose_test.cpp:36-109: create -> decompose returns
    # ((a1+a2)/2)^2 and the phase.  Exercised through a 1x1 search window
    # and 1x1 patch/scale, for which the filter is the identity.
    rng = np.random.default_rng(5)
    a1 = rng.gamma(2, 2, (12, 12)).astype(np.float32)
    a2 = rng.gamma(2, 2, (12, 12)).astype(np.float32)
    ph = rng.uniform(0, 1, (12, 12)).astype(np.float32)
    stats = {(1, 1): train_stats[(3, 1)]}
    ref, phase, coh = oracle.nlsar_insar(a1, a2, ph, 1, [1], [1], stats)
    np.testing.assert_allclose(ref, (0.5 * (a1 + a2)) ** 2, rtol=1e-4)
    np.testing.assert_allclose(phase, ph, atol=1e-5)
    np.testing.assert_allclose(coh, 1.0, atol=1e-4)


def test_rescale_gamma(oracle):
    # covmat_rescale_test.cpp: off-diagonals scaled by min(L/d,1)^0.33333
    assert oracle.lib().oracle_rescale_gamma() == np.float32(np.float32(0.5) ** np.float32(0.33333))


def test_spatial_average_kernel(oracle):
    # covmat_spatial_avg_test.cpp:37-165
    for s in (1, 3, 5, 7):
        g = oracle.gen_gauss(s).reshape(s, s)
        assert g.sum() == pytest.approx(1.0, abs=1e-6)
        np.testing.assert_array_equal(g, g.T)
        np.testing.assert_array_equal(g, g[::-1, ::-1])
    ones = np.ones((8, 20, 30), np.float32)
    out = oracle.covmat_spatial_avg(ones, 3, 5)
    np.testing.assert_allclose(out, 1.0, atol=1e-6)
    # scale 1 inside s_max 5 is a copy shifted by (5-1)/2
    rnd = np.random.default_rng(4).uniform(0, 1, (8, 20, 30)).astype(np.float32)
    out = oracle.covmat_spatial_avg(rnd, 1, 5)
    np.testing.assert_array_equal(out, rnd[:, 2:2 + 16, 2:2 + 26])


def test_filter_of_constant_scene_is_constant(oracle, train_stats):
    # compute_nl_statistics_test.cpp (ones -> sum w = 441, I = 1, var = 0)
    # and weighted_means_test.cpp (ones in -> ones out)
    a = np.ones((40, 50), np.float32)
    z = np.zeros((40, 50), np.float32)
    ref, phase, coh = oracle.nlsar_insar(a, a, z, 21, [3, 5, 7], [1, 3], train_stats)
    np.testing.assert_allclose(ref, 1.0, rtol=1e-5)
    np.testing.assert_allclose(phase, 0.0, atol=1e-6)
    np.testing.assert_allclose(coh, 1.0, rtol=1e-5)


def test_tile_iterator_matches_reference(oracle):
    ref = oracle.ref_pieces()
    if ref is None:
        pytest.skip("reference source tree absent: pieces not built")
    for H, W, th, tw, ov in [(512, 512, 128, 100, 14), (64, 80, 92, 108, 14), (37, 301, 40, 33, 3)]:
        cap = 4096
        h0 = (ctypes.c_int * cap)()
        w0 = (ctypes.c_int * cap)()
        n = ref.ref_tile_list(H, W, th, tw, ov, h0, w0, cap)
        assert oracle.tile_list(H, W, th, tw, ov) == list(zip(h0[:n], w0[:n]))


def test_best_params_reference_mode_matches_reference(oracle):
    # best_params.cpp:27-54 always returns the last key of the map for finite
    # ENLs; the oracle's reference mode does the same
    ref = oracle.ref_pieces()
    if ref is None:
        pytest.skip("reference source tree absent: pieces not built")
    keys = [(3, 1), (3, 3), (5, 1), (5, 3), (7, 1), (7, 3)]
    n = 50
    enl = np.random.default_rng(6).uniform(1, 400, (len(keys), n)).astype(np.float32)
    kk = (ctypes.c_int * (2 * len(keys)))(*[v for k in keys for v in k])
    out = (ctypes.c_int * (2 * n))()
    ref.ref_get_best_params(kk, len(keys), enl.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n, out)
    got = set(zip(out[0::2], out[1::2]))
    assert got == {(7, 3)}


def test_training_pair_counts(oracle):
    # patches.cpp / combinations.cpp: n = ceil(Hs/p)*ceil(Ws/p) patches, n(n-1)/2 pairs
    from despeckcl_b200 import synthetic

    a1, a2, ph = synthetic.training_area(64, seed=1)
    cov = oracle.covmat_create(a1, a2, ph)
    for p, s in [(3, 1), (5, 3), (7, 3)]:
        hs = 64 - s + 1
        n = (-(-hs // p)) ** 2
        assert oracle.training_dissims(cov, p, s).size == n * (n - 1) // 2


def _herm3(rng):
    """A random Hermitian positive-definite 3x3 matrix as its 9 unique reals
    {a00, a11, a22, Re a01, Im a01, Re a02, Im a02, Re a12, Im a12}."""
    z = rng.normal(size=(3, 4)) + 1j * rng.normal(size=(3, 4))
    m = z @ z.conj().T / 4
    return np.float32([m[0, 0].real, m[1, 1].real, m[2, 2].real, m[0, 1].real, m[0, 1].imag, m[0, 2].real,
                       m[0, 2].imag, m[1, 2].real, m[1, 2].imag])


def test_similarity_3x3_matches_reference_translation_unit(oracle):
    ref = oracle.ref_pieces()
    if ref is None:
        pytest.skip("reference source tree absent: pieces not built")
    rng = np.random.default_rng(5)
    fp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))  # noqa: E731
    for _ in range(2000):
        a, b = _herm3(rng), _herm3(rng)
        assert oracle.pixel_similarity_3x3(a, b) == ref.ref_pixel_similarity_3x3(fp(a), fp(b))
    # identical pixels: 0; a singular pixel next to a regular one: +inf
    a = _herm3(rng)
    assert oracle.pixel_similarity_3x3(a, a) == pytest.approx(0.0, abs=1e-4)
    s = np.float32([1, 1, 1, 1, 0, 1, 0, 1, 0])  # rank one: all-ones matrix
    assert np.isinf(oracle.pixel_similarity_3x3(s, a))


def test_rescale_gamma_3x3(oracle):
    # covmat_rescale.cl:25-26: (1/dim)^0.33333
    assert oracle.lib().oracle_rescale_gamma_dim(3) == pytest.approx((1 / 3) ** 0.33333, rel=1e-6)
    assert oracle.lib().oracle_rescale_gamma_dim(2) == oracle.lib().oracle_rescale_gamma()


def _cov18(m9, H, W):
    """A constant 18-plane covariance image from the 9 unique reals (the
    lower triangle the conjugate of the upper)."""
    a00, a11, a22, r01, i01, r02, i02, r12, i12 = [float(x) for x in m9]
    M = np.array([[a00, r01 + 1j * i01, r02 + 1j * i02],
                  [r01 - 1j * i01, a11, r12 + 1j * i12],
                  [r02 - 1j * i02, r12 - 1j * i12, a22]])
    cov = np.zeros((18, H, W), np.float32)
    for r in range(3):
        for c in range(3):
            cov[2 * (r * 3 + c)] = M[r, c].real
            cov[2 * (r * 3 + c) + 1] = M[r, c].imag
    return cov


def test_filter_of_constant_3x3_scene_is_constant(oracle):
    # compute_nl_statistics_test.cpp / weighted_means_test.cpp for 3x3: with
    # power-of-two entries every weighted mean is exact, the variance exactly
    # 0 and alpha 0, so a constant scene comes back unchanged
    rng = np.random.default_rng(6)
    m = np.float32([4, 2, 1, 0.5, 0.25, 0.25, -0.5, 0.125, 0.125])
    # training on a speckled 3-channel area gives LUTs with a sane spread
    z = (rng.normal(size=(3, 40, 40)) + 1j * rng.normal(size=(3, 40, 40))) / np.sqrt(2)
    train = np.zeros((18, 40, 40), np.float32)
    for r in range(3):
        for c in range(3):
            e = z[r] * z[c].conj()
            train[2 * (r * 3 + c)] = e.real
            train[2 * (r * 3 + c) + 1] = e.imag
    stats = oracle.training_covmat(train, [3, 5], [1, 3])
    cov = _cov18(m, 36, 40)
    for dbl in (False, True):
        out = oracle.nlsar_covmat(cov, 11, [3, 5], [1, 3], stats, select_mode=1, use_double=dbl)
        np.testing.assert_array_equal(out, cov)


def test_training_3x3_pair_counts(oracle):
    rng = np.random.default_rng(7)
    cov = _cov18(_herm3(rng), 30, 30) * rng.uniform(0.5, 1.5, (1, 30, 30)).astype(np.float32)
    for p, s in [(3, 1), (5, 3)]:
        n = -(-(30 - s + 1) // p)
        n = n * n
        d = oracle.training_dissims(cov, p, s)
        assert d.size == n * (n - 1) // 2
        assert np.isfinite(d).all()


@pytest.mark.parametrize("reference", [False, True])
@pytest.mark.parametrize("patch,pmax", [(3, 3), (3, 7), (5, 7)])
def test_patch_sums_of_constant_planes(oracle, reference, patch, pmax):
    # compute_patch_similarities_test.cpp:31-81: plane d of the pixel
    # similarities holds d everywhere; every patch sum of plane d is d * p^2
    # (20 x 30 similarities, search window 5).  reference=True runs the
    # reference's row and column pass kernels (oracle/_ref), when built.
    hs, ws, sws = 20, 30, 5
    U = sws * (sws // 2) + sws // 2
    pix = np.broadcast_to(np.arange(U, dtype=np.float32)[:, None, None], (U, hs, ws))
    got = oracle.patch_similarities(pix, sws, patch, pmax, reference=reference)
    if got is None:
        pytest.skip("reference pieces not built")
    want = np.broadcast_to((np.arange(U, dtype=np.float32) * patch * patch)[:, None, None], got.shape)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-4)


def test_patch_sums_oracle_equals_reference_kernels_on_random_planes(oracle):
    rng = np.random.default_rng(11)
    pix = rng.gamma(2.0, 1.0, (12, 23, 29)).astype(np.float32)
    for patch, pmax in [(3, 7), (5, 7), (7, 7), (9, 11)]:
        ref = oracle.patch_similarities(pix, 5, patch, pmax, reference=True)
        if ref is None:
            pytest.skip("reference pieces not built")
        np.testing.assert_array_equal(oracle.patch_similarities(pix, 5, patch, pmax), ref)


@pytest.mark.parametrize("reference", [False, True])
def test_copy_symm_weights_index_map(oracle, reference):
    # copy_symm_weights_test.cpp:33-128: random weights 0..9 on the upper half
    # window (70 x 30 pixels, search window 7); the full window holds the copied
    # upper half and, for the lower half, the value of the mirrored offset at
    # the shifted pixel.  reference=True runs the reference's kernel.
    ho, wo, sws = 70, 30, 7
    wsh = sws // 2
    U = sws * wsh + wsh
    rng = np.random.default_rng(5)
    wsymm = rng.integers(0, 10, (U, ho + wsh, wo + 2 * wsh)).astype(np.float32)
    full = oracle.copy_symm_weights(wsymm, ho, wo, sws, reference=reference)
    if full is None:
        pytest.skip("reference pieces not built")
    for i in range(U):
        np.testing.assert_array_equal(full[i], wsymm[i, :ho, wsh:wsh + wo])
    for hh in range(wsh, sws):
        for ww in range(wsh + 1 if hh == wsh else 0, sws):
            hhs, wws = sws - hh - 1, sws - ww - 1
            src = wsymm[hhs * sws + wws, hh - wsh:hh - wsh + ho, ww:ww + wo]
            np.testing.assert_array_equal(full[hh * sws + ww], src)
    if not reference:
        np.testing.assert_array_equal(full[U], np.ones((ho, wo), np.float32))  # self weight
