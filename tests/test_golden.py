"""The oracle against committed outputs of the reference's own code
(tests/golden/reference_pieces.npz, written by tests/golden/make_golden.py
from the reference sources compiled in place).  These run without the
reference tree: the fixtures are the record of what its code computes.
"""
import ctypes
import os

import numpy as np
import pytest
from nlsar_parity import REF_NLSAR, nlsar_cases, nlsar_stats

G = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_pieces.npz"))


def wrapped(d):
    return np.abs(np.angle(np.exp(1j * d.astype(np.float64))))


def test_pixel_similarity_2x2_matches_reference_bit_for_bit(oracle):
    f = oracle.lib().oracle_pixel_similarity_2x2
    got = np.float32([f(*[float(x) for x in r]) for r in G["sim2_args"]])
    ref = G["sim2_ref"]
    assert np.array_equal(np.isinf(got), np.isinf(ref))
    assert np.array_equal(got[np.isfinite(ref)], ref[np.isfinite(ref)])
    assert np.isinf(ref).any()  # the singular (single-look) cases are in the set


def test_pixel_similarity_3x3_matches_reference_bit_for_bit(oracle):
    got = np.float32([oracle.pixel_similarity_3x3(a, b) for a, b in zip(G["sim3_a"], G["sim3_b"])])
    assert np.array_equal(got, G["sim3_ref"])


def test_tile_iterator_matches_reference(oracle):
    tiles = G["tiles"]
    for i, (H, W, th, tw, ov) in enumerate(G["tile_cases"]):
        want = [tuple(t[1:]) for t in tiles if t[0] == i]
        assert oracle.tile_list(int(H), int(W), int(th), int(tw), int(ov)) == want


def test_reference_selection_takes_the_last_key():
    # best_params.cpp:27-54 never updates best_enl: every pixel gets the last
    # key of the (patch, scale)-ordered map, which DCL_SELECT_REFERENCE keeps
    last = G["best_keys"][-1]
    assert (G["best_ref"] == last).all()


def test_goldstein_restatement_matches_reference_kernels(oracle):
    a1, a2, ph = G["gold_in"]
    rd, pd = oracle.goldstein(a1, a2, ph, 32, 4, 0.5, True)
    rr, pr = G["gold_ref"]
    scale = np.abs(rd).mean()
    assert (np.abs(rr - rd) <= 1e-4 * np.maximum(np.abs(rd), 0.05 * scale)).all()
    assert wrapped(pr - pd)[rd > 0.05 * scale].max() < 1e-3


def test_nlinsar_fp32_restatement_matches_reference_bit_for_bit(oracle):
    a1, a2, ph = G["nl_in"]
    mine = oracle.nlinsar(a1, a2, ph, 21, 7, 2, 10, use_double=False)
    for m, r in zip(mine, G["nl_ref"]):
        assert np.array_equal(m, r)


# ---- end-to-end NL-SAR: the reference's own kernels (oracle/nlsar_ref_shim.cpp)

N = REF_NLSAR


@pytest.mark.parametrize("name,mode", list(nlsar_cases()))
def test_nlsar_fp32_oracle_matches_reference_kernels_bit_for_bit(oracle, name, mode):
    a1, a2, ph = N[f"{name}_in"]
    patches, scales = list(N[f"{name}_patches"]), list(N[f"{name}_scales"])
    st = nlsar_stats(oracle, patches, scales)
    o = oracle.nlsar_insar(a1, a2, ph, 21, patches, scales, st, select_mode=mode, use_double=False,
                           tile=tuple(int(t) for t in N[f"{name}_tile"]), diag=True)
    ref = N[f"{name}_m{mode}_out"]
    for i in range(3):
        assert np.array_equal(o[i], ref[i], equal_nan=True), (name, mode, i, np.argwhere(o[i] != ref[i])[:5])
    assert np.array_equal(o[3].sel, N[f"{name}_m{mode}_sel"])


@pytest.mark.parametrize("mode", [0, 1])
def test_nlsar_covariance_fp32_oracle_matches_reference_kernels_bit_for_bit(oracle, mode):
    st = nlsar_stats(oracle, [3, 5, 7], [1, 3])
    o = oracle.nlsar_covmat(N["cov_in"], 21, [3, 5, 7], [1, 3], st, select_mode=mode, use_double=False)
    assert np.array_equal(o, N[f"cov_m{mode}_out"], equal_nan=True)


def test_nlsar_reference_fixtures_cover_both_modes_and_the_boundary():
    # both selection modes differ somewhere, and the tiled case's tiles meet
    # inside the scene (70 x 90 with 60 x 60 tiles and overlap 14)
    a = N["s96x96_m0_out"]
    b = N["s96x96_m1_out"]
    assert not np.array_equal(a, b)
    assert len(np.unique(N["s96x96_m1_sel"])) > 1
    assert (N["s96x96_m0_sel"] == N["s96x96_m0_sel"].flat[0]).all()  # the last key everywhere
    assert tuple(N["tiled_tile"]) == (60, 60)
