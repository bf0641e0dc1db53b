"""The CUDA NL-SAR path against the reference's own kernels.

tests/golden/reference_nlsar.npz holds end-to-end outputs of the reference's
NL-SAR OpenCL kernels, compiled as C++ and driven the way its host code drives
them (oracle/nlsar_ref_shim.cpp, written by tests/golden/make_golden.py), on
seeded scenes in both selection modes, together with the statistics they
used.  The CUDA path must meet the tolerance of tests/test_gpu_nlsar.py
against those outputs: reflectivity and coherence within 1e-4 relative, phase
within 1e-3 rad on every well-conditioned pixel (conditioning from the FP64
oracle), 99 % of all pixels; and the per-pixel (patch, scale) selection must
agree wherever the ENL margin and every LUT bin margin are clear.
"""
import numpy as np
import pytest

from nlsar_parity import REF_NLSAR as N
from nlsar_parity import check_parity, nlsar_cases, nlsar_stats, run_gpu

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import despeckcl_b200 as dcl  # noqa: E402

MODES = {0: "reference", 1: "argmax_enl"}


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()


@pytest.mark.parametrize("name,mode", list(nlsar_cases()))
def test_cuda_path_matches_reference_kernels(oracle, name, mode):
    a1, a2, ph = N[f"{name}_in"]
    patches = [int(p) for p in N[f"{name}_patches"]]
    scales = [int(s) for s in N[f"{name}_scales"]]
    tile = tuple(int(t) for t in N[f"{name}_tile"])
    st = nlsar_stats(oracle, patches, scales)
    ref = N[f"{name}_m{mode}_out"]
    diag = oracle.nlsar_insar(a1, a2, ph, 21, patches, scales, st, select_mode=mode, use_double=True, tile=tile,
                              diag=True)[3]
    g = run_gpu(a1, a2, ph, st, MODES[mode], patches=patches, scales=scales, selection=True)
    check_parity(g, tuple(ref), diag, MODES[mode])
    sel_ref = N[f"{name}_m{mode}_sel"]
    if mode == 1:
        clear = (diag.enl_margin > 1e-4) & (diag.var_cond > 1e-4) & (diag.bin_margin_all > 1e-3)
    else:
        clear = np.ones(sel_ref.shape, bool)
    assert np.array_equal(g[3][clear], sel_ref[clear])
    assert (g[3] == sel_ref).mean() >= 0.995


@pytest.mark.parametrize("mode", [0, 1])
def test_cuda_covariance_path_matches_reference_kernels(oracle, mode):
    # the covariance overload (nlsar.cpp:171-194): 8 planes in and out.  Each
    # element is held to 1e-4 relative to its own magnitude, or to 1e-4 of the
    # pixel's diagonal where the element is much smaller than the diagonal
    # (an imaginary diagonal of noise, a near-zero off-diagonal): FP32 rounding
    # of a weighted sum scales with the magnitudes summed, not with the result.
    cov = N["cov_in"]
    st = nlsar_stats(oracle, [3, 5, 7], [1, 3])
    ref = N[f"cov_m{mode}_out"]
    H, W = cov.shape[1:]
    cplx = (cov[0::2] + 1j * cov[1::2]).reshape(2, 2, H, W)
    g = dcl.nlsar(cplx, 21, [3, 5, 7], [1, 3], st, select_mode=MODES[mode])
    gi = np.empty_like(ref)
    gi[0::2] = g.real.reshape(4, H, W)
    gi[1::2] = g.imag.reshape(4, H, W)
    diag_mag = np.maximum(np.abs(ref[0]), np.abs(ref[6]))
    scale = np.maximum(np.abs(ref), 1e-2 * diag_mag[None])
    assert (scale > 0).all()
    err = np.abs(gi - ref) / scale
    assert np.isfinite(err).all()
    assert (err <= 1e-4).mean() >= 0.99, err.max()
