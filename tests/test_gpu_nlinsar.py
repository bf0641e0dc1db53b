"""The GPU NL-InSAR filter against the oracle (pinned bit for bit to the
reference's code in test_nlinsar_oracle.py).

NL-InSAR is not Lipschitz in its inputs: a pixel whose number of looks sits at
lmin, or whose lmin-th and next weights are close, switches its smoothing on a
last-bit change, and later passes spread such switches.  FP32 and FP64 runs of
the oracle itself differ at about 1% of the pixels after one pass and at a
third of them after five.  So: one pass at a time from the same estimates, at
least 99% of the pixels within 1e-4 (reflectivity, coherence) / 1e-3 rad
(phase) of the FP32 oracle; over five passes the GPU must stay as close to the
FP64 oracle as the FP32 oracle does (median error and the fraction of pixels
within 1e-3).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import despeckcl_b200 as dcl  # noqa: E402
from despeckcl_b200 import synthetic  # noqa: E402


def wrapped(d):
    return np.abs(np.angle(np.exp(1j * d)))


def _ok(got, want):
    r = np.abs(got[0] - want[0]) <= 1e-4 * np.abs(want[0])
    p = wrapped(got[1] - want[1]) <= 1e-3
    c = np.abs(got[2] - want[2]) <= 1e-4 * np.maximum(np.abs(want[2]), 1e-3)
    return r & p & c


def _gpu(a1, a2, ph, niter, lmin, init=None):
    t = [torch.from_numpy(x).cuda() for x in (a1, a2, ph)]
    est = None if init is None else tuple(torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in init)
    out = dcl.nlinsar_device(*t, 21, 7, niter, lmin, estimates=est)
    torch.cuda.synchronize()
    return [o.cpu().numpy() for o in out]


@pytest.mark.parametrize("shape,seed", [((90, 90), 1), ((128, 75), 2), ((54, 54), 3), ((20, 33), 4)])
def test_first_pass_matches_oracle(oracle, shape, seed):
    a1, a2, ph = synthetic.insar_scene(*shape, seed)
    got = _gpu(a1, a2, ph, 1, 10)
    want = oracle.nlinsar(a1, a2, ph, 21, 7, 1, 10, use_double=False)
    ok = _ok(got, want)
    print("first pass: fraction within tolerance", ok.mean())
    assert ok.mean() >= 0.99


def test_one_pass_from_estimates_matches_oracle(oracle):
    a1, a2, ph = synthetic.insar_scene(100, 110, 5)
    init = oracle.nlinsar(a1, a2, ph, 21, 7, 2, 10, use_double=True)
    got = _gpu(a1, a2, ph, 1, 10, init=init)
    want = oracle.nlinsar(a1, a2, ph, 21, 7, 1, 10, use_double=False, init=init)
    ok = _ok(got, want)
    print("pass from estimates: fraction within tolerance", ok.mean())
    assert ok.mean() >= 0.99


def test_five_passes_as_close_to_fp64_as_the_fp32_oracle(oracle):
    a1, a2, ph = synthetic.insar_scene(120, 120, 8)
    got = _gpu(a1, a2, ph, 5, 10)
    d = oracle.nlinsar(a1, a2, ph, 21, 7, 5, 10, use_double=True)
    f = oracle.nlinsar(a1, a2, ph, 21, 7, 5, 10, use_double=False)
    eg = np.abs(got[0] - d[0]) / np.abs(d[0])
    ef = np.abs(f[0] - d[0]) / np.abs(d[0])
    print("five passes: median", np.median(eg), np.median(ef), "within 1e-3", (eg < 1e-3).mean(), (ef < 1e-3).mean())
    assert np.median(eg) <= max(3 * np.median(ef), 1e-5)
    assert (eg < 1e-3).mean() >= (ef < 1e-3).mean() - 0.05


def test_host_entry_point_equals_device_entry_point():
    a1, a2, ph = synthetic.insar_scene(70, 80, 9)
    host = dcl.nlinsar(a1, a2, ph, 21, 7, 2, 10)
    dev = _gpu(a1, a2, ph, 2, 10)
    for h, d in zip(host, dev):
        assert np.array_equal(h, d)
