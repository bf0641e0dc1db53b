"""The GPU Goldstein filter against the FP64 oracle (itself pinned to the
reference's kernels in test_goldstein_oracle.py).

Tolerance: the FFTs run in FP32 (as clFFT does in the reference), so the
amplitude is compared relative to max(|oracle|, 5% of the scene's mean
amplitude) at 1e-4 and the phase at 1e-3 rad where the amplitude is above 5%
of the mean (below that the phase of a near-zero sum is not defined to FP32
accuracy).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import despeckcl_b200 as dcl  # noqa: E402
from despeckcl_b200 import synthetic  # noqa: E402


def wrapped(d):
    return np.abs(np.angle(np.exp(1j * d)))


def _check(ref, ph, rd, pd):
    scale = np.abs(rd).mean()
    err = np.abs(ref - rd) / np.maximum(np.abs(rd), 0.05 * scale)
    assert err.max() <= 1e-4, err.max()
    strong = rd > 0.05 * scale
    assert wrapped(ph - pd)[strong].max() <= 1e-3


@pytest.mark.parametrize("shape,ov,alpha", [((48, 48), 4, 0.5), ((100, 73), 4, 0.5), ((257, 300), 4, 0.5),
                                            ((61, 40), 4, 0.5), ((85, 85), 4, 0.5), ((64, 200), 7, 0.3),
                                            ((90, 130), 2, 0.8), ((512, 512), 4, 0.5), ((37, 19), 4, 0.5),
                                            ((10, 12), 4, 0.5)])
def test_goldstein_matches_fp64_oracle(oracle, shape, ov, alpha):
    a1, a2, phi = synthetic.insar_scene(*shape, 21)
    ref, ph, coh = dcl.goldstein(a1, a2, phi, 32, ov, alpha)
    rd, pd = oracle.goldstein(a1, a2, phi, 32, ov, alpha, True)
    _check(ref, ph, rd, pd)
    assert (coh == 0).all()


def test_alpha_zero_is_raw_plus_raw():
    a1, a2, phi = synthetic.insar_scene(200, 150, 4)
    ref, ph, _ = dcl.goldstein(a1, a2, phi, 32, 4, 0.0)
    np.testing.assert_allclose(ref, a1 + a2, rtol=2e-6, atol=1e-6)
    assert wrapped(ph - phi).max() < 1e-5


def test_constant_interferogram_closed_form():
    a1 = np.full((77, 91), 1.3, np.float32)
    a2 = np.full((77, 91), 0.7, np.float32)
    phi = np.full((77, 91), -2.0, np.float32)
    ref, ph, _ = dcl.goldstein(a1, a2, phi, 32, 4, 0.5)
    np.testing.assert_allclose(ref, 1.0 * (1 + 1024 ** 0.5), rtol=1e-5)
    assert wrapped(ph + 2.0).max() < 1e-5


def test_device_entry_point_equals_host_entry_point():
    a1, a2, phi = synthetic.insar_scene(300, 333, 8)
    ref, ph, _ = dcl.goldstein(a1, a2, phi, 32, 4, 0.5)
    t = [torch.from_numpy(x).cuda() for x in (a1, a2, phi)]
    out = dcl.goldstein_device(*t, 32, 4, 0.5)
    torch.cuda.synchronize()
    assert np.array_equal(out[0].cpu().numpy(), ref)
    assert np.array_equal(out[1].cpu().numpy(), ph)


FUSED_VS_TWO_PASS = r'''
import os, sys
import numpy as np
sys.path.insert(0, os.environ["DCL_ROOT"])
import despeckcl_b200 as dcl
from despeckcl_b200 import synthetic
out = []
for (H, W, ov, alpha, seed) in [(48, 48, 4, 0.5, 1), (100, 73, 4, 0.5, 2), (257, 300, 4, 0.5, 3), (64, 200, 7, 0.3, 4),
                                (90, 130, 2, 0.8, 5), (700, 100, 4, 0.5, 6), (1, 1, 4, 0.5, 7), (5, 3, 0, 0.5, 8),
                                (33, 500, 5, 0.0, 9), (1000, 1000, 4, 0.5, 10), (61, 40, 4, 0.5, 11),
                                (85, 85, 4, 0.5, 12), (997, 997, 4, 0.5, 13), (37, 19, 4, 0.5, 14)]:
    a1, a2, ph = synthetic.insar_scene(H, W, seed)
    r, p, _ = dcl.goldstein(a1, a2, ph, 32, ov, alpha)
    out += [r, p]
np.savez(os.environ["DCL_OUT"], *out)
'''


def test_fused_kernel_equals_two_pass_path_bit_for_bit(tmp_path):
    # the fused kernel (DESPECKCL_B200_GOLDSTEIN_FUSED=1, patches kept in
    # shared memory) and the default two-kernel path (patches through HBM) run
    # the same FFT, weighting and parity-ordered overlap-add, so they agree
    # exactly; scenes include non-square ones, ones whose last row or column
    # comes from a second reference tile (61 x 40, 85 x 85, 997 x 997, 37 x 19),
    # overlaps 0..7 and alpha 0
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = []
    for name, fused in (("fused", "1"), ("two", "0")):
        env = dict(os.environ, DCL_ROOT=root, DCL_OUT=str(tmp_path / f"{name}.npz"),
                   DESPECKCL_B200_GOLDSTEIN_FUSED=fused)
        r = subprocess.run([sys.executable, "-c", FUSED_VS_TWO_PASS], env=env, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr[-3000:]
        z = np.load(tmp_path / f"{name}.npz")
        res.append([z[k] for k in sorted(z.files, key=lambda s: int(s.split("_")[1]))])
    for a, b in zip(*res):
        assert np.array_equal(a, b, equal_nan=True)
