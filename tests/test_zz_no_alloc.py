"""The allocation-free NL-SAR entry point against the allocating one.

dcl_nlsar_insar_device_noalloc serves callers that cannot allocate GPU memory
while they filter: its scratch is a static device array of this library.  Two
calls in a row on scenes of different sizes must reproduce
dcl_nlsar_insar_device bit for bit (the same kernels on the same data), and
a scene larger than the array must be refused before any device work.  This
file is collected last so that a failure here stops a run only after every
other test has run.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import despeckcl_b200 as dcl  # noqa: E402
from despeckcl_b200 import api, synthetic  # noqa: E402

SWS, PATCHES, SCALES = 21, [3, 5, 7], [1, 3]


def _stats():
    t1, t2, tp = synthetic.training_area(64, seed=7)
    return dcl.nlsar_train_insar(t1, t2, tp, PATCHES, SCALES)


def _call(fn, tensors, out, sel, stats, mode):
    H, W = tensors[0].shape
    pk, pp, npn = api._ints(PATCHES)
    sk, sp, nsn = api._ints(SCALES)
    arr, n, keep = api._entries(stats)
    p = [ctypes.c_void_p(t.data_ptr()) for t in list(tensors) + list(out)]
    rc = fn(*p, H, W, SWS, pp, npn, sp, nsn, arr, n, ctypes.c_float(15.0), ctypes.c_float(49.0),
            api.SELECT_MODES[mode], ctypes.c_void_p(sel.data_ptr()),
            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return rc


def test_noalloc_matches_allocating_entry_point_twice():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = dcl.lib()
    stats = _stats()
    for (H, W, seed, mode) in [(200, 300, 41, "argmax_enl"), (96, 128, 42, "reference")]:
        a = [torch.from_numpy(x).cuda() for x in synthetic.insar_scene(H, W, seed)]
        out_n = [torch.full((H, W), float("nan"), device="cuda") for _ in range(3)]
        out_r = [torch.empty((H, W), device="cuda") for _ in range(3)]
        sel_n = torch.full((H, W), -7, dtype=torch.int32, device="cuda")
        sel_r = torch.empty((H, W), dtype=torch.int32, device="cuda")
        assert _call(L.dcl_nlsar_insar_device_noalloc, a, out_n, sel_n, stats, mode) == 0, \
            L.dcl_last_error().decode()
        assert _call(L.dcl_nlsar_insar_device, a, out_r, sel_r, stats, mode) == 0, L.dcl_last_error().decode()
        torch.cuda.synchronize()
        n = [o.cpu().numpy() for o in out_n]
        r = [o.cpu().numpy() for o in out_r]
        for i in range(3):
            assert np.array_equal(n[i], r[i], equal_nan=True), i
        assert np.array_equal(sel_n.cpu().numpy(), sel_r.cpu().numpy())


def test_noalloc_refuses_scenes_beyond_its_scratch():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = dcl.lib()
    stats = _stats()
    H = W = 2048
    a = [torch.zeros((H, W), device="cuda") for _ in range(3)]
    out = [torch.zeros((H, W), device="cuda") for _ in range(3)]
    sel = torch.zeros((H, W), dtype=torch.int32, device="cuda")
    rc = _call(L.dcl_nlsar_insar_device_noalloc, a, out, sel, stats, "argmax_enl")
    assert rc == -1
    assert "allocation-free entry point holds" in L.dcl_last_error().decode()
    torch.cuda.synchronize()
    assert float(out[0].abs().max()) == 0.0
