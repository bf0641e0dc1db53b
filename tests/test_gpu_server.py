"""The NL-SAR request server (dcl_server_*) against one-scene calls.

A served request is filtered tile by tile in launches shared with other
requests (a large scene split over several launches, small ones joining
them), but every tile is computed from the scene's own frame and descriptor,
so the result must equal dcl_nlsar_insar_device on the same scene bit for bit,
whatever it was batched with.  Admission must keep the admitted memory within
the budget and refuse a scene that can never fit.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import despeckcl_b200 as dcl  # noqa: E402
from despeckcl_b200 import synthetic  # noqa: E402

SWS, PATCHES, SCALES = 21, [3, 5, 7], [1, 3]
SIZES = [(300, 280), (96, 700), (640, 512), (50, 60), (1100, 200), (257, 255)]


@pytest.fixture(scope="module")
def stats():
    t1, t2, tp = synthetic.training_area(64, seed=7)
    return dcl.nlsar_train_insar(t1, t2, tp, PATCHES, SCALES)


@pytest.fixture(scope="module")
def scenes():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return [tuple(torch.from_numpy(x).cuda() for x in synthetic.insar_scene(h, w, 500 + i))
            for i, (h, w) in enumerate(SIZES)]


@pytest.fixture(scope="module")
def alone(scenes, stats):
    out = [dcl.nlsar_insar_device(*s, SWS, PATCHES, SCALES, stats, select_mode="argmax_enl") for s in scenes]
    torch.cuda.synchronize()
    return [tuple(o.cpu().numpy() for o in r) for r in out]


def _equal(got, want):
    for g, w in zip(got, want):
        g = g.cpu().numpy() if hasattr(g, "cpu") else g
        assert np.array_equal(g, w, equal_nan=True)


@pytest.mark.parametrize("max_batch_tiles,max_inflight", [(64, 2), (37, 3), (100000, 1)])
def test_served_results_equal_alone(scenes, stats, alone, max_batch_tiles, max_inflight):
    srv = dcl.NlsarServer(SWS, PATCHES, SCALES, stats, hbm_budget_bytes=2 << 30, max_inflight=max_inflight,
                          max_batch_tiles=max_batch_tiles)
    try:
        ids = [srv.submit(*s) for s in scenes]
        infos = []
        for rid, want in zip(ids, alone):
            out, info = srv.wait(rid, timeout=120)
            _equal(out, want)
            infos.append(info)
        st = srv.stats()
        assert st["completed"] == len(scenes) and st["failed"] == 0
        assert st["admitted_bytes"] == 0
        if max_batch_tiles < 1000:
            # the large scenes were split, and some launch held more than one request
            assert max(i["chunks"] for i in infos) > 1
            spans = [(i["first_batch"], i["last_batch"]) for i in infos]
            assert any(a[1] >= b[0] and b[1] >= a[0] for k, a in enumerate(spans) for b in spans[k + 1:])
        for i in infos:
            assert i["submit_s"] <= i["admit_s"] <= i["launch_s"] <= i["done_s"]
    finally:
        srv.close()


def test_admission_keeps_within_budget(scenes, stats, alone):
    # a budget that holds the largest request's frame with little to spare:
    # requests are admitted as earlier ones free their memory
    srv0 = dcl.NlsarServer(SWS, PATCHES, SCALES, stats, hbm_budget_bytes=2 << 30)
    rid = srv0.submit(*scenes[2])
    srv0.wait(rid, timeout=120)
    need = srv0.stats()["peak_admitted_bytes"]
    srv0.close()
    budget = int(need * 1.3)
    srv = dcl.NlsarServer(SWS, PATCHES, SCALES, stats, hbm_budget_bytes=budget, max_inflight=2, max_batch_tiles=50)
    try:
        ids = [srv.submit(*s) for s in scenes]
        for rid, want in zip(ids, alone):
            out, _ = srv.wait(rid, timeout=120)
            _equal(out, want)
        st = srv.stats()
        assert 0 < st["peak_admitted_bytes"] <= budget
        assert st["completed"] == len(scenes)
    finally:
        srv.close()


def test_host_buffers_equal_host_entry_point(stats):
    a = synthetic.insar_scene(333, 222, 77)
    want = dcl.nlsar_insar(*a, SWS, PATCHES, SCALES, stats, select_mode="argmax_enl")
    srv = dcl.NlsarServer(SWS, PATCHES, SCALES, stats, hbm_budget_bytes=1 << 30, max_batch_tiles=30)
    try:
        out, info = srv.wait(srv.submit(*a), timeout=120)
        assert info["chunks"] > 1
        _equal(out, [np.asarray(w) for w in want])
    finally:
        srv.close()


def test_request_larger_than_budget_is_refused(scenes, stats):
    srv = dcl.NlsarServer(SWS, PATCHES, SCALES, stats, hbm_budget_bytes=1 << 20)
    try:
        with pytest.raises(dcl.DespeckclError) as e:
            srv.submit(*scenes[2])
        assert e.value.code == -3
        # a scene that fits is still served
        out, _ = srv.wait(srv.submit(*scenes[3]), timeout=120)
        assert torch.isfinite(out[0]).all()
    finally:
        srv.close()
