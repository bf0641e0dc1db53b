"""Reporting of staging timeouts (the bounded TMA staging wait running out).

The specialised NL-SAR kernel waits for its TMA staging copies with a bounded
wait; a thread block whose wait runs out leaves its tiles unwritten and is
counted.  DESPECKCL_B200_TEST_WITHHOLD_STAGING=1 makes every staging wait run
out without any fault: the kernel arms its barrier for the copies' bytes but
issues no copy (so nothing is left in flight), with a short poll limit.  In a
child process with that switch:
  * the host-pointer entry point returns DCL_ERR_TIMEOUT with its message;
  * the device entry point returns DCL_OK (its work is queued) and the
    device's ledger, read after synchronising, counts the thread blocks;
  * the request server fails the request with DCL_ERR_TIMEOUT;
  * with the switch cleared, the same process filters the scene again and the
    result equals a clean process's: the context stays usable.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import os, sys, json
import numpy as np
import torch
sys.path.insert(0, os.environ["DCL_ROOT"])
import despeckcl_b200 as dcl
from despeckcl_b200 import synthetic
t1, t2, tp = synthetic.training_area(64, seed=7)
stats = dcl.nlsar_train_insar(t1, t2, tp, [3, 5, 7], [1, 3])
a1, a2, ph = synthetic.insar_scene(64, 96, 5)
res = {}
os.environ["DESPECKCL_B200_TEST_WITHHOLD_STAGING"] = "1"
dcl.take_stage_timeouts()  # start from an empty ledger
try:
    dcl.nlsar_insar(a1, a2, ph, 21, [3, 5, 7], [1, 3], stats, select_mode="argmax_enl")
    res["host"] = [0, ""]
except dcl.DespeckclError as e:
    res["host"] = [e.code, str(e)]
res["ledger_after_host"] = dcl.take_stage_timeouts()
dev = [torch.from_numpy(x).cuda() for x in (a1, a2, ph)]
dcl.nlsar_insar_device(*dev, 21, [3, 5, 7], [1, 3], stats, select_mode="argmax_enl")
torch.cuda.synchronize()
res["ledger_after_device"] = dcl.take_stage_timeouts()
res["ledger_after_take"] = dcl.take_stage_timeouts()
srv = dcl.NlsarServer(21, [3, 5, 7], [1, 3], stats, hbm_budget_bytes=1 << 30, select_mode="argmax_enl")
rid = srv.submit(a1, a2, ph)
try:
    srv.wait(rid)
    res["server_status"] = 0
except dcl.DespeckclError as e:
    res["server_status"] = e.code
srv.close()
dcl.take_stage_timeouts()
os.environ["DESPECKCL_B200_TEST_WITHHOLD_STAGING"] = "0"
out = dcl.nlsar_insar(a1, a2, ph, 21, [3, 5, 7], [1, 3], stats, select_mode="argmax_enl")
np.save(os.environ["DCL_OUT"], np.stack(out))
res["ledger_after_clean"] = dcl.take_stage_timeouts()
print("RESULT " + json.dumps(res))
'''


def run_child(tmp_path, code, name):
    env = dict(os.environ, DCL_ROOT=ROOT, DCL_OUT=str(tmp_path / f"{name}.npy"))
    env.pop("DESPECKCL_B200_TEST_WITHHOLD_STAGING", None)
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return r.stdout


def test_staging_timeouts_are_reported_and_the_context_stays_usable(tmp_path):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import json

    out = run_child(tmp_path, CHILD, "after")
    res = json.loads([ln for ln in out.splitlines() if ln.startswith("RESULT ")][-1][7:])
    code, msg = res["host"]
    assert code == -6 and "gave up waiting" in msg, res["host"]
    # the ledger counts every launch's thread blocks that gave up, the host
    # call's included (it reported them itself as well)
    assert res["ledger_after_host"] > 0
    assert res["ledger_after_device"] > 0
    assert res["ledger_after_take"] == 0
    assert res["server_status"] == -6
    assert res["ledger_after_clean"] == 0
    # a clean process filters the same scene to the same bits
    clean = CHILD.replace('os.environ["DESPECKCL_B200_TEST_WITHHOLD_STAGING"] = "1"',
                          'os.environ["DESPECKCL_B200_TEST_WITHHOLD_STAGING"] = "0"')
    clean = clean[:clean.index("res = {}")] + (
        'out = dcl.nlsar_insar(a1, a2, ph, 21, [3, 5, 7], [1, 3], stats, select_mode="argmax_enl")\n'
        'np.save(os.environ["DCL_OUT"], np.stack(out))\n')
    run_child(tmp_path, clean, "clean")
    a = np.load(tmp_path / "after.npy")
    b = np.load(tmp_path / "clean.npy")
    assert np.array_equal(a, b, equal_nan=True)
