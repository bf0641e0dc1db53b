"""Host-side logic of the C ABI, without a GPU: the library loads, exports every
entry point its header declares, validates arguments before touching the
device, builds LUTs and reads/writes statistics files like the reference."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import despeckcl_b200 as dcl
from despeckcl_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "despeckcl_b200.h")).read()
    return sorted(set(re.findall(r"\b(dcl_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = dcl.lib()
    names = declared_symbols()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", api._LIBPATH], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(rf"\bT {n}\b", out), n


def _stats_entry(p, s):
    q = np.linspace(0, 1, 256).astype(np.float32)
    c = np.linspace(0, 100, 256).astype(np.float32)
    return dcl.Stats(256, 1.0, 10.0, q, c)


@pytest.mark.parametrize("kw,code", [
    (dict(sws=20), -1),                        # even search window
    (dict(patches=[4]), -1),                   # even patch size
    (dict(scales=[2]), -1),                    # even scale size
    (dict(scales=[11]), -1),                   # scale beyond 9
    (dict(stats_keys=[(3, 1)]), -2),           # (3, 3) missing
    (dict(h=0.0), -1),
])
def test_argument_validation_happens_on_the_host(kw, code):
    sws = kw.get("sws", 21)
    patches = kw.get("patches", [3])
    scales = kw.get("scales", [1, 3])
    keys = kw.get("stats_keys", [(p, s) for p in patches for s in scales])
    stats = {k: _stats_entry(*k) for k in keys}
    a = np.ones((8, 8), np.float32)
    with pytest.raises(dcl.DespeckclError) as e:
        dcl.nlsar_insar(a, a, a, sws, patches, scales, stats, h=kw.get("h", 15.0))
    assert e.value.code == code


@pytest.mark.parametrize("shape", [(0, 8), (8, 0), (0, 0)])
def test_empty_scene_is_rejected_on_the_host(shape):
    stats = {(3, s): _stats_entry(3, s) for s in (1, 3)}
    a = np.ones(shape, np.float32)
    with pytest.raises(dcl.DespeckclError) as e:
        dcl.nlsar_insar(a, a, a, 21, [3], [1, 3], stats)
    assert e.value.code == -1
    for fn, args in ((dcl.boxcar, (5,)), (dcl.goldstein, (32, 4, 0.5)), (dcl.nlinsar, (21, 7, 1, 10))):
        with pytest.raises(dcl.DespeckclError) as e:
            fn(a, a, a, *args)
        assert e.value.code == -1


def test_ragged_inputs_are_rejected():
    stats = {(3, s): _stats_entry(3, s) for s in (1, 3)}
    a, b = np.ones((8, 8), np.float32), np.ones((8, 9), np.float32)
    with pytest.raises((dcl.DespeckclError, ValueError)):
        dcl.nlsar_insar(a, b, a, 21, [3], [1, 3], stats)


@pytest.mark.parametrize("dim", [1, 4])
def test_covariance_dimension_outside_2_and_3_is_rejected(dim):
    # 2x2 and 3x3 covariances are filtered; any other size is an invalid
    # argument, reported before any device work
    cov = np.zeros((dim, dim, 4, 4), np.complex64)
    with pytest.raises(dcl.DespeckclError) as e:
        dcl.nlsar(cov, 21, [3], [1], {(3, 1): _stats_entry(3, 1)})
    assert e.value.code == -1


def test_lut_builder_matches_oracle(oracle):
    rng = np.random.default_rng(11)
    for n, L in [(5000, 256), (10001, 1000), (1234, 256)]:
        d = rng.gamma(2.0, 2.0, n).astype(np.float32)
        mine = dcl.stats_from_dissims(d, L)
        ref = oracle.stats_from_dissims(d, L)
        assert mine.dissims_min == ref.dissims_min and mine.dissims_max == ref.dissims_max
        np.testing.assert_array_equal(mine.quantilles, ref.quantilles)
        np.testing.assert_array_equal(mine.chi2cdf_inv, ref.chi2cdf_inv)


def test_chi2_table_matches_scipy():
    sps = pytest.importorskip("scipy.stats")
    st = dcl.stats_from_dissims(np.arange(100, dtype=np.float32), 256)
    ys = np.arange(255) / 256.0
    np.testing.assert_array_equal(st.chi2cdf_inv[:255], sps.chi2.ppf(ys, 49).astype(np.float32))
    assert st.chi2cdf_inv[255] == 100000


# tests/golden/nlsar_stats_boost.txt: the Boost text archive that the
# reference's store_nlsar_stats_collection (nlsar_training.cpp:99-104) writes
# for a map of two entries, laid out word by word from Boost.Serialization's
# save rules (not produced by Boost, which is absent here):
#   "22 serialization::archive 10"   signature and format version
#   "0 0"                            map: tracking 0, class version 0
#   "2 0"                            two elements, item version 0
#   "0 0" "0 0" "3 1"                pair and params class info, key (3, 1)
#   "0 0" "4 1.5 9.25"               stats class info, lut_size, dissims_min/max
#   "4 0 q0..q3" "4 0 c0..c3"        quantilles and chi2cdf_inv (count, item version)
#   "5 3 4 2 12 4 0 ... 4 0 ..."     second element: no class info any more
# Floats appear as Boost prints them (scientific, 9 digits after the point).
BOOST_GOLDEN = os.path.join(ROOT, "tests", "golden", "nlsar_stats_boost.txt")
BOOST_GOLDEN_STATS = {
    (3, 1): (4, 1.5, 9.25, [0, 0.25, 0.5, 1], [0, 30.5, 45, 100000]),
    (5, 3): (4, 2.0, 12.0, [0, 0.5, 0.75, 1], [0, 30.5, 45, 100000]),
}


def _golden_collection():
    return {k: dcl.Stats(L, lo, hi, np.array(q, np.float32), np.array(c, np.float32))
            for k, (L, lo, hi, q, c) in BOOST_GOLDEN_STATS.items()}


def _check_golden_values(back):
    assert list(back.keys()) == sorted(BOOST_GOLDEN_STATS)
    for k, (L, lo, hi, q, c) in BOOST_GOLDEN_STATS.items():
        assert (back[k].lut_size, back[k].dissims_min, back[k].dissims_max) == (L, lo, hi)
        np.testing.assert_array_equal(back[k].quantilles, q)
        np.testing.assert_array_equal(back[k].chi2cdf_inv, c)


def test_boost_text_archive_golden_read():
    _check_golden_values(dcl.load_nlsar_stats_collection(BOOST_GOLDEN))


def test_boost_text_archive_writer_matches_golden(tmp_path):
    f = tmp_path / "stats.txt"
    dcl.store_nlsar_stats_collection(_golden_collection(), str(f))
    assert f.read_text() == open(BOOST_GOLDEN).read()


def test_boost_text_archive_other_writers(tmp_path):
    # the same map as an older Boost prints it (default float format, another
    # format version) and in format version 3 (no item-version words)
    v17 = ("22 serialization::archive 17 0 0 2 0 0 0 0 0 3 1 0 0 4 1.5 9.25 4 0 0 0.25 0.5 1 4 0 0 30.5 45 100000 "
           "5 3 4 2 12 4 0 0 0.5 0.75 1 4 0 0 30.5 45 100000")
    v3 = ("22 serialization::archive 3 0 0 2 0 0 0 0 3 1 0 0 4 1.5 9.25 4 0 0.25 0.5 1 4 0 30.5 45 100000 "
          "5 3 4 2 12 4 0 0.5 0.75 1 4 0 30.5 45 100000")
    for text in (v17, v3):
        f = tmp_path / "a.txt"
        f.write_text(text + "\n")
        _check_golden_values(dcl.load_nlsar_stats_collection(str(f)))


def test_boost_text_archive_empty_map(tmp_path):
    # an empty map: class info of the map, count 0, item version, nothing else
    f = tmp_path / "empty.txt"
    dcl.store_nlsar_stats_collection({}, str(f))
    assert f.read_text() == "22 serialization::archive 10 0 0 0 0\n"
    assert dict(dcl.load_nlsar_stats_collection(str(f))) == {}


def test_boost_text_archive_malformed(tmp_path):
    words = open(BOOST_GOLDEN).read().split()
    bad = {
        "truncated": words[:-1],
        "trailing word": words + ["7"],
        "tracked map": words[:3] + ["1"] + words[4:],
        "lut_size against the tables": words[:15] + ["5"] + words[16:],
        "not a number": words[:20] + ["x"] + words[21:],
    }
    for name, w in bad.items():
        f = tmp_path / "bad.txt"
        f.write_text(" ".join(w) + "\n")
        with pytest.raises(dcl.DespeckclError, match="Boost text archive"):
            dcl.load_nlsar_stats_collection(str(f))


def test_stats_file_round_trip_both_formats(tmp_path, train_stats):
    coll = {k: dcl.Stats(v.lut_size, v.dissims_min, v.dissims_max, v.quantilles, v.chi2cdf_inv)
            for k, v in train_stats.items()}
    for fmt in ("boost", "native"):
        f = str(tmp_path / f"stats_{fmt}.txt")
        dcl.store_nlsar_stats_collection(coll, f, format=fmt)
        first = open(f).read().split()[:2]
        assert first == (["22", "serialization::archive"] if fmt == "boost" else ["despeckcl_b200-nlsar-stats", "1"])
        back = dcl.load_nlsar_stats_collection(f)
        assert list(back.keys()) == sorted(coll.keys())
        for k in coll:
            a, b = coll[k], back[k]
            assert (a.lut_size, a.dissims_min, a.dissims_max) == (b.lut_size, b.dissims_min, b.dissims_max)
            np.testing.assert_array_equal(a.quantilles, b.quantilles)
            np.testing.assert_array_equal(a.chi2cdf_inv, b.chi2cdf_inv)


def test_cpp_api_compiles_and_links(tmp_path):
    src = tmp_path / "use.cpp"
    src.write_text(r'''
#include "despeckcl.h"
#include <cstdio>
int main() {
  nlsar_stats_collection m;
  std::vector<float> d;
  for (int i = 0; i < 100; ++i) d.push_back((float)i);
  m[nlsar::params{3, 1}] = nlsar::stats(d, 256);
  despeckcl::store_nlsar_stats_collection(m, "s.txt");
  nlsar_stats_collection b = despeckcl::load_nlsar_stats_collection("s.txt");
  std::printf("%zu %u %g\n", b.size(), b[nlsar::params{3, 1}].lut_size, b[nlsar::params{3, 1}].dissims_max);
  return 0;
}
''')
    exe = tmp_path / "use"
    libdir = os.path.dirname(api._LIBPATH)
    subprocess.run(["/usr/bin/g++", "-std=c++17", str(src), "-I", os.path.join(ROOT, "include"), "-L", libdir,
                    "-ldespeckcl_b200", "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], cwd=tmp_path, capture_output=True, text=True, check=True).stdout
    assert out.split() == ["1", "256", "99"]


def test_stage_timeout_ledger_fails_loudly_without_a_device():
    # dcl_take_stage_timeouts: a null count is an argument error; without a
    # CUDA device the ledger cannot be read and the call says so (count 0)
    L = dcl.lib()
    assert L.dcl_take_stage_timeouts(None) == -1
    n = ctypes.c_int(7)
    rc = L.dcl_take_stage_timeouts(ctypes.byref(n))
    if rc == 0:
        pytest.skip("a CUDA device is present")
    assert rc == -4 and n.value == 0
    assert "CUDA" in L.dcl_last_error().decode() or "device" in L.dcl_last_error().decode()
    with pytest.raises(dcl.DespeckclError):
        dcl.take_stage_timeouts()
