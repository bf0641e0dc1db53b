"""The drop-in C++ API (include/despeckcl.h) executed on the GPU.

A C++ program compiled against include/despeckcl.h and linked with the
library trains NL-SAR statistics with despeckcl::nlsar_training, stores them
with despeckcl::store_nlsar_stats_collection, and filters host buffers with
despeckcl::nlsar (InSAR input and the covariance overload, both selection
modes through DESPECKCL_B200_SELECT), despeckcl::boxcar, despeckcl::goldstein
and despeckcl::nlinsar, the way a caller of the reference's despeckcl.h would
(include/despeckcl.h:30-123 of the reference).  Every output must equal the C
ABI's (dcl_nlsar_insar, dcl_nlsar_covmat, dcl_boxcar, dcl_goldstein,
dcl_nlinsar, reached through despeckcl_b200.api) bit for bit, and the
statistics it stored must load back equal to the C ABI's training.
"""
import os
import subprocess

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import despeckcl_b200 as dcl  # noqa: E402
from despeckcl_b200 import api, synthetic  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
H, W = 72, 88

PROGRAM = r'''
#include "despeckcl.h"
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

static std::vector<float> load(const std::string& f, size_t n) {
  std::vector<float> v(n);
  FILE* fp = std::fopen(f.c_str(), "rb");
  if (!fp || std::fread(v.data(), sizeof(float), n, fp) != n) { std::fprintf(stderr, "read %s\n", f.c_str()); std::exit(2); }
  std::fclose(fp);
  return v;
}
static void save(const std::string& f, const float* p, size_t n) {
  FILE* fp = std::fopen(f.c_str(), "wb");
  std::fwrite(p, sizeof(float), n, fp);
  std::fclose(fp);
}

int main(int argc, char** argv) {
  const int H = std::stoi(argv[1]), W = std::stoi(argv[2]), T = std::stoi(argv[3]);
  const std::string mode = argv[4];
  const size_t n = (size_t)H * W, nt = (size_t)T * T;
  std::vector<std::string> logs{"error"};
  std::vector<float> t1 = load("t1.bin", nt), t2 = load("t2.bin", nt), tp = load("tp.bin", nt);
  std::vector<float> a1 = load("a1.bin", n), a2 = load("a2.bin", n), ph = load("ph.bin", n);
  std::vector<float> cov = load("cov.bin", 8 * n);
  nlsar_stats_collection st = despeckcl::nlsar_training(t1.data(), t2.data(), tp.data(), T, T, {3, 5, 7}, {1, 3}, logs);
  despeckcl::store_nlsar_stats_collection(st, "stats.txt");
  std::vector<float> ref(n), phf(n), coh(n), cf(8 * n);
  if (despeckcl::nlsar(a1.data(), a2.data(), ph.data(), ref.data(), phf.data(), coh.data(), H, W, 21, {3, 5, 7},
                       {1, 3}, st, 15.0f, 49.0f, logs) != 0) return 3;
  save("nlsar_" + mode + ".bin", ref.data(), n);
  save("nlsar_" + mode + ".bin.1", phf.data(), n);
  save("nlsar_" + mode + ".bin.2", coh.data(), n);
  if (despeckcl::nlsar(cov.data(), cf.data(), H, W, 2, 21, {3, 5, 7}, {1, 3}, st, 15.0f, 49.0f, logs) != 0) return 4;
  save("cov_" + mode + ".bin", cf.data(), 8 * n);
  if (mode == "reference") {
    if (despeckcl::boxcar(a1.data(), a2.data(), ph.data(), ref.data(), phf.data(), coh.data(), H, W, 7, logs)) return 5;
    save("boxcar.bin", ref.data(), n); save("boxcar.bin.1", phf.data(), n); save("boxcar.bin.2", coh.data(), n);
    std::vector<float> z(n, 0.0f);
    ref = z; phf = z; coh = z;
    if (despeckcl::goldstein(a1.data(), a2.data(), ph.data(), ref.data(), phf.data(), coh.data(), (unsigned)H,
                             (unsigned)W, 32u, 4u, 0.5f, logs)) return 6;
    save("gold.bin", ref.data(), n); save("gold.bin.1", phf.data(), n); save("gold.bin.2", coh.data(), n);
    ref = z; phf = z; coh = z;
    if (despeckcl::nlinsar(a1.data(), a2.data(), ph.data(), ref.data(), phf.data(), coh.data(), H, W, 21, 7, 2, 10,
                           logs)) return 7;
    save("nlinsar.bin", ref.data(), n); save("nlinsar.bin.1", phf.data(), n); save("nlinsar.bin.2", coh.data(), n);
  }
  std::printf("ok\n");
  return 0;
}
'''


def _read(path, shape):
    return np.fromfile(path, np.float32).reshape(shape)


def _planes(d, name):
    return [_read(d / (name + s), (H, W)) for s in ("", ".1", ".2")]


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    d = tmp_path_factory.mktemp("cpp_api")
    (d / "use.cpp").write_text(PROGRAM)
    libdir = os.path.dirname(api._LIBPATH)
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O1", str(d / "use.cpp"), "-I", os.path.join(ROOT, "include"),
                    "-L", libdir, "-ldespeckcl_b200", "-Wl,-rpath," + libdir, "-o", str(d / "use")], check=True)
    t = synthetic.training_area(64, seed=7)
    s = synthetic.insar_scene(H, W, 21)
    for name, x in zip(("t1", "t2", "tp", "a1", "a2", "ph"), t + s):
        np.ascontiguousarray(x, np.float32).tofile(d / f"{name}.bin")
    cov = covariance(*s)
    cov.tofile(d / "cov.bin")
    for mode in ("reference", "argmax_enl"):
        env = dict(os.environ, DESPECKCL_B200_SELECT=mode)
        r = subprocess.run([str(d / "use"), str(H), str(W), "64", mode], cwd=d, env=env, capture_output=True,
                           text=True)
        assert r.returncode == 0 and r.stdout.strip() == "ok", (r.returncode, r.stdout, r.stderr)
    return d, t, s, cov


def covariance(a1, a2, ph):
    """A 2x2 covariance image [8][H][W] with all planes carrying data."""
    z2 = a2.astype(np.float64) * np.exp(-1j * ph.astype(np.float64))
    c01 = a1 * z2
    rng = np.random.default_rng(3)
    return np.stack([a1 * a1, rng.normal(0, 0.05, a1.shape), c01.real, c01.imag, 1.01 * c01.real, -c01.imag, a2 * a2,
                     rng.normal(0, 0.05, a1.shape)]).astype(np.float32)


def test_cpp_training_and_stored_stats_equal_the_c_abi(program):
    d, t, s, cov = program
    st_c = dcl.nlsar_train_insar(*t, [3, 5, 7], [1, 3])
    st_cpp = dcl.load_nlsar_stats_collection(str(d / "stats.txt"))
    assert sorted(st_cpp.keys()) == sorted(st_c.keys())
    for k in st_c:
        a, b = st_c[k], st_cpp[k]
        assert a.lut_size == b.lut_size and a.dissims_min == b.dissims_min and a.dissims_max == b.dissims_max
        np.testing.assert_array_equal(np.float32(a.quantilles), np.float32(b.quantilles))
        np.testing.assert_array_equal(np.float32(a.chi2cdf_inv), np.float32(b.chi2cdf_inv))


@pytest.mark.parametrize("mode", ["reference", "argmax_enl"])
def test_cpp_nlsar_equals_c_abi_bit_for_bit(program, mode):
    d, t, s, cov = program
    st = dcl.load_nlsar_stats_collection(str(d / "stats.txt"))
    want = dcl.nlsar_insar(*s, 21, [3, 5, 7], [1, 3], st, select_mode=mode)
    got = _planes(d, f"nlsar_{mode}.bin")
    for g, w in zip(got, want):
        assert np.array_equal(g, w, equal_nan=True)
    cplx = (cov[0::2] + 1j * cov[1::2]).reshape(2, 2, H, W)
    wc = dcl.nlsar(cplx, 21, [3, 5, 7], [1, 3], st, select_mode=mode)
    wi = np.empty_like(cov)
    wi[0::2] = wc.real.reshape(4, H, W)
    wi[1::2] = wc.imag.reshape(4, H, W)
    assert np.array_equal(_read(d / f"cov_{mode}.bin", (8, H, W)), wi, equal_nan=True)


def test_cpp_secondary_filters_equal_c_abi_bit_for_bit(program):
    d, t, s, cov = program
    for name, want in (("boxcar", dcl.boxcar(*s, 7)), ("gold", dcl.goldstein(*s, 32, 4, 0.5)),
                       ("nlinsar", dcl.nlinsar(*s, 21, 7, 2, 10))):
        got = _planes(d, f"{name}.bin")
        for g, w in zip(got, want):
            assert np.array_equal(g, w, equal_nan=True), name
