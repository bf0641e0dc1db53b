"""Writes the golden fixtures: outputs of the reference's own code, compiled
from the reference sources by oracle/Makefile into oracle/_ref/libref_pieces.so
(the translation units that build without OpenCL, GSL or Boost, and the
NL-SAR, Goldstein and NL-InSAR kernels compiled as C++).

    make -C oracle && python tests/golden/make_golden.py

tests/golden/reference_pieces.npz: pixel similarities (2x2 and 3x3,
sim_measures.h), the tile iterator (tile_iterator.cpp), the selection of
best_params.cpp, and the Goldstein and NL-InSAR outputs of the reference's
kernels on two small seeded scenes.

tests/golden/reference_nlsar.npz: end-to-end NL-SAR outputs of the
reference's kernels (oracle/nlsar_ref_shim.cpp) on seeded scenes, both
selection modes, with the statistics (LUTs) they used.

The fixtures let tests/test_golden.py pin the oracle, and
tests/test_gpu_reference_nlsar.py the CUDA path, without the reference tree.
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from despeckcl_b200 import synthetic  # noqa: E402
from oracle import pyoracle  # noqa: E402


def herm3(rng):
    z = rng.normal(size=(3, 4)) + 1j * rng.normal(size=(3, 4))
    m = z @ z.conj().T / 4
    return np.float32([m[0, 0].real, m[1, 1].real, m[2, 2].real, m[0, 1].real, m[0, 1].imag, m[0, 2].real,
                       m[0, 2].imag, m[1, 2].real, m[1, 2].imag])


def main():
    R = pyoracle.ref_pieces()
    if R is None:
        raise SystemExit("oracle/_ref/libref_pieces.so not built: run `make -C oracle` with the reference tree present")
    fp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))  # noqa: E731
    out = {}
    rng = np.random.default_rng(2026)
    # 2x2 pixel similarities: Hermitian PD pairs plus singular (single-look) pixels
    n2 = 400
    args2 = np.zeros((n2, 8), np.float32)
    for i in range(n2):
        a, b = rng.gamma(2.0, 2.0, 2), rng.gamma(2.0, 2.0, 2)
        ga, gb = (1.0, rng.uniform(0, 1)) if i % 5 == 0 else rng.uniform(0, 1, 2)
        pa, pb = rng.uniform(-np.pi, np.pi, 2)
        args2[i] = [a[0] ** 2, ga * a[0] * a[1] * np.cos(pa), ga * a[0] * a[1] * np.sin(pa), a[1] ** 2,
                    b[0] ** 2, gb * b[0] * b[1] * np.cos(pb), gb * b[0] * b[1] * np.sin(pb), b[1] ** 2]
    out["sim2_args"] = args2
    out["sim2_ref"] = np.float32([R.ref_pixel_similarity_2x2(*[float(x) for x in r]) for r in args2])
    # 3x3 pixel similarities
    n3 = 400
    a3 = np.stack([herm3(rng) for _ in range(n3)])
    b3 = np.stack([herm3(rng) for _ in range(n3)])
    out["sim3_a"], out["sim3_b"] = a3, b3
    out["sim3_ref"] = np.float32([R.ref_pixel_similarity_3x3(fp(np.ascontiguousarray(a3[i])),
                                                             fp(np.ascontiguousarray(b3[i]))) for i in range(n3)])
    # tile iterator
    cases = [(100, 73, 40, 40, 14), (512, 512, 124, 124, 14), (33, 200, 60, 60, 13), (1, 1, 30, 30, 14)]
    tiles = []
    for H, W, th, tw, ov in cases:
        cap = 1 << 14
        h0, w0 = np.zeros(cap, np.int32), np.zeros(cap, np.int32)
        n = R.ref_tile_list(H, W, th, tw, ov, h0.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                            w0.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), cap)
        tiles.append(np.stack([np.full(n, len(tiles)), h0[:n], w0[:n]], 1))
    out["tile_cases"] = np.int32(cases)
    out["tiles"] = np.concatenate(tiles).astype(np.int32)
    # best_params (reference selection): keys (patch, scale), ENL maps
    keys = np.int32([[3, 1], [3, 3], [5, 1], [5, 3], [7, 1], [7, 3]])
    enl = rng.uniform(0, 50, (len(keys), 64)).astype(np.float32)
    sel = np.zeros(2 * 64, np.int32)
    R.ref_get_best_params(keys.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(keys), fp(enl), 64,
                          sel.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    out["best_keys"], out["best_enl"], out["best_ref"] = keys, enl, sel.reshape(64, 2)
    # Goldstein (patch 32, overlap 4, alpha 0.5) on a 48 x 56 scene, seed 31
    a1, a2, ph = synthetic.insar_scene(48, 56, 31)
    g = pyoracle.ref_goldstein(a1, a2, ph, 32, 4, 0.5)
    out["gold_in"] = np.stack([a1, a2, ph])
    out["gold_ref"] = np.stack(g[:2])
    # NL-InSAR (search 21, patch 7, 2 passes, lmin 10) on a 40 x 44 scene, seed 32
    a1, a2, ph = synthetic.insar_scene(40, 44, 32)
    nl = pyoracle.ref_nlinsar(a1, a2, ph, 21, 7, 2, 10)
    out["nl_in"] = np.stack([a1, a2, ph])
    out["nl_ref"] = np.stack(nl)
    np.savez_compressed(os.path.join(HERE, "reference_pieces.npz"), **out)
    print("wrote", os.path.join(HERE, "reference_pieces.npz"))


# NL-SAR cases: (name, H, W, seed, patches, scales, select modes, tile or None)
NLSAR_CASES = [
    ("s64x80", 64, 80, 41, [3, 5, 7], [1, 3], (0, 1), None),
    ("s96x96", 96, 96, 42, [3, 5, 7], [1, 3], (0, 1), None),
    ("example", 40, 48, 43, [3, 5, 7, 9, 11], [1, 3, 5], (0, 1), None),
    ("tiled", 70, 90, 45, [3, 5, 7], [1, 3], (0, 1), (60, 60)),
]


def covariance_input(seed):
    """A generic 2x2 covariance image [8][H][W]: the covariance of an InSAR
    scene, 3x3 box-averaged, with an independent imaginary diagonal and a
    perturbed lower off-diagonal, so every plane carries its own data."""
    a1, a2, ph = synthetic.insar_scene(40, 48, seed)
    z1 = a1.astype(np.float64)
    z2 = a2.astype(np.float64) * np.exp(-1j * ph.astype(np.float64))
    pad = lambda x: np.pad(x, 1, mode="edge")  # noqa: E731
    box = lambda x: sum(pad(x)[i:i + 40, j:j + 48] for i in range(3) for j in range(3)) / 9  # noqa: E731
    c00, c11, c01 = box(np.abs(z1) ** 2), box(np.abs(z2) ** 2), box(z1 * np.conj(z2))
    rng = np.random.default_rng(seed)
    cov = np.stack([c00, rng.normal(0, 0.05, c00.shape), c01.real, c01.imag, 1.01 * c01.real, -c01.imag, c11,
                    rng.normal(0, 0.05, c00.shape)])
    return cov.astype(np.float32)


def nlsar_main():
    if pyoracle.ref_pieces() is None:
        raise SystemExit("oracle/_ref/libref_pieces.so not built: run `make -C oracle` with the reference tree present")
    t1, t2, tp = synthetic.training_area(128, seed=7)
    stats = pyoracle.training_insar(t1, t2, tp, [3, 5, 7, 9, 11], [1, 3, 5])
    keys = sorted(stats)
    out = {"stat_keys": np.int32(keys), "stat_lut_size": np.int32([stats[k].lut_size for k in keys]),
           "stat_dmin": np.float32([stats[k].dissims_min for k in keys]),
           "stat_dmax": np.float32([stats[k].dissims_max for k in keys]),
           "stat_quant": np.stack([np.float32(stats[k].quantilles) for k in keys]),
           "stat_chi2": np.stack([np.float32(stats[k].chi2cdf_inv) for k in keys])}
    names = []
    for name, H, W, seed, patches, scales, modes, tile in NLSAR_CASES:
        a1, a2, ph = synthetic.insar_scene(H, W, seed)
        st = {k: v for k, v in stats.items() if k[0] in patches and k[1] in scales}
        out[f"{name}_in"] = np.stack([a1, a2, ph])
        out[f"{name}_patches"] = np.int32(patches)
        out[f"{name}_scales"] = np.int32(scales)
        out[f"{name}_tile"] = np.int32(tile if tile else pyoracle.default_tile(H, W, 21, patches, scales))
        for m in modes:
            r = pyoracle.ref_nlsar_insar(a1, a2, ph, 21, patches, scales, st, select_mode=m, tile=tile)
            out[f"{name}_m{m}_out"] = np.stack(r[:3])
            out[f"{name}_m{m}_sel"] = r[3]
            print(name, "mode", m, "done")
        names.append(name)
    out["cases"] = np.array(names)
    cov = covariance_input(44)
    st = {k: v for k, v in stats.items() if k[0] in (3, 5, 7) and k[1] in (1, 3)}
    out["cov_in"] = cov
    for m in (0, 1):
        out[f"cov_m{m}_out"] = pyoracle.ref_nlsar_covmat(cov, 21, [3, 5, 7], [1, 3], st, select_mode=m)
    np.savez_compressed(os.path.join(HERE, "reference_nlsar.npz"), **out)
    print("wrote", os.path.join(HERE, "reference_nlsar.npz"))


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "nlsar":
        nlsar_main()
    elif len(sys.argv) > 1 and sys.argv[1] == "pieces":
        main()
    else:
        main()
        nlsar_main()
