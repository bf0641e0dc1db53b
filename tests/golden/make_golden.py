"""Writes tests/golden/reference_pieces.npz: outputs of the reference's own
code, compiled from the reference sources by oracle/Makefile into
oracle/_ref/libref_pieces.so (the translation units that build without
OpenCL, GSL or Boost, and the Goldstein / NL-InSAR kernels compiled as C++).

    make -C oracle && python tests/golden/make_golden.py

The fixtures let tests/test_golden.py pin the oracle without the reference
tree: pixel similarities (2x2 and 3x3, sim_measures.h), the tile iterator
(tile_iterator.cpp), the selection of best_params.cpp, and the Goldstein and
NL-InSAR outputs of the reference's kernels on two small seeded scenes.
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


if __name__ == "__main__":
    main()
