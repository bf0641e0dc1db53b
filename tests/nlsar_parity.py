"""Shared parity helpers of the NL-SAR tests (not a test module).

Tolerances (FP32 against the FP64 oracle): reflectivity and coherence within
1e-4 relative, phase within 1e-3 rad, asserted on every pixel whose FP64
result is well conditioned (see check_parity); at least 99 % of all pixels
must meet them.  The reference fixtures (tests/golden/reference_nlsar.npz)
are end-to-end outputs of the reference's own NL-SAR kernels
(oracle/nlsar_ref_shim.cpp, written by tests/golden/make_golden.py).
"""
import os

import numpy as np

REL_TOL, PHASE_TOL = 1e-4, 1e-3
KAPPA_MAX = 20.0

_GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REF_NLSAR = np.load(os.path.join(_GOLDEN, "reference_nlsar.npz"))


def wrapped(d):
    return np.abs(np.angle(np.exp(1j * d.astype(np.float64))))


def run_gpu(a1, a2, ph, stats, mode, sws=21, patches=(3, 5, 7), scales=(1, 3), selection=False):
    """The device entry point on cuda: (ref, phase, coh[, selection])."""
    import torch

    import despeckcl_b200 as dcl

    t = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (a1, a2, ph)]
    sel = torch.zeros(a1.shape, dtype=torch.int32, device="cuda") if selection else None
    out = dcl.nlsar_insar_device(*t, sws, list(patches), list(scales), stats, select_mode=mode, selection=sel)
    torch.cuda.synchronize()
    res = [o.cpu().numpy() for o in out]
    if selection:
        res.append(sel.cpu().numpy())
    return res


def check_parity(gpu, ora, diag, mode, min_all=0.99, min_stable=0.5):
    """Well-conditioned pixels: no weight of the selected combination within
    1e-3 LUT-index units of a weight-changing bin edge, no weighted intensity
    variance within 1e-4 of zero relative to the squared mean, and in ENL-argmax
    mode a bias-reduced ENL margin above 1e-4; coherence and phase also need the
    weighted complex mean to cancel by at most KAPPA_MAX (FP32 rounding of that
    sum scales with the factor, for any FP32 implementation)."""
    ref_g, ph_g, coh_g = gpu[:3]
    ref_o, ph_o, coh_o = ora
    stable = (diag.bin_margin > 1e-3) & (diag.var_cond > 1e-4)
    if mode == "argmax_enl":
        stable &= diag.enl_margin > 1e-4
    stable_c = stable & (diag.kappa <= KAPPA_MAX)
    with np.errstate(divide="ignore", invalid="ignore"):
        e_ref = np.abs(ref_g - ref_o) / np.abs(ref_o)
        e_coh = np.abs(coh_g - coh_o) / np.maximum(np.abs(coh_o), 1e-3)
    e_ph = wrapped(ph_g - ph_o)
    ok_ref = e_ref <= REL_TOL
    ok_c = (e_coh <= REL_TOL) & (e_ph <= PHASE_TOL)
    bad = (stable & ~ok_ref) | (stable_c & ~ok_c)
    assert not bad.any(), (
        f"{bad.sum()} well-conditioned pixels outside tolerance; worst rel ref {e_ref[stable].max():.3g}, "
        f"coh {e_coh[stable_c].max():.3g}, phase {e_ph[stable_c].max():.3g}; first at {np.argwhere(bad)[:5].tolist()}")
    ok = ok_ref & ok_c
    assert ok.mean() >= min_all, f"only {ok.mean():.4f} of all pixels within tolerance"
    assert stable.mean() >= min_stable
    return ok.mean(), stable.mean()


def nlsar_stats(oracle, patches, scales):
    """The statistics (LUTs) the reference fixtures were computed with."""
    N = REF_NLSAR
    st = {}
    for i, (p, s) in enumerate(N["stat_keys"]):
        if p in patches and s in scales:
            st[(int(p), int(s))] = oracle.OracleStats(int(N["stat_lut_size"][i]), float(N["stat_dmin"][i]),
                                                      float(N["stat_dmax"][i]), N["stat_quant"][i],
                                                      N["stat_chi2"][i])
    return st


def nlsar_cases():
    """(case name, selection mode) of every reference fixture."""
    for name in REF_NLSAR["cases"]:
        for m in (0, 1):
            if f"{name}_m{m}_out" in REF_NLSAR:
                yield str(name), m


def check_crops(oracle, stats, inputs, gpu, gpu_sel, mode, ncrops=4, crop=96, seed=0, sws=21, patches=(3, 5, 7),
                scales=(1, 3), min_stable=0.3):
    """Parity of a whole-scene GPU result on seeded crops: the FP64 oracle
    filters each crop with a margin of `overlap` pixels, so the crop's interior
    sees exactly its neighbourhood in the scene; the interiors are held to
    check_parity and to the selection agreement of clear pixels.  inputs, gpu:
    three host planes each (a1, a2, phase / ref, phase, coh)."""
    H, W = inputs[0].shape
    ov = oracle.overlap(sws, list(patches), list(scales))
    m = 0 if mode == "reference" else 1
    rng = np.random.default_rng(seed)
    g_all, o_all, d_all, s_all = [], [], [], []
    for _ in range(ncrops):
        y0 = int(rng.integers(ov, H - crop - ov))
        x0 = int(rng.integers(ov, W - crop - ov))
        ys, xs = slice(y0 - ov, y0 + crop + ov), slice(x0 - ov, x0 + crop + ov)
        o = oracle.nlsar_insar(*[x[ys, xs].copy() for x in inputs], sws, list(patches), list(scales), stats,
                               select_mode=m, use_double=True, diag=True)
        inner = (slice(ov, ov + crop), slice(ov, ov + crop))
        g_all.append([x[y0:y0 + crop, x0:x0 + crop] for x in gpu])
        s_all.append(gpu_sel[y0:y0 + crop, x0:x0 + crop])
        o_all.append([x[inner] for x in o[:3]])
        d = o[3]
        d_all.append({k: getattr(d, k)[inner] for k in ("sel", "bin_margin", "enl_margin", "var_cond", "kappa",
                                                        "bin_margin_all")})
    cat = lambda xs, i: np.concatenate([x[i] for x in xs])  # noqa: E731

    class D:
        pass

    diag = D()
    for k in d_all[0]:
        setattr(diag, k, np.concatenate([d[k] for d in d_all]))
    g = [cat(g_all, i) for i in range(3)]
    o = [cat(o_all, i) for i in range(3)]
    # about 43 % of the pixels of the benchmark scenes are well conditioned in
    # ENL-argmax mode (the 8192 x 8192 precision scene): with 441 weights of the
    # selected combination, one of them lies within 1e-3 index units of a LUT
    # bin edge for more than half of the pixels
    frac = check_parity(g, o, diag, mode, min_stable=min_stable)
    sel = np.concatenate(s_all)
    if m == 1:
        clear = (diag.enl_margin > 1e-4) & (diag.var_cond > 1e-4) & (diag.bin_margin_all > 1e-3)
    else:
        clear = np.ones(sel.shape, bool)
    assert np.array_equal(sel[clear], diag.sel[clear])
    assert (sel == diag.sel).mean() >= 0.995
    return frac
