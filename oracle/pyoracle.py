"""ctypes front end of the NL-SAR oracle -- TEST INFRASTRUCTURE ONLY.

The oracle is a CPU restatement of despeckCL's NL-SAR path (see
``nlsar_oracle.cpp``).  Only the tests, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` leg of ``bench.py`` load it, as the checker or as the timed
CPU baseline; the product library never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None


class _Lut(ctypes.Structure):
    _fields_ = [
        ("patch_size", ctypes.c_int),
        ("scale_size", ctypes.c_int),
        ("lut_size", ctypes.c_uint),
        ("dissims_min", ctypes.c_float),
        ("dissims_max", ctypes.c_float),
        ("quantilles", ctypes.POINTER(ctypes.c_float)),
        ("chi2cdf_inv", ctypes.POINTER(ctypes.c_float)),
    ]


def build() -> None:
    """Compile liboracle.so (and the reference pieces when the tree is present)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = ctypes.CDLL(path)
        _LIB.oracle_chi2_inv.restype = ctypes.c_double
        _LIB.oracle_chi2_inv.argtypes = [ctypes.c_double, ctypes.c_double]
        _LIB.oracle_training_dissims.restype = ctypes.c_long
        _LIB.oracle_pixel_similarity_2x2.restype = ctypes.c_float
        _LIB.oracle_pixel_similarity_2x2.argtypes = [ctypes.c_float] * 8
        _LIB.oracle_rescale_gamma.restype = ctypes.c_float
        _LIB.oracle_rescale_gamma_dim.restype = ctypes.c_float
        _LIB.oracle_pixel_similarity_3x3.restype = ctypes.c_float
        _LIB.oracle_lut_weight.restype = ctypes.c_float
        _LIB.oracle_alpha.restype = ctypes.c_float
        _LIB.oracle_enl_nobias.restype = ctypes.c_float
        _LIB.oracle_enl_nobias.argtypes = [ctypes.c_float] * 3
    return _LIB


def ref_pieces():
    """The reference's own compiled pieces (None when they were not built here)."""
    global _REF
    if _REF is None:
        path = os.path.join(_HERE, "_ref", "libref_pieces.so")
        if not os.path.exists(path):
            return None
        _REF = ctypes.CDLL(path)
        _REF.ref_pixel_similarity_2x2.restype = ctypes.c_float
        _REF.ref_pixel_similarity_2x2.argtypes = [ctypes.c_float] * 8
        _REF.ref_det_covmat_3x3.restype = ctypes.c_float
        _REF.ref_pixel_similarity_3x3.restype = ctypes.c_float
    return _REF


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _luts(stats):
    """stats: mapping (patch, scale) -> object with lut_size, dissims_min,
    dissims_max, quantilles, chi2cdf_inv."""
    keep = []
    arr = (_Lut * len(stats))()
    for i, (key, st) in enumerate(sorted(stats.items(), key=lambda kv: (kv[0][0], kv[0][1]))):
        q = _f32(st.quantilles)
        c = _f32(st.chi2cdf_inv)
        keep += [q, c]
        arr[i] = _Lut(int(key[0]), int(key[1]), int(st.lut_size), float(st.dissims_min), float(st.dissims_max),
                      _fp(q), _fp(c))
    return arr, keep


def overlap(sws, patches, scales) -> int:
    p = np.array(patches, np.int32)
    s = np.array(scales, np.int32)
    return lib().oracle_overlap(sws, _ip(p), len(p), _ip(s), len(s))


def default_tile(H, W, sws, patches, scales, core=96):
    ov = overlap(sws, patches, scales)
    return min(core, H) + 2 * ov, min(core, W) + 2 * ov


def nlsar_insar(a1, a2, phi, sws, patches, scales, stats, h=15.0, c=49.0, select_mode=0, use_double=False,
                tile=None, nthreads=0, diag=False):
    a1, a2, phi = _f32(a1), _f32(a2), _f32(phi)
    H, W = a1.shape
    ref = np.zeros((H, W), np.float32)
    ph = np.zeros((H, W), np.float32)
    coh = np.zeros((H, W), np.float32)
    p = np.array(patches, np.int32)
    s = np.array(scales, np.int32)
    luts, keep = _luts(stats)
    th, tw = tile if tile else default_tile(H, W, sws, patches, scales)
    sel = np.zeros((H, W), np.int32) if diag else None
    bm = np.zeros((H, W), np.float64) if diag else None
    em = np.zeros((H, W), np.float64) if diag else None
    vc = np.zeros((H, W), np.float64) if diag else None
    kp = np.zeros((H, W), np.float64) if diag else None
    ba = np.zeros((H, W), np.float64) if diag else None
    rc = lib().oracle_nlsar_insar(
        _fp(a1), _fp(a2), _fp(phi), _fp(ref), _fp(ph), _fp(coh), H, W, sws, _ip(p), len(p), _ip(s), len(s),
        luts, len(stats), ctypes.c_float(h), ctypes.c_float(c), select_mode, int(use_double), th, tw, nthreads,
        _ip(sel) if diag else None, _dp(bm) if diag else None, _dp(em) if diag else None,
        _dp(vc) if diag else None, _dp(kp) if diag else None, _dp(ba) if diag else None)
    if rc != 0:
        raise RuntimeError(f"oracle_nlsar_insar failed: {rc}")
    if diag:
        return ref, ph, coh, Diagnostics(sel, bm, em, vc, kp, ba)
    return ref, ph, coh


def nlsar_covmat(cov8, sws, patches, scales, stats, h=15.0, c=49.0, select_mode=0, use_double=False, tile=None,
                 nthreads=0):
    """cov8: [2*d*d][H][W] covariance planes (d = 2 or 3; even planes real,
    odd planes imaginary)."""
    cov8 = _f32(cov8)
    npl, H, W = cov8.shape
    dim = {8: 2, 18: 3}[npl]
    out = np.zeros_like(cov8)
    p = np.array(patches, np.int32)
    s = np.array(scales, np.int32)
    luts, keep = _luts(stats)
    th, tw = tile if tile else default_tile(H, W, sws, patches, scales)
    rc = lib().oracle_nlsar_covmat(_fp(cov8), _fp(out), H, W, dim, sws, _ip(p), len(p), _ip(s), len(s), luts,
                                   len(stats), ctypes.c_float(h), ctypes.c_float(c), select_mode, int(use_double),
                                   th, tw, nthreads)
    if rc != 0:
        raise RuntimeError(f"oracle_nlsar_covmat failed: {rc}")
    return out


class Diagnostics:
    """Per-pixel conditioning of the FP64 oracle's result.

    sel        selected combination (reference loop order: scale outer, patch inner)
    bin_margin distance, in LUT index units, from the nearest weight-changing
               LUT boundary over the pixel's weights of the selected combination
    enl_margin relative gap between the best and second-best ENL' (argmax mode)
    var_cond   min over the two intensities of |weighted variance| / mean^2;
               near 0 the reference's alpha formula is ill-conditioned
    kappa      sum w |C01| / |sum w C01| over the selected weights: the
               cancellation factor of the weighted complex mean, which scales
               the FP32 rounding error of coherence and phase
    bin_margin_all  bin_margin minimised over every combination (a flip in a
               non-selected combination moves its ENL' and can change the
               argmax selection)
    """

    def __init__(self, sel, bin_margin, enl_margin, var_cond, kappa, bin_margin_all):
        self.bin_margin_all = bin_margin_all
        self.sel = sel
        self.bin_margin = bin_margin
        self.enl_margin = enl_margin
        self.var_cond = var_cond
        self.kappa = kappa


class OracleStats:
    def __init__(self, lut_size, dmin, dmax, quant, chi2):
        self.lut_size = lut_size
        self.dissims_min = dmin
        self.dissims_max = dmax
        self.quantilles = quant
        self.chi2cdf_inv = chi2


def training_insar(a1, a2, phi, patches, scales):
    a1, a2, phi = _f32(a1), _f32(a2), _f32(phi)
    H, W = a1.shape
    n = len(patches) * len(scales)
    op = np.zeros(n, np.int32)
    osc = np.zeros(n, np.int32)
    dmin = np.zeros(n, np.float32)
    dmax = np.zeros(n, np.float32)
    q = np.zeros((n, 256), np.float32)
    ch = np.zeros((n, 256), np.float32)
    pp = np.array(patches, np.int32)
    ss = np.array(scales, np.int32)
    lib().oracle_nlsar_training_insar(_fp(a1), _fp(a2), _fp(phi), H, W, _ip(pp), len(pp), _ip(ss), len(ss),
                                      _ip(op), _ip(osc), _fp(dmin), _fp(dmax), _fp(q), _fp(ch))
    return {(int(op[i]), int(osc[i])): OracleStats(256, float(dmin[i]), float(dmax[i]), q[i].copy(), ch[i].copy())
            for i in range(n)}


def training_dissims(cov8, patch, scale):
    """cov8: [2*d*d][H][W] covariance planes, d = 2 or 3."""
    cov8 = _f32(cov8)
    npl, H, W = cov8.shape
    dim = {8: 2, 18: 3}[npl]
    n = lib().oracle_training_dissims(_fp(cov8), H, W, dim, patch, scale, None, ctypes.c_long(0))
    out = np.zeros(n, np.float32)
    lib().oracle_training_dissims(_fp(cov8), H, W, dim, patch, scale, _fp(out), ctypes.c_long(n))
    return out


def training_covmat(cov, patches, scales):
    """nlsar_training on a covariance image [2*d*d][H][W]: stats per (patch, scale)."""
    return {(int(p), int(s)): stats_from_dissims(training_dissims(cov, p, s)) for p in patches for s in scales}


def pixel_similarity_3x3(a, b):
    a = _f32(np.asarray(a).ravel())
    b = _f32(np.asarray(b).ravel())
    return lib().oracle_pixel_similarity_3x3(_fp(a), _fp(b))


def stats_from_dissims(d, lut_size=256):
    d = _f32(d)
    dmin = ctypes.c_float()
    dmax = ctypes.c_float()
    q = np.zeros(lut_size, np.float32)
    ch = np.zeros(lut_size, np.float32)
    lib().oracle_stats_from_dissims(_fp(d), ctypes.c_long(d.size), lut_size, ctypes.byref(dmin), ctypes.byref(dmax),
                                    _fp(q), _fp(ch))
    return OracleStats(lut_size, dmin.value, dmax.value, q, ch)


def chi2_inv(y, nu):
    return lib().oracle_chi2_inv(float(y), float(nu))


def covmat_create(a1, a2, phi):
    a1, a2, phi = _f32(a1), _f32(a2), _f32(phi)
    H, W = a1.shape
    out = np.zeros((8, H, W), np.float32)
    lib().oracle_covmat_create(_fp(a1), _fp(a2), _fp(phi), H, W, _fp(out))
    return out


def covmat_spatial_avg(cov8, s, smax):
    cov8 = _f32(cov8)
    _, H, W = cov8.shape
    out = np.zeros((8, H - smax + 1, W - smax + 1), np.float32)
    lib().oracle_covmat_spatial_avg(_fp(cov8), H, W, s, smax, _fp(out))
    return out


def gen_gauss(s):
    out = np.zeros(s * s, np.float32)
    lib().oracle_gen_gauss(s, _fp(out))
    return out


def tile_list(H, W, th, tw, ov):
    cap = 1 << 16
    h0 = np.zeros(cap, np.int32)
    w0 = np.zeros(cap, np.int32)
    n = lib().oracle_tile_list(H, W, th, tw, ov, _ip(h0), _ip(w0), cap)
    return list(zip(h0[:n].tolist(), w0[:n].tolist()))


def boxcar(a1, a2, phi, window_width, tile=512):
    a1, a2, phi = _f32(a1), _f32(a2), _f32(phi)
    H, W = a1.shape
    ref, ph, coh = (np.zeros((H, W), np.float32) for _ in range(3))
    rc = lib().oracle_boxcar(_fp(a1), _fp(a2), _fp(phi), _fp(ref), _fp(ph), _fp(coh), H, W, window_width, tile)
    if rc != 0:
        raise RuntimeError(f"oracle_boxcar failed: {rc}")
    return ref, ph, coh


def goldstein(a1, a2, phi, patch_size=32, overlap=4, alpha=0.5, use_double=True):
    """Goldstein filter restatement (goldstein_oracle.cpp): (ref, phase)."""
    a1, a2, phi = _f32(a1), _f32(a2), _f32(phi)
    H, W = a1.shape
    ref = np.zeros((H, W), np.float32)
    ph = np.zeros((H, W), np.float32)
    rc = lib().oracle_goldstein(_fp(a1), _fp(a2), _fp(phi), _fp(ref), _fp(ph), H, W, int(patch_size), int(overlap),
                                ctypes.c_float(alpha), int(bool(use_double)))
    if rc:
        raise ValueError("unsupported Goldstein parameters")
    return ref, ph


def ref_goldstein(a1, a2, phi, patch_size=32, overlap=4, alpha=0.5, coh=None):
    """The reference's own Goldstein kernels run on the CPU (oracle/_ref):
    (ref, phase, coh), or None when they were not built here."""
    R = ref_pieces()
    if R is None:
        return None
    a1, a2, phi = _f32(a1), _f32(a2), _f32(phi)
    H, W = a1.shape
    ref = np.zeros((H, W), np.float32)
    ph = np.zeros((H, W), np.float32)
    c = np.zeros((H, W), np.float32) if coh is None else _f32(coh).copy()
    rc = R.ref_goldstein(_fp(a1), _fp(a2), _fp(phi), _fp(ref), _fp(ph), _fp(c), H, W, int(patch_size),
                         int(overlap), ctypes.c_float(alpha))
    if rc:
        raise ValueError("scene smaller than two patches per side")
    return ref, ph, c


def nlinsar(a1, a2, phi, sws=21, patch_size=7, niter=5, lmin=10, use_double=True, init=None, threads=0):
    """NL-InSAR restatement (nlinsar_oracle.cpp): (ref, phase, coh); the
    initial estimates are zeros (as the Python binding passes) unless given."""
    a1, a2, phi = _f32(a1), _f32(a2), _f32(phi)
    H, W = a1.shape
    if init is None:
        ref, ph, coh = (np.zeros((H, W), np.float32) for _ in range(3))
    else:
        ref, ph, coh = (_f32(x).copy() for x in init)
    rc = lib().oracle_nlinsar(_fp(a1), _fp(a2), _fp(phi), _fp(ref), _fp(ph), _fp(coh), H, W, int(sws),
                              int(patch_size), int(niter), int(lmin), int(bool(use_double)),
                              int(threads or os.cpu_count() or 1))
    if rc:
        raise ValueError("unsupported NL-InSAR parameters")
    return ref, ph, coh


def ref_nlinsar(a1, a2, phi, sws=21, patch_size=7, niter=5, lmin=10, init=None):
    """The reference's own NL-InSAR pieces run on the CPU (oracle/_ref), or
    None when they were not built here."""
    R = ref_pieces()
    if R is None:
        return None
    a1, a2, phi = _f32(a1), _f32(a2), _f32(phi)
    H, W = a1.shape
    if init is None:
        ref, ph, coh = (np.zeros((H, W), np.float32) for _ in range(3))
    else:
        ref, ph, coh = (_f32(x).copy() for x in init)
    rc = R.ref_nlinsar(_fp(a1), _fp(a2), _fp(phi), _fp(ref), _fp(ph), _fp(coh), H, W, int(sws), int(patch_size),
                       int(niter), int(lmin))
    if rc:
        raise ValueError("unsupported NL-InSAR parameters")
    return ref, ph, coh


def _ref_stats_arrays(stats):
    """Flattened statistics for the reference shim: keys (patch, scale) in map
    order, LUT sizes, ranges and the concatenated LUTs."""
    items = sorted(stats.items(), key=lambda kv: (kv[0][0], kv[0][1]))
    keys = np.int32([[k[0], k[1]] for k, _ in items]).reshape(-1)
    sizes = np.int32([int(st.lut_size) for _, st in items])
    dmin = np.float32([st.dissims_min for _, st in items])
    dmax = np.float32([st.dissims_max for _, st in items])
    quant = np.concatenate([_f32(st.quantilles)[: int(st.lut_size)] for _, st in items])
    chi2 = np.concatenate([_f32(st.chi2cdf_inv)[: int(st.lut_size)] for _, st in items])
    return keys, sizes, dmin, dmax, _f32(quant), _f32(chi2)


def ref_nlsar_insar(a1, a2, phi, sws, patches, scales, stats, h=15.0, c=49.0, select_mode=0, tile=None):
    """The reference's own NL-SAR kernels run on the CPU (oracle/_ref,
    nlsar_ref_shim.cpp): (ref, phase, coh, sel), or None when they were not
    built here.  select_mode 0 is the reference's get_best_params, 1 the ENL
    argmax."""
    R = ref_pieces()
    if R is None:
        return None
    a1, a2, phi = _f32(a1), _f32(a2), _f32(phi)
    H, W = a1.shape
    out = [np.zeros((H, W), np.float32) for _ in range(3)]
    sel = np.zeros((H, W), np.int32)
    p = np.array(patches, np.int32)
    s = np.array(scales, np.int32)
    keys, sizes, dmin, dmax, quant, chi2 = _ref_stats_arrays(stats)
    th, tw = tile if tile else default_tile(H, W, sws, patches, scales)
    rc = R.ref_nlsar_insar(_fp(a1), _fp(a2), _fp(phi), _fp(out[0]), _fp(out[1]), _fp(out[2]), H, W, int(sws),
                           _ip(p), len(p), _ip(s), len(s), _ip(keys), len(sizes), _ip(sizes), _fp(dmin), _fp(dmax),
                           _fp(quant), _fp(chi2), ctypes.c_float(h), ctypes.c_float(c), int(select_mode), th, tw,
                           _ip(sel))
    if rc:
        raise ValueError(f"ref_nlsar_insar failed: {rc}")
    return out[0], out[1], out[2], sel


def ref_nlsar_covmat(cov8, sws, patches, scales, stats, h=15.0, c=49.0, select_mode=0, tile=None):
    """The reference's own NL-SAR kernels on an 8-plane 2x2 covariance image
    ([8][H][W]), or None when they were not built here."""
    R = ref_pieces()
    if R is None:
        return None
    cov8 = _f32(cov8)
    _, H, W = cov8.shape
    out = np.zeros_like(cov8)
    p = np.array(patches, np.int32)
    s = np.array(scales, np.int32)
    keys, sizes, dmin, dmax, quant, chi2 = _ref_stats_arrays(stats)
    th, tw = tile if tile else default_tile(H, W, sws, patches, scales)
    rc = R.ref_nlsar_covmat(_fp(cov8), _fp(out), H, W, int(sws), _ip(p), len(p), _ip(s), len(s), _ip(keys),
                            len(sizes), _ip(sizes), _fp(dmin), _fp(dmax), _fp(quant), _fp(chi2), ctypes.c_float(h),
                            ctypes.c_float(c), int(select_mode), th, tw)
    if rc:
        raise ValueError(f"ref_nlsar_covmat failed: {rc}")
    return out


def patch_similarities(pix, sws, patch_size, patch_size_max, reference=False):
    """Patch sums of U = sws*wsh + wsh pixel-similarity planes pix
    [U][height_sim][width_sim] (the oracle's stage, or with reference=True the
    reference's row and column pass kernels; None when those were not built)."""
    pix = _f32(pix)
    U, hs, ws = pix.shape
    out = np.zeros((U, hs - patch_size_max + 1, ws - patch_size_max + 1), np.float32)
    if reference:
        R = ref_pieces()
        if R is None:
            return None
        rc = R.ref_patch_similarities(_fp(pix), _fp(out), hs, ws, int(sws), int(patch_size), int(patch_size_max))
    else:
        rc = lib().oracle_patch_similarities(_fp(pix), _fp(out), hs, ws, int(sws), int(patch_size),
                                             int(patch_size_max))
    if rc:
        raise ValueError("bad patch-similarity arguments")
    return out


def copy_symm_weights(wsymm, height_ori, width_ori, sws, reference=False):
    """The upper half window of weights [U][height_ori + wsh][width_ori + 2 wsh]
    expanded to the full window [sws*sws][height_ori][width_ori] (the oracle's
    index map, or the reference's kernel with reference=True; None when that
    was not built)."""
    wsymm = _f32(wsymm)
    out = np.zeros((sws * sws, height_ori, width_ori), np.float32)
    if reference:
        R = ref_pieces()
        if R is None:
            return None
        rc = R.ref_copy_symm_weights(_fp(wsymm), _fp(out), int(height_ori), int(width_ori), int(sws))
    else:
        rc = lib().oracle_copy_symm_weights(_fp(wsymm), _fp(out), int(height_ori), int(width_ori), int(sws))
    if rc:
        raise ValueError("bad symmetric-copy arguments")
    return out
