"""Python API of the B200 NL-SAR engine.

The functions mirror despeckCL's Python bindings (swig/python/nlsar.i:44-258,
swig/python/boxcar.i in the reference): same names, argument order, defaults
(h=15, c=49) and return values, so scripts written for ``despeckcl`` run
unchanged.  Two keyword arguments are added: ``select_mode`` ("reference" --
the reference's behaviour, every pixel takes the last statistics key -- or
"argmax_enl", the largest bias-reduced ENL) and, on the device entry points,
``stream``.

Everything runs on the GPU through the C ABI of ``libdespeckcl_b200.so``;
there is no CPU fallback: if the library cannot be loaded, every call raises.
"""
from __future__ import annotations

import ctypes
import os
from collections import namedtuple
from typing import Iterable

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBPATH = os.path.join(_HERE, "libdespeckcl_b200.so")
_LIB = None

SELECT_MODES = {"reference": 0, "argmax_enl": 1}
DEFAULT_LOG_LEVELS = ["error", "warning", "fatal"]


class DespeckclError(RuntimeError):
    """A failed call of the C ABI; ``code`` is the negative dcl_status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{message} (dcl_status {code})")
        self.code = code


class StatsEntry(ctypes.Structure):
    """dcl_stats_entry (include/despeckcl_b200.h)."""

    _fields_ = [
        ("patch_size", ctypes.c_int),
        ("scale_size", ctypes.c_int),
        ("lut_size", ctypes.c_uint),
        ("dissims_min", ctypes.c_float),
        ("dissims_max", ctypes.c_float),
        ("quantilles", ctypes.POINTER(ctypes.c_float)),
        ("chi2cdf_inv", ctypes.POINTER(ctypes.c_float)),
    ]


class RequestInfo(ctypes.Structure):
    """dcl_request_info (include/despeckcl_b200.h)."""

    _fields_ = [("status", ctypes.c_int), ("chunks", ctypes.c_int), ("first_batch", ctypes.c_longlong),
                ("last_batch", ctypes.c_longlong), ("submit_s", ctypes.c_double), ("admit_s", ctypes.c_double),
                ("launch_s", ctypes.c_double), ("done_s", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerStats(ctypes.Structure):
    """dcl_server_stats (include/despeckcl_b200.h)."""

    _fields_ = [(k, ctypes.c_longlong) for k in ("submitted", "completed", "failed", "batches", "kernel_launches",
                                                   "tiles")] + \
        [(k, ctypes.c_ulonglong) for k in ("budget_bytes", "admitted_bytes", "peak_admitted_bytes")] + \
        [(k, ctypes.c_int) for k in ("queued", "admitted", "inflight", "peak_inflight")]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def lib() -> ctypes.CDLL:
    """The loaded native library (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(_LIBPATH):
            raise DespeckclError(-5, f"{_LIBPATH} not found: run `python -m despeckcl_b200.build`")
        L = ctypes.CDLL(_LIBPATH)
        L.dcl_last_error.restype = ctypes.c_char_p
        L.dcl_version.restype = ctypes.c_char_p
        for fn in ("dcl_nlsar_training_insar", "dcl_nlsar_training_covmat", "dcl_stats_load",
                   "dcl_stats_collection_from_entries", "dcl_stats_from_dissims", "dcl_nlsar_batch_create",
                   "dcl_server_create"):
            getattr(L, fn).restype = ctypes.c_void_p
        L.dcl_nlsar_batch_run.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.dcl_nlsar_batch_variant.argtypes = [ctypes.c_void_p]
        L.dcl_nlsar_batch_launches.argtypes = [ctypes.c_void_p]
        L.dcl_nlsar_batch_destroy.argtypes = [ctypes.c_void_p]
        L.dcl_stats_collection_size.argtypes = [ctypes.c_void_p]
        L.dcl_stats_collection_get.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(StatsEntry)]
        L.dcl_stats_collection_free.argtypes = [ctypes.c_void_p]
        L.dcl_stats_save.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.dcl_stats_save_boost_text.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.dcl_stats_load.argtypes = [ctypes.c_char_p]
        L.dcl_server_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(StatsEntry),
                                         ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                         ctypes.c_ulonglong, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.dcl_server_submit.restype = ctypes.c_longlong
        L.dcl_server_submit.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 6 + [ctypes.c_int] * 3 + \
            [ctypes.c_void_p]
        L.dcl_server_wait.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_double,
                                       ctypes.POINTER(RequestInfo)]
        L.dcl_server_poll.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.POINTER(RequestInfo)]
        L.dcl_server_now.restype = ctypes.c_double
        L.dcl_server_now.argtypes = [ctypes.c_void_p]
        L.dcl_server_get_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(ServerStats)]
        L.dcl_server_destroy.argtypes = [ctypes.c_void_p]
        _LIB = L
    return _LIB


def _check(rc: int) -> None:
    if rc != 0:
        raise DespeckclError(rc, lib().dcl_last_error().decode(errors="replace"))


def take_stage_timeouts() -> int:
    """Thread blocks of the NL-SAR kernels on the current device that gave up
    waiting for a TMA staging copy since the last call (their tiles are
    unwritten); reads and resets the device's ledger.  Call it after
    synchronising the streams whose launches it should cover."""
    n = ctypes.c_int(0)
    _check(lib().dcl_take_stage_timeouts(ctypes.byref(n)))
    return n.value


# ---------------------------------------------------------------------------
# statistics collections (std::map<nlsar::params, nlsar::stats>)
# ---------------------------------------------------------------------------

Params = namedtuple("Params", ["patch_size", "scale_size"])


class Stats:
    """nlsar::stats: LUTs of one (patch, scale) combination."""

    def __init__(self, lut_size, dissims_min, dissims_max, quantilles, chi2cdf_inv):
        self.lut_size = int(lut_size)
        self.dissims_min = float(dissims_min)
        self.dissims_max = float(dissims_max)
        self.quantilles = np.ascontiguousarray(quantilles, np.float32)
        self.chi2cdf_inv = np.ascontiguousarray(chi2cdf_inv, np.float32)

    def __repr__(self):
        return f"Stats(lut_size={self.lut_size}, dissims_min={self.dissims_min}, dissims_max={self.dissims_max})"


class StatsCollection(dict):
    """nlsar_stats_collection: a mapping Params -> Stats iterated in
    (patch, scale) order, like the SWIG-wrapped std::map."""

    def __iter__(self):
        return iter(sorted(super().keys()))

    def keys(self):
        return sorted(super().keys())

    def items(self):
        return [(k, self[k]) for k in self.keys()]

    def values(self):
        return [self[k] for k in self.keys()]


def _as_collection(stats) -> StatsCollection:
    if isinstance(stats, StatsCollection):
        return stats
    out = StatsCollection()
    for k, v in dict(stats).items():
        out[Params(int(k[0]), int(k[1]))] = v if isinstance(v, Stats) else Stats(
            v.lut_size, v.dissims_min, v.dissims_max, v.quantilles, v.chi2cdf_inv)
    return out


def _entries(stats):
    coll = _as_collection(stats)
    arr = (StatsEntry * max(1, len(coll)))()
    keep = []
    for i, (k, s) in enumerate(coll.items()):
        q = np.ascontiguousarray(s.quantilles, np.float32)
        c = np.ascontiguousarray(s.chi2cdf_inv, np.float32)
        lut = s.lut_size if (q.size >= s.lut_size and c.size >= s.lut_size) else 0
        keep += [q, c]
        arr[i] = StatsEntry(k[0], k[1], lut, s.dissims_min, s.dissims_max,
                            q.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                            c.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    return arr, len(coll), keep


def _from_handle(h) -> StatsCollection:
    if not h:
        raise DespeckclError(-1, lib().dcl_last_error().decode(errors="replace"))
    L = lib()
    try:
        out = StatsCollection()
        for i in range(L.dcl_stats_collection_size(h)):
            e = StatsEntry()
            _check(L.dcl_stats_collection_get(h, i, ctypes.byref(e)))
            n = e.lut_size
            q = np.ctypeslib.as_array(e.quantilles, shape=(n,)).copy()
            c = np.ctypeslib.as_array(e.chi2cdf_inv, shape=(n,)).copy()
            out[Params(e.patch_size, e.scale_size)] = Stats(n, e.dissims_min, e.dissims_max, q, c)
        return out
    finally:
        L.dcl_stats_collection_free(h)


def store_nlsar_stats_collection(nsc, filename: str, format: str = "boost") -> None:
    """Stores a statistics collection (nlsar.i:29-34).

    format="boost" writes the reference's file, a Boost text archive of
    std::map<nlsar::params, nlsar::stats> (nlsar_training.cpp:99-104), which
    the reference's load_nlsar_stats_collection reads; format="native" writes
    this library's own versioned text format.  load_nlsar_stats_collection
    reads both."""
    if format not in ("boost", "native"):
        raise ValueError(f"format must be 'boost' or 'native', not {format!r}")
    arr, n, keep = _entries(nsc)
    h = lib().dcl_stats_collection_from_entries(arr, n)
    if not h:
        raise DespeckclError(-1, lib().dcl_last_error().decode(errors="replace"))
    try:
        save = lib().dcl_stats_save_boost_text if format == "boost" else lib().dcl_stats_save
        _check(save(h, os.fsencode(filename)))
    finally:
        lib().dcl_stats_collection_free(h)


def load_nlsar_stats_collection(filename: str) -> StatsCollection:
    """Loads a statistics collection (nlsar.i:36-42)."""
    return _from_handle(lib().dcl_stats_load(os.fsencode(filename)))


# ---------------------------------------------------------------------------
# numpy helpers
# ---------------------------------------------------------------------------

def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _fp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _ints(v: Iterable[int]):
    a = np.ascontiguousarray(list(v), dtype=np.int32)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), a.size


def _mode(select_mode) -> int:
    if isinstance(select_mode, int):
        return select_mode
    if select_mode not in SELECT_MODES:
        raise ValueError(f"select_mode must be one of {sorted(SELECT_MODES)}")
    return SELECT_MODES[select_mode]


def _same_shape(*arrs):
    s = arrs[0].shape
    if len(s) != 2 or any(a.shape != s for a in arrs):
        raise ValueError("inputs must be 2-D arrays of the same shape")
    return s


# ---------------------------------------------------------------------------
# filters (host arrays)
# ---------------------------------------------------------------------------

def nlsar_insar(ampl_master, ampl_slave, phase, search_window_size, patch_sizes, scale_sizes, nlsar_stats,
                h=15.0, c=49.0, enabled_log_levels=DEFAULT_LOG_LEVELS, select_mode="reference"):
    """NL-SAR filter of an InSAR pair (nlsar.i:212-258): returns
    (reflectivity, phase, coherence) as float32 arrays."""
    a1, a2, ph = _f32(ampl_master), _f32(ampl_slave), _f32(phase)
    H, W = _same_shape(a1, a2, ph)
    ref, phf, coh = (np.zeros((H, W), np.float32) for _ in range(3))
    pk, pp, npn = _ints(patch_sizes)
    sk, sp, nsn = _ints(scale_sizes)
    arr, n, keep = _entries(nlsar_stats)
    _check(lib().dcl_nlsar_insar(_fp(a1), _fp(a2), _fp(ph), _fp(ref), _fp(phf), _fp(coh), H, W,
                                 int(search_window_size), pp, npn, sp, nsn, arr, n, ctypes.c_float(h),
                                 ctypes.c_float(c), _mode(select_mode)))
    return ref, phf, coh


def nlsar(covmat_raw, search_window_size, patch_sizes, scale_sizes, nlsar_stats, h=15.0, c=49.0,
          enabled_log_levels=DEFAULT_LOG_LEVELS, select_mode="reference"):
    """NL-SAR filter of a covariance image (nlsar.i:157-210): covmat_raw is a
    complex (d, d, height, width) array; returns the filtered array."""
    cov = np.asarray(covmat_raw)
    d, dd, H, W = cov.shape
    inter = np.empty((2 * d * d, H, W), np.float32)
    inter[::2] = cov.real.reshape((-1, H, W))
    inter[1::2] = cov.imag.reshape((-1, H, W))
    out = np.zeros_like(inter)
    pk, pp, npn = _ints(patch_sizes)
    sk, sp, nsn = _ints(scale_sizes)
    arr, n, keep = _entries(nlsar_stats)
    _check(lib().dcl_nlsar_covmat(_fp(inter), _fp(out), H, W, d, int(search_window_size), pp, npn, sp, nsn, arr, n,
                                  ctypes.c_float(h), ctypes.c_float(c), _mode(select_mode)))
    return out[::2].reshape((d, d, H, W)) + 1j * out[1::2].reshape((d, d, H, W))


def nlsar_train_insar(ampl_master, ampl_slave, phase, patch_sizes, scale_sizes,
                      enabled_log_levels=DEFAULT_LOG_LEVELS) -> StatsCollection:
    """Trains the weighting kernel on a homogeneous area (nlsar.i:45-60)."""
    a1, a2, ph = _f32(ampl_master), _f32(ampl_slave), _f32(phase)
    H, W = _same_shape(a1, a2, ph)
    pk, pp, npn = _ints(patch_sizes)
    sk, sp, nsn = _ints(scale_sizes)
    return _from_handle(lib().dcl_nlsar_training_insar(_fp(a1), _fp(a2), _fp(ph), H, W, pp, npn, sp, nsn))


def nlsar_train(covmat_raw, patch_sizes, scale_sizes, enabled_log_levels=DEFAULT_LOG_LEVELS) -> StatsCollection:
    """Trains on a complex (d, d, height, width) covariance image (nlsar.i:141-153)."""
    cov = np.asarray(covmat_raw)
    d, dd, H, W = cov.shape
    inter = np.empty((2 * d * d, H, W), np.float32)
    inter[::2] = cov.real.reshape((-1, H, W))
    inter[1::2] = cov.imag.reshape((-1, H, W))
    pk, pp, npn = _ints(patch_sizes)
    sk, sp, nsn = _ints(scale_sizes)
    return _from_handle(lib().dcl_nlsar_training_covmat(_fp(inter), H, W, d, pp, npn, sp, nsn))


def boxcar(ampl_master, ampl_slave, phase, window_width, enabled_log_levels=DEFAULT_LOG_LEVELS):
    """Boxcar filter (swig/python/boxcar.i): returns (reflectivity, phase, coherence)."""
    a1, a2, ph = _f32(ampl_master), _f32(ampl_slave), _f32(phase)
    H, W = _same_shape(a1, a2, ph)
    ref, phf, coh = (np.zeros((H, W), np.float32) for _ in range(3))
    _check(lib().dcl_boxcar(_fp(a1), _fp(a2), _fp(ph), _fp(ref), _fp(phf), _fp(coh), H, W, int(window_width)))
    return ref, phf, coh


def goldstein(ampl_master, ampl_slave, phase, patch_size, overlap, alpha, enabled_log_levels=DEFAULT_LOG_LEVELS):
    """Goldstein filter (swig/python/goldstein.i): returns (reflectivity,
    phase, coherence); the coherence stays zero as in the reference."""
    a1, a2, ph = _f32(ampl_master), _f32(ampl_slave), _f32(phase)
    H, W = _same_shape(a1, a2, ph)
    ref, phf, coh = (np.zeros((H, W), np.float32) for _ in range(3))
    _check(lib().dcl_goldstein(_fp(a1), _fp(a2), _fp(ph), _fp(ref), _fp(phf), _fp(coh), H, W, int(patch_size),
                               int(overlap), ctypes.c_float(alpha)))
    return ref, phf, coh


def nlinsar(ampl_master, ampl_slave, phase, search_window_size, patch_size, niter, lmin,
            enabled_log_levels=DEFAULT_LOG_LEVELS):
    """NL-InSAR filter (swig/python/nlinsar.i): returns (reflectivity, phase,
    coherence), starting from zero estimates as the reference's binding does."""
    a1, a2, ph = _f32(ampl_master), _f32(ampl_slave), _f32(phase)
    H, W = _same_shape(a1, a2, ph)
    ref, phf, coh = (np.zeros((H, W), np.float32) for _ in range(3))
    _check(lib().dcl_nlinsar(_fp(a1), _fp(a2), _fp(ph), _fp(ref), _fp(phf), _fp(coh), H, W, int(search_window_size),
                             int(patch_size), int(niter), int(lmin)))
    return ref, phf, coh


# ---------------------------------------------------------------------------
# device entry points (torch CUDA tensors; torch is only the allocator/stream)
# ---------------------------------------------------------------------------

def _dptr(t):
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("device entry points take contiguous CUDA tensors")
    return ctypes.c_void_p(t.data_ptr())


def _stream(stream):
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def nlsar_insar_device(a1, a2, phase, search_window_size, patch_sizes, scale_sizes, nlsar_stats, h=15.0, c=49.0,
                       select_mode="reference", out=None, selection=None, stream=None):
    """NL-SAR on float32 CUDA tensors, asynchronous on `stream` (default: the
    current torch stream).  `out` = (ref, phase, coh) tensors to fill;
    `selection` = int32 tensor receiving the selected combination index."""
    import torch

    H, W = a1.shape
    if out is None:
        out = tuple(torch.empty((H, W), dtype=torch.float32, device=a1.device) for _ in range(3))
    pk, pp, npn = _ints(patch_sizes)
    sk, sp, nsn = _ints(scale_sizes)
    arr, n, keep = _entries(nlsar_stats)
    sel = _dptr(selection) if selection is not None else None
    _check(lib().dcl_nlsar_insar_device(_dptr(a1), _dptr(a2), _dptr(phase), _dptr(out[0]), _dptr(out[1]),
                                        _dptr(out[2]), H, W, int(search_window_size), pp, npn, sp, nsn, arr, n,
                                        ctypes.c_float(h), ctypes.c_float(c), _mode(select_mode), sel,
                                        _stream(stream)))
    return out


def nlsar_insar_batch_device(scenes, search_window_size, patch_sizes, scale_sizes, nlsar_stats, h=15.0, c=49.0,
                             select_mode="argmax_enl", outs=None, stream=None):
    """Batched NL-SAR: `scenes` is a list of (a1, a2, phase) CUDA tensors of
    possibly different shapes, filtered in one persistent launch."""
    import torch

    n = len(scenes)
    if outs is None:
        outs = [tuple(torch.empty(s[0].shape, dtype=torch.float32, device=s[0].device) for _ in range(3))
                for s in scenes]
    P = ctypes.c_void_p * n
    a1 = P(*[_dptr(s[0]) for s in scenes])
    a2 = P(*[_dptr(s[1]) for s in scenes])
    ph = P(*[_dptr(s[2]) for s in scenes])
    r = P(*[_dptr(o[0]) for o in outs])
    p = P(*[_dptr(o[1]) for o in outs])
    co = P(*[_dptr(o[2]) for o in outs])
    hs = (ctypes.c_int * n)(*[s[0].shape[0] for s in scenes])
    ws = (ctypes.c_int * n)(*[s[0].shape[1] for s in scenes])
    pk, pp, npn = _ints(patch_sizes)
    sk, sp, nsn = _ints(scale_sizes)
    arr, ns, keep = _entries(nlsar_stats)
    _check(lib().dcl_nlsar_insar_batch_device(n, a1, a2, ph, r, p, co, hs, ws, int(search_window_size), pp, npn, sp,
                                              nsn, arr, ns, ctypes.c_float(h), ctypes.c_float(c), _mode(select_mode),
                                              _stream(stream)))
    return outs


class NlsarBatch:
    """A prepared batch (dcl_nlsar_batch_*): scenes of uneven size filtered by
    one fused launch per run, optionally replayed as a CUDA graph and with the
    kernel instantiation picked by the autotuner."""

    def __init__(self, scenes, search_window_size, patch_sizes, scale_sizes, nlsar_stats, h=15.0, c=49.0,
                 select_mode="argmax_enl", outs=None, graph=True, autotune=True, variant=None, stream=None):
        import torch

        n = len(scenes)
        self.scenes = scenes
        self.outs = outs if outs is not None else [
            tuple(torch.empty(s[0].shape, dtype=torch.float32, device=s[0].device) for _ in range(3)) for s in scenes]
        P = ctypes.c_void_p * n
        ptr = lambda i, j, src: _dptr(src[i][j])
        args = [P(*[ptr(i, j, scenes) for i in range(n)]) for j in range(3)]
        args += [P(*[ptr(i, j, self.outs) for i in range(n)]) for j in range(3)]
        hs = (ctypes.c_int * n)(*[s[0].shape[0] for s in scenes])
        ws = (ctypes.c_int * n)(*[s[0].shape[1] for s in scenes])
        pk, pp, npn = _ints(patch_sizes)
        sk, sp, nsn = _ints(scale_sizes)
        arr, ns, keep = _entries(nlsar_stats)
        flags = (1 if graph else 0) | (2 if autotune else 0) | (4 if variant == 1 else 0) | (8 if variant == 2 else 0)
        h_ = lib().dcl_nlsar_batch_create(n, *args, hs, ws, int(search_window_size), pp, npn, sp, nsn, arr, ns,
                                          ctypes.c_float(h), ctypes.c_float(c), _mode(select_mode), flags,
                                          _stream(stream))
        if not h_:
            raise DespeckclError(-1, lib().dcl_last_error().decode(errors="replace"))
        self.handle = h_

    def run(self, stream=None):
        _check(lib().dcl_nlsar_batch_run(self.handle, _stream(stream)))
        return self.outs

    @property
    def variant(self):
        return lib().dcl_nlsar_batch_variant(self.handle)

    @property
    def launches(self):
        return lib().dcl_nlsar_batch_launches(self.handle)

    def close(self):
        if getattr(self, "handle", None):
            lib().dcl_nlsar_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class NlsarServer:
    """NL-SAR request server (dcl_server_*): scenes are admitted by a device
    memory budget and filtered with continuous batching on the current device.

    submit() takes CUDA tensors (read after the work queued so far on the
    current stream) or numpy arrays (staged through the budget) and returns a
    request id; wait() returns the request's (ref, phase, coh) and its timing.
    """

    def __init__(self, search_window_size, patch_sizes, scale_sizes, nlsar_stats, h=15.0, c=49.0,
                 select_mode="argmax_enl", hbm_budget_bytes=8 << 30, max_inflight=2, max_batch_tiles=148 * 8,
                 variant=0):
        pk, pp, npn = _ints(patch_sizes)
        sk, sp, nsn = _ints(scale_sizes)
        arr, ns, keep = _entries(nlsar_stats)
        h_ = lib().dcl_server_create(int(search_window_size), pp, npn, sp, nsn, arr, ns, ctypes.c_float(h),
                                     ctypes.c_float(c), _mode(select_mode), int(hbm_budget_bytes),
                                     int(max_inflight), int(max_batch_tiles), 4 if variant == 1 else 0)
        if not h_:
            raise DespeckclError(-1, lib().dcl_last_error().decode(errors="replace"))
        self.handle = h_
        self._live = {}  # request id -> buffers (and event) kept alive until waited for

    def submit(self, a1, a2, phase, out=None):
        H, W = a1.shape
        if isinstance(a1, np.ndarray):
            ins = tuple(_f32(x) for x in (a1, a2, phase))
            if out is None:
                out = tuple(np.empty((H, W), dtype=np.float32) for _ in range(3))
            ptrs = [ctypes.c_void_p(x.ctypes.data) for x in ins + tuple(out)]
            host, ev = 1, None
        else:
            import torch

            ins = (a1, a2, phase)
            if out is None:
                out = tuple(torch.empty((H, W), dtype=torch.float32, device=a1.device) for _ in range(3))
            ptrs = [_dptr(x) for x in ins + tuple(out)]
            ev = torch.cuda.Event()
            ev.record()
            host = 0
        rid = lib().dcl_server_submit(self.handle, *ptrs, H, W, host,
                                      ctypes.c_void_p(ev.cuda_event) if ev is not None else None)
        if rid < 0:
            raise DespeckclError(int(rid), lib().dcl_last_error().decode(errors="replace"))
        self._live[rid] = (ins, out, ev)
        return rid

    def wait(self, rid, timeout=None):
        info = RequestInfo()
        _check(lib().dcl_server_wait(self.handle, rid, -1.0 if timeout is None else float(timeout),
                                     ctypes.byref(info)))
        _, out, _ = self._live.pop(rid)
        if info.status != 0:
            raise DespeckclError(info.status, f"request {rid} failed: " +
                                 lib().dcl_last_error().decode(errors="replace"))
        return out, info.as_dict()

    def poll(self, rid):
        info = RequestInfo()
        rc = lib().dcl_server_poll(self.handle, rid, ctypes.byref(info))
        if rc < 0:
            _check(rc)
        if rc == 0:
            return None
        _, out, _ = self._live.pop(rid)
        if info.status != 0:
            raise DespeckclError(info.status, f"request {rid} failed")
        return out, info.as_dict()

    def now(self):
        return lib().dcl_server_now(self.handle)

    def stats(self):
        s = ServerStats()
        _check(lib().dcl_server_get_stats(self.handle, ctypes.byref(s)))
        return s.as_dict()

    def close(self):
        if getattr(self, "handle", None):
            lib().dcl_server_destroy(self.handle)
            self.handle = None
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def nlinsar_device(a1, a2, phase, search_window_size, patch_size, niter, lmin, estimates=None, stream=None):
    """NL-InSAR on CUDA tensors: `estimates` = (ref, phase, coh) tensors with
    the initial estimates (zeros when omitted), overwritten with the results."""
    import torch

    H, W = a1.shape
    if estimates is None:
        estimates = tuple(torch.zeros((H, W), dtype=torch.float32, device=a1.device) for _ in range(3))
    _check(lib().dcl_nlinsar_device(_dptr(a1), _dptr(a2), _dptr(phase), _dptr(estimates[0]), _dptr(estimates[1]),
                                    _dptr(estimates[2]), H, W, int(search_window_size), int(patch_size), int(niter),
                                    int(lmin), _stream(stream)))
    return estimates


def goldstein_device(a1, a2, phase, patch_size, overlap, alpha, out=None, stream=None):
    """Goldstein filter on CUDA tensors: fills and returns (ref, phase) tensors."""
    import torch

    H, W = a1.shape
    if out is None:
        out = tuple(torch.empty((H, W), dtype=torch.float32, device=a1.device) for _ in range(2))
    _check(lib().dcl_goldstein_device(_dptr(a1), _dptr(a2), _dptr(phase), _dptr(out[0]), _dptr(out[1]), None, H, W,
                                      int(patch_size), int(overlap), ctypes.c_float(alpha), _stream(stream)))
    return out


def boxcar_device(a1, a2, phase, window_width, out=None, stream=None):
    import torch

    H, W = a1.shape
    if out is None:
        out = tuple(torch.empty((H, W), dtype=torch.float32, device=a1.device) for _ in range(3))
    _check(lib().dcl_boxcar_device(_dptr(a1), _dptr(a2), _dptr(phase), _dptr(out[0]), _dptr(out[1]), _dptr(out[2]),
                                   H, W, int(window_width), _stream(stream)))
    return out


def stats_from_dissims(dissims, lut_size=256, patch_size=1, scale_size=1) -> Stats:
    """nlsar::stats(dissims, lut_size) (src/compute/nlsar/stats.cpp:28-80)."""
    d = _f32(dissims).ravel()
    h = lib().dcl_stats_from_dissims(int(patch_size), int(scale_size), _fp(d), ctypes.c_long(d.size), int(lut_size))
    return _from_handle(h)[Params(int(patch_size), int(scale_size))]
