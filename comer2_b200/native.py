"""ctypes binding of the C ABI in ``include/comer2_b200.h``.

The shared library is built in-tree (``comer2_b200/_lib/libcomer2_b200.so``,
see ``build.py``).  There is no fallback: if the library cannot be loaded,
every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from .params import SearchParams
from .synth import ProfileSet

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libcomer2_b200.so")

C2_OK = 0
STATUS_NAMES = {0: "C2_OK", 1: "C2_ERR_ARG", 2: "C2_ERR_CUDA", 3: "C2_ERR_NOMEM", 4: "C2_ERR_STATE",
                5: "C2_ERR_CAPACITY", 6: "C2_ERR_DEVICE"}

# every symbol include/comer2_b200.h declares
EXPORTS = [
    "c2_create", "c2_destroy", "c2_last_error", "c2_upload_db", "c2_set_query", "c2_run_phase1",
    "c2_get_phase1", "c2_run_finalize", "c2_get_finalize", "c2_get_thresholds", "c2_set_stream", "c2_sync",
    "c2_launch_count", "c2_run_stats", "c2_run_map", "c2_get_hits", "c2_search", "c2_get_search_space",
    "c2_run_phase1_static", "c2_set_score_mode", "c2_logz_fwd", "c2_logz_bwd", "c2_logz_cells",
    "c2_db2bin_info", "c2_db2bin_read", "c2_share_db", "c2_search_batch", "c2_format_report",
    "c2_set_wait_limit", "c2_get_pair_scores", "c2_db2bin_descriptions", "c2_set_device_memory_limit",
    "c2_db2bin_lengths", "c2_db2bin_read_range", "c2_get_device_memory_info", "c2_db_device_bytes",
    "c2_logz_fwd_batch", "c2_set_query_batch", "c2_set_batch_sm_reserve", "c2_get_device_count",
    "c2_get_query_limits",
    "c2_get_device_memory_use", "c2_get_search_groups",
]

REPORT_PLAIN = 0
REPORT_JSON = 1

# c2_batch_cb
BATCH_CB = C.CFUNCTYPE(None, C.c_void_p, C.c_int32, C.c_int, C.c_void_p, C.c_int32, C.c_void_p, C.c_size_t)

SCORE_FP32 = 0
SCORE_BF16_TC = 1

_fp = C.POINTER(C.c_float)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)
_u8p = C.POINTER(C.c_uint8)


class c2_params(C.Structure):
    _fields_ = [
        ("ungapped_lambda", C.c_float), ("ungapped_K", C.c_float), ("ungapped_H", C.c_float),
        ("gapped_lambda", C.c_float), ("gapped_K", C.c_float), ("gapped_H", C.c_float),
        ("gapped_alpha", C.c_float), ("gapped_beta", C.c_float),
        ("eval", C.c_float), ("ssswgt", C.c_float), ("cvswgt", C.c_float), ("minpp", C.c_float),
        ("mapaln", C.c_int32), ("x_uninf", C.c_int32), ("ssemodel", C.c_int32),
        ("ssss", _fp), ("ssss_card", C.c_int32),
        ("cvs2s_keys", _fp), ("cvs2s_values", _fp), ("cvs2s_card", C.c_int32), ("cvs2s_shift", C.c_int32),
        ("sse_nn_weights", _fp), ("n_sse_nn_weights", C.c_int32),
    ]


class c2_profiles(C.Structure):
    _fields_ = [
        ("nprofiles", C.c_int32), ("npositions", C.c_int64),
        ("lengths", _i32p), ("offsets", _i64p), ("bkg", _fp), ("eno", _fp), ("trn", _fp),
        ("trg", _fp), ("cv", _fp), ("cvprior", _fp), ("cvnorm2", _fp), ("ss", _fp),
        ("ssstate", _u8p), ("aa", _u8p),
    ]


class c2_p1_result(C.Structure):
    _fields_ = [("best", C.c_float), ("coords", C.c_uint32)]


class c2_dp_result(C.Structure):
    _fields_ = [("score", C.c_float), ("profile", C.c_int32), ("psts", C.c_int32),
                ("beg", C.c_uint32), ("end", C.c_uint32), ("passed", C.c_int32)]


class c2_hit(C.Structure):
    _fields_ = [("profile", C.c_int32), ("score", C.c_float), ("logE", C.c_float), ("logEpA", C.c_float),
                ("lambda_", C.c_float), ("K", C.c_float), ("lambda_est", C.c_float), ("K_est", C.c_float),
                ("E", C.c_float), ("H", C.c_float), ("smin", C.c_int32), ("smax", C.c_int32),
                ("psts", C.c_int32), ("idts", C.c_int32), ("gaps", C.c_int32), ("alnlen", C.c_int32),
                ("beg", C.c_uint32), ("end", C.c_uint32), ("aln_offset", C.c_int64)]


HIT_DTYPE = np.dtype([(k, {C.c_int32: np.int32, C.c_float: np.float32, C.c_uint32: np.uint32,
                           C.c_int64: np.int64}[t]) for k, t in c2_hit._fields_], align=True)
assert HIT_DTYPE.itemsize == C.sizeof(c2_hit)


class c2_report_info(C.Structure):
    _fields_ = [
        ("progname", C.c_char_p), ("progversion", C.c_char_p), ("references", C.POINTER(C.c_char_p)),
        ("query_desc", C.c_char_p), ("query_length", C.c_int32), ("query_eno", C.c_float),
        ("query_has_ss", C.c_int32), ("db_names", C.POINTER(C.c_char_p)), ("n_db_names", C.c_int32),
        ("db_positions", C.c_uint64), ("db_profiles", C.c_uint64), ("logevthld", C.c_float),
        ("searchspace", C.c_double), ("deltalen", C.c_int32), ("ref_lambda", C.c_float), ("ref_K", C.c_float),
        ("gapped_lambda", C.c_float), ("gapped_K", C.c_float), ("print_ss", C.c_int32), ("dsclen", C.c_int32),
        ("dscwidth", C.c_int32), ("alnwidth", C.c_int32), ("show", C.c_int32), ("nhits", C.c_int32),
        ("nalns", C.c_int32), ("db_desc", C.POINTER(C.c_char_p)), ("db_lengths", C.POINTER(C.c_int32)),
        ("db_eno", C.POINTER(C.c_float)), ("db_has_ss", C.POINTER(C.c_uint8)),
    ]


def _cstrs(seq, terminate=False):
    arr = (C.c_char_p * (len(seq) + (1 if terminate else 0)))()
    for i, x in enumerate(seq):
        arr[i] = None if x is None else x.encode()
    return arr


def format_report(fmt: int, hits: np.ndarray, alns: np.ndarray, *, query_length: int, query_eno: float,
                  db_lengths, db_eno, db_desc=None, db_has_ss=None, query_desc=None, query_has_ss=True,
                  db_names=("db",), db_positions=0, db_profiles=0, logevthld=0.0, searchspace=0.0, deltalen=0,
                  ref_lambda=0.0, ref_K=0.0, gapped_lambda=0.0, gapped_K=0.0, print_ss=True, dsclen=1024,
                  dscwidth=80, alnwidth=60, show=1, nhits=700, nalns=700, progname=None, progversion=None,
                  references=None) -> str:
    """One query's result file in the reference's Plain (REPORT_PLAIN) or JSON
    (REPORT_JSON) format from hits_arrays()-style records (c2_format_report)."""
    lib = load()
    keep = []
    r = c2_report_info()
    r.progname = progname.encode() if progname else None
    r.progversion = progversion.encode() if progversion else None
    if references is not None:
        refs = _cstrs(list(references), terminate=True)
        keep.append(refs)
        r.references = refs
    r.query_desc = query_desc.encode() if query_desc is not None else None
    r.query_length, r.query_eno, r.query_has_ss = int(query_length), float(query_eno), int(bool(query_has_ss))
    names = _cstrs(list(db_names))
    keep.append(names)
    r.db_names, r.n_db_names = names, len(db_names)
    r.db_positions, r.db_profiles = int(db_positions), int(db_profiles)
    r.logevthld, r.searchspace, r.deltalen = float(logevthld), float(searchspace), int(deltalen)
    r.ref_lambda, r.ref_K, r.gapped_lambda, r.gapped_K = (float(ref_lambda), float(ref_K), float(gapped_lambda),
                                                          float(gapped_K))
    r.print_ss, r.dsclen, r.dscwidth, r.alnwidth = int(bool(print_ss)), int(dsclen), int(dscwidth), int(alnwidth)
    r.show, r.nhits, r.nalns = int(show), int(nhits), int(nalns)
    dl = np.ascontiguousarray(db_lengths, np.int32)
    de = np.ascontiguousarray(db_eno, np.float32)
    keep += [dl, de]
    r.db_lengths, r.db_eno = _ptr(dl, _i32p), _ptr(de, _fp)
    if db_desc is not None:
        dd = _cstrs(list(db_desc))
        keep.append(dd)
        r.db_desc = dd
    if db_has_ss is not None:
        ds = np.ascontiguousarray(db_has_ss, np.uint8)
        keep.append(ds)
        r.db_has_ss = _ptr(ds, _u8p)
    hits = np.ascontiguousarray(hits, HIT_DTYPE)
    alns = np.ascontiguousarray(alns, np.uint8)
    n = C.c_size_t(0)
    st = lib.c2_format_report(int(fmt), C.byref(r), hits.ctypes.data, len(hits), alns.ctypes.data, None, C.byref(n))
    if st != C2_OK:
        raise C2Error("c2_format_report(size): %s" % STATUS_NAMES.get(st, st))
    buf = C.create_string_buffer(n.value)
    st = lib.c2_format_report(int(fmt), C.byref(r), hits.ctypes.data, len(hits), alns.ctypes.data, buf, C.byref(n))
    if st != C2_OK:
        raise C2Error("c2_format_report: %s" % STATUS_NAMES.get(st, st))
    return buf.value.decode("latin-1")

_lib: Optional[C.CDLL] = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load the CUDA library (raises OSError when it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError("comer2_b200 CUDA library not built: %s (run comer2_b200/build.py)" % path)
    lib = C.CDLL(path)
    P = C.POINTER
    lib.c2_create.argtypes = [C.c_int, P(c2_params), P(C.c_void_p)]
    lib.c2_destroy.argtypes = [C.c_void_p]
    lib.c2_last_error.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t]
    lib.c2_upload_db.argtypes = [C.c_void_p, P(c2_profiles), C.c_uint64, C.c_uint64]
    lib.c2_set_query.argtypes = [C.c_void_p, P(c2_profiles)]
    lib.c2_run_phase1.argtypes = [C.c_void_p]
    lib.c2_get_phase1.argtypes = [C.c_void_p, P(c2_p1_result), C.c_int32]
    lib.c2_run_finalize.argtypes = [C.c_void_p, P(C.c_int32)]
    lib.c2_get_finalize.argtypes = [C.c_void_p, P(c2_dp_result), C.c_int32]
    lib.c2_get_thresholds.argtypes = [C.c_void_p, P(C.c_float), P(C.c_float)]
    lib.c2_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    lib.c2_sync.argtypes = [C.c_void_p]
    lib.c2_launch_count.argtypes = [C.c_void_p, P(C.c_uint64)]
    lib.c2_run_stats.argtypes = [C.c_void_p, P(C.c_int32)]
    lib.c2_run_map.argtypes = [C.c_void_p, P(C.c_int32)]
    lib.c2_get_hits.argtypes = [C.c_void_p, P(c2_hit), C.c_int32, C.c_char_p, P(C.c_size_t)]
    lib.c2_search.argtypes = [C.c_void_p, P(c2_profiles), P(C.c_int32)]
    lib.c2_get_search_space.argtypes = [C.c_void_p, P(C.c_uint64), P(C.c_uint64)]
    lib.c2_run_phase1_static.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.c2_set_score_mode.argtypes = [C.c_void_p, C.c_int32]
    lib.c2_set_wait_limit.argtypes = [C.c_void_p, C.c_uint32]
    lib.c2_set_device_memory_limit.argtypes = [C.c_void_p, C.c_uint64]
    lib.c2_get_device_memory_use.argtypes = [C.c_void_p, P(C.c_uint64)]
    lib.c2_get_search_groups.argtypes = [C.c_void_p, P(C.c_int32)]
    lib.c2_get_pair_scores.argtypes = [C.c_void_p, C.c_int32, _fp, _fp]
    lib.c2_db2bin_descriptions.argtypes = [C.c_char_p, C.c_void_p, P(C.c_size_t), _i64p, C.c_char_p, C.c_size_t]
    lib.c2_logz_fwd.argtypes = [C.c_void_p, _i32p, C.c_int32, _fp, C.c_float, C.c_float, _fp]
    lib.c2_logz_bwd.argtypes = [C.c_void_p, _fp]
    lib.c2_set_query_batch.argtypes = [C.c_void_p, P(c2_profiles)]
    lib.c2_set_batch_sm_reserve.argtypes = [C.c_void_p, C.c_int32]
    lib.c2_get_device_count.argtypes = [_i32p]
    lib.c2_get_query_limits.argtypes = [C.c_void_p, C.c_int32, P(C.c_uint64), P(C.c_uint64), P(C.c_float),
                                        P(C.c_float)]
    lib.c2_logz_fwd_batch.argtypes = [C.c_void_p, _i32p, _i32p, C.c_int32, _fp, C.c_float, C.c_float, _fp]
    lib.c2_logz_cells.argtypes = [C.c_void_p, C.c_int32, _fp, _fp]
    lib.c2_db2bin_info.argtypes = [C.c_char_p, _i32p, _i64p, C.c_char_p, C.c_size_t]
    lib.c2_db2bin_read.argtypes = [C.c_char_p, _i32p, _i64p, _fp, _fp, _fp, _fp, _fp, _fp, _fp, _fp, _u8p, _u8p,
                                   C.c_char_p, C.c_size_t]
    lib.c2_get_device_memory_info.argtypes = [C.c_void_p, P(C.c_uint64), P(C.c_uint64)]
    lib.c2_db_device_bytes.argtypes = [C.c_void_p, C.c_int64, C.c_int32, C.c_int32, P(C.c_uint64)]
    lib.c2_db2bin_lengths.argtypes = [C.c_char_p, _i32p, C.c_char_p, C.c_size_t]
    lib.c2_db2bin_read_range.argtypes = [C.c_char_p, C.c_int32, C.c_int32, _i32p, _i64p, _fp, _fp, _fp, _fp, _fp,
                                         _fp, _fp, _fp, _u8p, _u8p, C.c_char_p, C.c_size_t]
    lib.c2_format_report.argtypes = [C.c_int32, P(c2_report_info), C.c_void_p, C.c_int32, C.c_void_p, C.c_char_p,
                                     P(C.c_size_t)]
    lib.c2_share_db.argtypes = [C.c_void_p, C.c_void_p]
    lib.c2_search_batch.argtypes = [C.c_void_p, P(c2_profiles), C.c_int32, BATCH_CB, C.c_void_p]
    for n in EXPORTS:
        getattr(lib, n).restype = C.c_int
    _lib = lib
    return lib


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


class _Keep:
    """Holds numpy arrays alive while a ctypes struct points into them."""

    def __init__(self):
        self.arrs = []

    def f32(self, x):
        a = np.ascontiguousarray(x, np.float32)
        self.arrs.append(a)
        return _ptr(a, _fp)

    def i32(self, x):
        a = np.ascontiguousarray(x, np.int32)
        self.arrs.append(a)
        return _ptr(a, _i32p)

    def i64(self, x):
        a = np.ascontiguousarray(x, np.int64)
        self.arrs.append(a)
        return _ptr(a, _i64p)

    def u8(self, x):
        a = np.ascontiguousarray(x, np.uint8)
        self.arrs.append(a)
        return _ptr(a, _u8p)


def make_params(p: SearchParams, keep: _Keep) -> c2_params:
    s = c2_params()
    for k in ("ungapped_lambda", "ungapped_K", "ungapped_H", "gapped_lambda", "gapped_K", "gapped_H",
              "gapped_alpha", "gapped_beta", "eval", "ssswgt", "cvswgt", "minpp"):
        setattr(s, k, float(getattr(p, k)))
    s.mapaln, s.x_uninf, s.ssemodel = int(p.mapaln), int(p.x_uninf), int(p.ssemodel)
    s.ssss = keep.f32(p.ssss.reshape(-1))
    s.ssss_card = int(p.ssss_card)
    s.cvs2s_keys = keep.f32(p.cvs2s_keys)
    s.cvs2s_values = keep.f32(p.cvs2s_values)
    s.cvs2s_card = int(p.cvs2s_card)
    s.cvs2s_shift = int(p.cvs2s_shift)
    s.sse_nn_weights = keep.f32(p.sse_nn_weights)
    s.n_sse_nn_weights = int(p.sse_nn_weights.shape[0])
    return s


def make_profiles(ps: ProfileSet, keep: _Keep) -> c2_profiles:
    s = c2_profiles()
    s.nprofiles = ps.nprofiles
    s.npositions = ps.npositions
    s.lengths = keep.i32(ps.lengths)
    s.offsets = keep.i64(ps.offsets)
    s.bkg = keep.f32(ps.bkg)
    s.eno = keep.f32(ps.eno)
    s.trn = keep.f32(ps.trn)
    s.trg = keep.f32(ps.trg)
    s.cv = keep.f32(ps.cv)
    s.cvprior = keep.f32(ps.cvprior)
    s.cvnorm2 = keep.f32(ps.cvnorm2)
    s.ss = keep.f32(ps.ss)
    s.ssstate = keep.u8(ps.ssstate)
    s.aa = keep.u8(ps.aa)
    return s


class C2Error(RuntimeError):
    pass


class Handle:
    """One search context on one GPU (wraps a ``c2_handle``)."""

    def __init__(self, params: SearchParams, device: int = 0):
        self.lib = load()
        self._keep = _Keep()
        self.params = params
        self._h = C.c_void_p()
        sp = make_params(params, self._keep)
        st = self.lib.c2_create(device, C.byref(sp), C.byref(self._h))
        if st != C2_OK:
            raise C2Error("c2_create failed: %s" % STATUS_NAMES.get(st, st))
        self.nprof = 0

    def _ck(self, st, what):
        if st != C2_OK:
            buf = C.create_string_buffer(512)
            self.lib.c2_last_error(self._h, buf, 512)
            raise C2Error("%s: %s: %s" % (what, STATUS_NAMES.get(st, st), buf.value.decode()))

    def close(self):
        if self._h:
            self.lib.c2_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload_db(self, db: ProfileSet, total_positions: int = 0, total_profiles: int = 0):
        k = _Keep()
        s = make_profiles(db, k)
        self._ck(self.lib.c2_upload_db(self._h, C.byref(s), total_positions, total_profiles), "c2_upload_db")
        self.nprof = db.nprofiles

    def set_query(self, q: ProfileSet):
        k = _Keep()
        s = make_profiles(q, k)
        self._ck(self.lib.c2_set_query(self._h, C.byref(s)), "c2_set_query")
        self.Lq = int(q.lengths[0])

    def thresholds(self):
        a, b = C.c_float(), C.c_float()
        self._ck(self.lib.c2_get_thresholds(self._h, C.byref(a), C.byref(b)), "c2_get_thresholds")
        return a.value, b.value

    def run_phase1(self):
        self._ck(self.lib.c2_run_phase1(self._h), "c2_run_phase1")

    def set_stream(self, stream_ptr: int):
        """Issue work on a caller-owned cudaStream_t (e.g. torch.cuda.current_stream().cuda_stream)."""
        self._ck(self.lib.c2_set_stream(self._h, C.c_void_p(stream_ptr)), "c2_set_stream")

    def sync(self):
        self._ck(self.lib.c2_sync(self._h), "c2_sync")

    def logz_fwd(self, profiles, theta=None, wss: float = 0.0, wcv: float = 0.0) -> np.ndarray:
        """Log-partition of the MAP forward model for the current query vs db profiles (c2_logz_fwd)."""
        pr = np.ascontiguousarray(profiles, np.int32)
        th = np.zeros(7, np.float32) if theta is None else np.ascontiguousarray(theta, np.float32)
        out = np.zeros(pr.shape[0], np.float32)
        self._ck(self.lib.c2_logz_fwd(self._h, _ptr(pr, _i32p), int(pr.shape[0]), _ptr(th, _fp),
                                      float(wss), float(wcv), _ptr(out, _fp)), "c2_logz_fwd")
        self._adj_n = int(pr.shape[0])
        self._adj_Lq = np.full(pr.shape[0], self.Lq, np.int64)
        return out

    def set_query_batch(self, queries: ProfileSet):
        """Pack and upload the queries of logz_fwd_batch (c2_set_query_batch)."""
        k = _Keep()
        qs = make_profiles(queries, k)
        self._ck(self.lib.c2_set_query_batch(self._h, C.byref(qs)), "c2_set_query_batch")
        self._adj_qlen = np.asarray(queries.lengths, np.int64).copy()

    def logz_fwd_batch(self, query_of_pair, profiles, theta=None, wss: float = 0.0, wcv: float = 0.0) -> np.ndarray:
        """Log-partition of independent pairs: query query_of_pair[k] of the set_query_batch
        queries vs db profile profiles[k] (c2_logz_fwd_batch)."""
        qi = np.ascontiguousarray(query_of_pair, np.int32)
        pr = np.ascontiguousarray(profiles, np.int32)
        if qi.shape != pr.shape:
            raise C2Error("logz_fwd_batch: query_of_pair and profiles differ in length")
        th = np.zeros(7, np.float32) if theta is None else np.ascontiguousarray(theta, np.float32)
        out = np.zeros(pr.shape[0], np.float32)
        self._ck(self.lib.c2_logz_fwd_batch(self._h, _ptr(qi, _i32p), _ptr(pr, _i32p), int(pr.shape[0]),
                                            _ptr(th, _fp), float(wss), float(wcv), _ptr(out, _fp)),
                 "c2_logz_fwd_batch")
        self._adj_n = int(pr.shape[0])
        self._adj_Lq = self._adj_qlen[qi]
        return out

    def logz_bwd(self) -> np.ndarray:
        """[npairs, 9]: dlogZ/dtheta (7), dlogZ/dwss, dlogZ/dwcv of the last logz_fwd."""
        g = np.zeros((self._adj_n, 9), np.float32)
        self._ck(self.lib.c2_logz_bwd(self._h, _ptr(g, _fp)), "c2_logz_bwd")
        return g

    def logz_cells(self, k: int, L: int):
        """(dlogZ/dS, MM posterior) of pair k, each [Lq][L] (Lq: the pair's query length, L: its db
        profile length)."""
        lq = int(self._adj_Lq[k])
        ds = np.zeros((lq, L), np.float32)
        po = np.zeros((lq, L), np.float32)
        self._ck(self.lib.c2_logz_cells(self._h, int(k), _ptr(ds, _fp), _ptr(po, _fp)), "c2_logz_cells")
        return ds, po

    def set_score_mode(self, mode: int):
        """SCORE_FP32 (CUDA cores) or SCORE_BF16_TC (split-BF16 tensor-core contractions)."""
        self._ck(self.lib.c2_set_score_mode(self._h, mode), "c2_set_score_mode")

    def set_memory_limit(self, nbytes: int):
        """Device memory budget of the handle in bytes, 0 for none (c2_set_device_memory_limit)."""
        self._ck(self.lib.c2_set_device_memory_limit(self._h, int(nbytes)), "c2_set_device_memory_limit")

    def memory_use(self) -> int:
        n = C.c_uint64()
        self._ck(self.lib.c2_get_device_memory_use(self._h, C.byref(n)), "c2_get_device_memory_use")
        return n.value

    def memory_info(self):
        """(free, total) bytes of the handle's device (c2_get_device_memory_info)."""
        f, t = C.c_uint64(), C.c_uint64()
        self._ck(self.lib.c2_get_device_memory_info(self._h, C.byref(f), C.byref(t)), "c2_get_device_memory_info")
        return f.value, t.value

    def db_device_bytes(self, npositions: int, nprofiles: int, max_length: int) -> int:
        """Device bytes an upload of a database of these sizes holds (c2_db_device_bytes)."""
        n = C.c_uint64()
        self._ck(self.lib.c2_db_device_bytes(self._h, npositions, nprofiles, max_length, C.byref(n)),
                 "c2_db_device_bytes")
        return n.value

    def search_groups(self) -> int:
        """Candidate groups the last search ran its phase 2 in (c2_get_search_groups)."""
        n = C.c_int32()
        self._ck(self.lib.c2_get_search_groups(self._h, C.byref(n)), "c2_get_search_groups")
        return n.value

    def set_wait_limit(self, polls: int):
        """Polls before a phase-2 strip wait gives up (0: the default; c2_set_wait_limit)."""
        self._ck(self.lib.c2_set_wait_limit(self._h, int(polls)), "c2_set_wait_limit")

    def phase1(self):
        out = (c2_p1_result * self.nprof)()
        self._ck(self.lib.c2_get_phase1(self._h, out, self.nprof), "c2_get_phase1")
        arr = np.frombuffer(out, dtype=np.dtype([("best", np.float32), ("coords", np.uint32)]), count=self.nprof)
        return arr["best"].copy(), arr["coords"].copy()

    def run_finalize(self) -> int:
        n = C.c_int32()
        self._ck(self.lib.c2_run_finalize(self._h, C.byref(n)), "c2_run_finalize")
        return n.value

    def finalize(self, n: int):
        out = (c2_dp_result * max(n, 1))()
        self._ck(self.lib.c2_get_finalize(self._h, out, n), "c2_get_finalize")
        dt = np.dtype([("score", np.float32), ("profile", np.int32), ("psts", np.int32),
                       ("beg", np.uint32), ("end", np.uint32), ("passed", np.int32)])
        return np.frombuffer(out, dtype=dt, count=n).copy()

    def pair_scores(self, profile: int, L: int):
        """(scores, modular scores), each [Lq][L] float32, of a finalised pair
        of the current query as the device computed them (c2_get_pair_scores)."""
        sm = np.zeros((self.Lq, L), np.float32)
        mm = np.zeros((self.Lq, L), np.float32)
        self._ck(self.lib.c2_get_pair_scores(self._h, int(profile), _ptr(sm, _fp), _ptr(mm, _fp)),
                 "c2_get_pair_scores")
        return sm, mm

    def run_stats(self) -> int:
        n = C.c_int32()
        self._ck(self.lib.c2_run_stats(self._h, C.byref(n)), "c2_run_stats")
        return n.value

    def run_map(self) -> int:
        n = C.c_int32()
        self._ck(self.lib.c2_run_map(self._h, C.byref(n)), "c2_run_map")
        return n.value

    def query_limits(self, query_length: int):
        """(search space, length adjustment, score threshold, log E threshold) of a query
        of this length against the uploaded database (c2_get_query_limits)."""
        a, b = C.c_uint64(), C.c_uint64()
        c, d = C.c_float(), C.c_float()
        self._ck(self.lib.c2_get_query_limits(self._h, int(query_length), C.byref(a), C.byref(b), C.byref(c),
                                              C.byref(d)), "c2_get_query_limits")
        return a.value, b.value, c.value, d.value

    def search_space(self):
        a, b = C.c_uint64(), C.c_uint64()
        self._ck(self.lib.c2_get_search_space(self._h, C.byref(a), C.byref(b)), "c2_get_search_space")
        return a.value, b.value

    def hits(self, n: int):
        """The current hits as a list of dicts (sorted by log E-value), with alignment strings."""
        sz = C.c_size_t(0)
        self._ck(self.lib.c2_get_hits(self._h, None, 0, None, C.byref(sz)), "c2_get_hits(size)")
        arr = (c2_hit * max(n, 1))()
        buf = C.create_string_buffer(max(sz.value, 1))
        self._ck(self.lib.c2_get_hits(self._h, arr, n, buf, C.byref(sz)), "c2_get_hits")
        raw = buf.raw
        out = []
        for i in range(n):
            h = arr[i]
            d = {k: getattr(h, k) for k, _ in c2_hit._fields_}
            o = d.pop("aln_offset")
            L = d["alnlen"]
            d["strings"] = [raw[o + r * (L + 1):o + r * (L + 1) + L].decode() for r in range(5)]
            out.append(d)
        return out

    def hits_arrays(self, n: int):
        """The current hits as (records, alignments): a numpy structured array with
        the c2_hit fields (sorted by log E-value) and the bytes holding each hit's
        five NUL-terminated alignment strings from its aln_offset."""
        sz = C.c_size_t(0)
        self._ck(self.lib.c2_get_hits(self._h, None, 0, None, C.byref(sz)), "c2_get_hits(size)")
        rec = np.zeros(max(n, 1), dtype=HIT_DTYPE)
        buf = np.zeros(max(sz.value, 1), np.uint8)
        self._ck(self.lib.c2_get_hits(self._h, rec.ctypes.data_as(C.POINTER(c2_hit)), n,
                                      buf.ctypes.data_as(C.c_char_p), C.byref(sz)), "c2_get_hits")
        return rec[:n], buf

    def search(self, q: ProfileSet, arrays: bool = False):
        """Complete search of query q over the uploaded database; returns the hits
        as a list of dicts, or with arrays=True as hits_arrays() does."""
        k = _Keep()
        s = make_profiles(q, k)
        n = C.c_int32()
        self._ck(self.lib.c2_search(self._h, C.byref(s), C.byref(n)), "c2_search")
        self.Lq = int(q.lengths[0])
        return self.hits_arrays(n.value) if arrays else self.hits(n.value)

    def search_batch(self, queries: ProfileSet, nworkers: int = 2):
        """Search every profile of queries over the uploaded database with nworkers
        worker handles sharing it (c2_search_batch).  Returns one (records,
        alignments) pair per query, as hits_arrays() gives them."""
        k = _Keep()
        s = make_profiles(queries, k)
        out = [None] * queries.nprofiles
        errs = []

        def cb(user, q, status, hits, nhits, alns, nbytes):
            if status != C2_OK:
                errs.append((q, status))
                return
            rec = np.zeros(nhits, dtype=HIT_DTYPE)
            if nhits:
                C.memmove(rec.ctypes.data, hits, nhits * HIT_DTYPE.itemsize)
            buf = np.zeros(nbytes, np.uint8)
            if nbytes:
                C.memmove(buf.ctypes.data, alns, nbytes)
            out[q] = (rec, buf)

        fn = BATCH_CB(cb)
        self._ck(self.lib.c2_search_batch(self._h, C.byref(s), int(nworkers), fn, None), "c2_search_batch")
        if errs:
            raise C2Error("c2_search_batch: queries failed: %s" % errs)
        return out

    def set_batch_sm_reserve(self, nsm: int):
        """SMs phase 1 leaves to phase 2 in a multi-worker search_batch (-1: default)."""
        self._ck(self.lib.c2_set_batch_sm_reserve(self._h, int(nsm)), "c2_set_batch_sm_reserve")

    def share_db(self, src: "Handle"):
        """Search the database uploaded to src from this handle as well (c2_share_db)."""
        self._ck(self.lib.c2_share_db(self._h, src._h), "c2_share_db")
        self.nprof = src.nprof

    def launch_count(self) -> int:
        n = C.c_uint64()
        self._ck(self.lib.c2_launch_count(self._h, C.byref(n)), "c2_launch_count")
        return n.value


def read_db2bin(path: str, k0: int = 0, k1: int = None):
    """Read a database written by the reference's db2bin (format v2.2), or its
    profiles [k0, k1) only, into a synth.ProfileSet (c2_db2bin_info /
    c2_db2bin_read / c2_db2bin_read_range; no GPU needed)."""
    from .synth import ProfileSet
    lib = load()
    P, N = C.c_int32(), C.c_int64()
    err = C.create_string_buffer(512)
    st = lib.c2_db2bin_info(path.encode(), C.byref(P), C.byref(N), err, 512)
    if st != C2_OK:
        raise C2Error("c2_db2bin_info: %s" % err.value.decode())
    P, N = P.value, N.value
    whole = k0 == 0 and (k1 is None or k1 == P)
    if not whole:
        k1 = P if k1 is None else k1
        if not 0 <= k0 < k1 <= P:
            raise C2Error("profile range [%d, %d) outside the database's %d profiles" % (k0, k1, P))
        every = np.zeros(P, np.int32)
        st = lib.c2_db2bin_lengths(path.encode(), _ptr(every, _i32p), err, 512)
        if st != C2_OK:
            raise C2Error("c2_db2bin_lengths: %s" % err.value.decode())
        P, N = k1 - k0, int(every[k0:k1].astype(np.int64).sum())
    lengths = np.zeros(P, np.int32)
    offsets = np.zeros(P, np.int64)
    bkg = np.zeros((P, 20), np.float32)
    eno = np.zeros(P, np.float32)
    trn = np.zeros((N + P, 7), np.float32)
    trg = np.zeros((N, 20), np.float32)
    cv = np.zeros((N, 19), np.float32)
    cvp = np.zeros(N, np.float32)
    cvn = np.zeros(N, np.float32)
    ss = np.zeros((N, 3), np.float32)
    sss = np.zeros(N, np.uint8)
    aa = np.zeros(N, np.uint8)
    arrays = (_ptr(lengths, _i32p), _ptr(offsets, _i64p), _ptr(bkg, _fp), _ptr(eno, _fp), _ptr(trn, _fp),
              _ptr(trg, _fp), _ptr(cv, _fp), _ptr(cvp, _fp), _ptr(cvn, _fp), _ptr(ss, _fp), _ptr(sss, _u8p),
              _ptr(aa, _u8p), err, 512)
    if whole:
        st = lib.c2_db2bin_read(path.encode(), *arrays)
    else:
        st = lib.c2_db2bin_read_range(path.encode(), k0, k1, *arrays)
    if st != C2_OK:
        raise C2Error("c2_db2bin_read: %s" % err.value.decode())
    return ProfileSet(lengths, offsets, bkg, eno, trn, trg, cv, cvp, cvn, ss, sss, aa,
                      np.zeros((N + P, 7), np.int32), np.zeros((N, 20), np.int32))


def read_db2bin_descriptions(path: str):
    """Profile descriptions of a database written by the reference's db2bin
    (c2_db2bin_descriptions), in the database's profile order."""
    lib = load()
    err = C.create_string_buffer(512)
    n = C.c_size_t(0)
    st = lib.c2_db2bin_descriptions(path.encode(), None, C.byref(n), None, err, 512)
    if st != C2_OK:
        raise C2Error("c2_db2bin_descriptions: %s" % err.value.decode())
    P, N = C.c_int32(), C.c_int64()
    st = lib.c2_db2bin_info(path.encode(), C.byref(P), C.byref(N), err, 512)
    if st != C2_OK:
        raise C2Error("c2_db2bin_info: %s" % err.value.decode())
    buf = C.create_string_buffer(max(n.value, 1))
    off = np.zeros(P.value, np.int64)
    st = lib.c2_db2bin_descriptions(path.encode(), buf, C.byref(n), _ptr(off, _i64p), err, 512)
    if st != C2_OK:
        raise C2Error("c2_db2bin_descriptions: %s" % err.value.decode())
    raw = buf.raw
    return [raw[o:raw.index(b"\0", o)].decode() for o in off]
