"""ctypes binding of the CPU oracle (test infrastructure only).

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
checker; the product never imports this module.  ``build()`` compiles the two
oracle variants (float: reference operation order; double: FP64 error
reference) with the Makefile next to this file.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")


def build():
    """Build the oracle; with COMER2_REFERENCE naming the reference's source
    tree, also the helpers compiled from its own sources (oracle/_ref)."""
    cmd = ["make", "-s", "-C", HERE]
    if os.environ.get("COMER2_REFERENCE"):
        cmd.append("REF=" + os.environ["COMER2_REFERENCE"])
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)


_fp = C.POINTER(C.c_float)
_u8p = C.POINTER(C.c_uint8)


class orc_params(C.Structure):
    _fields_ = [("ssswgt", C.c_float), ("cvswgt", C.c_float), ("mapaln", C.c_int),
                ("ssss", _fp), ("ssss_card", C.c_int), ("cvkeys", _fp), ("cvvals", _fp),
                ("cvcard", C.c_int), ("cvshift", C.c_int),
                ("cv_lokappa0", C.c_float), ("cv_pownu0", C.c_float), ("cv_cterm", C.c_float)]


class orc_profile(C.Structure):
    _fields_ = [("len", C.c_int), ("eno", C.c_float), ("bkg", _fp), ("trn", _fp), ("trg", _fp),
                ("cv", _fp), ("cvprior", _fp), ("cvnorm2", _fp), ("ss", _fp), ("aa", _u8p)]


class orc_stats_in(C.Structure):
    _fields_ = [("ssemodel", C.c_int), ("nq", C.c_int), ("nd", C.c_int), ("qeno", C.c_float),
                ("deno", C.c_float), ("searchspace", C.c_float), ("reflambda", C.c_float),
                ("refK", C.c_float), ("expglambda", C.c_float), ("expgK", C.c_float),
                ("nnw", _fp), ("score", C.c_float), ("psts", C.c_float)]


def _stats_out(rt):
    class orc_stats_out(C.Structure):
        _fields_ = [(n, rt) for n in ("min", "max", "E", "H", "lambda_", "K", "lambda_est", "K_est",
                                      "logE", "logEpA", "mu", "scale")]
    return orc_stats_out


def _map_out(rt):
    class orc_map_out(C.Structure):
        _fields_ = [("logZ", rt), ("maxF", rt), ("mapmax", rt)] + [
            (n, C.c_int) for n in ("endx", "endy", "begx", "begy", "alnlen", "idts", "psts", "gaps")]
    return orc_map_out


class Oracle:
    """One oracle variant: bits=32 (float) or bits=64 (double)."""

    def __init__(self, params, bits: int = 32):
        path = os.path.join(BUILD, "liborc%d.so" % bits)
        if not os.path.exists(path):
            build()
        self.lib = C.CDLL(path)
        self.bits = bits
        self.rt = np.float32 if bits == 32 else np.float64
        self.crt = C.c_float if bits == 32 else C.c_double
        rp = C.POINTER(self.crt)
        L = self.lib
        L.orc_cv_constants.argtypes = [_fp, _fp, _fp]
        L.orc_score_matrix.argtypes = [C.POINTER(orc_params), C.POINTER(orc_profile), C.POINTER(orc_profile), rp, rp]
        L.orc_score_cell.argtypes = [C.POINTER(orc_params), C.POINTER(orc_profile), C.POINTER(orc_profile),
                                     C.c_int, C.c_int, rp, rp, rp, rp, rp]
        L.orc_dp.argtypes = [C.POINTER(orc_params), C.POINTER(orc_profile), C.POINTER(orc_profile), rp,
                             rp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                             C.POINTER(C.c_int8)]
        L.orc_finalize.argtypes = [rp, C.POINTER(C.c_int8), C.c_int, C.c_int, self.crt, C.c_int, C.c_int,
                                   rp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_score_threshold.argtypes = [C.c_size_t, C.c_size_t, C.c_float, C.c_float, C.c_float, _fp, _fp]
        L.orc_length_adjustment.argtypes = [C.c_float, C.c_float, C.c_float, C.c_float, C.c_size_t,
                                            C.c_ulonglong, C.c_size_t, C.POINTER(C.c_ulonglong),
                                            C.POINTER(C.c_ulonglong)]
        L.orc_logz.argtypes = [C.POINTER(orc_profile), C.POINTER(orc_profile), rp, rp]
        L.orc_logz.restype = self.crt
        L.orc_score_parts.argtypes = [C.POINTER(orc_params), C.POINTER(orc_profile), C.POINTER(orc_profile),
                                      rp, rp, rp]
        self.StatsOut = _stats_out(self.crt)
        self.MapOut = _map_out(self.crt)
        L.orc_stats.argtypes = [C.POINTER(orc_stats_in), rp, _u8p, _u8p, C.c_int, C.POINTER(self.StatsOut)]
        L.orc_significance.argtypes = [C.POINTER(orc_stats_in), self.crt, self.crt, C.POINTER(self.StatsOut)]
        L.orc_map.argtypes = [C.POINTER(orc_profile), C.POINTER(orc_profile), rp, rp, self.crt, self.crt,
                              C.c_int, _u8p, _u8p, rp, C.c_char_p, C.POINTER(self.MapOut)]
        L.orc_set_map_exact.argtypes = [C.c_int]
        L.orc_lbetainc.argtypes = [self.crt] * 3
        L.orc_lbetainc.restype = self.crt
        L.orc_lgammainc_Q.argtypes = [self.crt] * 2
        L.orc_lgammainc_Q.restype = self.crt
        L.orc_batch_phase1.argtypes = [C.POINTER(orc_params), C.POINTER(orc_profile), C.POINTER(orc_profile),
                                       C.c_int, C.c_int, self.crt, rp, rp]
        self._keep = []
        self.params = params
        self.P = self._make_params(params)

    def _f32(self, a):
        a = np.ascontiguousarray(a, np.float32)
        self._keep.append(a)
        return a.ctypes.data_as(_fp)

    def _make_params(self, p):
        s = orc_params()
        s.ssswgt, s.cvswgt, s.mapaln = float(p.ssswgt), float(p.cvswgt), int(p.mapaln)
        s.ssss = self._f32(p.ssss.reshape(-1))
        s.ssss_card = int(p.ssss_card)
        s.cvkeys = self._f32(p.cvs2s_keys)
        s.cvvals = self._f32(p.cvs2s_values)
        s.cvcard, s.cvshift = int(p.cvs2s_card), int(p.cvs2s_shift)
        a, b, c = C.c_float(), C.c_float(), C.c_float()
        self.lib.orc_cv_constants(C.byref(a), C.byref(b), C.byref(c))
        s.cv_lokappa0, s.cv_pownu0, s.cv_cterm = a.value, b.value, c.value
        return s

    def profile(self, ps, k: int = 0):
        """orc_profile view of profile k of a ProfileSet (arrays kept alive)."""
        L = int(ps.lengths[k])
        o = int(ps.offsets[k])
        keep = []

        def f(a):
            a = np.ascontiguousarray(a, np.float32)
            keep.append(a)
            return a.ctypes.data_as(_fp)

        s = orc_profile()
        s.len = L
        s.eno = float(ps.eno[k])
        s.bkg = f(ps.bkg[k])
        s.trn = f(ps.trn[o + k:o + k + L + 1])
        s.trg = f(ps.trg[o:o + L])
        s.cv = f(ps.cv[o:o + L])
        s.cvprior = f(ps.cvprior[o:o + L])
        s.cvnorm2 = f(ps.cvnorm2[o:o + L])
        s.ss = f(ps.ss[o:o + L])
        aa = np.ascontiguousarray(ps.aa[o:o + L], np.uint8)
        keep.append(aa)
        s.aa = aa.ctypes.data_as(_u8p)
        s._keep = keep
        return s

    def score_matrix(self, q, d):
        Lq, Ld = q.len, d.len
        S = np.zeros((Lq, Ld), self.rt)
        M = np.zeros((Lq, Ld), self.rt)
        rp = C.POINTER(self.crt)
        self.lib.orc_score_matrix(C.byref(self.P), C.byref(q), C.byref(d), S.ctypes.data_as(rp),
                                  M.ctypes.data_as(rp))
        return S, M

    def score_parts(self, q, d):
        """Amino-acid score and the SS and CV terms before their weights, [Lq][Ld] each."""
        sh = (q.len, d.len)
        S0, SS, CV = (np.zeros(sh, self.rt) for _ in range(3))
        rp = C.POINTER(self.crt)
        self.lib.orc_score_parts(C.byref(self.P), C.byref(q), C.byref(d), S0.ctypes.data_as(rp),
                                 SS.ctypes.data_as(rp), CV.ctypes.data_as(rp))
        return S0, SS, CV

    def logz(self, q, d, S, theta=None):
        """Exact log-partition of the MAP forward model over S (theta: 7 query transition offsets)."""
        S = np.ascontiguousarray(S, self.rt)
        th = np.zeros(7, self.rt) if theta is None else np.ascontiguousarray(theta, self.rt)
        rp = C.POINTER(self.crt)
        return float(self.lib.orc_logz(C.byref(q), C.byref(d), S.ctypes.data_as(rp), th.ctypes.data_as(rp)))

    def dp(self, q, d, S, with_btck: bool = False):
        S = np.ascontiguousarray(S, self.rt)
        best = self.crt()
        x, y, nt = C.c_int(), C.c_int(), C.c_int()
        bt = np.zeros((q.len, d.len), np.int8) if with_btck else None
        btp = bt.ctypes.data_as(C.POINTER(C.c_int8)) if with_btck else None
        self.lib.orc_dp(C.byref(self.P), C.byref(q), C.byref(d), S.ctypes.data_as(C.POINTER(self.crt)),
                        C.byref(best), C.byref(x), C.byref(y), C.byref(nt), btp)
        return best.value, x.value, y.value, nt.value, bt

    def finalize(self, S, bt, maxsc, x, y):
        S = np.ascontiguousarray(S, self.rt)
        Lq, Ld = S.shape
        sc = self.crt()
        ps, bx, by = C.c_int(), C.c_int(), C.c_int()
        self.lib.orc_finalize(S.ctypes.data_as(C.POINTER(self.crt)), bt.ctypes.data_as(C.POINTER(C.c_int8)),
                              Lq, Ld, maxsc, x, y, C.byref(sc), C.byref(ps), C.byref(bx), C.byref(by))
        return sc.value, ps.value, bx.value, by.value

    def pair(self, q, d):
        """Phase 1 + finalisation of one pair: dict of results."""
        S, M = self.score_matrix(q, d)
        best, x, y, nt, bt = self.dp(q, d, S, with_btck=True)
        out = {"S": S, "MOD": M, "best": best, "x": x, "y": y, "nties": nt, "btck": bt}
        if best > 0:
            sc, ps, bx, by = self.finalize(S, bt, best, x, y)
            out.update(score=sc, psts=ps, begx=bx, begy=by)
        return out

    def stats(self, S, qaa, daa, score, psts, qeno, deno, searchspace, xuninf=1):
        """Statistics of one passed pair; S is the pair's [nq, nd] score matrix."""
        p = self.params
        S = np.ascontiguousarray(S, self.rt)
        nq, nd = S.shape
        si = orc_stats_in(int(p.ssemodel), nq, nd, float(qeno), float(deno), float(searchspace),
                          float(p.ungapped_lambda), float(p.ungapped_K), float(p.gapped_lambda),
                          float(p.gapped_K), self._f32(p.sse_nn_weights), float(score), float(psts))
        qa = np.ascontiguousarray(qaa, np.uint8)
        da = np.ascontiguousarray(daa, np.uint8)
        o = self.StatsOut()
        self.lib.orc_stats(C.byref(si), S.ctypes.data_as(C.POINTER(self.crt)), qa.ctypes.data_as(_u8p),
                           da.ctypes.data_as(_u8p), xuninf, C.byref(o))
        return {k: getattr(o, k) for k, _ in o._fields_}

    def significance(self, nq, nd, score, psts, qeno, deno, searchspace, lambda_, K):
        """log E-values of one pair from given computed ungapped lambda and K
        (<= 0: failed): dict with lambda_est, K_est, logEpA, mu, scale, logE."""
        p = self.params
        si = orc_stats_in(int(p.ssemodel), int(nq), int(nd), float(qeno), float(deno), float(searchspace),
                          float(p.ungapped_lambda), float(p.ungapped_K), float(p.gapped_lambda),
                          float(p.gapped_K), self._f32(p.sse_nn_weights), float(score), float(psts))
        o = self.StatsOut()
        self.lib.orc_significance(C.byref(si), lambda_, K, C.byref(o))
        return {k: getattr(o, k) for k in ("lambda_est", "K_est", "logEpA", "mu", "scale", "logE")}

    def map(self, q, d, S, MOD, logepa, qss=None, dss=None, exact=False, with_post=False):
        """MAP alignment of one pair: dict with logZ, coordinates, counts and strings."""
        p = self.params
        S = np.ascontiguousarray(S, self.rt)
        MOD = np.ascontiguousarray(MOD, self.rt)
        nq, nd = S.shape
        post = np.zeros((nq, nd), self.rt) if with_post else None
        cap = nq + nd + 1
        aln = C.create_string_buffer(5 * cap)
        keep = []

        def u8(a):
            if a is None:
                return None
            a = np.ascontiguousarray(a, np.uint8)
            keep.append(a)
            return a.ctypes.data_as(_u8p)

        self.lib.orc_set_map_exact(1 if exact else 0)
        o = self.MapOut()
        rp = C.POINTER(self.crt)
        self.lib.orc_map(C.byref(q), C.byref(d), S.ctypes.data_as(rp), MOD.ctypes.data_as(rp), logepa,
                         float(p.minpp), 1, u8(qss), u8(dss), post.ctypes.data_as(rp) if with_post else None,
                         aln, C.byref(o))
        self.lib.orc_set_map_exact(0)
        out = {k: getattr(o, k) for k, _ in o._fields_}
        raw = aln.raw
        out["strings"] = [raw[r * cap:r * cap + out["alnlen"]].decode() for r in range(5)]
        if with_post:
            out["post"] = post
        return out

    def batch_phase1(self, q, db, ks, nthreads, thld):
        """Phase 1 + finalisation of query q against db profiles ks on nthreads host threads."""
        profs = (orc_profile * len(ks))()
        keep = []
        for i, k in enumerate(ks):
            pr = self.profile(db, int(k))
            keep.append(pr)
            profs[i] = pr
        best = np.zeros(len(ks), self.rt)
        score = np.zeros(len(ks), self.rt)
        rp = C.POINTER(self.crt)
        self.lib.orc_batch_phase1(C.byref(self.P), C.byref(q), profs, len(ks), int(nthreads), thld,
                                  best.ctypes.data_as(rp), score.ctypes.data_as(rp))
        return best, score

    def score_threshold(self, nq, dbsize, eval_, gK, glambda):
        a, b = C.c_float(), C.c_float()
        self.lib.orc_score_threshold(nq, dbsize, eval_, gK, glambda, C.byref(a), C.byref(b))
        return a.value, b.value

    def length_adjustment(self, lam, K, alpha, beta, m, n, N):
        ss, dl = C.c_ulonglong(), C.c_ulonglong()
        self.lib.orc_length_adjustment(lam, K, alpha, beta, m, n, N, C.byref(ss), C.byref(dl))
        return ss.value, dl.value
