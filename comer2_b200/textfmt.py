"""COMER text profile format (v2.0, condensed), writer.

Writes a ``ProfileSet`` profile in the layout of the reference's
``TextWriteProfileCondensed`` (src/libpro/srcpro/PMProfileModel.cpp:2295-2512),
which both of its readers accept (``TextReadProfile``,
src/libpro/srcpro/PMProfileModel.cpp:2756-3960, used by ``makedb``; and
``TextReadProfileHD``-style reading in src/libmycu/cupro/IOProfileModelTxt.cu,
used by ``comer`` for queries).  Values are the integers the synthetic
generator drew (probabilities x 10000), so the reference's readers recover
exactly the float values this package searches with.

Fields this implementation does not use are written with neutral values:
posterior composition = background, MID-state observation counts = 1, one HDP
cluster entry with probability 0 and index -1 (the reference's own entry for
masked positions), and the statistics footer.
"""
from __future__ import annotations

from typing import TextIO

import numpy as np

from .synth import AA, ProfileSet, SCALE

INTSCALE = 1000   # MID-state expected observations scale of the format


def _ints(xs) -> str:
    return "".join(" %d" % int(v) for v in xs)


def write_profile(fp: TextIO, ps: ProfileSet, k: int, name: str, desc: str) -> None:
    L = int(ps.lengths[k])
    o = int(ps.offsets[k])
    t0 = o + k
    bkg = np.rint(ps.bkg[k].astype(np.float64) * SCALE).astype(np.int64)
    fp.write("COMER profile v2.0\n")
    fp.write("DESC: %s\n" % desc)
    fp.write("FILE: %s\n" % name)
    fp.write("CMD: \n")
    fp.write("LEN: %d\n" % L)
    fp.write("NOS: %d\n" % 10)
    fp.write("EFFNOS: %.1f\n" % float(ps.eno[k]))
    fp.write("SCALE: %d\n" % SCALE)
    fp.write("".join(" %c" % c for c in AA.decode()) + "\n")
    fp.write("NULL" + _ints(bkg) + "\n")
    fp.write("POST" + _ints(bkg) + "\n")
    # beginning transitions: 9 values MM MI MD IM II ID DM DI DD (ID, DI = 0)
    def trn9(row):
        t = ps.trn_int[row]
        return [t[0], t[1], t[2], t[3], t[4], 0, t[5], 0, t[6]]
    fp.write(_ints(trn9(t0)) + "\n")
    fp.write(_ints([INTSCALE] * 3))
    for i in range(L):
        pos = o + i
        fp.write("\n%d %c" % (i + 1, chr(ps.aa[pos])) + _ints(ps.trg_int[pos]) + "\n")
        fp.write(_ints(trn9(t0 + i + 1)) + "\n")
        fp.write(_ints([INTSCALE] * 3) + "\n")
        fp.write(" 0 1\n 0\n -1\n")   # one HDP cluster entry, probability 0, index -1
        cv = np.rint(ps.cv[pos].astype(np.float64) * SCALE).astype(np.int64)
        pr = int(np.rint(float(ps.cvprior[pos]) * SCALE))
        n2 = int(np.rint(float(ps.cvnorm2[pos]) * SCALE))
        fp.write(" CV: %d %d %d" % (pr, n2, cv.shape[0]) + _ints(cv) + "\n")
        ss = np.rint(ps.ss[pos].astype(np.float64) * SCALE).astype(np.int64)
        fp.write(" SS:%c" % chr(ps.ssstate[pos]) + _ints(ss))
    fp.write("\n")
    fp.write("K, Lambda:\n")
    fp.write("Computed  ungapped, %6.4f %6.4f\n" % (0.1, 1.0))
    fp.write("Reference ungapped, %6.4f %6.4f\n" % (0.1158, 1.1163))
    fp.write("Entropy, %6.4f; Expected, %6.4f\n" % (0.2, -1.0))
    fp.write("*\n")


def _ivals(line: str):
    return [int(t) for t in line.split()]


def read_profiles(text: str) -> ProfileSet:
    """Read one or more COMER v2.0 text profiles (full or condensed layout).

    Conversions follow the reference's reader (src/libmycu/cupro/IOProfileModelTxt.cu:
    336-371, 480-515, 860-960): probability = int / scale in float32; transition
    value = logf(p) (x 0.4 for IM, II, DM, DD), -32768 for p = 0; ID and DI
    columns are dropped.  HDP and posterior fields are skipped.
    """
    from . import synth as S
    lines = [ln.rstrip("\n") for ln in text.splitlines()]
    profs = []
    i = 0
    n = len(lines)
    while i < n:
        if not lines[i].startswith("COMER profile v"):
            i += 1
            continue
        hdr = {}
        i += 1
        while i < n and not lines[i].startswith("NULL"):
            ln = lines[i].strip()
            for key in ("DESC:", "FILE:", "LEN:", "NOS:", "EFFNOS:", "SCALE:"):
                if ln.startswith(key):
                    hdr[key] = ln[len(key):].strip()
            i += 1
        scale = int(hdr.get("SCALE:", "10000"))
        L = int(hdr["LEN:"])
        bkg = _ivals(lines[i][4:])
        i += 1  # POST
        i += 1
        beg = _ivals(lines[i]); i += 1
        i += 1  # beginning MID observations
        trg = np.zeros((L, 20), np.int64)
        trn = np.zeros((L + 1, 7), np.int64)
        trn[0] = [beg[0], beg[1], beg[2], beg[3], beg[4], beg[6], beg[8]]
        cv = np.zeros((L, 19), np.int64)
        prior = np.zeros(L, np.int64)
        norm2 = np.zeros(L, np.int64)
        ss = np.zeros((L, 3), np.int64)
        sss = np.full(L, ord("C"), np.uint8)
        aa = np.zeros(L, np.uint8)
        for m in range(L):
            while not lines[i].strip():
                i += 1
            toks = lines[i].split()
            assert int(toks[0]) == m + 1, "bad numbering at position %d" % m
            aa[m] = ord(toks[1])
            trg[m] = [int(t) for t in toks[2:22]]
            i += 1
            t9 = _ivals(lines[i]); i += 1
            trn[m + 1] = [t9[0], t9[1], t9[2], t9[3], t9[4], t9[6], t9[8]]
            i += 1  # MID observations (+ weight, information in the full layout)
            nop = _ivals(lines[i])[1]; i += 1
            if nop > 0:
                i += 2
            while i < n and (lines[i].lstrip().startswith("CT:") or lines[i].lstrip().startswith("CV:")
                             or lines[i].lstrip().startswith("SS:")):
                s = lines[i].strip()
                if s.startswith("CV:"):
                    v = _ivals(s[3:])
                    prior[m], norm2[m] = v[0], v[1]
                    cv[m] = v[3:3 + v[2]]
                elif s.startswith("SS:"):
                    sss[m] = ord(s[3])
                    ss[m] = _ivals(s[4:])[:3]
                i += 1
        while i < n and not lines[i].startswith("*"):
            i += 1
        i += 1
        f = lambda q: (q.astype(np.float32) / np.float32(scale)).astype(np.float32)
        P = S.ProfileSet(np.array([L], np.int32), np.zeros(1, np.int64),
                         f(np.array([bkg[:20]])), np.array([float(hdr.get("EFFNOS:", "0"))], np.float32),
                         S._trn_values(trn.astype(np.int32)), f(trg), f(cv), f(prior), f(norm2), f(ss), sss, aa,
                         trn.astype(np.int32), trg.astype(np.int32))
        profs.append(P)
    return S.concat(profs)
