"""Search parameters: statistical constants, option values and score tables.

The search needs four parameter sources, the same ones the reference ``comer``
program reads at start-up:

* ``comer.par`` -- ungapped and gapped Karlin-Altschul constants
  (reference: ``src/env/comer.par``, read by ``Configuration`` /
  ``JobDispatcher::ReadConfiguration``, ``src/libmycu/cualn/JobDispatcher.cpp:152-167``);
* ``options.txt`` -- option keys (``src/libpro/srcpro/MOptions.h:25-76``);
* ``ssss`` -- the secondary-structure state score table, lower-triangular,
  cardinality 30 (parsed as in ``src/libpro/srcpro/SSSScores.cpp`` and
  ``VirtScores::ReadScoresHelper``, ``src/libpro/srcpro/VirtScores.cpp:44-133``);
* ``cvs2s`` -- the context-vector score-to-score map (keys step 0.5), which the
  reader smooths with a 5-wide moving average before use
  (``CVS2Scores::ReadScoresHelper`` / ``SmoothScores``,
  ``src/libpro/srcpro/CVS2Scores.cpp``).

The parsers below accept those file formats, so a user's own ``var/`` files can
be loaded.  The package ships the numbers of the reference's default files in
``data/comer2_params.json`` (GPL-3 data of the COMER2 project; see
``data/gen_params.py``), and ``load_default()`` reads them.
"""
from __future__ import annotations

import json
import math
import os
import re
from dataclasses import dataclass, field
from typing import Dict, List, Sequence, Tuple

import numpy as np

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "comer2_params.json")

# value the cvs2s reader assigns to a '+' entry (CVS2Scores::plusval_)
CVS2S_PLUS = 9999.0
CVS2S_NA = -9999.0


@dataclass
class SearchParams:
    # [UNGAPPED] and [GAPPED_A_1] sections of comer.par
    ungapped_lambda: float = 1.116276
    ungapped_K: float = 0.115812
    ungapped_H: float = 0.218508
    gapped_lambda: float = 0.561132
    gapped_K: float = 0.001488
    gapped_H: float = 0.158085
    gapped_alpha: float = 0.5
    gapped_beta: float = -1.0
    # options.txt keys on the search path
    eval: float = 10.0
    ssswgt: float = 0.12
    cvswgt: float = 0.15
    mapaln: int = 1
    minpp: float = 0.28
    x_uninf: int = 1
    ssemodel: int = 2
    nohits: int = 700
    noalns: int = 700
    # SS score table: full symmetric card x card matrix (row-major, float32)
    ssss_card: int = 30
    ssss: np.ndarray = field(default_factory=lambda: np.zeros((30, 30), np.float32))
    # context-vector score map after smoothing (keys step 0.5)
    cvs2s_keys: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    cvs2s_values: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    cvs2s_shift: int = 0
    # SS18 E-value model: NN weights and adjustment constants, in the order the
    # statistics kernels index them
    sse_nn_weights: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))

    @property
    def cvs2s_card(self) -> int:
        return int(self.cvs2s_keys.shape[0])


# ---------------------------------------------------------------------------
# tokenisation helpers: the reference's readers skip lines whose first
# non-blank character is '#'
def _lines(text: str) -> List[str]:
    out = []
    for ln in text.splitlines():
        s = ln.strip()
        if not s or s.startswith("#"):
            continue
        out.append(s)
    return out


def parse_comer_par(text: str) -> Dict[str, Dict[str, float]]:
    """Parse ``comer.par`` into {section: {key: value}}."""
    sec = None
    res: Dict[str, Dict[str, float]] = {}
    for s in _lines(text):
        m = re.match(r"^\[(\w+)\]$", s)
        if m:
            sec = m.group(1)
            res[sec] = {}
            continue
        if sec is None or "=" not in s:
            continue
        k, v = s.split("=", 1)
        try:
            res[sec][k.strip()] = float(v.split()[0])
        except ValueError:
            pass
    return res


def parse_options(text: str) -> Dict[str, str]:
    """Parse an ``options.txt`` file into {KEY: value-string}."""
    res: Dict[str, str] = {}
    for s in _lines(text):
        if s.startswith("["):
            continue
        if "=" in s:
            k, v = s.split("=", 1)
            res[k.strip()] = v.split()[0] if v.split() else ""
    return res


def parse_ssss(text: str) -> Tuple[int, List[float]]:
    """Parse the single-table ``ssss`` file.

    Returns the cardinality and the lower-triangular entries in file order
    (row r holds r+1 values), as ``VirtScores::ReadScoresHelper`` reads them.
    """
    ls = _lines(text)
    i = 0
    while i < len(ls) and "Cardinality" not in ls[i]:
        i += 1
    if i == len(ls):
        raise ValueError("ssss: no Cardinality line")
    card = int(ls[i].split("=")[1].split()[0])
    tri: List[float] = []
    for r in range(card):
        toks = ls[i + 1 + r].split()
        if len(toks) < r + 1:
            raise ValueError("ssss: short row %d" % r)
        tri.extend(CVS2S_NA if t == "NA" else float(t) for t in toks[: r + 1])
    return card, tri


def ssss_full(card: int, tri: Sequence[float]) -> np.ndarray:
    """Expand the triangular table into a symmetric card x card matrix.

    Index rule of ``SerializedScoresSM::GetScoreP1E1``
    (``src/libmycu/cupro/SerializedScoresSM.cuh:103-120``): with row >= col the
    entry is tri[row*(row+1)/2 + col].
    """
    m = np.zeros((card, card), np.float32)
    for r in range(card):
        for c in range(r + 1):
            v = np.float32(tri[r * (r + 1) // 2 + c])
            m[r, c] = v
            m[c, r] = v
    return m


def parse_cvs2s(text: str) -> Tuple[List[float], List[float]]:
    """Parse the single-table ``cvs2s`` file: keys and raw scores ('+' -> 9999)."""
    ls = _lines(text)
    i = 0
    while i < len(ls) and "Cardinality" not in ls[i]:
        i += 1
    if i == len(ls):
        raise ValueError("cvs2s: no Cardinality line")
    card = int(ls[i].split("=")[1].split()[0])
    keys = [float(t) for t in ls[i + 1].split()[:card]]
    vals = [CVS2S_PLUS if t == "+" else float(t) for t in ls[i + 2].split()[:card]]
    if len(keys) != card or len(vals) != card:
        raise ValueError("cvs2s: short key/score rows")
    return keys, vals


def smooth_cvs2s(keys: Sequence[float], vals: Sequence[float], step: int = 2):
    """Smooth the CV score map as ``CVS2Scores::SmoothScores`` does.

    A 5-wide running mean (float32 arithmetic) over the scores that are not '+',
    assigned back to every entry (the reference keeps the smoothed value for
    all entries, nSLAST=9999), then missing keys are inserted at ``1/step``
    spacing, '+' entries take the smoothed value, and the shift is the number
    of negative keys.  Returns (keys, values, shift) as float32 arrays.
    """
    f32 = np.float32
    keys = [f32(k) for k in keys]
    scos = [f32(v) for v in vals]
    n_el = len(scos)
    incr = f32(1.0) / f32(step)
    nswin, nswinh = 5, 2
    smth = [f32(0.0)] * n_el
    rwin = [f32(0.0)] * nswin
    rsum = f32(0.0)
    avg = f32(0.0)
    nv = rn = nn = 0

    def plus(v):
        return v >= f32(CVS2S_PLUS)

    for n in range(n_el):
        sc = scos[n]
        if sc <= f32(CVS2S_NA):
            raise ValueError("cvs2s: NA score")
        if nv < nswinh:
            nn += 1
        if not plus(sc):
            if nswin <= rn:
                rn = 0
            rsum = f32(rsum - rwin[rn])
            rwin[rn] = sc
            rn += 1
            rsum = f32(rsum + sc)
            avg = f32(rsum / f32(nswin))
            nv += 1
        if nswin <= nv:
            if not plus(sc):
                if nswin == nv:
                    for p in range(nn):
                        smth[p] = avg
                smth[nn] = avg
                nn += 1
                while nn < n and plus(scos[nn]):
                    smth[nn] = avg
                    nn += 1
            if n_el == n + 1:
                for p in range(nn, n_el):
                    smth[p] = avg
    # every entry takes its smoothed value; sm ends as smth[0]
    sm = f32(0.0)
    for n in range(n_el - 1, -1, -1):
        sm = smth[n]
        scos[n] = sm
    # insert missing keys
    out_k, out_v = [], []
    pkk = f32(0.0)
    n = 0
    k_list, v_list, s_list = list(keys), list(scos), list(smth)
    while n < len(k_list):
        kk, sc = k_list[n], v_list[n]
        if n and kk <= pkk:
            raise ValueError("cvs2s: keys not sorted")
        if n and incr < f32(kk - pkk):
            pkk = f32(pkk + incr)
            k_list.insert(n, pkk)
            v_list.insert(n, sm)
            s_list.insert(n, sm)
            n += 1
            continue
        pkk = kk
        sm = s_list[n]
        if plus(sc):
            v_list[n] = sm
        n += 1
    shift = 0
    for k in k_list:
        if f32(0.0) <= k:
            break
        shift += 1
    return np.array(k_list, np.float32), np.array(v_list, np.float32), shift


def from_dict(d: dict) -> SearchParams:
    p = SearchParams()
    un, ga = d["comer_par"]["UNGAPPED"], d["comer_par"]["GAPPED_A_1"]
    p.ungapped_lambda, p.ungapped_K, p.ungapped_H = un["Lambda"], un["K"], un["H"]
    p.gapped_lambda, p.gapped_K, p.gapped_H = ga["Lambda"], ga["K"], ga["H"]
    p.gapped_alpha, p.gapped_beta = ga["Alpha"], ga["Beta"]
    o = d["options"]
    p.eval = float(o.get("EVAL", p.eval))
    p.ssswgt = float(o.get("SSSWGT", p.ssswgt))
    p.cvswgt = float(o.get("CVSWGT", p.cvswgt))
    p.mapaln = int(o.get("MAPALN", p.mapaln))
    p.minpp = float(o.get("MINPP", p.minpp))
    p.x_uninf = int(o.get("X_UNINF", p.x_uninf))
    p.ssemodel = int(o.get("SSEMODEL", p.ssemodel))
    p.nohits = int(o.get("NOHITS", p.nohits))
    p.noalns = int(o.get("NOALNS", p.noalns))
    p.ssss_card = int(d["ssss"]["card"])
    p.ssss = ssss_full(p.ssss_card, d["ssss"]["tri"])
    k, v, s = smooth_cvs2s(d["cvs2s"]["keys"], d["cvs2s"]["values"])
    p.cvs2s_keys, p.cvs2s_values, p.cvs2s_shift = k, v, s
    p.sse_nn_weights = np.array(d["sse_nn_weights"], np.float32)
    return p


def load_default() -> SearchParams:
    """Parameters of the reference's default install (with SCOADJ = no)."""
    with open(_DATA) as fh:
        return from_dict(json.load(fh))


def load_files(comer_par: str, options: str, ssss: str, cvs2s: str, base: SearchParams = None) -> SearchParams:
    """Build parameters from reference-format files (a ``var/`` directory)."""
    def rd(p):
        with open(p) as fh:
            return fh.read()
    d = {
        "comer_par": parse_comer_par(rd(comer_par)),
        "options": parse_options(rd(options)),
    }
    card, tri = parse_ssss(rd(ssss))
    d["ssss"] = {"card": card, "tri": tri}
    kk, vv = parse_cvs2s(rd(cvs2s))
    d["cvs2s"] = {"keys": kk, "values": vv}
    d["sse_nn_weights"] = list((base or load_default()).sse_nn_weights)
    return from_dict(d)
