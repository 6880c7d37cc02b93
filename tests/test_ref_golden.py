"""Golden results of the reference itself: its own comer program, built for
sm_100a from its sources (oracle/build_ref.sh) and run on a B200 on three
seeded workloads (tests/golden/make_ref_fixtures.py: prepare, run, collect).

On this hardware and toolkit that build gives valid results only with the
secondary-structure and context-vector score terms off (SSSWGT = CVSWGT = 0;
tests/golden/ref_b200_outcome.json: with the SS term on, its score matrix
holds invalid cells and every reported score is non-finite), and even then
its computed ungapped lambda, K and entropy of a pair are not valid: most are
reported as failed ("n/a"), the others implausible (entropy 222.9 where the
score distribution gives 1.80), and two runs of the same input report
different values.  The fixtures (ref_<case>_w00_plain.json, its Plain result
files, every field of every hit) therefore pin the method stage by stage:

* DP score (phase 1 + finalisation, printed %.2f): within 0.006;
* expected score and score range of the pair's score distribution: exact to
  the printed digits;
* given the lambda and K the reference computed for the pair (as printed;
  "n/a" = its failure values), the E-value (SS18 model) and bit score within
  the printed precision, and the MAP alignment -- query, middle and target
  rows, identities, positives, gaps, coordinates -- identical.

Here the oracle (the CPU restatement every GPU test checks against) is
pinned that way; tests/test_gpu_search.py checks the CUDA path against the
same fixtures."""
import copy
import json
import math
import os

import numpy as np
import pytest

from comer2_b200 import synth as S

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ("c1_s2", "c1_s9", "c0_s4")
LAMBDA_FAIL, K_FAIL = -32.0, -1.0   # a failed computation: -1 in scaled units, times the scale 32; K -1


VARIANTS = ("w00", "w00aln0")   # SS and CV weights 0; MAP alignments / MAPALN 0 (Viterbi alignments)


def load_fixture(case, variant="w00"):
    with open(os.path.join(HERE, "golden", "ref_%s_%s_plain.json" % (case, variant))) as fh:
        return json.load(fh)


def fixture_params(params, fx):
    p = copy.deepcopy(params)
    p.ssswgt = np.float32(fx["ssswgt"])
    p.cvswgt = np.float32(fx["cvswgt"])
    p.mapaln = int(fx.get("mapaln", 1))
    return p


def fixture_workload(fx):
    n, seed, scale = fx["config"]
    return S.config(n, seed=seed, scale=scale)


def ref_lambda_K(r):
    lam = r["computed_lambda_ungapped"]
    K = r["computed_K_ungapped"]
    return (LAMBDA_FAIL if lam == "n/a" else float(lam)), (K_FAIL if K == "n/a" else float(K))


def search_space(orc, prm, w):
    q = w.queries[0]
    return orc.length_adjustment(prm.gapped_lambda, prm.gapped_K, prm.gapped_alpha, prm.gapped_beta,
                                 int(q.lengths[0]), int(w.db.lengths.sum()), int(w.db.nprofiles))[0]


def viterbi_alignment(bt, S, qaa, daa, qss, dss, x, y):
    """The Viterbi DP's own alignment (MAPALN 0): the walk from the DP
    maximum (x, y) through the traceback codes, as FinalizeDP_ALN draws it
    (src/libmycu/cudp/CuBatchDP_aln_final.cu:240-360): query, middle and
    target rows and the SS rows, identities, non-identical positives, gaps,
    0-based first cell and the end cell.  bt, S: [Lq][L]."""
    STOP, LEFT, UP = 0, 1, 2
    end = (x, y)
    q, m, t, sq, st = [], [], [], [], []
    idts = psts = gaps = 0
    while x >= 0 and y >= 0:
        b = int(bt[y, x])
        if b == STOP:
            break
        if b == UP:
            gaps += 1
            q.append(chr(qaa[y])); t.append("-"); m.append(" "); sq.append(chr(qss[y])); st.append(" ")
            y -= 1
            continue
        if b == LEFT:
            gaps += 1
            q.append("-"); t.append(chr(daa[x])); m.append(" "); sq.append(" "); st.append(chr(dss[x]))
            x -= 1
            continue
        cq, cd = chr(qaa[y]), chr(daa[x])
        q.append(cq); t.append(cd); sq.append(chr(qss[y])); st.append(chr(dss[x]))
        if cq == cd:
            m.append(cq)
            idts += 1
        elif S[y, x] > 0:
            m.append("+")
            psts += 1
        else:
            m.append(" ")
        x -= 1
        y -= 1
    rows = ["".join(reversed(r)) for r in (q, m, t, sq, st)]
    return rows, len(q), idts, psts, gaps, (x + 1, y + 1), end


def check_alignment(r, strings, alnlen, idts, psts, gaps, beg, end):
    """One hit's MAP alignment against the fixture record (beg/end: (x, y)
    of the first and last aligned cells, 0-based; the Plain file prints
    1-based first and last residues)."""
    k = r["profile"]
    assert (strings[0], strings[1], strings[2]) == (r["query_aln"], r["middle"], r["target_aln"]), k
    assert (alnlen, idts, psts, gaps) == (r["aln_length"], r["n_identities"], r["n_positives"], r["n_gaps"]), k
    assert (beg[1] + 1, beg[0] + 1) == (r["query_from"], r["target_from"]), k
    assert (end[1] + 1, end[0] + 1) == (r["query_to"], r["target_to"]), k


def check_evalue(r, logE, searchspace):
    k = r["profile"]
    assert math.exp(logE) == pytest.approx(r["evalue"], rel=0.051), (k, math.exp(logE), r["evalue"])
    bits = (math.log(np.float32(searchspace)) - logE) / math.log(2.0)
    assert abs(bits - r["bit_score"]) <= 0.051, (k, bits, r["bit_score"])


def oracle_alignment(orc, prm, qo, do, x, q, w, off, nd, logepa):
    """The hit's alignment as the reference's configuration draws it: MAP
    (MAPALN 1) or the Viterbi DP's own (MAPALN 0)."""
    if prm.mapaln:
        m = orc.map(qo, do, x["S"], x["MOD"], logepa, qss=q.ssstate, dss=w.db.ssstate[off:off + nd])
        return m["strings"], m["alnlen"], m["idts"], m["psts"], m["gaps"], (m["begx"], m["begy"]), (m["endx"], m["endy"])
    return viterbi_alignment(x["btck"], x["S"], q.aa, w.db.aa[off:off + nd], q.ssstate, w.db.ssstate[off:off + nd],
                             x["x"], x["y"])


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_the_reference_run(params, case, variant):
    from oracle_py import Oracle
    fx = load_fixture(case, variant)
    assert fx["n_hits"] == len(fx["hits"]) > 0
    prm = fixture_params(params, fx)
    w = fixture_workload(fx)
    orc = Oracle(prm, 32)
    q = w.queries[0]
    qo = orc.profile(q)
    Lq = int(q.lengths[0])
    ss = search_space(orc, prm, w)
    for r in fx["hits"]:
        k = r["profile"]
        off, nd = int(w.db.offsets[k]), int(w.db.lengths[k])
        assert (nd, round(float(w.db.eno[k]), 1)) == (r["target_length"], r["target_eno"])
        do = orc.profile(w.db, k)
        x = orc.pair(qo, do)
        assert abs(x["score"] - r["score"]) <= 0.006, (k, x["score"], r["score"])
        st = orc.stats(x["S"], q.aa, w.db.aa[off:off + nd], x["score"], x["psts"], q.eno[0], w.db.eno[k], float(ss),
                       prm.x_uninf)
        assert abs(st["E"] - r["expected_score"]) <= 6e-5, (k, st["E"], r["expected_score"])
        assert (st["min"], st["max"]) == (r["min_score"], r["max_score"]), k
        lam, K = ref_lambda_K(r)
        sg = orc.significance(Lq, nd, x["score"], x["psts"], q.eno[0], w.db.eno[k], ss, lam, K)
        check_evalue(r, sg["logE"], ss)
        check_alignment(r, *oracle_alignment(orc, prm, qo, do, x, q, w, off, nd, sg["logEpA"]))


@pytest.mark.parametrize("case", CASES)
def test_oracle_statistics_are_valid_where_the_reference_failed(params, case):
    """The oracle's own lambda, K and entropy of the same pairs: positive,
    finite and plausible for natural-log-odds scores (lambda near 1), where
    the reference's run reported failures or implausible values."""
    from oracle_py import Oracle
    fx = load_fixture(case)
    prm = fixture_params(params, fx)
    w = fixture_workload(fx)
    orc = Oracle(prm, 32)
    q = w.queries[0]
    qo = orc.profile(q)
    ss = search_space(orc, prm, w)
    for r in fx["hits"]:
        k = r["profile"]
        off, nd = int(w.db.offsets[k]), int(w.db.lengths[k])
        x = orc.pair(qo, orc.profile(w.db, k))
        st = orc.stats(x["S"], q.aa, w.db.aa[off:off + nd], x["score"], x["psts"], q.eno[0], w.db.eno[k], float(ss),
                       prm.x_uninf)
        assert 0.9 < st["lambda_"] < 1.1 and 0.3 < st["K"] < 0.6 and 1.5 < st["H"] < 2.1, (k, st)


def _sig_interval(x, digits):
    """[lo, hi) of the values that %.<digits>g prints as the string x (which
    drops trailing zeros, so x alone does not give the precision)."""
    ex = int(("%e" % float(x)).split("e")[1])
    half = 0.5 * 10 ** (ex - (digits - 1))
    return float(x) - half, float(x) + half


def _interval_logE(r, searchspace, summary_e):
    """A log E-value consistent with every printed value the reference derived
    from it: the bit score (%.1f), the E-value (%.2g), the P-value (%.2g) and
    the summary list's E-value (%.1g)."""
    ln2 = math.log(2.0)
    lss = math.log(np.float32(searchspace))
    los = [lss - (r["bit_score"] + 0.05) * ln2]
    his = [lss - (r["bit_score"] - 0.05) * ln2]
    for s_, dg in (("%.2g" % r["evalue"], 2), (summary_e, 1)):
        lo, hi = _sig_interval(s_, dg)
        los.append(math.log(lo))
        his.append(math.log(hi))
    if r["evalue"] >= 0.01:
        lo, hi = _sig_interval("%.2g" % r["pvalue"], 2)
        los.append(math.log(-math.log1p(-lo)))
        if hi < 1.0:
            his.append(math.log(-math.log1p(-hi)))
    lo, hi = max(los), min(his)
    assert lo < hi, (r["profile"], los, his)
    return 0.5 * (lo + hi)


def _summary_evalues(text):
    """profile -> E-value string of the reference file's summary list."""
    out = {}
    for ln in text.splitlines():
        t = ln.split()
        if len(t) == 3 and t[0].startswith("p0") and ln.startswith("p0"):
            out[int(t[0][1:])] = t[2]
    return out


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("case", CASES)
def test_plain_writer_reproduces_the_reference_file(params, case, variant):
    """c2_format_report against the reference's own Plain result file, byte
    for byte: the hit records are rebuilt from the oracle (scores, MAP
    alignments on the reference's lambda and K) and the printed statistics
    of the reference's run (its lambda, K and entropy values as printed, and
    a log E-value consistent with its printed E-value and bit score)."""
    from oracle_py import Oracle
    from comer2_b200 import native as N
    fx = load_fixture(case, variant)
    prm = fixture_params(params, fx)
    w = fixture_workload(fx)
    orc = Oracle(prm, 32)
    q = w.queries[0]
    qo = orc.profile(q)
    Lq = int(q.lengths[0])
    ss, dl = orc.length_adjustment(prm.gapped_lambda, prm.gapped_K, prm.gapped_alpha, prm.gapped_beta, Lq,
                                   int(w.db.lengths.sum()), int(w.db.nprofiles))
    with open(os.path.join(HERE, "golden", "ref_%s_%s.out" % (case, variant))) as fh:
        ref = fh.read()
    summ = _summary_evalues(ref)
    hits = np.zeros(len(fx["hits"]), N.HIT_DTYPE)
    alns = []
    pos = 0

    def printed(v, tiny):
        # the writer prints K / lambda values > 0 with 4 decimals and "n/a" otherwise
        return -1.0 if v == "n/a" else (float(v) if float(v) > 0 else tiny)

    for i, r in enumerate(fx["hits"]):
        k = r["profile"]
        off, nd = int(w.db.offsets[k]), int(w.db.lengths[k])
        do = orc.profile(w.db, k)
        x = orc.pair(qo, do)
        lam, K = ref_lambda_K(r)
        sg = orc.significance(Lq, nd, x["score"], x["psts"], q.eno[0], w.db.eno[k], ss, lam, K)
        strings, alnlen, idts, psts, gaps, beg, end = oracle_alignment(orc, prm, qo, do, x, q, w, off, nd,
                                                                         sg["logEpA"])
        h = hits[i]
        h["profile"], h["score"], h["logE"] = k, x["score"], _interval_logE(r, ss, summ[k])
        h["lambda_"], h["K"] = printed(r["computed_lambda_ungapped"], 1e-6), printed(r["computed_K_ungapped"], 1e-6)
        h["lambda_est"] = printed(r["estimated_lambda_gapped"], 1e-6)
        h["K_est"] = printed(r["estimated_K_gapped"], 1e-6)
        h["E"], h["H"] = r["expected_score"], r["entropy"]
        h["smin"], h["smax"] = r["min_score"], r["max_score"]
        h["alnlen"], h["idts"], h["psts"], h["gaps"] = alnlen, idts, psts, gaps
        h["beg"] = (beg[0] << 16) | beg[1]
        h["end"] = (end[0] << 16) | end[1]
        h["aln_offset"] = pos
        for sgl in strings:
            alns.append(sgl.encode() + b"\0")
            pos += len(sgl) + 1
    text = N.format_report(
        N.REPORT_PLAIN, hits, np.frombuffer(b"".join(alns), np.uint8), query_length=Lq,
        query_eno=float(q.eno[0]), query_desc="query", query_has_ss=True,
        db_lengths=w.db.lengths, db_eno=w.db.eno, db_desc=["p%06d" % k for k in range(w.db.nprofiles)],
        db_names=["db"], db_positions=int(w.db.lengths.sum()), db_profiles=int(w.db.nprofiles),
        logevthld=math.log(prm.eval), searchspace=float(ss), deltalen=int(dl), ref_lambda=prm.ungapped_lambda,
        ref_K=prm.ungapped_K, gapped_lambda=prm.gapped_lambda, gapped_K=prm.gapped_K, print_ss=False,
        dsclen=1024, dscwidth=80, alnwidth=60, show=1, nhits=700, nalns=700, progname="comer",
        progversion="2.03.03", references=REFERENCES)
    if text != ref:
        import difflib
        diff = "".join(list(difflib.unified_diff(ref.splitlines(True), text.splitlines(True), "reference",
                                                 "c2_format_report"))[:60])
        pytest.fail("Plain file differs from the reference's:\n" + diff)


REFERENCES = [
    "Margelevicius, M. (2020). COMER2: GPU-accelerated sensitive and specific homology searches. "
    "Bioinformatics 36, 3570-3572.",
    "Margelevicius, M. (2016). Bayesian nonparametrics in protein remote homology search. "
    "Bioinformatics 32, 2744-2752.",
]
