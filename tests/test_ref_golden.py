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


def load_fixture(case):
    with open(os.path.join(HERE, "golden", "ref_%s_w00_plain.json" % case)) as fh:
        return json.load(fh)


def fixture_params(params, fx):
    p = copy.deepcopy(params)
    p.ssswgt = np.float32(fx["ssswgt"])
    p.cvswgt = np.float32(fx["cvswgt"])
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


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_the_reference_run(params, case):
    from oracle_py import Oracle
    fx = load_fixture(case)
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
        m = orc.map(qo, do, x["S"], x["MOD"], sg["logEpA"], qss=q.ssstate, dss=w.db.ssstate[off:off + nd])
        check_alignment(r, m["strings"], m["alnlen"], m["idts"], m["psts"], m["gaps"], (m["begx"], m["begy"]),
                        (m["endx"], m["endy"]))


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
