"""GPU parity of the complete search (phase 1, finalisation, statistics, MAP)
against the CPU oracle, through the C ABI.

Tolerances: DP scores 1e-4 relative, log E-values 1e-3 absolute, hit lists
identical, MAP alignment strings identical.  A context-vector score near a
map-bin edge can round differently on the two sides (one cell moves by one
table step, ~0.01); pairs affected that way are counted and must be rare.
"""
import math

import numpy as np
import pytest

from comer2_b200 import synth as S

pytestmark = pytest.mark.gpu


def _oracle_search(orc, prm, w, searchspace, thld, logevthld):
    """The oracle's hit list: {profile: record}."""
    q = w.queries[0]
    qo = orc.profile(q)
    out = {}
    for k in range(w.db.nprofiles):
        do = orc.profile(w.db, k)
        r = orc.pair(qo, do)
        if not (r["best"] > thld) or not (r["score"] > thld):
            continue
        off, nd = int(w.db.offsets[k]), int(w.db.lengths[k])
        st = orc.stats(r["S"], q.aa, w.db.aa[off:off + nd], r["score"], r["psts"], q.eno[0], w.db.eno[k],
                       float(searchspace), prm.x_uninf)
        rec = {"score": r["score"], "stats": st}
        if not (logevthld < st["logE"]):
            m = orc.map(qo, do, r["S"], r["MOD"], st["logEpA"], qss=q.ssstate, dss=w.db.ssstate[off:off + nd])
            rec["map"] = m
        out[k] = rec
    return out


def _recheck_on_device_scores(h, orc, prm, w, x, searchspace, logevthld):
    """Every stage after the score matrix, checked on the device's own FP32
    score and modular-score matrices of the hit's pair (c2_get_pair_scores):
    the oracle's DP, finalisation, statistics and MAP run on exactly the
    scores the GPU used, so no rounding of the score terms can excuse a
    difference.  DP scores within 1e-5 relative, log E within 1e-3, the
    alignment (strings, counts, coordinates) identical."""
    q = w.queries[0]
    k = int(x["profile"])
    off, nd = int(w.db.offsets[k]), int(w.db.lengths[k])
    sm, mm = h.pair_scores(k, nd)
    qo, do = orc.profile(q), orc.profile(w.db, k)
    best, bx, by, nt, bt = orc.dp(qo, do, sm, with_btck=True)
    score, psts, _, _ = orc.finalize(sm, bt, best, bx, by)
    assert x["score"] == pytest.approx(score, rel=1e-5, abs=1e-5), k
    st = orc.stats(sm, q.aa, w.db.aa[off:off + nd], score, psts, q.eno[0], w.db.eno[k], float(searchspace),
                   prm.x_uninf)
    assert (x["smin"], x["smax"]) == (st["min"], st["max"]), k
    assert x["logE"] == pytest.approx(st["logE"], abs=1e-3), k
    assert x["logEpA"] == pytest.approx(st["logEpA"], abs=1e-3), k
    assert x["lambda_"] == pytest.approx(st["lambda_"], rel=1e-3, abs=1e-5), k
    assert x["K"] == pytest.approx(st["K"], rel=1e-3, abs=1e-6), k
    assert not (logevthld < st["logE"]), k
    m = orc.map(qo, do, sm, mm, st["logEpA"], qss=q.ssstate, dss=w.db.ssstate[off:off + nd])
    assert x["strings"] == m["strings"], k
    assert (x["alnlen"], x["idts"], x["psts"], x["gaps"]) == (m["alnlen"], m["idts"], m["psts"], m["gaps"]), k
    assert (x["beg"] >> 16, x["beg"] & 0xFFFF) == (m["begx"], m["begy"]), k
    assert (x["end"] >> 16, x["end"] & 0xFFFF) == (m["endx"], m["endy"]), k


def _run(params, w, mode=0):
    from comer2_b200.native import Handle
    h = Handle(params, 0)
    h.set_score_mode(mode)
    h.upload_db(w.db)
    hits = h.search(w.queries[0])
    thld, logevthld = h.thresholds()
    ss, _ = h.search_space()
    return h, hits, thld, logevthld, ss


@pytest.mark.parametrize("mode", [0, 1])   # FP32 scores; split-BF16 tensor-core scores
@pytest.mark.parametrize("seed", [2, 9])
def test_search_matches_oracle(params, orc32, seed, mode):
    w = S.config(1, seed=seed, scale=0.003)   # 300 profiles, 6 planted homologs
    h, hits, thld, logevthld, ss = _run(params, w, mode)
    ref = _oracle_search(orc32, params, w, ss, thld, logevthld)
    ref_hits = sorted(k for k, v in ref.items() if "map" in v)
    got = sorted(int(x["profile"]) for x in hits)
    assert got == ref_hits
    # hits are sorted by log E-value
    le = [x["logE"] for x in hits]
    assert le == sorted(le)
    flips = 0
    for x in hits:
        k = int(x["profile"])
        r = ref[k]
        st, m = r["stats"], r["map"]
        _recheck_on_device_scores(h, orc32, params, w, x, ss, logevthld)
        dscore = abs(x["score"] - r["score"])
        if dscore > 1e-4 * max(1.0, abs(r["score"])):
            # a context-vector bin edge moved a cell by one table step: the
            # hit was checked above on the device's scores
            flips += 1
            assert dscore < 0.1
            continue
        assert x["logE"] == pytest.approx(st["logE"], abs=1e-3), k
        assert x["logEpA"] == pytest.approx(st["logEpA"], abs=1e-3), k
        assert x["lambda_"] == pytest.approx(st["lambda_"], rel=1e-3, abs=1e-5), k
        assert x["K"] == pytest.approx(st["K"], rel=1e-3, abs=1e-6), k
        assert (x["smin"], x["smax"]) == (st["min"], st["max"])
        assert x["strings"][:3] == m["strings"][:3], k
        assert x["strings"][3:] == m["strings"][3:], k
        assert (x["alnlen"], x["idts"], x["psts"], x["gaps"]) == (m["alnlen"], m["idts"], m["psts"], m["gaps"])
        assert (x["beg"] >> 16, x["beg"] & 0xFFFF) == (m["begx"], m["begy"])
        assert (x["end"] >> 16, x["end"] & 0xFFFF) == (m["endx"], m["endy"])
    assert flips <= max(1, len(hits) // 20)
    # every planted homolog is found with a small E-value
    for k in w.homologs:
        assert k in got
    h.close()


@pytest.mark.parametrize("mode", [0, 1])
def test_long_query_matches_oracle(params, orc32, mode):
    """A 3,000-position query of six domains (94 strips) against 30 profiles
    with planted single-domain homologs: the same hits, E-values and
    alignments as the oracle."""
    w = S.config(4, seed=5, scale=0.0006)
    h, hits, thld, logevthld, ss = _run(params, w, mode)
    ref = _oracle_search(orc32, params, w, ss, thld, logevthld)
    ref_hits = sorted(k for k, v in ref.items() if "map" in v)
    assert sorted(int(x["profile"]) for x in hits) == ref_hits
    for x in hits:
        r = ref[int(x["profile"])]
        _recheck_on_device_scores(h, orc32, params, w, x, ss, logevthld)
        if abs(x["score"] - r["score"]) > 1e-4 * max(1.0, abs(r["score"])):
            continue
        assert x["logE"] == pytest.approx(r["stats"]["logE"], abs=1e-3)
        assert x["strings"][:3] == r["map"]["strings"][:3]
    for k in w.homologs:
        assert k in [int(x["profile"]) for x in hits]
    h.close()


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("lq", [20, 33, 64, 97])
def test_query_strip_edges_match_oracle(params, orc32, lq, mode):
    """Queries of one partial strip, a one-row last strip, whole strips and
    three strips plus one row, against short (< 32 columns) and long profiles
    with planted homologs: the strip pipelines of the traceback and MAP
    sweeps at their edges give the oracle's hits, E-values and alignments."""
    rng = np.random.default_rng(500 + lq)
    q = S.random_profiles(rng, [lq])
    lens = np.concatenate([rng.integers(8, 32, 12), rng.integers(32, 400, 28)])
    db, hom = S.make_db(rng, lens, q, 0.2)
    w = S.Workload("edge", [q], db, hom)
    h, hits, thld, logevthld, ss = _run(params, w, mode)
    ref = _oracle_search(orc32, params, w, ss, thld, logevthld)
    ref_hits = sorted(k for k, v in ref.items() if "map" in v)
    assert sorted(int(x["profile"]) for x in hits) == ref_hits
    flips = 0
    for x in hits:
        r = ref[int(x["profile"])]
        _recheck_on_device_scores(h, orc32, params, w, x, ss, logevthld)
        if abs(x["score"] - r["score"]) > 1e-4 * max(1.0, abs(r["score"])):
            flips += 1
            continue
        assert x["logE"] == pytest.approx(r["stats"]["logE"], abs=1e-3)
        assert x["strings"] == r["map"]["strings"]
        m = r["map"]
        assert (x["beg"] >> 16, x["beg"] & 0xFFFF) == (m["begx"], m["begy"])
        assert (x["end"] >> 16, x["end"] & 0xFFFF) == (m["endx"], m["endy"])
    assert flips <= max(1, len(hits) // 20)
    h.close()


def test_search_space_matches_oracle(params, orc32):
    w = S.config(0, seed=4, scale=0.05)
    from comer2_b200.native import Handle
    h = Handle(params, 0)
    h.upload_db(w.db, total_positions=5_000_000, total_profiles=20_000)
    h.set_query(w.queries[0])
    ss, dl = h.search_space()
    ref = orc32.length_adjustment(params.gapped_lambda, params.gapped_K, params.gapped_alpha,
                                  params.gapped_beta, int(w.queries[0].lengths[0]), 5_000_000, 20_000)
    assert (ss, dl) == ref
    thld, le = h.thresholds()
    rt, rl = orc32.score_threshold(int(w.queries[0].lengths[0]), 5_000_000, params.eval, params.gapped_K,
                                   params.gapped_lambda)
    assert thld == rt and le == rl
    h.close()


def test_no_hits_db(params):
    """A database of unrelated short profiles: the search completes with few or no hits."""
    rng = np.random.default_rng(77)
    q = S.random_profiles(rng, [60])
    db = S.random_profiles(rng, [40] * 30)
    from comer2_b200.native import Handle
    h = Handle(params, 0)
    h.upload_db(db, total_positions=10_000_000, total_profiles=50_000)
    hits = h.search(q)
    assert len(hits) == 0
    h.close()


def test_hits_arrays_match_dicts(params):
    """search(arrays=True) returns the same records and alignment strings as the dict form."""
    from comer2_b200.native import Handle
    w = S.config(1, seed=2, scale=0.002)
    h = Handle(params, 0)
    h.upload_db(w.db)
    hits = h.search(w.queries[0])
    rec, buf = h.search(w.queries[0], arrays=True)
    assert rec.shape[0] == len(hits) > 0
    raw = buf.tobytes()
    for x, r in zip(hits, rec):
        assert int(r["profile"]) == x["profile"] and float(r["logE"]) == x["logE"]
        o, L = int(r["aln_offset"]), int(r["alnlen"])
        assert [raw[o + k * (L + 1):o + k * (L + 1) + L].decode() for k in range(5)] == x["strings"]
    h.close()


def test_bf16_form_with_a_cv_table_off_its_index_range(params):
    """A CV table whose key range is narrower than its index clamp (keys moved
    by +1) takes the tensor kernel's explicit range tests; its hits must equal
    the FP32 form's."""
    import copy
    from comer2_b200.native import Handle
    p = copy.deepcopy(params)
    p.cvs2s_keys = np.asarray(p.cvs2s_keys, np.float32) + np.float32(1.0)
    w = S.config(1, seed=4, scale=0.003)
    out = []
    for mode in (0, 1):
        h = Handle(p, 0)
        h.set_score_mode(mode)
        h.upload_db(w.db)
        rec, alns = h.search(w.queries[0], arrays=True)
        out.append((rec, bytes(alns)))
    (r0, a0), (r1, a1) = out
    assert len(r0) > 0
    assert list(r0["profile"]) == list(r1["profile"])
    assert np.allclose(r0["score"], r1["score"], rtol=1e-4, atol=1e-4)
    assert np.allclose(r0["logE"], r1["logE"], atol=1e-3)
    assert a0 == a1


def test_observed_statistics_model_matches_oracle(params, orc32):
    """SSEMODEL 0 (E-values from the expected gapped lambda and K over the
    search space, the reference's CalcSignificanceObsDynPlmProfile): hit
    list, log E-values and alignments equal the oracle's."""
    import copy
    from oracle_py import Oracle
    p = copy.deepcopy(params)
    p.ssemodel = 0
    orc = Oracle(p, 32)   # the oracle's statistics follow its own parameters
    w = S.config(1, seed=9, scale=0.003)
    h, hits, thld, logevthld, ss = _run(p, w, 1)
    ref = _oracle_search(orc, p, w, ss, thld, logevthld)
    assert sorted(int(x["profile"]) for x in hits) == sorted(k for k, v in ref.items() if "map" in v)
    assert len(hits) > 0
    for x in hits:
        _recheck_on_device_scores(h, orc, p, w, x, ss, logevthld)
        st = ref[int(x["profile"])]["stats"]
        expect = np.log(np.float32(p.gapped_K) * np.float32(ss)) - np.float32(p.gapped_lambda) * x["score"]
        assert x["logE"] == pytest.approx(float(expect), abs=1e-3)
        assert x["logE"] == pytest.approx(st["logE"], abs=1e-3)
    h.close()


def test_config0_in_full_matches_oracle(params, orc32):
    """The plain-method workload at full size (1 x 150 vs 2,000 profiles of
    U[50,500]): the oracle's hit list, and every hit checked through all
    stages on the device's own scores."""
    w = S.config(0, seed=0, scale=1.0)
    assert w.db.nprofiles == 2000
    h, hits, thld, logevthld, ss = _run(params, w, 1)
    ref = _oracle_search(orc32, params, w, ss, thld, logevthld)
    assert sorted(int(x["profile"]) for x in hits) == sorted(k for k, v in ref.items() if "map" in v)
    for x in hits:
        _recheck_on_device_scores(h, orc32, params, w, x, ss, logevthld)
    h.close()


def test_config1_sample_with_all_homologs_matches_oracle(params, orc32):
    """A 2,500-profile sample of the database-scan workload (1 x 400,
    lognormal lengths) holding all its planted homologs, searched with the
    full database's size for the thresholds and search space: the oracle's
    hit list, and every hit checked on the device's own scores."""
    w = S.config(1, seed=1, scale=0.025)
    assert w.db.nprofiles == 2500 and len(w.homologs) >= 40
    from comer2_b200.native import Handle
    h = Handle(params, 0)
    h.set_score_mode(1)
    h.upload_db(w.db, total_positions=24_000_000, total_profiles=100_000)
    hits = h.search(w.queries[0])
    thld, logevthld = h.thresholds()
    ss, _ = h.search_space()
    ref = _oracle_search(orc32, params, w, ss, thld, logevthld)
    assert sorted(int(x["profile"]) for x in hits) == sorted(k for k, v in ref.items() if "map" in v)
    for k in w.homologs:
        assert k in [int(x["profile"]) for x in hits]
    for x in hits:
        _recheck_on_device_scores(h, orc32, params, w, x, ss, logevthld)
    h.close()


def test_masked_residues_matches_oracle(params, orc32):
    """'X' residues in the query and the database: with X_UNINF their cells
    are left out of the score statistics (the reference's
    CalcScoreProbsXuninfDynPlmProfile) and 'X' pairs count as identities in
    the alignment middle line like any letter; hits, statistics and
    alignments equal the oracle's."""
    w = S.config(1, seed=2, scale=0.003)
    rng = np.random.default_rng(123)
    for ps in (w.queries[0], w.db):
        idx = rng.choice(ps.npositions, size=max(1, ps.npositions // 15), replace=False)
        ps.aa[idx] = ord("X")
    assert params.x_uninf == 1
    h, hits, thld, logevthld, ss = _run(params, w, 1)
    ref = _oracle_search(orc32, params, w, ss, thld, logevthld)
    assert sorted(int(x["profile"]) for x in hits) == sorted(k for k, v in ref.items() if "map" in v)
    assert len(hits) > 0
    assert any("X" in x["strings"][0] for x in hits)
    for x in hits:
        _recheck_on_device_scores(h, orc32, params, w, x, ss, logevthld)
    h.close()


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("variant", ["w00", "w00aln0"])
@pytest.mark.parametrize("case", ["c1_s2", "c1_s9", "c0_s4"])
def test_matches_the_reference_run(params, case, variant, mode):
    """The CUDA path against the reference's own results on a B200 (the
    fixtures of tests/test_ref_golden.py; SS and CV weights 0, the only
    setting in which that build's results are valid; MAP or, with MAPALN 0,
    Viterbi alignments and that setting's score shift): for every hit the
    reference reported, the DP score within the printed 0.006, and the
    expected score and score range of the pair's score distribution to the
    printed digits.  The E-value threshold is raised so that every pair gets
    its statistics; the E-values and MAP alignments follow the statistics,
    which are checked against the oracle elsewhere (the reference's own
    lambda and K are not valid on this build)."""
    import copy
    from test_ref_golden import fixture_params, fixture_workload, load_fixture
    from comer2_b200.native import Handle
    fx = load_fixture(case, variant)
    p = fixture_params(params, fx)
    p = copy.deepcopy(p)
    p.eval = 1e12
    w = fixture_workload(fx)
    h = Handle(p, 0)
    h.set_score_mode(mode)
    h.upload_db(w.db)
    got = {int(x["profile"]): x for x in h.search(w.queries[0])}
    for r in fx["hits"]:
        k = r["profile"]
        assert k in got, k
        x = got[k]
        assert abs(x["score"] - r["score"]) <= 0.006, (k, x["score"], r["score"])
        assert abs(x["E"] - r["expected_score"]) <= 6e-5, (k, x["E"], r["expected_score"])
        assert (x["smin"], x["smax"]) == (r["min_score"], r["max_score"]), k
    h.close()


@pytest.mark.parametrize("mode", [0, 1])
def test_viterbi_alignments_match_oracle(params, mode):
    """MAPALN 0: the hits carry the Viterbi DP's own alignments (the
    reference's FinalizeDP_ALN instead of the MAP stage), with the
    MAPALN-0 score shift (0.0003) and integer context-vector priors of the
    score matrix: hit list, scores, E-values and alignments equal the
    oracle's (which applies the same MAPALN-0 score terms)."""
    import copy
    from oracle_py import Oracle
    from test_ref_golden import viterbi_alignment
    p = copy.deepcopy(params)
    p.mapaln = 0
    orc = Oracle(p, 32)
    w = S.config(1, seed=2, scale=0.003)
    h, hits, thld, logevthld, ss = _run(p, w, mode)
    q = w.queries[0]
    qo = orc.profile(q)
    ref = {}
    for k in range(w.db.nprofiles):
        do = orc.profile(w.db, k)
        r = orc.pair(qo, do)
        if not (r["best"] > thld and r["score"] > thld):
            continue
        off, nd = int(w.db.offsets[k]), int(w.db.lengths[k])
        st = orc.stats(r["S"], q.aa, w.db.aa[off:off + nd], r["score"], r["psts"], q.eno[0], w.db.eno[k],
                       float(ss), p.x_uninf)
        if not (logevthld < st["logE"]):
            ref[k] = (r, st, off, nd)
    assert sorted(int(x["profile"]) for x in hits) == sorted(ref)
    assert len(hits) > 0
    for x in hits:
        k = int(x["profile"])
        r, st, off, nd = ref[k]
        if abs(x["score"] - r["score"]) > 1e-4 * max(1.0, abs(r["score"])):
            continue   # a context-vector bin edge: checked below on the device's scores
        assert x["logE"] == pytest.approx(st["logE"], abs=1e-3), k
        rows, alnlen, idts, psts, gaps, beg, end = viterbi_alignment(
            r["btck"], r["S"], q.aa, w.db.aa[off:off + nd], q.ssstate, w.db.ssstate[off:off + nd], r["x"], r["y"])
        assert x["strings"] == rows, k
        assert (x["alnlen"], x["idts"], x["psts"], x["gaps"]) == (alnlen, idts, psts, gaps), k
        assert (x["beg"] >> 16, x["beg"] & 0xFFFF) == beg, k
        assert (x["end"] >> 16, x["end"] & 0xFFFF) == end, k
    h.close()
