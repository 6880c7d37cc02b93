"""GPU parity of phase 1 (fused score + Viterbi DP) and the DP finalisation
against the CPU oracle, called through the C ABI.

Both score modes are checked: FP32 on the CUDA cores and the split-BF16
tensor-core contractions (mode 1), against the same FP32 oracle.

Tolerance: DP maxima within 1e-4 relative.  The context-vector term maps a
continuous value through a step table (rint(2x) bins), so a rounding
difference near a bin edge moves one cell's score by one table step
(about 0.01 after weighting); pairs whose path crosses such a cell are
allowed up to 0.05 absolute, and must be rare.
"""
import numpy as np
import pytest

from comer2_b200 import synth as S

pytestmark = pytest.mark.gpu


MODES = [0, 1]   # native.SCORE_FP32, native.SCORE_BF16_TC


def _handle(params, mode=0):
    from comer2_b200.native import Handle
    h = Handle(params, 0)
    h.set_score_mode(mode)
    return h


def _oracle_all(orc, q, db, ks):
    qo = orc.profile(q)
    return {k: orc.pair(qo, orc.profile(db, k)) for k in ks}


def _check_phase1(best, coords, ref, ks):
    rel_ok = 0
    for k in ks:
        r = ref[k]
        tol = 1e-4 * max(1.0, abs(r["best"]))
        d = abs(float(best[k]) - r["best"])
        assert d <= tol + 0.05, (k, best[k], r["best"])
        if d <= tol:
            rel_ok += 1
            if r["best"] > 0 and r["nties"] == 1:
                x, y = int(coords[k]) >> 16, int(coords[k]) & 0xFFFF
                assert (x, y) == (r["x"], r["y"]), (k, (x, y), (r["x"], r["y"]))
    return rel_ok


@pytest.mark.parametrize("mode", MODES)
def test_phase1_small_db(params, orc32, mode):
    w = S.config(1, seed=3, scale=0.002)  # 200 profiles, 4 planted homologs
    h = _handle(params, mode)
    h.upload_db(w.db)
    h.set_query(w.queries[0])
    h.run_phase1()
    best, coords = h.phase1()
    ks = list(range(w.db.nprofiles))
    ref = _oracle_all(orc32, w.queries[0], w.db, ks)
    ok = _check_phase1(best, coords, ref, ks)
    assert ok >= 0.98 * len(ks)
    for k in w.homologs:
        assert best[k] > 100.0


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("lq", [1, 5, 31, 32, 33, 64, 65, 97])
def test_phase1_edge_lengths(params, orc32, lq, mode):
    rng = np.random.default_rng(100 + lq)
    q = S.random_profiles(rng, [lq])
    lens = [1, 2, 5, 31, 32, 33, 63, 64, 65, 96, 130, 257]
    db = S.random_profiles(rng, lens)
    h = _handle(params, mode)
    h.upload_db(db)
    h.set_query(q)
    h.run_phase1()
    best, coords = h.phase1()
    ks = list(range(db.nprofiles))
    ref = _oracle_all(orc32, q, db, ks)
    ok = _check_phase1(best, coords, ref, ks)
    assert ok >= len(ks) - 1


@pytest.mark.parametrize("mode", MODES)
def test_phase1_homolog_long_alignments(params, orc32, mode):
    """Planted homologs give maxima in the hundreds; their paths cross many
    strips, so the strip hand-off and the column -1 boundary are exercised."""
    rng = np.random.default_rng(11)
    q = S.random_profiles(rng, [300])
    parts = [S.planted_homolog(rng, q, L) for L in (40, 77, 128, 200, 333, 600)]
    db = S.concat(parts)
    h = _handle(params, mode)
    h.upload_db(db)
    h.set_query(q)
    h.run_phase1()
    best, coords = h.phase1()
    ks = list(range(db.nprofiles))
    ref = _oracle_all(orc32, q, db, ks)
    ok = _check_phase1(best, coords, ref, ks)
    assert ok >= len(ks) - 1
    assert (best > 50).all()


def test_finalize_matches_oracle(params, orc32):
    w = S.config(1, seed=5, scale=0.003)
    h = _handle(params)
    h.upload_db(w.db)
    h.set_query(w.queries[0])
    thld, _ = h.thresholds()
    h.run_phase1()
    best, coords = h.phase1()
    n = h.run_finalize()
    fin = h.finalize(n)
    cand = np.nonzero(best > thld)[0]
    assert list(fin["profile"]) == list(cand)
    assert n >= len(w.homologs)
    qo = orc32.profile(w.queries[0])
    agree = 0
    for rec in fin:
        k = int(rec["profile"])
        r = orc32.pair(qo, orc32.profile(w.db, k))
        tol = 1e-4 * max(1.0, abs(r["score"]))
        d = abs(float(rec["score"]) - r["score"])
        assert d <= tol + 0.1, (k, rec["score"], r["score"])
        if d <= tol and r["nties"] == 1:
            agree += 1
            assert rec["psts"] == r["psts"]
            assert (rec["beg"] >> 16, rec["beg"] & 0xFFFF) == (r["begx"], r["begy"])
            assert (rec["end"] >> 16, rec["end"] & 0xFFFF) == (r["x"], r["y"])
        assert rec["passed"] == int(rec["score"] > thld)
    assert agree >= 0.9 * n
    assert h.launch_count() >= 3
