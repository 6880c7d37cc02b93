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


@pytest.mark.parametrize("mode", MODES)
def test_phase1_and_finalize_on_device_scores(params, orc32, mode):
    """With an E-value threshold that makes every pair with a positive
    maximum a candidate, the device's own FP32 score matrix of every pair is
    available (c2_get_pair_scores).  On it the oracle's DP must reproduce the
    phase-1 maximum (FP32 form: to 1e-6 relative with the same cell; BF16
    form: within its 2e-3 relative candidate margin) and the finalisation
    (score to 1e-5 relative, positive count, path ends); and the device's
    scores must equal the oracle's cell by cell (5e-5 absolute: CUDA's fast
    logarithm against the C library's), except
    cells where the context-vector score crosses a table bin edge (one table
    step, < 0.05), which must be rare."""
    import copy
    p = copy.deepcopy(params)
    p.eval = 1e12
    w = S.config(1, seed=3, scale=0.002)
    h = _handle(p, mode)
    h.upload_db(w.db)
    h.set_query(w.queries[0])
    thld, _ = h.thresholds()
    assert thld == 0.0
    h.run_phase1()
    best, coords = h.phase1()
    n = h.run_finalize()
    fin = {int(r["profile"]): r for r in h.finalize(n)}
    qo = orc32.profile(w.queries[0])
    ncell = nedge = 0
    for k in range(w.db.nprofiles):
        if not best[k] > 0:
            continue
        assert k in fin
        L = int(w.db.lengths[k])
        do = orc32.profile(w.db, k)
        sm, mm = h.pair_scores(k, L)
        rs, rm = orc32.score_matrix(qo, do)
        d = np.abs(sm - rs)
        edge = d > 5e-5
        assert (d[edge] < 0.05).all(), (k, float(d.max()))
        assert np.abs(mm - rm)[~edge].max(initial=0.0) <= 5e-5
        ncell += d.size
        nedge += int(edge.sum())
        ob, ox, oy, nt, bt = orc32.dp(qo, do, sm, with_btck=True)
        if mode == 0:
            assert float(best[k]) == pytest.approx(ob, rel=1e-6, abs=1e-6), k
            if nt == 1:
                assert (int(coords[k]) >> 16, int(coords[k]) & 0xFFFF) == (ox, oy), k
        else:
            assert abs(float(best[k]) - ob) <= 2e-3 * max(1.0, abs(ob)), k
        sc, ps, bx, by = orc32.finalize(sm, bt, ob, ox, oy)
        r = fin[k]
        assert float(r["score"]) == pytest.approx(sc, rel=1e-5, abs=1e-5), k
        if nt == 1:
            assert int(r["psts"]) == ps, k
            assert (int(r["beg"]) >> 16, int(r["beg"]) & 0xFFFF) == (bx, by), k
            assert (int(r["end"]) >> 16, int(r["end"]) & 0xFFFF) == (ox, oy), k
    assert ncell > 1_000_000
    assert nedge <= 1e-4 * ncell, (nedge, ncell)
    h.close()
