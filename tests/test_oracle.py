"""CPU tests of the oracle (the checker) and of the host-side logic.

The C oracle is cross-checked against an independent pure-Python restatement
of the reference's DP on small cases, and its float build against its double
build; the threshold and length-adjustment formulas against direct formulas.
"""
import math
import os

import numpy as np
import pytest

from comer2_b200 import synth as S

NEG = -32768.0


def _q7(ps, k, i):
    """DP transitions of position i of profile k (MMp MIc MDp IMp IIc DMp DDp)."""
    L = int(ps.lengths[k])
    if i < 0 or i >= L:
        return [NEG] * 7
    o = int(ps.offsets[k]) + k
    a, b = ps.trn[o + i], ps.trn[o + i + 1]
    return [float(a[0]), float(b[1]), float(a[2]), float(a[3]), float(b[4]), float(a[5]), float(a[6])]


def py_dp(qs, ds, Smat):
    """Pure-Python restatement of the reference's Viterbi DP with its
    row-dependent column -1 boundary (src/libmycu/cudp/CuBatchDP_init_btck.cu:117-360)."""
    Lq, Ld = Smat.shape
    MM, MI, MD, IM, II, DM, DD = range(7)
    Z = (0.0, 0.0, 0.0, 0.0, 0.0)
    C = []
    for r in range(Lq):
        t = _q7(qs, 0, r)
        U = Z if r % 32 == 0 else C[r - 1]
        mi = max(U[0] + t[MM] + NEG, U[1] + t[MM] + NEG)
        im = max(t[MI] + NEG, t[II] + NEG) if r % 32 == 0 else t[MI] + NEG
        dn = max(U[0] + t[MD], U[3] + t[DD])
        C.append((0.0, mi, im, dn, NEG))
    e = min(60, int(round(0.34 * max(Lq, Ld))))
    prev = [Z] * Ld
    best, bi, bj = 0.0, -1, -1
    bt = np.zeros((Lq, Ld), np.int8)
    for i in range(Lq):
        q = _q7(qs, 0, i)
        cur = [None] * Ld
        for j in range(Ld):
            d = _q7(ds, 0, j)
            up = Z if i == 0 else prev[j]
            if j == 0:
                left = Z if i % 32 == 31 else C[i]
                diag = Z if i % 32 in (0, 31) else C[i - 1]
            else:
                left = cur[j - 1]
                diag = Z if i == 0 else prev[j - 1]
            corner = (Lq <= i + e and j <= e + i - Lq) or (Ld - e + i <= j and i < e)
            sc = -9.0 if corner else float(Smat[i, j])
            v = max(diag[1] + q[MM] + d[IM], diag[2] + q[IM] + d[MM], diag[3] + q[DM] + d[MM],
                    diag[4] + q[MM] + d[DM], diag[0] + q[MM] + d[MM])
            mm = max(v + sc, 0.0)
            mi = max(up[0] + q[MM] + d[MI], up[1] + q[MM] + d[II])
            im = max(left[0] + q[MI] + d[MM], left[2] + q[II] + d[MM])
            dn = max(up[0] + q[MD], up[3] + q[DD])
            nd = max(left[0] + d[MD], left[4] + d[DD])
            cur[j] = (mm, mi, im, dn, nd)
            b, mx = 0, mm
            if mm != 0:
                b = 3
            for val, code in ((mi, 2), (im, 1), (dn, 2), (nd, 1)):
                if mx < val:
                    mx, b = val, code
            bt[i, j] = b
            if best < mm:
                best, bi, bj = mm, i, j
        prev = cur
    return best, bj, bi, bt


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_dp_matches_python_restatement(orc64, seed):
    rng = np.random.default_rng(seed)
    Lq, Ld = int(rng.integers(20, 75)), int(rng.integers(20, 70))
    qs = S.random_profiles(rng, [Lq])
    ds = S.random_profiles(rng, [Ld])
    q, d = orc64.profile(qs), orc64.profile(ds)
    Smat, _ = orc64.score_matrix(q, d)
    Smat = Smat + 2.5  # make alignments long enough to cross row blocks and the boundary
    best, x, y, nt, bt = orc64.dp(q, d, Smat, with_btck=True)
    pb, px, py, pbt = py_dp(qs, ds, Smat)
    assert best == pytest.approx(pb, rel=1e-12, abs=1e-12)
    assert (x, y) == (px, py)
    assert np.array_equal(bt, pbt)


def test_float_oracle_close_to_double(orc32, orc64):
    w = S.config(1, seed=7, scale=0.0006)
    q32, q64 = orc32.profile(w.queries[0]), orc64.profile(w.queries[0])
    ks = list(w.homologs[:2]) + [0, 1, 2]
    for k in ks:
        r32 = orc32.pair(q32, orc32.profile(w.db, k))
        r64 = orc64.pair(q64, orc64.profile(w.db, k))
        # scores: equal to rounding except rare context-vector map bin flips
        dS = np.abs(r32["S"].astype(np.float64) - r64["S"])
        assert np.mean(dS < 1e-5) > 0.999
        assert dS.max() < 0.05
        assert abs(r32["best"] - r64["best"]) <= 1e-4 * max(1.0, abs(r64["best"])) + 0.05


def test_finalize_known_path(orc64):
    # a 6x6 score matrix with a straight diagonal path from (5,5) to (1,1)
    Smat = np.full((6, 6), -1.0)
    bt = np.zeros((6, 6), np.int8)
    vals = [1.0, 2.0, -0.5, 3.0, 1.5]
    for k, v in enumerate(vals):
        Smat[5 - k, 5 - k] = v
        bt[5 - k, 5 - k] = 3
    score, psts, bx, by = orc64.finalize(Smat, bt, 10.0, 5, 5)
    # correlation over the collected scores s_k (traceback order) with s_{-1..-4} = 0
    s = vals
    c = sum(s[k] * sum(s[max(0, k - 4):k]) for k in range(len(s)))
    adj = math.copysign(math.sqrt(abs(c / 2)), c)
    assert score == pytest.approx(10.0 + adj, rel=1e-12)
    assert psts == 4
    assert (bx, by) == (1, 1)


def test_score_threshold_formula(orc32, params):
    nq, dbsize = 400, 22_000_000
    thld, le = orc32.score_threshold(nq, dbsize, 10.0, params.gapped_K, params.gapped_lambda)
    ref = -math.log(30.0 / (params.gapped_K * nq * dbsize)) / params.gapped_lambda
    assert thld == pytest.approx(ref, rel=1e-5)
    assert le == pytest.approx(math.log(10.0), rel=1e-6)
    thld, le = orc32.score_threshold(nq, dbsize, 0.5, params.gapped_K, params.gapped_lambda)
    ref = -math.log(5.0 / (params.gapped_K * nq * dbsize)) / params.gapped_lambda
    assert thld == pytest.approx(ref, rel=1e-5)


def test_length_adjustment(orc32, params):
    # small databases: Gertz iteration converges to a positive length
    ss, dl = orc32.length_adjustment(params.gapped_lambda, params.gapped_K, params.gapped_alpha,
                                     params.gapped_beta, 1000, 1_000_000, 5000)
    assert 0 < dl < 1000
    m, n, N = 1000, 1_000_000, 5000
    assert ss == pytest.approx((m - dl) * (n - N * dl), rel=1e-2)
    # large search spaces with this K leave the space unadjusted (c < 0 branch)
    ss, dl = orc32.length_adjustment(params.gapped_lambda, params.gapped_K, params.gapped_alpha,
                                     params.gapped_beta, 400, 22_000_000, 100_000)
    assert (ss, dl) == (400 * 22_000_000, 0)


LENADJ = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "ref_lenadj")


@pytest.mark.skipif(not os.path.exists(LENADJ), reason="reference harness not built (no reference tree)")
def test_length_adjustment_matches_reference_code(orc32, params):
    """The oracle's search space and length adjustment equal those of the
    reference's own AbstractScoreMatrix::ComputeLengthAdjustment (built from
    its source by oracle/Makefile) over seeded query and database sizes,
    adjusted and unadjusted branches included."""
    import subprocess
    rng = np.random.default_rng(11)
    cases = [(400, 24_010_873, 100_000), (3000, 15_000_000, 50_000), (2000, 1000, 3), (1, 100, 1),
             (150, 680_000, 2000), (1000, 1_000_000, 5000)]
    for _ in range(200):
        m = int(rng.integers(1, 5000))
        N = int(rng.integers(1, 200_000))
        n = int(N * rng.integers(30, 2000))
        cases.append((m, n, N))
    inp = "".join("%d %d %d\n" % c for c in cases)
    out = subprocess.run([LENADJ, repr(params.gapped_lambda), repr(params.gapped_K), repr(params.gapped_alpha),
                          repr(params.gapped_beta)], input=inp, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    got = [tuple(int(x) for x in ln.split()) for ln in out.stdout.strip().splitlines()]
    assert len(got) == len(cases)
    nadj = 0
    for c, r in zip(cases, got):
        o = tuple(orc32.length_adjustment(params.gapped_lambda, params.gapped_K, params.gapped_alpha,
                                          params.gapped_beta, *c))
        assert o == r, (c, o, r)
        nadj += r[1] > 0
    assert nadj >= 5   # the Gertz iteration itself is exercised


def test_logz_model_is_the_map_forward(params, orc64):
    """The log-partition of the differentiable-alignment model at theta = 0 is
    the MAP stage's total probability (exact exp/log, unadjusted scores)."""
    rng = np.random.default_rng(21)
    q = S.random_profiles(rng, [45])
    d = S.random_profiles(rng, [38])
    qo, do = orc64.profile(q), orc64.profile(d)
    s0, ss, cv = orc64.score_parts(qo, do)
    Sk = s0 + params.ssswgt * ss + params.cvswgt * cv
    full, _ = orc64.score_matrix(qo, do)
    assert np.allclose(Sk, full, atol=1e-6)
    m = orc64.map(qo, do, Sk, np.zeros_like(Sk), -500.0, exact=True)
    assert orc64.logz(qo, do, Sk) == pytest.approx(m["logZ"], rel=1e-12)
