"""Differentiable alignment on the GPU (c2_logz_fwd / c2_logz_bwd) against
the FP64 oracle: log-partition values, gradients against central finite
differences of the oracle's log-partition (step 1e-4), per-cell gradients,
the MM state posteriors against the oracle's MAP posteriors (exact exp/log,
no log-E-value score adjustment), and the torch.autograd wrapper.

Tolerances: logZ 2e-4 relative; gradients 2e-3 relative to max(1, |g|)
(FP32 sweeps against FP64 differences); posteriors 2e-4 absolute.
"""
import numpy as np
import pytest

from comer2_b200 import synth as S

pytestmark = pytest.mark.gpu

THETA = np.array([0.05, -0.1, 0.02, 0.0, 0.1, -0.05, 0.03])


def _setup(params, seed=7, lq=70, lens=(33, 64, 90, 41)):
    from comer2_b200.native import Handle
    rng = np.random.default_rng(seed)
    q = S.random_profiles(rng, [lq])
    parts = [S.planted_homolog(rng, q, L, seg_lo=20, seg_hi=40) for L in lens]
    db = S.concat(parts)
    h = Handle(params, 0)
    h.upload_db(db)
    h.set_query(q)
    return h, q, db


def _corners(lq, ld):
    """Cells of the two far corner triangles (the DP and MAP stages' corner masking)."""
    e = min(60, int(np.rint(0.34 * max(lq, ld))))
    y, x = np.mgrid[0:lq, 0:ld]
    return ((lq <= y + e) & (x <= e + y - lq)) | ((ld - e + y <= x) & (y < e))


def _oracle_S(orc, qo, do, wss, wcv):
    s0, ss, cv = orc.score_parts(qo, do)
    return s0 + wss * ss + wcv * cv, ss, cv


def test_logz_and_gradients(params, orc64):
    h, q, db = _setup(params)
    ks = list(range(db.nprofiles))
    wss, wcv = params.ssswgt, params.cvswgt
    z = h.logz_fwd(ks, THETA, wss, wcv)
    g = h.logz_bwd()
    qo = orc64.profile(q)
    hstep = 1e-4
    for k in ks:
        do = orc64.profile(db, k)
        Sk, ss, cv = _oracle_S(orc64, qo, do, wss, wcv)
        zr = orc64.logz(qo, do, Sk, THETA)
        assert z[k] == pytest.approx(zr, rel=2e-4), k
        for t in range(7):
            tp = THETA.copy(); tp[t] += hstep
            tm = THETA.copy(); tm[t] -= hstep
            fd = (orc64.logz(qo, do, Sk, tp) - orc64.logz(qo, do, Sk, tm)) / (2 * hstep)
            assert abs(g[k, t] - fd) <= 2e-3 * max(1.0, abs(fd)), (k, t, g[k, t], fd)
        fss = (orc64.logz(qo, do, Sk + hstep * ss, THETA) - orc64.logz(qo, do, Sk - hstep * ss, THETA)) / (2 * hstep)
        fcv = (orc64.logz(qo, do, Sk + hstep * cv, THETA) - orc64.logz(qo, do, Sk - hstep * cv, THETA)) / (2 * hstep)
        assert abs(g[k, 7] - fss) <= 2e-3 * max(1.0, abs(fss)), (k, g[k, 7], fss)
        assert abs(g[k, 8] - fcv) <= 2e-3 * max(1.0, abs(fcv)), (k, g[k, 8], fcv)
    h.close()


def test_cell_gradients_and_posteriors(params, orc64):
    h, q, db = _setup(params, seed=8, lq=45, lens=(38, 52))
    wss, wcv = params.ssswgt, params.cvswgt
    h.logz_fwd([0, 1], None, wss, wcv)
    h.logz_bwd()
    qo = orc64.profile(q)
    rng = np.random.default_rng(3)
    for k in (0, 1):
        L = int(db.lengths[k])
        ds, post = h.logz_cells(k, L)
        do = orc64.profile(db, k)
        Sk, _, _ = _oracle_S(orc64, qo, do, wss, wcv)
        # dlogZ/dS at sampled cells by central differences
        hstep = 1e-4
        for _ in range(12):
            i, j = int(rng.integers(0, q.lengths[0])), int(rng.integers(0, L))
            Sp = Sk.copy(); Sp[i, j] += hstep
            Sm = Sk.copy(); Sm[i, j] -= hstep
            fd = (orc64.logz(qo, do, Sp) - orc64.logz(qo, do, Sm)) / (2 * hstep)
            assert abs(ds[i, j] - fd) <= 2e-4 + 2e-3 * abs(fd), (k, i, j, ds[i, j], fd)
        # the MM posterior is the MAP stage's posterior of the same model
        m = orc64.map(qo, do, Sk, np.zeros_like(Sk), -500.0, exact=True, with_post=True)
        keep = ~_corners(int(q.lengths[0]), L)   # the MAP stage masks the two far corners
        assert np.abs(post - m["post"])[keep].max() <= 2e-4
        # expected emissions never exceed the posterior mass of the cell
        assert (ds <= post + 1e-5).all() and (ds >= -1e-6).all()
    h.close()


def test_torch_autograd_wrapper(params):
    import torch
    from comer2_b200.adjoint import logz
    h, q, db = _setup(params, seed=9)
    ks = list(range(db.nprofiles))
    theta = torch.tensor(THETA, dtype=torch.float32, requires_grad=True)
    wss = torch.tensor(float(params.ssswgt), requires_grad=True)
    wcv = torch.tensor(float(params.cvswgt), requires_grad=True)
    z = logz(h, ks, theta, wss, wcv)
    weights = torch.arange(1, len(ks) + 1, dtype=torch.float32)
    (weights * z).sum().backward()
    h.logz_fwd(ks, THETA, float(params.ssswgt), float(params.cvswgt))
    g = h.logz_bwd()
    want = (weights.numpy()[:, None] * g).sum(0)
    assert np.allclose(theta.grad.numpy(), want[:7], rtol=1e-5, atol=1e-5)
    assert wss.grad.item() == pytest.approx(want[7], rel=1e-5, abs=1e-5)
    assert wcv.grad.item() == pytest.approx(want[8], rel=1e-5, abs=1e-5)
    h.close()


def test_batch_of_independent_pairs(params, orc64):
    """c2_logz_fwd_batch: pairs with their own queries (lengths 20, 45, 70
    and 33; one strip, and several with a partial last strip), query 1 used
    twice, against the oracle's log-partition and finite-difference
    gradients of each pair, and the same values as the one-query call for
    the pairs of one query."""
    from comer2_b200.native import Handle
    rng = np.random.default_rng(12)
    qs = [S.random_profiles(rng, [n]) for n in (20, 45, 70, 33)]
    parts = [S.planted_homolog(rng, qs[i], L, seg_lo=10, seg_hi=18) for i, L in ((0, 50), (1, 36), (2, 64), (3, 27))]
    db = S.concat(parts + [S.random_profiles(rng, [58])])
    Q = S.concat(qs)
    qof = np.array([0, 1, 2, 3, 1], np.int32)
    prof = np.array([0, 1, 2, 3, 4], np.int32)
    wss, wcv = params.ssswgt, params.cvswgt
    h = Handle(params, 0)
    h.upload_db(db)
    h.set_query_batch(Q)
    z = h.logz_fwd_batch(qof, prof, THETA, wss, wcv)
    g = h.logz_bwd()
    hstep = 1e-4
    for k in range(len(prof)):
        qo, do = orc64.profile(qs[qof[k]]), orc64.profile(db, int(prof[k]))
        Sk, ss, cv = _oracle_S(orc64, qo, do, wss, wcv)
        assert z[k] == pytest.approx(orc64.logz(qo, do, Sk, THETA), rel=2e-4), k
        for t in (0, 2, 4):
            tp = THETA.copy(); tp[t] += hstep
            tm = THETA.copy(); tm[t] -= hstep
            fd = (orc64.logz(qo, do, Sk, tp) - orc64.logz(qo, do, Sk, tm)) / (2 * hstep)
            assert abs(g[k, t] - fd) <= 2e-3 * max(1.0, abs(fd)), (k, t, g[k, t], fd)
        fcv = (orc64.logz(qo, do, Sk + hstep * cv, THETA) - orc64.logz(qo, do, Sk - hstep * cv, THETA)) / (2 * hstep)
        assert abs(g[k, 8] - fcv) <= 2e-3 * max(1.0, abs(fcv)), (k, g[k, 8], fcv)
    ds, post = h.logz_cells(2, int(db.lengths[2]))
    assert ds.shape == (70, int(db.lengths[2])) and (ds <= post + 1e-5).all()
    # pairs 1 and 4 share query 1: the one-query call gives the same values
    h.set_query(qs[1])
    z1 = h.logz_fwd([1, 4], THETA, wss, wcv)
    g1 = h.logz_bwd()
    assert np.array_equal(z1, z[[1, 4]])
    assert np.array_equal(g1, g[[1, 4]])
    h.close()


def test_checkpointed_backward_matches_kept_states(params):
    """With room for every forward state the backward sweep reads them; under
    a device memory budget that leaves no room for them it recomputes each
    strip's states from the checkpoint row above (strip-row checkpointing).
    Both give the same log-partitions, gradients and per-cell values, bit for
    bit (the recomputation is the same arithmetic)."""
    from comer2_b200.native import Handle
    rng = np.random.default_rng(21)
    qs = [S.random_profiles(rng, [n]) for n in (70, 41)]
    parts = [S.planted_homolog(rng, qs[i % 2], L, seg_lo=15, seg_hi=30) for i, L in enumerate((64, 90, 57))]
    db = S.concat(parts)
    Q = S.concat(qs)
    qof, prof = np.array([0, 1, 0], np.int32), np.array([0, 1, 2], np.int32)
    wss, wcv = params.ssswgt, params.cvswgt
    res = []
    limit = 0
    for run in range(2):
        h = Handle(params, 0)
        h.upload_db(db)
        h.set_query_batch(Q)
        if run == 1:
            h.set_memory_limit(limit)
        z = h.logz_fwd_batch(qof, prof, THETA, wss, wcv)
        g = h.logz_bwd()
        cells = [h.logz_cells(k, int(db.lengths[prof[k]])) for k in range(3)]
        res.append((z, g, cells))
        if run == 0:
            # every budget byte the first run used, less the forward states
            # (5 floats a cell in wavefront order), plus one backward CTA's
            # scratch and a margin smaller than the forward states
            nc = sum(((int(Q.lengths[q]) + 31) // 32) * (int(db.lengths[p]) + 31) * 32 for q, p in zip(qof, prof))
            lmax = int(db.lengths.max())
            one_cta = 4 * (lmax + 31) * 160 * 4
            fbytes = 20 * nc
            assert fbytes > one_cta + (64 << 10)
            limit = h.memory_use() - fbytes + one_cta + (64 << 10)
        else:
            assert h.memory_use() <= limit
        h.close()
    (z0, g0, c0), (z1, g1, c1) = res
    assert np.array_equal(z0, z1)
    assert np.array_equal(g0, g1)
    for (a0, b0), (a1, b1) in zip(c0, c1):
        assert np.array_equal(a0, a1) and np.array_equal(b0, b1)
