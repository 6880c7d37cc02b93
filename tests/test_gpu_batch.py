"""Multi-query search (c2_search_batch) and database sharing (c2_share_db) on
the GPU: every query's hits from a batch spread over worker handles equal
those of the same query searched alone, field for field and byte for byte
(same kernels, same data; only the scheduling differs)."""
import numpy as np
import pytest

from comer2_b200 import synth as S

pytestmark = pytest.mark.gpu


def _same(a, b):
    (ra, ba), (rb, bb) = a, b
    assert len(ra) == len(rb)
    for name in ra.dtype.names:
        assert np.array_equal(ra[name], rb[name]), name
    assert bytes(ba[:len(bb)]) == bytes(bb[:len(ba)])


@pytest.mark.parametrize("mode", [0, 1])   # FP32 scores; split-BF16 tensor-core scores
def test_batch_matches_single_searches(params, mode):
    from comer2_b200.native import Handle
    w = S.config(2, seed=5, scale=0.025)   # 6 queries LN(250, 0.6) vs 500 profiles, homologs of query 0
    assert len(w.queries) == 6
    h = Handle(params, 0)
    h.set_score_mode(mode)
    h.upload_db(w.db)
    alone = [h.search(q, arrays=True) for q in w.queries]
    assert len(alone[0][0]) > 0
    batch = h.search_batch(S.concat(w.queries), nworkers=3)
    assert len(batch) == len(alone)
    for a, b in zip(alone, batch):
        _same(a, b)
    # more workers than queries, and one worker
    for nw in (8, 1):
        again = h.search_batch(S.concat(w.queries[:2]), nworkers=nw)
        for a, b in zip(alone[:2], again):
            _same(a, b)


def test_shared_database_and_reupload(params):
    from comer2_b200.native import Handle
    w = S.config(2, seed=6, scale=0.025)
    h = Handle(params, 0)
    h.upload_db(w.db)
    h2 = Handle(params, 0)
    h2.share_db(h)
    q = w.queries[0]
    _same(h.search(q, arrays=True), h2.search(q, arrays=True))
    # a new database on h: workers made for the old one are remade, and h2
    # keeps searching the old one
    w2 = S.config(2, seed=7, scale=0.025)
    before = h2.search(q, arrays=True)
    h.search_batch(S.concat(w.queries[:2]), nworkers=2)
    h.upload_db(w2.db)
    _same(h2.search(q, arrays=True), before)
    b = h.search_batch(S.concat(w2.queries[:2]), nworkers=2)
    for qq, got in zip(w2.queries[:2], b):
        _same(h.search(qq, arrays=True), got)


def test_search_to_result_files(params):
    """A search's hits written in both reference formats: the JSON parses and
    carries every hit's alignment; the Plain file lists the same hits."""
    import json
    from comer2_b200 import native as N
    w = S.config(1, seed=3, scale=0.003)
    h = N.Handle(params, 0)
    h.upload_db(w.db)
    q = w.queries[0]
    rec, alns = h.search(q, arrays=True)
    assert len(rec) > 0
    ss, dl = h.search_space()
    thld, logevthld = h.thresholds()
    kw = dict(query_length=int(q.lengths[0]), query_eno=float(q.eno[0]), db_lengths=w.db.lengths,
              db_eno=w.db.eno, db_desc=["profile %d" % k for k in range(w.db.nprofiles)],
              db_positions=int(w.db.npositions), db_profiles=int(w.db.nprofiles), logevthld=logevthld,
              searchspace=float(ss), deltalen=int(dl), ref_lambda=params.ungapped_lambda, ref_K=params.ungapped_K,
              gapped_lambda=params.gapped_lambda, gapped_K=params.gapped_K)
    d = json.loads(N.format_report(N.REPORT_JSON, rec, alns, **kw))["comer_search"]
    assert len(d["search_hits"]) == len(rec)
    for r, hit in zip(d["search_hits"], rec):
        a = r["hit_record"]["alignment"]
        o = int(hit["aln_offset"])
        L = int(hit["alnlen"])
        assert a["query_aln"] == bytes(alns[o:o + L]).decode()
        assert r["hit_record"]["target_description"] == "profile %d" % int(hit["profile"])
    plain = N.format_report(N.REPORT_PLAIN, rec, alns, **kw)
    assert plain.count("\n>profile ") == len(rec)
