"""Device memory budget (c2_set_device_memory_limit, the reference's
--dev-mem): a budget too small for the database is refused with
C2_ERR_NOMEM before any allocation beyond it; a budget that holds the
database but not the phase-2 scratch of all candidate pairs makes c2_search
run phase 2 in candidate groups, with the same hits, statistics and
alignments as the unbounded search, and the handle's device memory never
above the budget."""
import numpy as np
import pytest

from comer2_b200 import synth as S

pytestmark = pytest.mark.gpu


def _pair_scratch_bytes(Lq, L, Lmax):
    """The library's estimate of one candidate pair's phase-2 device bytes
    (pair_scratch_bytes in c2_host.cu)."""
    ns = (Lq + 31) // 32
    return (9 * Lq * L + 2 * 10 * 4 * L + 2 * 4 * ns + 4 * ns * 2 + 2 * 4 * 32 * ns * (L + 31)
            + 2 * 5 * (Lq + Lmax + 1) + 512)


def _key(rec, buf):
    raw = bytes(buf)
    out = []
    for r in rec:
        o, L = int(r["aln_offset"]), int(r["alnlen"])
        out.append((int(r["profile"]), float(r["score"]), float(r["logE"]), float(r["lambda_"]), float(r["K"]),
                    int(r["beg"]), int(r["end"]), raw[o:o + 5 * (L + 1)]))
    return out


@pytest.mark.parametrize("mode", [0, 1])
def test_budget_groups_give_the_same_hits(params, mode):
    from comer2_b200.native import Handle
    w = S.config(4, seed=3, scale=0.0008)   # 1 x 3000 vs 40 profiles, 2 planted homologs
    h = Handle(params, 0)
    h.set_score_mode(mode)
    h.upload_db(w.db, total_positions=18_000_000, total_profiles=50_000)
    ref = _key(*h.search(w.queries[0], arrays=True))
    assert h.search_groups() == 1 and len(ref) >= 2
    h.close()
    h = Handle(params, 0)
    h.set_score_mode(mode)
    h.upload_db(w.db, total_positions=18_000_000, total_profiles=50_000)
    h.set_query(w.queries[0])
    h.run_phase1()
    h.sync()
    base = h.memory_use()
    # room for the phase-2 scratch of the longest hit's pair and a little
    # more, so that the candidates go in several groups
    Lq = int(w.queries[0].lengths[0])
    longest = max(int(w.db.lengths[x[0]]) for x in ref)
    limit = base + (2 << 20) + int(1.3 * _pair_scratch_bytes(Lq, longest, int(w.db.lengths.max())) / 0.9)
    h.set_memory_limit(limit)
    got = _key(*h.search(w.queries[0], arrays=True))
    assert h.search_groups() >= 2
    assert h.memory_use() <= limit
    assert got == ref
    h.close()


def test_budget_below_the_database_is_refused(params):
    from comer2_b200.native import C2Error, Handle
    w = S.config(1, seed=4, scale=0.002)
    h = Handle(params, 0)
    h.set_memory_limit(h.memory_use() + 1 * 2**20)
    with pytest.raises(C2Error, match="C2_ERR_NOMEM"):
        h.upload_db(w.db)
    assert h.memory_use() <= h.memory_use() + 2**20
    h.set_memory_limit(0)
    h.upload_db(w.db)
    assert len(h.search(w.queries[0])) >= 1
    h.close()
