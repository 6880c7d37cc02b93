"""Failure handling on the GPU without faulting it: the bounded waits of the
phase-2 strip pipelines give up after the poll limit set with
c2_set_wait_limit, the sweep returns, and the call reports the device status
(C2_ERR_DEVICE) instead of hanging; the handle then serves the next search."""
import pytest

from comer2_b200 import synth as S

pytestmark = pytest.mark.gpu


def _strip_key(hits):
    return [(int(x["profile"]), round(float(x["score"]), 4), x["strings"][0]) for x in hits]


def test_traceback_sweep_wait_timeout(params):
    """One poll per wait: strips started beside their predecessor give up at
    once in the traceback sweep (c2_run_finalize); c2_run_stats reports it."""
    from comer2_b200.native import C2Error, Handle
    w = S.config(1, seed=2, scale=0.003)   # 1 x 400 (13 strips) vs 300 profiles
    h = Handle(params, 0)
    h.upload_db(w.db)
    good = h.search(w.queries[0])
    assert len(good) > 0
    h.set_wait_limit(1)
    with pytest.raises(C2Error, match="timed out"):
        h.search(w.queries[0])
    h.set_wait_limit(0)
    again = h.search(w.queries[0])
    assert _strip_key(again) == _strip_key(good)
    h.close()


def test_map_sweep_wait_timeout(params):
    """The same in the MAP forward-backward and MAP DP sweeps: phase 1,
    finalisation and statistics run with the default limit, MAP with one
    poll per wait; c2_get_hits reports the timeout."""
    from comer2_b200.native import C2Error, Handle
    w = S.config(1, seed=9, scale=0.003)
    h = Handle(params, 0)
    h.upload_db(w.db)
    h.set_query(w.queries[0])
    h.run_phase1()
    h.run_finalize()
    h.run_stats()
    h.set_wait_limit(1)
    n = h.run_map()
    assert n > 0
    with pytest.raises(C2Error, match="timed out"):
        h.hits(n)
    h.set_wait_limit(0)
    assert len(h.search(w.queries[0])) == n
    h.close()
