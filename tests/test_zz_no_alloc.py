"""The allocation-free phase-1 entry point c2_run_phase1_static, through the
C ABI: its results equal c2_run_phase1's on the same database and query, on
two calls in a row (the second reuses the static scratch); a database
beyond its compiled scratch limit, and a handle in the tensor-core score
mode, are refused before any launch."""
import ctypes as C

import numpy as np
import pytest

from comer2_b200 import synth as S

pytestmark = pytest.mark.gpu

C2_ERR_STATE = 4
C2_ERR_CAPACITY = 5


def _call(h, d_best, d_coords):
    return h.lib.c2_run_phase1_static(h._h, C.c_void_p(d_best.data_ptr()), C.c_void_p(d_coords.data_ptr()))


def test_phase1_static_matches_phase1(params):
    import torch
    from comer2_b200.native import Handle
    w = S.config(1, seed=5, scale=0.002)   # 200 profiles, lengths 30..2000
    h = Handle(params, 0)
    h.upload_db(w.db)
    h.set_query(w.queries[0])
    h.run_phase1()
    h.sync()
    best, coords = h.phase1()
    n = w.db.nprofiles
    for _ in range(2):
        d_best = torch.full((n,), -1.0, dtype=torch.float32, device="cuda:0")
        d_coords = torch.full((n,), -1, dtype=torch.int32, device="cuda:0")
        torch.cuda.synchronize()
        h._ck(_call(h, d_best, d_coords), "c2_run_phase1_static")
        h.sync()
        got_b = d_best.cpu().numpy()
        got_c = d_coords.cpu().numpy().view(np.uint32)
        assert np.array_equal(got_b.view(np.uint32), best.view(np.uint32))
        assert np.array_equal(got_c, coords)
    h.close()


def test_phase1_static_limit_boundary(params):
    """A longest profile of 52,416 positions fits the scratch (and gives
    c2_run_phase1's maxima); 52,417 is refused before any launch, and the
    message names the longest profile and the limit."""
    import torch
    from comer2_b200.native import Handle
    rng = np.random.default_rng(3)
    q = S.random_profiles(rng, [40])
    for L, ok in ((52_416, True), (52_417, False)):
        db = S.random_profiles(rng, [L])
        h = Handle(params, 0)
        h.upload_db(db)
        h.set_query(q)
        d_best = torch.zeros(1, dtype=torch.float32, device="cuda:0")
        d_coords = torch.zeros(1, dtype=torch.int32, device="cuda:0")
        torch.cuda.synchronize()
        before = h.launch_count()
        if ok:
            h._ck(_call(h, d_best, d_coords), "c2_run_phase1_static")
            h.sync()
            h.run_phase1()
            h.sync()
            best, coords = h.phase1()
            assert np.array_equal(d_best.cpu().numpy().view(np.uint32), best.view(np.uint32))
            assert np.array_equal(d_coords.cpu().numpy().view(np.uint32), coords)
        else:
            assert _call(h, d_best, d_coords) == C2_ERR_CAPACITY
            buf = C.create_string_buffer(512)
            h.lib.c2_last_error(h._h, buf, 512)
            assert b"static scratch limit" in buf.value
            assert b"(52417 positions)" in buf.value and b"(52416 positions)" in buf.value, buf.value
            assert h.launch_count() == before
        h.close()


def test_phase1_static_refuses_tensor_core_mode(params):
    """The static entry scores in FP32 only: a handle in the tensor-core
    score mode gets C2_ERR_STATE, not maxima of another arithmetic."""
    import torch
    from comer2_b200.native import Handle
    w = S.config(1, seed=6, scale=0.0005)
    h = Handle(params, 0)
    h.set_score_mode(1)
    h.upload_db(w.db)
    h.set_query(w.queries[0])
    n = w.db.nprofiles
    d_best = torch.zeros(n, dtype=torch.float32, device="cuda:0")
    d_coords = torch.zeros(n, dtype=torch.int32, device="cuda:0")
    torch.cuda.synchronize()
    before = h.launch_count()
    assert _call(h, d_best, d_coords) == C2_ERR_STATE
    assert h.launch_count() == before
    h.set_score_mode(0)
    h._ck(_call(h, d_best, d_coords), "c2_run_phase1_static")
    h.sync()
    h.close()
