"""Host-side parameter parsing, smoothing and the C-ABI surface (CPU only)."""
import ctypes
import os
import re

import numpy as np
import pytest

from comer2_b200 import params as P
from comer2_b200 import synth as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_default_tables(params):
    assert params.ssss.shape == (30, 30)
    assert np.array_equal(params.ssss, params.ssss.T)
    assert params.cvs2s_card == 93 and params.cvs2s_shift == 5
    assert np.all(np.diff(params.cvs2s_keys) > 0)
    assert params.cvs2s_keys[params.cvs2s_shift] == 0.0
    assert len(params.sse_nn_weights) == 93
    assert (params.ssswgt, params.cvswgt, params.mapaln, params.eval) == (np.float32(0.12), np.float32(0.15), 1, 10.0)


def test_cvs2s_smoothing_running_mean():
    keys = [-1.0, -0.5, 0.0, 0.5, 1.0, 1.5, 2.0]
    vals = [1.0, 2.0, 3.0, 4.0, 5.0, 6.0, P.CVS2S_PLUS]
    k, v, shift = P.smooth_cvs2s(keys, vals)
    assert shift == 2
    # first full window (5 values) mean = 3, assigned to the first three entries
    assert v[0] == v[1] == v[2] == np.float32(3.0)
    # next window (2..6) mean = 4 for index 3; the '+' tail takes the last mean
    assert v[3] == np.float32(4.0)
    assert v[4] == v[5] == v[6] == np.float32(4.0)


def test_cvs2s_inserts_missing_keys():
    keys = [0.0, 0.5, 1.5, 2.0, 2.5, 3.0]
    vals = [1.0, 1.0, 1.0, 1.0, 1.0, 1.0]
    k, v, shift = P.smooth_cvs2s(keys, vals)
    assert list(k) == [0.0, 0.5, 1.0, 1.5, 2.0, 2.5, 3.0]
    assert np.all(v == np.float32(1.0))


def test_parse_ssss_layout():
    txt = "ssss= 0 +1\n0000 11\nCardinality = 3\n 1\n 2 3\n 4 5 6\n"
    card, tri = P.parse_ssss(txt)
    m = P.ssss_full(card, tri)
    assert m.tolist() == [[1, 2, 4], [2, 3, 5], [4, 5, 6]]


def test_synth_quantisation():
    rng = np.random.default_rng(0)
    ps = S.random_profiles(rng, [40, 30])
    assert ps.trg_int.sum(1).tolist() == [10000] * 70
    assert (ps.trg_int >= 1).all()
    t = ps.trn_int
    assert (t[:, 0:3].sum(1) == 10000).all() and (t[:, 3:5].sum(1) == 10000).all() and (t[:, 5:7].sum(1) == 10000).all()
    # working values as the text reader computes them
    assert np.allclose(ps.trn[:, :3], np.log(t[:, :3] / 10000.0), atol=1e-6)
    assert np.allclose(ps.trn[:, 3:], 0.4 * np.log(t[:, 3:] / 10000.0), atol=1e-6)
    assert ps.trn.shape[0] == ps.npositions + ps.nprofiles


def test_library_exports_header_symbols():
    """The built C-ABI library exports every function include/comer2_b200.h declares."""
    from comer2_b200 import native
    hdr = open(os.path.join(ROOT, "include", "comer2_b200.h")).read()
    declared = sorted(set(re.findall(r"\b(c2_[a-z0-9_]+)\s*\(", hdr)))
    assert declared, "no declarations found"
    lib = ctypes.CDLL(native.LIB_PATH)
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(native.EXPORTS) == declared


def test_create_rejects_cv_maps_beyond_shared_memory(params):
    """c2_create refuses, before touching a device, a CV map larger than the
    FP32 score kernels' shared-memory tables hold (256 entries; the
    reference's map has 93)."""
    import copy
    from comer2_b200 import native
    lib = native.load()
    p = copy.deepcopy(params)
    card = 300
    p.cvs2s_keys = np.arange(card, dtype=np.float32) * 0.5 - 2.5
    p.cvs2s_values = np.zeros(card, np.float32)
    assert p.cvs2s_card == card
    keep = native._Keep()
    sp = native.make_params(p, keep)
    h = ctypes.c_void_p()
    st = lib.c2_create(0, ctypes.byref(sp), ctypes.byref(h))
    assert native.STATUS_NAMES.get(st) == "C2_ERR_ARG"
    assert not h.value


REFTAB = os.path.join(ROOT, "oracle", "_ref", "ref_tables")


@pytest.mark.skipif(not os.path.exists(REFTAB), reason="reference table harness not built (no reference tree)")
def test_tables_match_reference_readers(params):
    """The SS table and the smoothed CV map that the loader hands to the
    kernels equal what the reference's own readers (SSSScores, CVS2Scores,
    built from its source by oracle/Makefile) make of its parameter files."""
    import subprocess
    # the harness reads the reference tree's parameter files (the directory is
    # fixed when oracle/Makefile builds it)
    out = subprocess.run([REFTAB], capture_output=True, text=True, timeout=60)
    if out.returncode != 0 and "reading the tables failed" in out.stderr:
        pytest.skip("the reference tree's parameter files are not on this machine")
    assert out.returncode == 0, out.stderr
    lines = {ln.split()[0]: ln for ln in out.stdout.splitlines()}
    ss, cv = lines["ssss"], lines["cvs2s"]
    a = ss.split()
    card, n = int(a[1]), int(a[2])
    tri = np.array([float(x) for x in a[3:3 + n]], np.float32)
    assert card == params.ssss_card and n == card * (card + 1) // 2
    # VirtScores::GetScore: entry (r, c), r >= c, at c + r (r + 1) / 2
    full = np.zeros((card, card), np.float32)
    for r in range(card):
        for c in range(card):
            hi, lo = max(r, c), min(r, c)
            full[r, c] = tri[lo + hi * (hi + 1) // 2]
    assert np.array_equal(full, np.asarray(params.ssss, np.float32).reshape(card, card))
    b = cv.split()
    shift, m = int(b[2]), int(b[3])
    kv = np.array([float(x) for x in b[4:4 + 2 * m]], np.float32).reshape(m, 2)
    assert (m, shift) == (params.cvs2s_card, params.cvs2s_shift)
    assert np.array_equal(kv[:, 0], params.cvs2s_keys)
    assert np.array_equal(kv[:, 1], params.cvs2s_values)


@pytest.mark.skipif(not os.path.exists(REFTAB), reason="reference table harness not built (no reference tree)")
def test_cv_constants_match_reference(orc32):
    """1/kappa0, PowerNU0 and CTERM of the CV score as the oracle computes
    them (c2_host.cu's cv_constants follows the same float steps) equal the
    reference's _TCTXVECT object's values."""
    import subprocess
    out = subprocess.run([REFTAB], capture_output=True, text=True, timeout=60)
    if out.returncode != 0 and "reading the tables failed" in out.stderr:
        pytest.skip("the reference tree's parameter files are not on this machine")
    assert out.returncode == 0, out.stderr
    line = [ln for ln in out.stdout.splitlines() if ln.startswith("cvconst ")][0].split()
    ref = [np.float32(float(x)) for x in line[1:4]]
    a, b, c = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
    orc32.lib.orc_cv_constants(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
    assert [np.float32(a.value), np.float32(b.value), np.float32(c.value)] == ref


def test_create_refuses_unknown_options(params):
    """MAPALN outside {0, 1}, SSEMODEL outside 0..2 and negative score-term
    weights are refused by c2_create with C2_ERR_ARG before any device call,
    rather than answered with results of another configuration."""
    import copy
    from comer2_b200.native import C2Error, Handle
    for field, value in (("mapaln", 2), ("mapaln", -1), ("ssemodel", 3), ("ssemodel", -1), ("ssswgt", -0.1),
                         ("cvswgt", -0.5)):
        p = copy.deepcopy(params)
        setattr(p, field, value)
        with pytest.raises(C2Error, match="C2_ERR_ARG"):
            Handle(p, 0)
