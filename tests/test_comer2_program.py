"""The comer2 search program (comer2_b200/host/comer2.cpp): the reference
comer's command line over the C ABI.  On the CPU its input side is checked:
the parameter tables it loads (context-vector map smoothing included) against
the Python loader, which is pinned to the reference's own table readers; its
text-profile reader against comer2_b200.textfmt.read_profiles (both follow the
reference's reader); its database reader against c2_db2bin_read; and the
option file overriding the packaged option values."""
import os
import subprocess

import numpy as np
import pytest

from comer2_b200 import build as B
from comer2_b200 import synth as S
from comer2_b200 import textfmt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
needs_ref = pytest.mark.skipif(not os.path.exists(os.path.join(REF, "db2bin")),
                               reason="reference tools not built (oracle/build_ref.sh)")


def _prog():
    if not os.path.exists(B.PROG):
        B.build()
    return B.PROG


def _parse(out):
    d = {}
    for ln in out.splitlines():
        tag, _, rest = ln.partition(" ")
        if tag.endswith(".aa") or tag.endswith(".ssstate"):
            d[tag] = rest
        elif tag.endswith(".desc"):
            k, _, txt = rest.partition(" ")
            d.setdefault(tag, {})[int(k)] = txt
        elif tag in ("ints", "q.n", "d.n"):
            d[tag] = [int(x) for x in rest.split()]
        else:
            v = rest.split()
            d[tag] = np.array([float(x) for x in v[1:]], np.float32)
            assert int(v[0]) == d[tag].shape[0]
    return d


def _make_db(tmp, ps, names):
    pro = tmp / "pro"
    pro.mkdir()
    for k in range(ps.nprofiles):
        with open(pro / ("%s.pro" % names[k]), "w") as fh:
            textfmt.write_profile(fh, ps, k, names[k], names[k])
    opts = os.path.join(REF, "var", "options.txt")
    subprocess.run([os.path.join(REF, "makedb"), "-o", str(tmp / "db"), "-p", opts, "-d", str(pro)], check=True,
                   capture_output=True)
    subprocess.run([os.path.join(REF, "db2bin"), "-d", str(tmp / "db"), "-p", opts], check=True, capture_output=True)
    return str(tmp / "db")


@needs_ref
def test_program_inputs_match_the_readers(tmp_path, params):
    from comer2_b200.native import read_db2bin, read_db2bin_descriptions
    rng = np.random.default_rng(21)
    qs = S.concat([S.random_profiles(rng, [37]), S.random_profiles(rng, [80])])
    qf = tmp_path / "queries.pro"
    with open(qf, "w") as fh:
        for k in range(qs.nprofiles):
            textfmt.write_profile(fh, qs, k, "q%d" % k, "query number %d" % k)
    ps = S.random_profiles(rng, [31, 12, 140])
    db = _make_db(tmp_path, ps, ["pa", "pb", "pc"])
    opt = tmp_path / "opts.txt"
    opt.write_text("# test options\n[OPTIONS]\nEVAL = 3.5\nSSEMODEL = 1\n")
    r = subprocess.run([_prog(), "--print-inputs", "-i", str(qf), "-d", db, "-p", str(opt)], capture_output=True,
                       text=True, check=True)
    d = _parse(r.stdout)
    # parameters
    p = params
    sc = [p.ungapped_lambda, p.ungapped_K, p.ungapped_H, p.gapped_lambda, p.gapped_K, p.gapped_H, p.gapped_alpha,
          p.gapped_beta, 3.5, p.ssswgt, p.cvswgt, p.minpp]
    assert np.array_equal(d["scalars"], np.array(sc, np.float32))
    assert d["ints"] == [p.mapaln, p.x_uninf, 1, p.ssss_card, p.cvs2s_shift]
    assert np.array_equal(d["ssss"], p.ssss.reshape(-1))
    assert np.array_equal(d["cvkeys"], p.cvs2s_keys)
    assert np.array_equal(d["cvvals"], p.cvs2s_values)
    assert np.array_equal(d["nnw"], p.sse_nn_weights)
    # stacked text queries, as the Python reader reads them
    T = textfmt.read_profiles(qf.read_text())
    assert d["q.n"] == [2, int(T.npositions)]
    for f in ("bkg", "eno", "trn", "trg", "cv", "cvprior", "cvnorm2", "ss"):
        assert np.array_equal(d["q." + f], getattr(T, f).reshape(-1)), f
    assert d["q.aa"] == bytes(T.aa).decode() and d["q.ssstate"] == bytes(T.ssstate).decode()
    assert d["q.desc"] == {0: "query number 0", 1: "query number 1"}
    # the database, as c2_db2bin_read gives it
    D = read_db2bin(db + ".bin")
    for f in ("bkg", "eno", "trn", "trg", "cv", "cvprior", "cvnorm2", "ss"):
        assert np.array_equal(d["d." + f], getattr(D, f).reshape(-1)), f
    assert np.array_equal(d["d.lengths"], D.lengths.astype(np.float32))
    assert d["d.desc"] == dict(enumerate(read_db2bin_descriptions(db + ".bin")))


def test_program_usage_and_argument_errors(tmp_path):
    r = subprocess.run([_prog(), "-h"], capture_output=True, text=True)
    assert r.returncode == 0 and "-i <query_profiles>" in r.stdout
    r = subprocess.run([_prog(), "-i", "x.pro"], capture_output=True, text=True)
    assert r.returncode == 1 and "both -i and -d are required" in r.stderr
    bad = tmp_path / "bad.pro"
    bad.write_text("COMER profile v2.0\nLEN: 3\nNULL 1 2\n")
    r = subprocess.run([_prog(), "-i", str(bad), "-d", str(tmp_path / "nodb"), "--print-inputs"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "ERROR" in r.stderr
