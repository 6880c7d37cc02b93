"""The comer2 program end to end on the GPU: a query file of two stacked
text profiles against a database made by the reference's makedb + db2bin,
result files in both formats.  Its hits equal the C ABI search of the same
profiles (as the library's readers read them), in the order and with the
scores, E-values and alignments the JSON file reports."""
import json
import os
import subprocess

import numpy as np
import pytest

from comer2_b200 import synth as S
from comer2_b200 import textfmt

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
needs_ref = pytest.mark.skipif(not os.path.exists(os.path.join(REF, "db2bin")),
                               reason="reference tools not built (oracle/build_ref.sh)")


@needs_ref
def test_program_matches_the_library(tmp_path, params):
    from comer2_b200 import build as B
    from comer2_b200.native import Handle, read_db2bin, read_db2bin_descriptions
    rng = np.random.default_rng(31)
    w = S.config(1, seed=6, scale=0.0015)   # 150 profiles, 3 planted homologs of query 0
    q2 = S.random_profiles(rng, [120])
    pro = tmp_path / "pro"
    pro.mkdir()
    for k in range(w.db.nprofiles):
        with open(pro / ("p%04d.pro" % k), "w") as fh:
            textfmt.write_profile(fh, w.db, k, "p%04d" % k, "profile %d of the test database" % k)
    opts = os.path.join(REF, "var", "options.txt")
    subprocess.run([os.path.join(REF, "makedb"), "-o", str(tmp_path / "tdb"), "-p", opts, "-d", str(pro)],
                   check=True, capture_output=True)
    subprocess.run([os.path.join(REF, "db2bin"), "-d", str(tmp_path / "tdb"), "-p", opts], check=True,
                   capture_output=True)
    qf = tmp_path / "two.pro"
    with open(qf, "w") as fh:
        textfmt.write_profile(fh, w.queries[0], 0, "q0", "first query")
        textfmt.write_profile(fh, q2, 0, "q1", "second query")
    out = tmp_path / "out"
    for fmt in ("1", "0"):
        r = subprocess.run([B.PROG, "-i", str(qf), "-d", str(tmp_path / "tdb"), "-o", str(out), "-f", fmt, "-v"],
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
    assert sorted(os.listdir(out)) == ["two__0.json", "two__0.out", "two__1.json", "two__1.out"]
    # the same search through the library
    D = read_db2bin(str(tmp_path / "tdb.bin"))
    desc = read_db2bin_descriptions(str(tmp_path / "tdb.bin"))
    Q = textfmt.read_profiles(qf.read_text())
    h = Handle(params, 0)
    h.upload_db(D)
    for qn in range(2):
        hits = h.search(_one(Q, qn))
        doc = json.loads(open(out / ("two__%d.json" % qn)).read())["comer_search"]
        assert doc["query"]["description"] == ("first query", "second query")[qn]
        recs = [x["hit_record"] for x in doc["search_hits"]]
        assert [x["target_description"] for x in recs] == [desc[x["profile"]] for x in hits]
        for x, r in zip(hits, recs):
            a = r["alignment"]
            assert a["score"] == pytest.approx(x["score"], abs=0.01)
            assert a["evalue"] == pytest.approx(float(np.exp(np.float64(x["logE"]))), rel=0.06, abs=1e-300)
        plain = open(out / ("two__%d.out" % qn)).read()
        for x in hits[:5]:
            assert desc[x["profile"]] in plain
    assert len(json.loads(open(out / "two__0.json").read())["comer_search"]["search_hits"]) >= 3
    h.close()


def _one(P, k):
    L, o = int(P.lengths[k]), int(P.offsets[k])
    return S.ProfileSet(np.array([L], np.int32), np.zeros(1, np.int64), P.bkg[k:k + 1], P.eno[k:k + 1],
                        P.trn[o + k:o + k + L + 1], P.trg[o:o + L], P.cv[o:o + L], P.cvprior[o:o + L],
                        P.cvnorm2[o:o + L], P.ss[o:o + L], P.ssstate[o:o + L], P.aa[o:o + L],
                        P.trn_int[o + k:o + k + L + 1], P.trg_int[o:o + L])


def _makedb(tmp, name, ps, ks):
    pro = tmp / (name + "_pro")
    pro.mkdir()
    for k in ks:
        with open(pro / ("p%04d.pro" % k), "w") as fh:
            textfmt.write_profile(fh, ps, k, "p%04d" % k, "profile %d of the test database" % k)
    opts = os.path.join(REF, "var", "options.txt")
    subprocess.run([os.path.join(REF, "makedb"), "-o", str(tmp / name), "-p", opts, "-d", str(pro)],
                   check=True, capture_output=True)
    subprocess.run([os.path.join(REF, "db2bin"), "-d", str(tmp / name), "-p", opts], check=True,
                   capture_output=True)
    return str(tmp / name)


@needs_ref
def test_program_in_database_chunks_writes_the_same_files(tmp_path, params):
    """The same queries against two databases (4,000 short profiles, a few
    homologs planted) three ways: whole on one GPU; under a --dev-mem limit
    that splits them into chunks spanning both files, double-buffered (the
    next chunk uploaded on a second handle while the current one is
    searched); and split across two GPU workers (--dev-N=,0,0, both on GPU
    0 here).  Every chunk is uploaded with the totals of both databases, so
    the result files are the same byte for byte."""
    from comer2_b200 import build as B
    from comer2_b200.native import Handle, read_db2bin
    rng = np.random.default_rng(32)
    q0 = S.random_profiles(rng, [110])
    q1 = S.random_profiles(rng, [90])
    hom = [S.planted_homolog(rng, q0, int(L), seg_lo=25, seg_hi=40) for L in (45, 52, 60)]
    db = S.concat([S.random_profiles(rng, list(rng.integers(30, 61, 1997)))] + hom +
                  [S.random_profiles(rng, list(rng.integers(30, 61, 2000)))])
    n = db.nprofiles
    dbs = [_makedb(tmp_path, "da", db, range(0, n // 2)), _makedb(tmp_path, "db", db, range(n // 2, n))]
    qf = tmp_path / "two.pro"
    with open(qf, "w") as fh:
        textfmt.write_profile(fh, q0, 0, "q0", "first query")
        textfmt.write_profile(fh, q1, 0, "q1", "second query")
    # the program's chunk plan: one handle's database bytes within half of
    # what it does not hold, two handles per GPU (each half the limit) once
    # there is more than one chunk; the limit is set for chunks of about a
    # quarter of the positions
    D = [read_db2bin(d + ".bin") for d in dbs]
    N = sum(int(x.lengths.sum()) for x in D)
    P = sum(x.nprofiles for x in D)
    lmax = max(int(x.lengths.max()) for x in D)
    h = Handle(params, 0)
    used0 = h.memory_use()
    fixed = h.db_device_bytes(0, 0, lmax)
    whole = h.db_device_bytes(N, P, lmax)
    h.close()
    cap2 = fixed + (whole - fixed) // 4
    limit = 2 * (2 * cap2 + used0)
    assert (limit - used0) // 2 < whole   # one handle cannot hold the whole database
    mb = -(-limit // 2**20)
    outs, nchunks = {}, {}
    for tag, extra in (("whole", []), ("dbuf", ["--dev-mem=%d" % mb]), ("gpus", ["--dev-N=,0,0"])):
        out = tmp_path / tag
        for fmt in ("1", "0"):
            r = subprocess.run([B.PROG, "-i", str(qf), "-d", ",".join(dbs), "-o", str(out), "-f", fmt, "-v"] + extra,
                               capture_output=True, text=True, timeout=600)
            assert r.returncode == 0, r.stderr
            nchunks[tag] = int(r.stderr.split("database in ")[1].split(" chunk")[0])
        outs[tag] = {f: open(out / f, "rb").read() for f in sorted(os.listdir(out))}
    assert nchunks["whole"] == 1 and 3 <= nchunks["dbuf"] <= 6 and nchunks["gpus"] >= 2, nchunks
    assert list(outs["whole"]) == ["two__0.json", "two__0.out", "two__1.json", "two__1.out"]
    assert outs["whole"] == outs["dbuf"]
    assert outs["whole"] == outs["gpus"]
    doc = json.loads(outs["whole"]["two__0.json"])["comer_search"]
    assert len(doc["search_hits"]) >= 3
