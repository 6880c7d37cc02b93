"""Result files in the reference's Plain and JSON formats (c2_format_report,
no GPU).  Description wrapping and escaping are pinned to the reference's
own FormatDescription / FormatDescriptionJSON (src/liblib/fmtdescription.h)
through oracle/_ref/ref_fmtdesc, built from the reference tree; the rest of
the layout is checked against the hit records it prints."""
import json
import os
import re
import subprocess

import numpy as np
import pytest

from comer2_b200 import native as N

HERE = os.path.dirname(os.path.abspath(__file__))
REFBIN = os.path.join(HERE, "..", "oracle", "_ref", "ref_fmtdesc")
WORDS = ["alpha", "beta", "sp|P12345|KINASE_HUMAN", "protein", "x" * 37, "a/b", 'say"hi"', "back\\slash", "",
         "domain-containing", "(fragment)", "1.2.3"]


def _desc(rng, nwords):
    out = []
    for _ in range(nwords):
        out.append(WORDS[rng.integers(len(WORDS))])
        out.append(rng.choice([" ", "  ", "\t", " \t "]))
    return "".join(out).strip(" \t") or "x"


def _ref_format(cases):
    """[(mode, maxoutlen, indent, width, addsep, desc)] -> formatted strings (reference code)."""
    inp = "".join("%d %d %d %d %d\t%s\n" % c for c in cases)
    r = subprocess.run([REFBIN], input=inp.encode("latin-1"), capture_output=True, check=True)
    parts = r.stdout.decode("latin-1").split("\x1e\n")
    assert parts[-1] == ""
    return parts[:-1]


def _one_hit(desc_len=10, alnlen=130, profile=0):
    h = np.zeros(1, N.HIT_DTYPE)
    h["profile"] = profile
    h["score"] = 87.25
    h["logE"] = -12.3
    h["alnlen"] = alnlen
    h["idts"], h["psts"], h["gaps"] = 40, 20, 9
    h["beg"] = (5 << 16) | 11
    h["E"], h["H"], h["K"], h["lambda_"], h["K_est"], h["lambda_est"] = -0.7, 0.5, 0.12, 0.31, 0.05, 0.27
    h["smin"], h["smax"] = -9, 11
    rng = np.random.default_rng(alnlen)
    aa = np.frombuffer(b"ACDEFGHIKLMNPQRSTVWY", np.uint8)
    q = aa[rng.integers(0, 20, alnlen)].copy()
    t = aa[rng.integers(0, 20, alnlen)].copy()
    q[rng.random(alnlen) < 0.05] = ord("-")
    t[rng.random(alnlen) < 0.05] = ord("-")
    m = np.where(q == t, q, ord(" ")).astype(np.uint8)
    qs = np.frombuffer(b"CEH", np.uint8)[rng.integers(0, 3, alnlen)]
    ts = np.frombuffer(b"CEH", np.uint8)[rng.integers(0, 3, alnlen)]
    z = np.zeros(1, np.uint8)
    alns = np.concatenate([q, z, m, z, t, z, qs, z, ts, z])
    return h, alns, (q.tobytes().decode(), m.tobytes().decode(), t.tobytes().decode(), qs.tobytes().decode(),
                     ts.tobytes().decode())


def _report(fmt, hits, alns, descs, **kw):
    n = max(1, int(hits["profile"].max()) + 1 if len(hits) else 1)
    args = dict(query_length=300, query_eno=8.4, db_lengths=[200] * n, db_eno=[6.1] * n, db_desc=descs,
                query_desc="test query", db_positions=123456, db_profiles=789, logevthld=np.log(10.0),
                searchspace=2.5e7, deltalen=21, ref_lambda=0.3176, ref_K=0.1342, gapped_lambda=0.2688,
                gapped_K=0.0411, progname="comer", progversion="2.30")
    args.update(kw)
    return N.format_report(fmt, hits, alns, **args)


@pytest.mark.skipif(not os.path.exists(REFBIN), reason="reference harness not built (no reference tree)")
@pytest.mark.parametrize("seed", range(4))
def test_descriptions_match_reference_formatters(seed):
    rng = np.random.default_rng(seed)
    h, alns, _ = _one_hit()
    for trial in range(12):
        desc = _desc(rng, int(rng.integers(1, 120)))
        dsclen = int(rng.choice([20, 64, 200, 1024]))
        dscwidth = int(rng.choice([10, 13, 40, 80, 300]))
        plain = _report(N.REPORT_PLAIN, h, alns, [desc], dsclen=dsclen, dscwidth=dscwidth)
        js = _report(N.REPORT_JSON, h, alns, [desc], dsclen=dsclen, dscwidth=dscwidth)
        width = dscwidth if 13 < dscwidth else 1
        ref_hit, ref_ann, ref_jhit, ref_jann = _ref_format([
            (0, dsclen, 13, width, ord(">"), desc), (0, 75, 0, 75, 0, desc),
            (1, dsclen, 0, 0, 0, desc), (1, 75, 0, 0, 0, desc)])
        # the hit record's description line(s), from '>' to the scores
        i = plain.index("\n\n\n\n>") + 4
        j = plain.index("\n  Length/ENO:", i)
        assert plain[i:j] == ref_hit, (desc, dsclen, dscwidth)
        # the annotation: description padded to 75, score, E-value
        k = plain.index("E-value\n\n") + len("E-value\n\n")
        line = plain[k:plain.index("\n", k)]
        assert line[:75] == ref_ann.ljust(75)[:max(75, len(ref_ann))][:75], (desc,)
        assert line[75:] == " %7.0f %7.1g" % (87.25, np.exp(np.float32(-12.3)))
        # JSON strings
        m = re.search(r'"target_description": "(.*?)",\n      "query_length"', js, re.S)
        assert m and m.group(1) == ref_jhit, (desc,)
        m = re.search(r'"summary_entry": \{\n      "description": "(.*?)",\n      "score"', js, re.S)
        assert m and m.group(1) == ref_jann, (desc,)


@pytest.mark.skipif(not os.path.exists(REFBIN), reason="reference harness not built (no reference tree)")
def test_query_description_budget_matches_reference():
    rng = np.random.default_rng(11)
    h, alns, _ = _one_hit()
    for _ in range(10):
        qd = _desc(rng, int(rng.integers(50, 400)))
        for dsclen, dscwidth in ((1024, 80), (100, 40), (3000, 60)):
            plain = _report(N.REPORT_PLAIN, h, alns, ["d"], query_desc=qd, dsclen=dsclen, dscwidth=dscwidth)
            head = "comer 2.30\n\n\n"
            assert plain.startswith(head)
            qh = "\n Query (300 positions):\n"
            budget = min(4096 - len(head), dsclen) - len(qh)
            ref, = _ref_format([(0, budget, 0, dscwidth, 0, qd)])
            i = plain.index(qh) + len(qh)
            j = plain.index("\n\n Database(s):", i)
            assert plain[i:j] == ref


def test_plain_alignment_fragments_and_scores():
    h, alns, (q, m, t, qs, ts) = _one_hit(alnlen=130)
    txt = _report(N.REPORT_PLAIN, h, alns, ["target one"], alnwidth=60)
    assert " Score = 87.25 (" in txt and "Expect = " in txt
    assert " Identities = 40/130 (30%), Positives = 20/130 (15%), Gaps = 9/130 (6%)" in txt
    qlines = re.findall(r"^Query: +(\d+) (\S+) (\d+) *$", txt, re.M)
    tlines = re.findall(r"^Sbjct: +(\d+) (\S+) (\d+) *$", txt, re.M)
    assert len(qlines) == len(tlines) == 3   # 130 columns in fragments of 60
    assert "".join(x[1] for x in qlines) == q and "".join(x[1] for x in tlines) == t
    # coordinates: 1-based starts, ends counted without gaps, consecutive fragments
    pos = 12
    for beg, frag, end in qlines:
        assert int(beg) == pos
        pos += len(frag) - frag.count("-")
        assert int(end) == pos - 1 or (frag.count("-") == len(frag) and int(end) == pos)
    ss = re.findall(r"^struct {7}(\S+)$", txt, re.M)
    assert "".join(ss[0::2]) == qs and "".join(ss[1::2]) == ts
    # no SS lines without the SS weight
    assert "struct" not in _report(N.REPORT_PLAIN, h, alns, ["t"], print_ss=False)
    assert "Computed  ungapped,        0.1200   0.3100" in txt
    assert "Effective search space, 25000000" in txt


def test_json_parses_and_carries_the_records():
    h1, a1, s1 = _one_hit(alnlen=70, profile=0)
    h2, a2, s2 = _one_hit(alnlen=45, profile=1)
    h2["aln_offset"] = len(a1)
    hits = np.concatenate([h1, h2])
    alns = np.concatenate([a1, a2])
    js = _report(N.REPORT_JSON, hits, alns, ["one", "two"])
    d = json.loads(js)["comer_search"]
    assert d["query"]["length"] == 300 and d["database"]["number_of_profiles"] == 789
    assert [e["summary_entry"]["description"] for e in d["search_summary"]] == ["one", "two"]
    recs = [r["hit_record"] for r in d["search_hits"]]
    for r, s, n in zip(recs, (s1, s2), (70, 45)):
        a = r["alignment"]
        assert (a["query_aln"], a["middle"], a["target_aln"]) == (s[0], s[1], s[2])
        assert a["aln_length"] == n and a["query_from"] == 12 and a["target_from"] == 6
        assert a["query_to"] == 12 + n - s[0].count("-") - 1
    assert d["search_statistics"]["effective_query_length"] == 300 - 21
    assert d["search_statistics"]["effective_database_size"] == 123456 - 789 * 21
    # NOALNS below NOHITS: the reference's writer puts a record separator after
    # the last alignment record (its separator test uses the hit-list bound)
    js1 = _report(N.REPORT_JSON, hits, alns, ["one", "two"], nalns=1)
    assert js1.count('"hit_record"') == 1 and '    }},\n  ],\n  "search_statistics"' in js1


def test_no_hits_messages():
    h = np.zeros(0, N.HIT_DTYPE)
    a = np.zeros(1, np.uint8)
    plain = N.format_report(N.REPORT_PLAIN, h, a, query_length=50, query_eno=3.0, db_lengths=[1], db_eno=[1.0],
                            logevthld=np.log(10.0), db_positions=10, db_profiles=1)
    assert " No profiles found below an e-value threshold of 10." in plain
    js = json.loads(N.format_report(N.REPORT_JSON, h, a, query_length=50, query_eno=3.0, db_lengths=[1],
                                    db_eno=[1.0], logevthld=np.log(10.0), db_positions=10, db_profiles=1))
    assert js["comer_search"]["search_hits"] == [] and js["comer_search"]["search_summary"] == []
    assert js["comer_search"]["message"].startswith("No profiles found below an e-value threshold of 10")
