"""Golden fixtures from the reference COMER2 itself.

The reference has no tests or golden vectors, so this script pins the oracle
and the GPU path to outputs of the reference's own ``comer`` program (built
for sm_100a by ``oracle/build_ref.sh``) run on a B200:

  prepare  (here)       seeded workloads -> COMER text profiles -> the
                        reference's makedb + db2bin -> oracle/_ref/inputs/
  run      (B200 host)  comer -i q.pro -d db -o out -f 1 (JSON output),
                        options with SCOADJ = no -> OUT (argument; default
                        oracle/_ref/out/)
  collect  (here)       JSON outputs -> tests/golden/ref_<case>.json

The workloads are regenerated from their seeds by comer2_b200.synth, so the
fixtures hold only the reference's results (hit list, scores, E-values,
alignments).
"""
import glob
import json
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
REF = os.path.join(ROOT, "oracle", "_ref")
INP = os.path.join(REF, "inputs")

# case name -> (config, seed, scale)
CASES = {
    "c1_s2": (1, 2, 0.003),
    "c1_s9": (1, 9, 0.003),
    "c0_s4": (0, 4, 0.05),
}


def workload(case):
    from comer2_b200 import synth as S
    n, seed, scale = CASES[case]
    return S.config(n, seed=seed, scale=scale)


def prepare():
    from comer2_b200 import textfmt
    for case in CASES:
        w = workload(case)
        d = os.path.join(INP, case)
        shutil.rmtree(d, ignore_errors=True)
        os.makedirs(os.path.join(d, "pro"))
        with open(os.path.join(d, "q.pro"), "w") as fh:
            textfmt.write_profile(fh, w.queries[0], 0, "query", "query")
        files = []
        for k in range(w.db.nprofiles):
            f = os.path.join(d, "pro", "p%06d.pro" % k)
            with open(f, "w") as fh:
                textfmt.write_profile(fh, w.db, k, "p%06d" % k, "p%06d" % k)
            files.append(f)
        opts = os.path.join(REF, "var", "options.txt")
        subprocess.run([os.path.join(REF, "makedb"), "-o", os.path.join(d, "db"), "-p", opts, "-d",
                        os.path.join(d, "pro")], check=True, capture_output=True)
        subprocess.run([os.path.join(REF, "db2bin"), "-d", os.path.join(d, "db"), "-p", opts], check=True,
                       capture_output=True)
        shutil.rmtree(os.path.join(d, "pro"))
        print("prepared", case, w.db.nprofiles, "profiles")


def run(outroot):
    opts = os.path.join(REF, "var", "options.txt")
    for case in CASES:
        d = os.path.join(INP, case)
        out = os.path.join(outroot, case)
        os.makedirs(out, exist_ok=True)
        # --dev-mem bounds the reference's device heap (its default takes all
        # memory, which leaves none for loading its kernels' module)
        env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
        r = subprocess.run(["timeout", "300", os.path.join(REF, "comer"), "-i", os.path.join(d, "q.pro"), "-d",
                            os.path.join(d, "db"), "-o", out, "-p", opts, "-f", "1", "--dev-N=1",
                            "--dev-mem=16000"],
                           capture_output=True, text=True, env=env)
        with open(os.path.join(out, "comer.log"), "w") as fh:
            fh.write(r.stdout + "\n---stderr---\n" + r.stderr + "\nrc=%d\n" % r.returncode)
        print(case, "rc", r.returncode)


def collect(outroot):
    """Summarise the reference's JSON output per case into ref_b200_outcome.json:
    the number of reported hits, how many have a finite score and E-value, and
    the first hits' fields."""
    summary = {}
    for case in CASES:
        files = glob.glob(os.path.join(outroot, case, "*.json"))
        if not files:
            summary[case] = {"error": "no output"}
            continue
        t = open(files[0]).read().replace("-nan", "NaN").replace("nan", "NaN").replace("inf", "Infinity")
        hits = json.loads(t)["comer_search"]["search_hits"]
        recs = []
        for h in hits:
            r = h["hit_record"]
            a = r["alignment"]
            recs.append({"target": r["target_description"], "score": a["score"], "evalue": a["evalue"],
                         "expected_score": a["expected_score"], "aln_length": a["aln_length"],
                         "min_score": a["min_score"], "max_score": a["max_score"]})
        import math
        finite = sum(1 for x in recs if math.isfinite(x["score"]) and math.isfinite(x["evalue"])
                     and abs(x["score"]) < 1e6)
        summary[case] = {"config": CASES[case], "n_hits": len(recs), "n_finite": finite, "first": recs[:5]}
    with open(os.path.join(HERE, "ref_b200_outcome.json"), "w") as fh:
        json.dump(summary, fh, indent=1)
    print(json.dumps({k: (v.get("n_hits"), v.get("n_finite")) for k, v in summary.items()}))


# option variants of the reference runs: name -> (SSSWGT, CVSWGT)
VARIANTS = {"w00": (0.0, 0.0), "w0cv": (0.0, 0.15), "wss0": (0.12, 0.0), "w00aln0": (0.0, 0.0)}
# options besides the weights: MAPALN 0 (Viterbi alignments) for the aln0 runs
VARIANT_MAPALN = {"w00aln0": 0}
HIT_FIELDS = ("score", "bit_score", "evalue", "pvalue", "n_identities", "n_positives", "n_gaps", "aln_length",
              "query_from", "query_to", "target_from", "target_to", "query_secstr", "target_secstr", "query_aln",
              "target_aln", "middle", "computed_K_ungapped", "computed_lambda_ungapped", "estimated_K_gapped",
              "estimated_lambda_gapped", "entropy", "expected_score", "min_score", "max_score")


def _load_ref_json(path):
    """The reference's JSON result file as {search_statistics, database, hits}.
    Read field by field: its writer prints inf / nan tokens, and with the SS
    weight at 0 it ends every hit record after the "query_secstr" key (the
    record's remaining fields are not written), so the file is not JSON.
    Each hit holds the fields its record has."""
    import re
    t = open(path).read()
    num = r"(-?(?:\d+(?:\.\d*)?(?:[eE][-+]?\d+)?|nan|inf))"

    def val(x):
        x = x.strip()
        if x.startswith('"'):
            return x[1:-1]
        if x in ("nan", "-nan"):
            return float("nan")
        if x in ("inf", "-inf"):
            return float(x)
        return float(x) if any(c in x for c in ".eE") else int(x)

    out = {"hits": []}
    for blk in re.split(r'\{"hit_record": \{', t)[1:]:
        rec = {}
        for m in re.finditer(r'"(\w+)": ("[^"\n]*"|' + num + r')\s*[,\n}]', blk):
            rec.setdefault(m.group(1), val(m.group(2)))
        out["hits"].append(rec)
    ss = re.search(r'"search_statistics": \{(.*?)\}', t, re.S)
    out["search_statistics"] = {m.group(1): val(m.group(2)) for m in
                                re.finditer(r'"(\w+)": ' + num, ss.group(1))} if ss else {}
    db = re.search(r'"number_of_profiles": (\d+),\s*"number_of_positions": (\d+)', t)
    out["database"] = {"number_of_profiles": int(db.group(1)), "number_of_positions": int(db.group(2))} if db else {}
    return out


def collect_variants(outroot):
    """The reference's results with score-term weights switched off
    (options SSSWGT / CVSWGT = 0, run by the variant runs) -> one fixture per
    case and variant, tests/golden/ref_<case>_<variant>.json: the search
    statistics and, per reported hit, the fields of its JSON record with the
    db profile index (descriptions are p%06d)."""
    import math
    summary = {}
    for case in CASES:
        for var, (wss, wcv) in VARIANTS.items():
            files = glob.glob(os.path.join(outroot, "%s_%s" % (case, var), "*.json"))
            if not files:
                summary["%s_%s" % (case, var)] = "no output"
                continue
            d = _load_ref_json(files[0])
            hits = []
            for r in d["hits"]:
                rec = {"profile": int(r["target_description"][1:]), "target_length": r["target_length"],
                       "target_eno": r["target_eno"]}
                rec.update({k: r[k] for k in HIT_FIELDS if k in r})
                hits.append(rec)
            finite = sum(1 for x in hits if math.isfinite(float(x["score"])) and math.isfinite(float(x["evalue"])))
            fx = {"case": case, "config": CASES[case], "variant": var, "ssswgt": wss, "cvswgt": wcv,
                  "search_statistics": d["search_statistics"], "database": d["database"],
                  "n_hits": len(hits), "n_finite": finite, "hits": hits}
            with open(os.path.join(HERE, "ref_%s_%s.json" % (case, var)), "w") as fh:
                json.dump(fx, fh, indent=0, allow_nan=True)
            summary["%s_%s" % (case, var)] = (len(hits), finite)
    print(json.dumps(summary))


def _load_ref_plain(path):
    """Hit records of the reference's Plain result file (-f 0): per hit the
    profile, lengths/ENOs, score, bits, E-value, identities, positives,
    gaps, the alignment rows (query, middle, target) with their first and
    last positions, and the statistics lines (K and lambda computed and
    estimated, entropy, expected score, score range)."""
    import re
    lines = open(path).read().split("\n")
    hits = []
    i = 0
    while i < len(lines):
        if not lines[i].startswith(">"):
            i += 1
            continue
        h = {"profile": int(lines[i][1:].strip()[1:]), "query_aln": "", "middle": "", "target_aln": ""}
        i += 1
        m = re.search(r"Query = (\d+)/([\d.]+), Sbjct = (\d+)/([\d.]+)", lines[i])
        h["target_length"], h["target_eno"] = int(m.group(3)), float(m.group(4))
        i += 1
        while not lines[i].startswith(" Score"):
            i += 1
        m = re.search(r"Score = (\S+) \((\S+) bits\),\s+Expect = (\S+), P-value = (\S+)", lines[i])
        h["score"], h["bit_score"], h["evalue"], h["pvalue"] = (float(m.group(1)), float(m.group(2)),
                                                              float(m.group(3)), float(m.group(4)))
        i += 1
        m = re.search(r"Identities = (\d+)/(\d+)", lines[i])
        h["n_identities"], h["aln_length"] = int(m.group(1)), int(m.group(2))
        ps = re.search(r"Positives = (\d+)/", lines[i])   # not printed when 0
        h["n_positives"] = int(ps.group(1)) if ps else 0
        g = re.search(r"Gaps = (\d+)/", lines[i])
        h["n_gaps"] = int(g.group(1)) if g else 0
        i += 1
        first = True
        while i < len(lines) and not lines[i].strip().startswith("K") and not lines[i].startswith(">"):
            ln = lines[i]
            if ln.startswith("Query:"):
                m = re.match(r"(Query:\s+(\d+) )(\S+) (\d+)", ln)
                col, seg = len(m.group(1)), m.group(3)
                if first:
                    h["query_from"] = int(m.group(2))
                h["query_to"] = int(m.group(4))
                h["query_aln"] += seg
                h["middle"] += lines[i + 1][col:col + len(seg)].ljust(len(seg))
                t = re.match(r"Sbjct:\s+(\d+) (\S+) (\d+)", lines[i + 2])
                if first:
                    h["target_from"] = int(t.group(1))
                h["target_to"] = int(t.group(3))
                h["target_aln"] += t.group(2)
                first = False
                i += 3
                continue
            i += 1
        if i < len(lines) and lines[i].strip().startswith("K"):
            cu = lines[i + 1].split()
            eg = lines[i + 2].split()
            h["computed_K_ungapped"], h["computed_lambda_ungapped"] = cu[-2], cu[-1]
            h["estimated_K_gapped"], h["estimated_lambda_gapped"] = eg[-2], eg[-1]
            m = re.search(r"Entropy, (\S+); Expected, (\S+); Min/Max, (-?\d+)/(-?\d+)", lines[i + 3])
            h["entropy"], h["expected_score"] = float(m.group(1)), float(m.group(2))
            h["min_score"], h["max_score"] = int(m.group(3)), int(m.group(4))
            i += 4
        hits.append(h)
    return hits


def collect_plain(outroot, variant="w00"):
    """The Plain result files of the weight-0 runs -> tests/golden/
    ref_<case>_<variant>_plain.json (every field the Plain records hold,
    alignments and statistics lines included)."""
    summary = {}
    for case in CASES:
        files = glob.glob(os.path.join(outroot, "%s_%s_f0" % (case, variant), "*.out"))
        if not files:
            summary[case] = "no output"
            continue
        hits = _load_ref_plain(files[0])
        wss, wcv = VARIANTS[variant]
        fx = {"case": case, "config": CASES[case], "variant": variant, "ssswgt": wss, "cvswgt": wcv,
              "mapaln": VARIANT_MAPALN.get(variant, 1), "format": "plain", "n_hits": len(hits), "hits": hits}
        with open(os.path.join(HERE, "ref_%s_%s_plain.json" % (case, variant)), "w") as fh:
            json.dump(fx, fh, indent=0)
        # the file itself, for the writers' byte-for-byte comparison
        shutil.copyfile(files[0], os.path.join(HERE, "ref_%s_%s.out" % (case, variant)))
        summary[case] = len(hits)
    print(json.dumps(summary))


# the runs of the reference on a B200 and their options (besides -f, --dev-N=1
# and --dev-mem=4000): folder -> (options file, extra arguments)
RUNS = {
    "default": ("options.txt", ""),
    "w00": ("options_w00.txt", ""),
    "w0cv": ("options_w0cv.txt", ""),
    "wss0": ("options_wss0.txt", ""),
    "el200": ("options.txt", "--dev-expected-length=200"),
    "wss0_el200": ("options_wss0.txt", "--dev-expected-length=200"),
}


def summarize(outroots):
    """Per case and run: reported hits, how many have a finite score and
    E-value -> tests/golden/ref_b200_outcome.json."""
    import math
    out = {"runs": {k: {"options": v[0], "args": v[1]} for k, v in RUNS.items()}, "cases": {}}
    for case in CASES:
        row = {}
        for run in RUNS:
            for root in outroots:
                files = glob.glob(os.path.join(root, "%s_%s" % (case, run), "*.json"))
                if run == "default":
                    files = files or glob.glob(os.path.join(root, case, "*.json"))
                if files:
                    hits = _load_ref_json(files[0])["hits"]
                    fin = sum(1 for h in hits if math.isfinite(float(h.get("score", float("nan"))))
                              and math.isfinite(float(h.get("evalue", float("nan")))) and abs(h["score"]) < 1e6)
                    row[run] = {"n_hits": len(hits), "n_finite": fin}
                    break
        out["cases"][case] = row
    with open(os.path.join(HERE, "ref_b200_outcome.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print(json.dumps(out["cases"]))


if __name__ == "__main__":
    cmd = sys.argv[1]
    if cmd == "prepare":
        prepare()
    elif cmd == "run":
        run(sys.argv[2] if len(sys.argv) > 2 else os.path.join(REF, "out"))
    elif cmd == "collect":
        collect(sys.argv[2] if len(sys.argv) > 2 else os.path.join(REF, "out"))
    elif cmd == "collect_variants":
        collect_variants(sys.argv[2])
    elif cmd == "collect_plain":
        collect_plain(sys.argv[2], sys.argv[3] if len(sys.argv) > 3 else "w00")
    elif cmd == "summarize":
        summarize(sys.argv[2:])
