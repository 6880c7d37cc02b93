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


if __name__ == "__main__":
    cmd = sys.argv[1]
    if cmd == "prepare":
        prepare()
    elif cmd == "run":
        run(sys.argv[2] if len(sys.argv) > 2 else os.path.join(REF, "out"))
    elif cmd == "collect":
        collect(sys.argv[2] if len(sys.argv) > 2 else os.path.join(REF, "out"))
