"""Benchmark of the COMER2 search hot path on B200.

Workload: one query profile of length 400 against 100,000 database profiles
(lengths lognormal, median 200, sigma 0.6, clipped to [30, 2000]; 2% planted
homologs), seeded synthetic data (no public profile database is used).  One
step = one complete search: fused score + Viterbi DP over all pairs, DP
finalisation, statistics and E-values, MAP alignment of the hits.

  value : GCUPS = L_q * sum(L_d) / step time, database and query resident in
          HBM, timed with CUDA events on the launching stream;
  e2e   : the same metric through the C ABI with host buffers: query upload,
          the search, and the hits (records and alignments) back to the host.

With --impl reference the line reports the CPU implementation of the same
method (the C restatement, float, one thread per host core) on a bounded
sample of the same workload; the reference has no CPU search path of its own.
Multi-GPU runs (torchrun) give every rank its own database of the same size
(weak scaling, no collective on the data path); times are the max over ranks.
--workload 0 / 4 measure the other single-query configurations the same way;
--workload 2 times the 64-query configuration end to end through the batch call.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GCUPS (score+DP+MAP)"
UNIT = "GCUPS"
WORKLOAD = "1 query L=400 vs 100000 db profiles LN(200,0.6)[30,2000], 2% planted homologs"
# --workload n: the synthetic configuration n (synth.config); 1 is the headline
WORKLOADS = {
    0: "1 query L=150 vs 2000 db profiles U[50,500]",
    1: WORKLOAD,
    2: "64 queries LN(250,0.6)[50,1500] vs 20000 db profiles LN(200,0.6)[30,2000], 2% homologs of query 0",
    3: "differentiable alignment: log-partition forward + adjoint, 256 independent pairs, query and db lengths U[100,600]",
    4: "1 query L=3000 (6 domains) vs 50000 db profiles LN(300,0.6)[30,2000], 5% planted homologs",
}


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def _bf16_peak():
    """Dense BF16 tensor throughput (TFLOP/s): measured burst figure, else the fallback."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            return float(json.load(fh).get("bf16_tflops", 1590.0))
    return 1590.0


def _traffic_per_position():
    """DRAM bytes per db position of the phase-1 kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "p1_kernel_traffic.json")
    if os.path.exists(p):
        with open(p) as fh:
            return float(json.load(fh)["dram_bytes_per_db_position"])
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def start(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _max_over_ranks(x, world, backend):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if backend == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_port_gcups(w, params, seconds=12.0, threads=None):
    """The C restatement of the whole method (float) on the host cores, on a
    bounded sample of the workload: phase 1 + DP finalisation over a random
    sample of db profiles (one POSIX thread per core inside the oracle), then,
    for the sampled pairs that pass the whole database's score threshold, the
    statistics and E-values and, for those within the E-value threshold, the
    MAP alignment (a thread pool over pairs).  Returns GCUPS over the whole
    sample time, the thread count, a description of the sample and the
    per-stage seconds."""
    from concurrent.futures import ThreadPoolExecutor
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle_py import Oracle
    threads = threads or os.cpu_count()
    orc = Oracle(params, 32)
    qs = w.queries[0]
    q = orc.profile(qs)
    Lq = int(qs.lengths[0])
    N, P = int(w.db.lengths.sum()), int(w.db.nprofiles)
    thld, logevthld = orc.score_threshold(Lq, N, params.eval, params.gapped_K, params.gapped_lambda)
    sspace, _ = orc.length_adjustment(params.gapped_lambda, params.gapped_K, params.gapped_alpha,
                                      params.gapped_beta, Lq, N, P)
    rng = np.random.default_rng(123)
    order = rng.permutation(w.db.nprofiles)
    # calibrate phase 1 on a small sample, then size the sample to ~`seconds`
    cal = order[:200]
    t0 = time.perf_counter()
    orc.batch_phase1(q, w.db, cal, threads, 1e9)
    dt = time.perf_counter() - t0
    rate = Lq * float(w.db.lengths[cal].sum()) / max(dt, 1e-6)
    want = rate * seconds
    lens = w.db.lengths[order].astype(np.float64) * Lq
    n = int(np.searchsorted(np.cumsum(lens), want)) + 1
    ks = order[:max(1, min(n, w.db.nprofiles))]
    cells = Lq * float(w.db.lengths[ks].sum())
    t0 = time.perf_counter()
    best, score = orc.batch_phase1(q, w.db, ks, threads, thld)
    t_p1 = time.perf_counter() - t0
    passed = [int(k) for k, b, sc in zip(ks, best, score) if b > thld and sc > thld]

    def stats_of(k):
        d = orc.profile(w.db, k)
        r = orc.pair(q, d)
        off, nd = int(w.db.offsets[k]), int(w.db.lengths[k])
        st = orc.stats(r["S"], qs.aa, w.db.aa[off:off + nd], r["score"], r["psts"], qs.eno[0], w.db.eno[k],
                       float(sspace), params.x_uninf)
        return k, d, r, st

    def map_of(item):
        k, d, r, st = item
        off, nd = int(w.db.offsets[k]), int(w.db.lengths[k])
        return orc.map(q, d, r["S"], r["MOD"], st["logEpA"], qss=qs.ssstate, dss=w.db.ssstate[off:off + nd])

    with ThreadPoolExecutor(threads) as ex:
        t0 = time.perf_counter()
        st = list(ex.map(stats_of, passed))
        t_st = time.perf_counter() - t0
        hits = [x for x in st if not (logevthld < x[3]["logE"])]
        t0 = time.perf_counter()
        list(ex.map(map_of, hits))
        t_map = time.perf_counter() - t0
    total = t_p1 + t_st + t_map
    stages = {"phase1+finalize_s": t_p1, "stats_s": t_st, "map_s": t_map, "pairs_passed": len(passed),
              "pairs_mapped": len(hits)}
    return cells / total / 1e9, threads, (
        "%d of %d db profiles (%.3g cells): phase 1 + DP finalisation, then statistics of the %d pairs over the "
        "full database's score threshold and MAP of the %d within the E-value threshold" % (
            len(ks), w.db.nprofiles, cells, len(passed), len(hits))), stages


def fp64_error(w, params, hits_rec, searchspace, nmax=24):
    """Error of the reported hits against the FP64 oracle (the same method in
    double): for up to nmax hits, |DP score - FP64| / |FP64| and |log E -
    FP64 log E|; maxima and medians."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle_py import Oracle
    orc = Oracle(params, 64)
    qs = w.queries[0]
    q = orc.profile(qs)
    ds, de = [], []
    for rec in hits_rec[:nmax]:
        k = int(rec["profile"])
        r = orc.pair(q, orc.profile(w.db, k))
        off, nd = int(w.db.offsets[k]), int(w.db.lengths[k])
        st = orc.stats(r["S"], qs.aa, w.db.aa[off:off + nd], r["score"], r["psts"], qs.eno[0], w.db.eno[k],
                       float(searchspace), params.x_uninf)
        ds.append(abs(float(rec["score"]) - r["score"]) / max(1e-30, abs(r["score"])))
        de.append(abs(float(rec["logE"]) - st["logE"]))
    if not ds:
        return None
    return {"hits_checked": len(ds), "score_rel_max": max(ds), "score_rel_median": float(np.median(ds)),
            "logE_abs_max": max(de), "logE_abs_median": float(np.median(de)),
            "note": "device results (phase 1 in the bench's score form, FP32 finalisation, statistics and MAP) "
                    "against the oracle in double precision on the same pairs"}


def batch_workload(args):
    """Configuration 2: 64 queries through c2_search_batch, timed end to end
    (queries from host memory, every query's hits and alignments back)."""
    import torch
    from comer2_b200 import params as P, synth as S
    from comer2_b200.native import Handle, SCORE_BF16_TC, SCORE_FP32, C2Error  # noqa: F401
    prm = P.load_default()
    w = S.config(2, seed=0, scale=args.scale)
    qs = S.concat(w.queries)
    cells = float(qs.npositions) * float(w.db.npositions)
    h = Handle(prm, 0)
    h.upload_db(w.db)
    out = {}
    for name, mode in (("bf16", SCORE_BF16_TC), ("fp32", SCORE_FP32)):
        h.set_score_mode(mode)
        for _ in range(max(1, args.warmup)):
            h.search_batch(qs, nworkers=2)
        ts, nh = [], 0
        for _ in range(max(1, args.steps)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = h.search_batch(qs, nworkers=2)
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
            nh = int(sum(len(x[0]) for x in r))
        out[name] = {"value": cells / float(np.mean(ts)) / 1e9, "s_per_step": float(np.mean(ts)), "hits": nh}
    main_r = out[args.score_mode]
    line = {"metric": METRIC, "value": main_r["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": main_r["s_per_step"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16" if args.score_mode == "bf16" else "f32",
            "data": "synthetic",
            "config": {"workload": WORKLOADS[2], "queries": len(w.queries), "cells": cells, "scale": args.scale,
                       "timing": "end to end through c2_search_batch (two workers: a query's phase 2 beside "
                                 "the next query's phase 1)"},
            "e2e": {"value": main_r["value"], "unit": UNIT}, "hits": main_r["hits"],
            "score_forms": out}
    print(json.dumps(line))
    h.close()


def adjoint_workload(args):
    """Configuration 3: the log-partition of the MAP forward model and its
    hand-written adjoint (c2_logz_fwd_batch + c2_logz_bwd: dlogZ/dtheta,
    dlogZ/dwss, dlogZ/dwcv per pair) over 256 independent pairs, query and db
    profile lengths each U[100,600]; cells = forward cells of the 256 pairs,
    device-timed per forward + backward step (CUDA events)."""
    import torch
    from comer2_b200 import params as P, synth as S
    from comer2_b200.native import Handle
    prm = P.load_default()
    w = S.config(3, seed=0, scale=args.scale)
    Q = S.concat(w.queries)
    npair = w.db.nprofiles
    qof = np.arange(npair, dtype=np.int32)
    pairs = np.arange(npair, dtype=np.int32)
    cells = float((Q.lengths.astype(np.float64) * w.db.lengths.astype(np.float64)).sum())
    h = Handle(prm, 0)
    st = torch.cuda.Stream()
    h.set_stream(st.cuda_stream)
    h.upload_db(w.db)
    theta = np.zeros(7, np.float32)
    h.set_query_batch(Q)
    for _ in range(max(3, args.warmup)):
        h.logz_fwd_batch(qof, pairs, theta, 0.12, 0.15)
        h.logz_bwd()
    n0 = h.launch_count()
    ts = []
    for _ in range(max(1, args.steps)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        z = h.logz_fwd_batch(qof, pairs, theta, 0.12, 0.15)
        g = h.logz_bwd()
        e1.record(st)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    launches = h.launch_count() - n0
    ms = float(np.mean(ts))
    # end to end: the queries packed and uploaded from host memory each step too
    te = []
    for _ in range(max(1, args.steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        h.set_query_batch(Q)
        h.logz_fwd_batch(qof, pairs, theta, 0.12, 0.15)
        h.logz_bwd()
        te.append(time.perf_counter() - t0)
    e2e_s = float(np.mean(te))
    line = {"metric": "GCUPS (log-partition forward + adjoint)", "value": cells / (ms * 1e-3) / 1e9, "unit": UNIT,
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOADS[3], "pairs": int(npair), "cells": cells,
                       "timing": "device (CUDA events), queries resident; logZ and the 9 gradients per pair copied "
                                 "to the host each step"},
            "e2e": {"value": cells / e2e_s / 1e9, "unit": UNIT,
                    "h2d_bytes_per_step": int(Q.npositions * (64 + 6) * 4 + (Q.npositions + Q.nprofiles) * 28
                                              + Q.nprofiles * 80 + npair * 8),
                    "d2h_bytes_per_step": int(npair * 40),
                    "note": "wall clock: the queries packed on the host and uploaded, forward, backward"},
            "gpu_launches": int(launches),
            "finite": bool(np.isfinite(z).all() and np.isfinite(g).all())}
    print(json.dumps(line))
    h.close()


def kernel_list(args):
    """Device time of every kernel (and copy / set) of one search of a
    single-query workload, BF16 score form, database and query resident, from
    the CUDA activity records of torch.profiler (CUPTI): real launch times of a
    normal run, not a replaying profiler's.  One JSON line per kernel name."""
    import collections
    import torch
    from torch.profiler import ProfilerActivity, profile
    from comer2_b200 import params as P, synth as S
    from comer2_b200.native import Handle, SCORE_BF16_TC
    if args.workload not in (0, 1, 4):
        raise SystemExit("--kernel-list: workloads 0, 1 and 4")
    w = S.config(args.workload, seed=0, scale=args.scale)
    q = w.queries[0]
    h = Handle(P.load_default(), 0)
    h.upload_db(w.db)
    h.set_score_mode(SCORE_BF16_TC)
    h.search(q)
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        h.search(q)
        torch.cuda.synchronize()
    agg = collections.OrderedDict()
    for e in prof.events():
        if e.device_type.name != "CUDA":
            continue
        nm = e.name.split("(")[0]
        low = nm.lower()
        if "memset" in low or "memcpy" in low:
            nm = "[memset]" if "memset" in low else "[memcpy]"
        a = agg.setdefault(nm, [0, 0.0])
        a[0] += 1
        a[1] += e.device_time_total
    tot = sum(v[1] for v in agg.values())
    for k, (n, t) in sorted(agg.items(), key=lambda x: -x[1][1]):
        print(json.dumps({"workload": args.workload, "kernel": k, "launches": n, "ms": round(t / 1e3, 3),
                          "share": round(t / tot, 4)}))
    h.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="database size factor (1.0 = 100k profiles)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (profiling runs)")
    ap.add_argument("--score-mode", default="bf16", choices=["fp32", "bf16"],
                    help="phase-1 score contractions: FP32 CUDA cores or split-BF16 tensor cores")
    ap.add_argument("--kernel-list", action="store_true",
                    help="instead of the bench line: the device time of every kernel of one search of the "
                         "workload (0, 1 or 4), from a CUPTI activity trace (torch.profiler), one JSON line each")
    ap.add_argument("--workload", type=int, default=1, choices=sorted(WORKLOADS),
                    help="synthetic configuration (1: the headline; 2: 64 queries through the batch call)")
    args = ap.parse_args()
    if args.kernel_list:
        return kernel_list(args)
    if args.workload == 2:
        return batch_workload(args)
    if args.workload == 3:
        return adjoint_workload(args)
    if args.workload != 1:
        global WORKLOAD
        WORKLOAD = WORKLOADS[args.workload]
    world, rank, local = _dist()
    from comer2_b200 import params as P, synth as S
    prm = P.load_default()

    if args.impl == "reference":
        if rank != 0:
            return
        w = S.config(args.workload, seed=0, scale=args.scale)
        vals = []
        thr = samp = stages = None
        for _ in range(max(1, args.steps)):
            g, thr, samp, stages = cpu_port_gcups(w, prm, seconds=args.cpu_seconds / max(1, args.steps))
            vals.append(g)
        v = float(np.median(vals))
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "f32",
                "data": "synthetic", "config": {"workload": WORKLOAD, "scale": args.scale},
                "cpu_baseline": {"value": v, "unit": UNIT, "cores": thr, "kind": "port", "sample": samp,
                                 "stages": stages},
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "note": "the reference has no CPU search path; this is the C restatement of its method"}
        print(json.dumps(line))
        return

    import torch
    backend = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl"
        torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    from comer2_b200.native import Handle

    w = S.config(args.workload, seed=rank, scale=args.scale)
    q = w.queries[0]
    Lq = int(q.lengths[0])
    cells = Lq * int(w.db.lengths.sum())
    h = Handle(prm, local)
    from comer2_b200.native import SCORE_BF16_TC, SCORE_FP32
    h.set_score_mode(SCORE_BF16_TC if args.score_mode == "bf16" else SCORE_FP32)
    st = torch.cuda.Stream()
    h.set_stream(st.cuda_stream)
    t0 = time.perf_counter()
    h.upload_db(w.db)
    upload_s = time.perf_counter() - t0

    def device_step():
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        with torch.cuda.stream(st):
            e[0].record(st)
            h.run_phase1()
            e[1].record(st)
            h.run_finalize()
            h.run_stats()
            nh = h.run_map()
            e[2].record(st)
        e[2].synchronize()
        return e[0].elapsed_time(e[2]), e[0].elapsed_time(e[1]), nh

    def measure(mode):
        """Device-timed search (inputs resident) and end-to-end search through
        the C ABI (query from host memory, hits and alignments back) in one
        score mode."""
        h.set_score_mode(mode)
        h.set_query(q)
        for _ in range(args.warmup):
            device_step()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        l0 = h.launch_count()
        tot, p1 = [], []
        for _ in range(args.steps):
            a, b, _ = device_step()
            tot.append(a)
            p1.append(b)
        torch.cuda.synchronize()
        launches = h.launch_count() - l0
        if world > 1:
            torch.distributed.barrier()
        ms = _max_over_ranks(float(np.mean(tot)), world, backend)
        p1ms = _max_over_ranks(float(np.mean(p1)), world, backend)
        e2e = []
        hits = []
        # untimed end-to-end searches first: the first one after a mode change
        # allocates the host-transfer buffers of the alignment read-back
        for _ in range(args.warmup):
            h.search(q, arrays=True)
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            hits = h.search(q, arrays=True)
            torch.cuda.synchronize()
            e2e.append((time.perf_counter() - t0) * 1e3)
        e2e_ms = _max_over_ranks(float(np.mean(e2e)), world, backend)
        return {"ms": ms, "p1ms": p1ms, "e2e_ms": e2e_ms, "launches": launches, "hits": hits}

    from comer2_b200.native import SCORE_BF16_TC, SCORE_FP32
    clk = ClockSampler(local)
    clk.start()
    res = {"bf16": measure(SCORE_BF16_TC), "fp32": measure(SCORE_FP32)}
    clocks = clk.stop()
    main_r = res[args.score_mode]
    ms, p1ms, e2e_ms, launches, hits = (main_r["ms"], main_r["p1ms"], main_r["e2e_ms"], main_r["launches"],
                                        main_r["hits"])

    def hitset(hs):
        rec, _ = hs
        return [(int(p), round(float(e), 3)) for p, e in zip(rec["profile"], rec["logE"])]

    same_hits = hitset(res["bf16"]["hits"]) == hitset(res["fp32"]["hits"])
    nprof = w.db.nprofiles
    h2d = Lq * (64 + 6) * 4 + (Lq + 1) * 7 * 4 + 2 * Lq + 20 * 4
    hrec, hbuf = hits
    d2h = nprof * 4 + int(hbuf.nbytes) + hrec.nbytes
    hbm_peak, peak_kind = _peaks()
    npos = int(w.db.lengths.sum())
    alg_bytes = 209.0 * npos                      # FP32 profile fields streamed per query pass
    achieved = alg_bytes / (p1ms * 1e-3) / 1e9
    tpp = _traffic_per_position()
    gc = lambda t: world * cells / (t * 1e-3) / 1e9   # noqa: E731
    bf, fp = res["bf16"], res["fp32"]
    line = {
        "metric": METRIC, "value": gc(ms), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16" if args.score_mode == "bf16" else "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "cells_per_gpu": cells, "db_profiles": nprof, "db_positions": npos,
                   "scale": args.scale, "l2": "inputs larger than L2 (db records %.1f GB)" % (npos * 224 / 1e9),
                   "parallelism": "db replicas, one per GPU" if world > 1 else "single GPU"},
        "e2e": {"value": world * cells / (e2e_ms * 1e-3) / 1e9, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "e2e_with_db_upload": {"value": world * cells / (e2e_ms * 1e-3 + upload_s) / 1e9, "unit": UNIT,
                               "db_upload_s": upload_s, "db_h2d_bytes": npos * (224 + 28 + 2) + nprof * (20 + 7 + 4 + 4),
                               "note": "one search with the database's upload (packing and host-to-device copies "
                                       "of every profile) counted in its time"},
        "hits_per_s": int(hrec.shape[0]) / (e2e_ms * 1e-3),
        "gpu_launches": launches,
        "hits": int(hrec.shape[0]), "homologs_found": int(np.isin(hrec["profile"], w.homologs).sum()),
        "stage_ms": {"phase1": p1ms, "finalize+stats+map": ms - p1ms},
        "score_forms": {
            "bf16": {"what": "score contractions as split-BF16 (hi+lo) tensor-core mma.sync, FP32 accumulate and DP",
                     "value": gc(bf["ms"]), "e2e": gc(bf["e2e_ms"]), "phase1_ms": bf["p1ms"],
                     "ms_per_step": bf["ms"]},
            "fp32": {"what": "score contractions in FP32 on the CUDA cores, FP32 DP",
                     "value": gc(fp["ms"]), "e2e": gc(fp["e2e_ms"]), "phase1_ms": fp["p1ms"],
                     "ms_per_step": fp["ms"]},
            "bf16_over_fp32_e2e": fp["e2e_ms"] / bf["e2e_ms"],
            "same_hit_lists": same_hits},
        "tensor_pipe": {"kernel": "p1t_kernel", "useful_flops_per_cell": 40,
                        "achieved_tflops": 40.0 * cells / (bf["p1ms"] * 1e-3) / 1e12,
                        "peak_tflops": _bf16_peak(), "frac": 40.0 * cells / (bf["p1ms"] * 1e-3) / 1e12 / _bf16_peak(),
                        "note": "40 flops/cell = the amino-acid contraction (20 multiply-adds); executed tensor "
                                "work is 3 split products x 3 contractions x K 32"},
        "roofline": {"kernel": ("p1t_kernel" if args.score_mode == "bf16" else "p1c_kernel")
                               + " (fused score + Viterbi DP)", "bound": "hbm",
                     "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                     "peak_kind": peak_kind,
                     "traffic": (tpp * npos) if tpp else None,
                     "note": "algorithmic bytes = 209 B x db positions per query pass; traffic = DRAM bytes per "
                             "position from an ncu capture of the 20,000-profile case x positions; "
                             "the kernel is issue/latency bound, not HBM bound"},
        "clocks": clocks,
        "db_upload_s": upload_s,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            g, thr, samp, stages = cpu_port_gcups(w, prm, seconds=args.cpu_seconds)
            line["cpu_baseline"] = {"value": g, "unit": UNIT, "cores": thr, "kind": "port", "sample": samp,
                                    "stages": stages}
        except Exception as ex:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                                    "sample": "failed: %s" % ex}
        try:
            line["error_vs_fp64"] = fp64_error(w, prm, hrec, h.search_space()[0])
        except Exception as ex:
            line["error_vs_fp64"] = {"failed": str(ex)}
    if rank == 0:
        print(json.dumps(line))
    h.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
