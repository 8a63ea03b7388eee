#!/usr/bin/env python
"""Benchmark of the banded pair-HMM path: DP cells/s of the batched FP32 form on the 256-read batch
(seeded synthetic reads, reference spans ~U(2 kb, 20 kb), 6-mer ACGT Gaussian table, anchors every
50 positions, diagonal expansion 50, threshold 0.01), with the plain FP64 one-read-per-launch form,
the CPU oracle and accuracy against the oracle reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0.  A step is one pass of the hot path over the whole batch: the persistent
FP32 launch over all 256 reads with inputs resident in HBM (`value`), or the C-ABI calls from host
buffers (plan, upload, launch, download: `e2e`, measured on a stream of batches with the next
batch planned and uploaded while the current one runs, and as one synchronous call per step in
`e2e.sequential`).  With N > 1 (torchrun) every rank aligns its own 256-read batch (weak scaling, no
collective on the data path); times are the max over ranks.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "dp_cells_per_sec"
UNIT = "cells/s"
FLOP_PER_CELL = 74.0   # forward + backward + posterior incl. emissions, FP32 form (per band cell)
# the worker kernel's share: transitions of both sweeps (2 x 16) and the posterior (2); the two
# emissions per cell (~2 x 10 FLOP per pass in the reference) are computed once by emission_kernel
WORKER_FLOP_PER_CELL = 34.0
EMISSION_BYTES_PER_CELL = 8.0   # emission_kernel writes match + extra-event emission per cell
# the whole path's FP32 work per band cell in the scaled-probability accounting: both sweeps'
# transitions (2 x 16), two emissions per sweep (2 x 2 x ~10) and the posterior (~2)
PATH_FLOP_PER_CELL = 74.0
WORKLOAD = "256 reads x U(2kb,20kb) spans, 6-mer ACGT Gaussian table, expansion 50, threshold 0.01"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--reads", type=int, default=256)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--quick", action="store_true", help="skip the CPU baseline and accuracy legs")
    ap.add_argument("--config", type=int, default=1, choices=[1, 2, 3],
                    help="1: the 256-read Gaussian batch (default); 2: 128 HDP reads (6-mer ACEGT, 2000-point "
                         "grid); 3: 512 2D reads x {C, E} hypotheses, Gaussian and HDP mixed")
    ap.add_argument("--expectations", action="store_true",
                    help="EM expectations run instead: the reads' expectations in one batched call, against the CPU "
                         "oracle on a bounded sample")
    ap.add_argument("--route", default="substitute", choices=["substitute", "degenerate"],
                    help="config 3: all-C and all-E references, or one reference with X (C or E) at the sites")
    ap.add_argument("--segments", type=int, default=None, metavar="DIAGS",
                    help="forward-segment cap for the batches (sa_setSegmentPolicy: -1 whole regions, 0 automatic)")
    ap.add_argument("--saturate", type=int, default=0, metavar="N",
                    help="device throughput with N reads in one batch (the 256-read set repeated), no e2e legs")
    ap.add_argument("--serve", action="store_true",
                    help="serving run instead: Poisson arrivals at --load of the measured capacity, p50/p99 latency")
    ap.add_argument("--serve-requests", type=int, default=400)
    ap.add_argument("--load", type=float, default=0.8)
    ap.add_argument("--serve-budget", type=int, default=200_000_000, help="band cells in flight")
    ap.add_argument("--serve-streams", type=int, default=8, help="micro-batches in flight")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def model_and_reads(n_reads, seed):
    """The synthetic reads and their .model text (6-mer ACGT Gaussian table, nanopore transitions)."""
    from signalalign_b200 import synth
    cfg = synth.config1(seed=seed, n_reads=n_reads)
    return cfg, synth.model_text(cfg["alphabet"], cfg["k"], cfg["table"])


def oracle_model_dict(text):
    """The checker's own reading of the .model text (the oracle's restated loader)."""
    from oracle import formats
    return formats.parse_model_lines(*text.split("\n")[:3])


def load_product_model(text, device=0):
    """The product's loader on the .model file (stateMachine3_loadFromFile + getStateMachine3_descaled)."""
    import tempfile
    from signalalign_b200 import api
    with tempfile.NamedTemporaryFile("w", suffix=".model", delete=False) as fh:
        fh.write(text)
        path = fh.name
    try:
        return api.StateMachine.load(path, api.THREE_STATE, api.EMIT_DESCALED, device=device)
    finally:
        os.unlink(path)


def accuracy_vs_oracle(m, reads, got_pairs, got_ll, threshold, threads, emission=None, hdp=None, options="CEO"):
    """Every read's pairs and log-likelihood against the FP64 oracle, one read per host thread.
    Returns the largest posterior error over the union of each read's pairs (a pair on one side only
    counts as its posterior minus the threshold), the largest |log-likelihood| error (absolute and
    relative to |log-likelihood|), and the pairs present on one side only with a posterior more than
    the FP32 bound (1e-4) above the threshold."""
    from oracle import oracle as orc
    emission = orc.EMIT_DESCALED if emission is None else emission
    p = orc.params(threshold=threshold, expansion=50)

    def one(i):
        rd = reads[i]
        om = orc.OracleModel(m if not isinstance(m, list) else m[i], emission, rd["scale"], rd["shift"],
                             rd.get("var", 1.0), hdp=hdp)
        want, tps = orc.aligned_pairs(om, rd["reference"], rd["events"], rd["anchors"], p, options=options,
                                      with_total_probs=True)
        got = got_pairs(i)
        ma = {(int(r["x"]), int(r["y"])): r["score"] / 1e7 for r in want}
        mg = {(int(r["x"]), int(r["y"])): r["score"] / 1e7 for r in got}
        err, outside = 0.0, 0
        for key in set(ma) | set(mg):
            if key in ma and key in mg:
                err = max(err, abs(ma[key] - mg[key]))
            else:
                present = ma.get(key) or mg.get(key)
                err = max(err, present - threshold)
                outside += present - threshold > 1e-4
        k = 6
        top = [v for d, v in tps if d == len(rd["reference"]) - (k - 1) + len(rd["events"])]
        ll_abs = abs(got_ll(i) - top[0]) if top else 0.0
        ll_rel = ll_abs / max(1.0, abs(top[0])) if top else 0.0
        return err, ll_abs, ll_rel, outside, len(want)

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        res = list(ex.map(one, range(len(reads))))
    return {"max_posterior_err": max(r[0] for r in res), "max_loglik_abs_err": max(r[1] for r in res),
            "max_loglik_rel_err": max(r[2] for r in res),
            "pairs_outside_threshold_tolerance": int(sum(r[3] for r in res)),
            "oracle_pairs": int(sum(r[4] for r in res)), "reads": len(reads),
            "longest_read_antidiagonals": int(max(len(rd["reference"]) - 5 + len(rd["events"]) for rd in reads)),
            "oracle_seconds": time.perf_counter() - t0, "vs": "FP64 CPU oracle, every read of the batch"}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while the timed region runs."""
    FIELDS = ["index", "clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + ",".join(self.FIELDS),
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < len(self.FIELDS):
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def time_oracle(m, reads, budget_s, threads):
    """CPU oracle (FP64 restatement of the reference path) over a bounded sample of the reads, one read
    per thread; returns (cells/s, cells, seconds, reads used)."""
    from oracle import oracle as orc
    p = orc.params(threshold=0.01, expansion=50)
    oms = [orc.OracleModel(m, orc.EMIT_DESCALED, rd["scale"], rd["shift"], 1.0) for rd in reads]
    cells = []
    for rd in reads:
        L, R = orc.band(rd["anchors"], len(rd["reference"]) - 5, len(rd["events"]), 50)
        cells.append(int(np.sum((R - L) // 2 + 1)))
    # the oracle runs ~2-3 M cells/s per thread: size the sample to the budget
    per_thread = 2.5e6 * budget_s
    order = np.argsort(cells)
    chosen, tot = [], 0
    for i in order:
        if tot + cells[i] > per_thread * threads and chosen:
            break
        chosen.append(int(i))
        tot += cells[i]
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(lambda i: orc.aligned_pairs(oms[i], reads[i]["reference"], reads[i]["events"],
                                               reads[i]["anchors"], p), chosen))
    dt = time.perf_counter() - t0
    return tot / dt, tot, dt, len(chosen)


def launch_source(device):
    """where the worker's launch configuration came from: the tuner's table row for this device, or
    the library's defaults"""
    import torch
    from signalalign_b200 import api, tune
    name = torch.cuda.get_device_name(device)
    rows = tune.read_table(api.LAUNCH_CONFIGS)
    return "tuned (python -m signalalign_b200.tune, %s)" % name if (name, 1) in rows else "defaults"


def run_reference(args):
    """`--impl reference`: the reference path on the host cores.  signalAlign's C sources need the
    un-vendored sonLib library, so the reference arm is the FP64 CPU restatement (the oracle), which
    follows the same recursion and reproduces the reference's golden outputs."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    cfg, text = model_and_reads(args.reads, args.seed)
    m = oracle_model_dict(text)
    threads = os.cpu_count() or 1
    vals = []
    for s in range(args.warmup + args.steps):
        v, cells, dt, nr = time_oracle(m, cfg["reads"], 2.0, threads)
        if s >= args.warmup:
            vals.append((v, cells, dt, nr))
    value = sum(c for _, c, _, _ in vals) / sum(d for _, _, d, _ in vals)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(d for _, _, d, _ in vals),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "global_batch": args.reads, "parallelism": "host threads"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": "%d reads per step (smallest bands first), one read per thread" % vals[0][3]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_serve(args):
    """Serving workload: log-normal spans (median 8 kb, clipped to 500 bp - 100 kb), per-request model
    choice (6-mer ACGT or 6-mer ACEGT Gaussian table), Poisson arrivals.  Capacity is measured first
    (all requests of a saturation set submitted at once); the timed run offers --load of it.  Latency
    is submission to completion as the server records it (planning, upload, kernels, download)."""
    import torch
    from signalalign_b200 import api, synth
    torch.cuda.set_device(0)
    r = np.random.Generator(np.random.PCG64(args.seed + 404))
    models = []
    for alphabet in ("ACGT", "ACEGT"):
        table = synth.gaussian_table(alphabet, 6, 1000 + len(alphabet))
        sm = load_product_model(synth.model_text(alphabet, 6, table))
        models.append((alphabet, table, sm))
    n = args.serve_requests
    spans = np.clip(np.exp(np.log(8000.0) + 0.6 * r.standard_normal(n)), 500, 100000).astype(int)
    reqs = []
    for L in spans:
        alphabet, table, sm = models[int(r.integers(0, 2))]
        seq = synth.random_reference(int(L), r, alphabet)
        rd = synth.make_read(seq, alphabet, 6, table[:, 0], table[:, 1], table[:, 2], table[:, 3], r)
        lo, hi = api.band_construct(rd["anchors"], len(seq) - 5, len(rd["events"]), 50)
        reqs.append((api.ReadInput(sm=sm, reference=rd["reference"], events=rd["events"], anchors=rd["anchors"],
                                   scale=rd["scale"], shift=rd["shift"]), int(L), int(np.sum((hi - lo) // 2 + 1))))
    p = api.pairwiseAlignmentBandingParameters_construct()
    srv = api.Server(device=0, max_inflight_cells=args.serve_budget, max_batches=args.serve_streams)
    try:
        for q, _, _ in reqs[:8]:                       # warm-up: tables resident, pools filled
            t = srv.submit(q, p)
            srv.wait(t)
            srv.result(t)
        sat = reqs[: max(16, n // 2)]
        t0 = time.perf_counter()
        ts = [srv.submit(q, p) for q, _, _ in sat]
        for t in ts:
            srv.wait(t)
            srv.result(t)
        cap = len(sat) / (time.perf_counter() - t0)
        rate = args.load * cap

        def offer(items, arrivals):
            out = []
            t_start = time.perf_counter()
            for (q, L, c), at in zip(items, arrivals):
                while True:
                    dt = at - (time.perf_counter() - t_start)
                    if dt <= 0:
                        break
                    time.sleep(min(dt, 0.0005))
                out.append((srv.submit(q, p), L, c))
            return out, t_start

        # untimed: the same arrival process for a while, so the memory pools hold the block sizes
        # of this load's micro-batches (a server in steady state allocates nothing)
        warm = reqs
        wt, _ = offer(warm, np.cumsum(r.exponential(1.0 / rate, len(warm))))
        for t, _, _ in wt:
            srv.wait(t, 600000.0)
            srv.result(t)
        arrivals = np.cumsum(r.exponential(1.0 / rate, n))
        stats0 = srv.stats()
        allocs0, alloc_ms0 = api.allocation_count(), api.allocation_ms()
        sampler = ClockSampler(0)
        sampler.start()
        tickets, t0 = offer(reqs, arrivals)
        res = []
        for t, L, c in tickets:
            srv.wait(t, 600000.0)
            st, pairs, ll, lat = srv.result(t, release=False)
            q, l = srv.timing(t)
            srv.release(t)
            res.append((st, L, c, lat, q, l))
        wall = time.perf_counter() - t0
        clocks = sampler.stop()
        stats = {k: v - stats0[k] for k, v in srv.stats().items()}
        allocs, alloc_ms = api.allocation_count() - allocs0, api.allocation_ms() - alloc_ms0
        blog = srv.batch_log()
    finally:
        srv.close()
    # micro-batches on the device at once (device event times of their kernels)
    ev = sorted([(b[0], 1) for b in blog] + [(b[1], -1) for b in blog], key=lambda e: (e[0], e[1]))
    conc = peak = 0
    for _, d in ev:
        conc += d
        peak = max(peak, conc)
    lat = np.array([x[3] for x in res])
    spans_ok = np.array([x[1] for x in res])
    sel = (spans_ok >= 8000) & (spans_ok <= 12000)
    ten = lat[sel]
    # where the 8-12 kb reads' time went: waiting for a stream and budget, planning and upload of
    # their micro-batch, and the rest (kernels until the read was published, copy of its pairs)
    queue = np.array([x[4] for x in res])[sel]
    launch = np.array([x[5] for x in res])[sel]
    run = ten - queue - launch

    def pct(v):
        return {"p50": float(np.percentile(v, 50)), "p99": float(np.percentile(v, 99)), "max": float(np.max(v))} \
            if len(v) else None
    worst = int(np.argmax(ten)) if len(ten) else None
    cells = sum(x[2] for x in res)
    line = {"metric": "serving_p99_latency_ms", "value": float(np.percentile(lat, 99)), "unit": "ms",
            "higher_is_better": False, "n_gpus": 1, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "%d requests, log-normal spans (median 8 kb, sigma 0.6, clipped 500 bp-100 kb), "
                                   "6-mer ACGT / ACEGT Gaussian tables per request, Poisson arrivals at %.0f%% of "
                                   "measured capacity" % (n, 100 * args.load),
                       "band_cell_budget": args.serve_budget, "streams": args.serve_streams},
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "p50_ms_8to12kb": float(np.percentile(ten, 50)) if len(ten) else None,
            "p99_ms_8to12kb": float(np.percentile(ten, 99)) if len(ten) else None,
            "reads_8to12kb": int(len(ten)),
            "capacity_reads_per_sec": cap, "offered_reads_per_sec": rate,
            "achieved_reads_per_sec": n / wall, "cells_per_sec": cells / wall,
            "errors": int(sum(1 for x in res if x[0] != 0)),
            "reads_finished_on_publication": stats["reads_early"],
            "reads_finished_at_batch_end": stats["reads_at_batch_end"],
            "micro_batches": stats["batches"], "max_concurrent_micro_batches": peak,
            "breakdown_8to12kb_ms": {"queue": pct(queue), "plan_upload_launch": pct(launch), "kernels_and_copy": pct(run),
                                     "slowest": None if worst is None else
                                     {"total": float(ten[worst]), "queue": float(queue[worst]),
                                      "plan_upload_launch": float(launch[worst]), "kernels_and_copy": float(run[worst])}},
            "dispatcher_ms": {"admit": stats["admit_ms"], "plan": stats["plan_ms"], "upload": stats["upload_ms"],
                              "fetch": stats["fetch_ms"], "finish": stats["finish_ms"], "wall": 1000.0 * wall},
            "allocations_in_timed_run": {"count": allocs, "ms": alloc_ms},
            "clocks": clocks}
    print(json.dumps(line), flush=True)


def run_saturate(args):
    """Device throughput of one batch of N reads (the bench's 256 reads repeated to N): many more
    forward segments and windows than worker CTAs, so the worker runs at its throughput, not at a
    chain's latency.  Device time of sa_batch_run by CUDA events; no host legs."""
    import torch
    from signalalign_b200 import api
    torch.cuda.set_device(0)
    cfg, text = model_and_reads(256, args.seed)
    sm = load_product_model(text)
    p = api.pairwiseAlignmentBandingParameters_construct(diagonal_expansion=50, threshold=0.01)
    base = [api.ReadInput(sm=sm, reference=rd["reference"], events=rd["events"], anchors=rd["anchors"],
                          scale=rd["scale"], shift=rd["shift"]) for rd in cfg["reads"]]
    reads = [base[i % len(base)] for i in range(args.saturate)]
    b = api.Batch(reads, p)
    b.upload()
    cells = b.cells
    for _ in range(max(3, args.warmup)):
        b.run()
    torch.cuda.synchronize()
    ms, kern = [], []
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        b.run()
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
        kern.append(b.kernel_ms())
    b.download()
    bad = sum(1 for i in range(len(reads)) if b.status(i) != 0)
    t = statistics.mean(ms)
    wk = statistics.mean(k[1] for k in kern)
    peak = api.measure_fp32_peak(0)
    achieved = WORKER_FLOP_PER_CELL * cells / (wk / 1e3) / 1e12
    line = {"metric": METRIC, "value": cells / (t / 1e3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": t, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic", "config": {"workload": "%d reads (the 256-read bench set repeated), expansion 50"
                                                   % len(reads), "cells_per_step": cells,
                                            "launch_config": api.get_launch_config(0, 1),
                                            "forward_segments": b.segment_info()},
            "reads_per_sec": len(reads) / (t / 1e3), "read_errors": bad,
            "kernels_ms": {"emission_kernel": statistics.mean(k[0] for k in kern), "worker_kernel": wk,
                           "gather_pairs": statistics.mean(k[2] for k in kern)},
            "roofline": {"kernel": "worker_kernel", "bound": "fp32", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak}}
    print(json.dumps(line), flush=True)


def run_config(args):
    """Configs 2 and 3 on one GPU: the device time of sa_batch_run over every alignment (config 3 in
    sub-batches of 512 alignments, which bounds the stores to ~40 GB), the end-to-end time of
    sa_align_batch, and the posterior error against the FP64 oracle on the shortest alignments."""
    import torch
    from oracle import formats
    from oracle import oracle as orc
    from signalalign_b200 import api, synth
    torch.cuda.set_device(0)
    tests_dir = os.path.join(ROOT, "tests")
    sys.path.insert(0, tests_dir)
    import workloads as W
    if args.config == 2:
        cfg = synth.config2(seed=args.seed + 1)
        hdp = W.hdp_dict(cfg["hdp"], 5 ** 6)
        m = formats.parse_model_lines(*synth.model_text("ACEGT", 6, cfg["table"]).split("\n")[:3])
        sm = W.gpu_model(api, m, orc.EMIT_HDP, None, hdp)
        als = [dict(rd, model="hdp") for rd in cfg["reads"]]
        models = {"hdp": (sm, m, orc.EMIT_HDP, hdp)}
        workload = "128 reads x U(5kb,15kb), 6-mer ACEGT HDP (15,625 k-mers, 2000-point grid), expansion 50"
        sub = len(als)
    else:
        cfg = synth.config3(seed=args.seed + 2, route=args.route)
        hdp = W.hdp_dict(cfg["hdp"], 5 ** 6)
        gm = formats.parse_model_lines(*synth.model_text("ACEGT", 6, cfg["gauss_table"]).split("\n")[:3])
        hm = formats.parse_model_lines(*synth.model_text("ACEGT", 6, cfg["hdp_table"]).split("\n")[:3])
        models = {"gauss": (load_product_model(synth.model_text("ACEGT", 6, cfg["gauss_table"])), gm,
                            orc.EMIT_DESCALED, None),
                  "hdp": (W.gpu_model(api, hm, orc.EMIT_HDP, None, hdp), hm, orc.EMIT_HDP, hdp)}
        als = cfg["alignments"]
        if args.route == "substitute":
            workload = ("512 reads x U(1kb,30kb) x {template, complement} x {all-C, all-E} at CCWGG sites = 2048 "
                        "alignments, 6-mer ACEGT Gaussian and HDP machines mixed")
        else:
            workload = ("512 reads x U(1kb,30kb) x {template, complement}, X (C or E) at CCWGG sites = 1024 "
                        "alignments with two-path cells over the sites (plain FP64 form), 6-mer ACEGT Gaussian "
                        "and HDP machines mixed")
        sub = 512
    p = api.pairwiseAlignmentBandingParameters_construct(diagonal_expansion=50, threshold=0.01)
    degen = api.CYTOSINE_METHYLATION2 if args.config == 3 and args.route == "degenerate" else api.CYTOSINE_METHYLATION3
    options = "CE" if degen == api.CYTOSINE_METHYLATION2 else "CEO"
    inputs = [api.ReadInput(sm=models[a["model"]][0], reference=a["reference"], events=a["events"],
                            anchors=a["anchors"], scale=a["scale"], shift=a["shift"], degenerate=degen) for a in als]
    groups = [inputs[i:i + sub] for i in range(0, len(inputs), sub)]
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    cells, dev_ms, e2e_ms = 0, 0.0, 0.0
    launches0 = api.kernel_launch_count()
    for g in groups:
        b = api.Batch(g, p)
        b.upload(sptr)
        for _ in range(max(3, args.warmup)):
            b.run(sptr)
        torch.cuda.synchronize()
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.run(sptr)
            e1.record(stream)
            e1.synchronize()
            dev_ms += e0.elapsed_time(e1) / args.steps
        cells += b.cells
        del b
        t0 = time.perf_counter()
        bb = api.align_batch(g, p, sptr)
        torch.cuda.synchronize()
        e2e_ms += (time.perf_counter() - t0) * 1e3
        del bb
    # accuracy against the FP64 oracle: every alignment of config 2; for config 3 the longest
    # alignment of each model and a spread of the others (about 20 s of host work)
    n_al = len(als)
    if args.config == 2:
        chosen = list(range(n_al))
    else:
        order = [int(i) for i in np.argsort([len(a["events"]) for a in als])]
        chosen = sorted(set(order[::max(1, n_al // 48)]) |
                        {max((i for i in range(n_al) if als[i]["model"] == mk), key=lambda i: len(als[i]["events"]))
                         for mk in models})
    bb = api.align_batch([inputs[i] for i in chosen], p, sptr)
    sub_reads = [als[i] for i in chosen]
    ms = [models[a["model"]][1] for a in sub_reads]
    acc = {}
    for mk, (_, mm, emis, hh) in models.items():
        idx = [j for j, a in enumerate(sub_reads) if a["model"] == mk]
        if not idx:
            continue
        a_k = accuracy_vs_oracle(mm, [sub_reads[j] for j in idx], lambda q: bb.pairs(idx[q]),
                                 lambda q: bb.log_likelihood(idx[q]), 0.01, os.cpu_count() or 1, emission=emis, hdp=hh,
                                 options=options)
        acc[mk] = a_k
    del ms
    line = {"metric": METRIC, "value": cells / (dev_ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": dev_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload, "alignments": len(als), "cells": cells, "sub_batches": len(groups)},
            "e2e": {"value": cells / (e2e_ms / 1e3), "unit": UNIT, "ms_per_step": e2e_ms},
            "accuracy": acc,
            "gpu_launches": api.kernel_launch_count() - launches0}
    print(json.dumps(line), flush=True)


def run_expectations(args):
    """EM expectations on the 256-read workload: every read's expectations (transitions, per-k-mer
    emission expectations, likelihood) in one sa_getExpectationsBatch call (the plain FP64 form, one
    CTA per read walking its regions in order), timed end to end from host buffers (planning, H2D,
    kernel, D2H); the CPU oracle's expectations on a bounded sample, one read per host thread."""
    import torch
    from oracle import oracle as orc
    from signalalign_b200 import api
    torch.cuda.set_device(0)
    cfg, text = model_and_reads(args.reads, args.seed)
    m = oracle_model_dict(text)
    sm = load_product_model(text)
    p = api.pairwiseAlignmentBandingParameters_construct(diagonal_expansion=50, threshold=0.01)
    reads = [api.ReadInput(sm=sm, reference=rd["reference"], events=rd["events"], anchors=rd["anchors"],
                           scale=rd["scale"], shift=rd["shift"]) for rd in cfg["reads"]]
    cells = []
    for rd in cfg["reads"]:
        L, R = orc.band(rd["anchors"], len(rd["reference"]) - 5, len(rd["events"]), 50)
        cells.append(int(np.sum((R - L) // 2 + 1)))
    for _ in range(max(1, args.warmup)):
        api.getExpectationsBatch(reads[:4], p)
    sampler = ClockSampler(0)
    sampler.start()
    launches0 = api.kernel_launch_count()
    times, errors = [], 0
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, status = api.getExpectationsBatch(reads, p)
        times.append(time.perf_counter() - t0)
        errors += sum(1 for v in status if v)
    launches = api.kernel_launch_count() - launches0
    clocks = sampler.stop()
    value = sum(cells) * args.steps / sum(times)
    # CPU: the oracle's expectations, smallest reads first, about 10 s of work over the host threads
    threads = os.cpu_count() or 1
    oms = [orc.OracleModel(m, orc.EMIT_DESCALED, rd["scale"], rd["shift"], 1.0) for rd in cfg["reads"]]
    op = orc.params(threshold=0.01, expansion=50)
    chosen, tot = [], 0
    for i in np.argsort(cells):
        if tot + cells[i] > 1.0e6 * 10.0 * threads and chosen:
            break
        chosen.append(int(i))
        tot += cells[i]
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(lambda i: orc.expectations(oms[i], cfg["reads"][i]["reference"], cfg["reads"][i]["events"],
                                               cfg["reads"][i]["anchors"], op), chosen))
    cpu_dt = time.perf_counter() - t0
    line = {"metric": "em_expectation_cells_per_sec", "value": value, "unit": "cells/s", "n_gpus": 1,
            "steps": args.steps, "warmup": max(1, args.warmup), "ms_per_step": 1e3 * statistics.mean(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD + ", expectations (pseudocounts 0.001)", "global_batch": len(reads),
                       "cells_per_step": int(sum(cells))},
            "e2e": {"value": value, "unit": "cells/s", "mode": "one sa_getExpectationsBatch call per step from host "
                    "buffers: planning, H2D, kernel, D2H of every read's accumulators"},
            "gpu_launches": launches, "errors": errors, "clocks": clocks,
            "cpu_baseline": {"value": tot / cpu_dt, "unit": "cells/s", "cores": threads, "kind": "port",
                             "sample": "%d reads (%d cells, smallest bands first), one read per thread, %.1f s"
                                       % (len(chosen), tot, cpu_dt)}}
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.segments is not None:
        from signalalign_b200 import api
        api.set_segment_policy(args.segments, api.get_segment_policy()[1])
    if args.expectations:
        run_expectations(args)
        return
    if args.serve:
        run_serve(args)
        return
    if args.saturate:
        run_saturate(args)
        return
    if args.config != 1 and args.impl == "ours":
        run_config(args)
        return
    if args.impl == "reference":
        run_reference(args)
        return
    rank, world, local = dist_env()
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    from signalalign_b200 import api

    cfg, text = model_and_reads(args.reads, args.seed + 1000 * rank)
    m = oracle_model_dict(text)
    sm = load_product_model(text, device=local)
    p = api.pairwiseAlignmentBandingParameters_construct(diagonal_expansion=50, threshold=0.01)
    reads = [api.ReadInput(sm=sm, reference=rd["reference"], events=rd["events"], anchors=rd["anchors"],
                           scale=rd["scale"], shift=rd["shift"]) for rd in cfg["reads"]]
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    b = api.Batch(reads, p)
    b.upload(sptr)
    cells = b.cells
    torch.cuda.synchronize()
    for _ in range(max(3, args.warmup)):
        b.run(sptr)
    torch.cuda.synchronize()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    sampler = ClockSampler(local)
    sampler.start()
    launches0 = api.kernel_launch_count()
    step_ms = []
    kern_ms = []
    barrier()
    for _ in range(args.steps):
        flush.fill_(1)                       # L2 flush between timed steps (outside the events)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.run(sptr)
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        kern_ms.append(b.kernel_ms())        # per-kernel CUDA events on the launching stream
    barrier()
    launches = api.kernel_launch_count() - launches0
    clocks = sampler.stop()
    t_local = sum(step_ms)
    t = torch.tensor([t_local], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    t_max = float(t.item())
    value = cells * args.steps * world / (t_max / 1e3)
    reads_per_s = len(reads) * args.steps * world / (t_max / 1e3)

    # e2e: the whole C-ABI call from host buffers (plan + upload + launch + download), wall clock
    e2e_ms = []
    h2d = d2h = 0
    for i in range(max(2, min(args.steps, 3)) + 1):
        barrier()
        t0 = time.perf_counter()
        bb = api.align_batch(reads, p, sptr)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) * 1e3
        if i > 0:
            e2e_ms.append(dt)
        h2d, d2h = bb.transfer_bytes()
        del bb
    te = torch.tensor([statistics.mean(e2e_ms)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_seq_value = cells * world / (float(te.item()) / 1e3)

    # e2e, pipelined: the same public calls on a stream of batches, as a pipeline uses them, three
    # batches in flight: batch k is planned on the host and uploaded on an H2D stream while batch
    # k-1's kernels run, and batch k-2 is downloaded on a D2H stream; events order the copies against
    # the kernels.  Every batch's planning, H2D, kernels and D2H are inside the timed region.
    h2d_stream, d2h_stream = torch.cuda.Stream(), torch.cuda.Stream()
    hptr, dptr = h2d_stream.cuda_stream, d2h_stream.cuda_stream

    def pipeline(n):
        inflight = []   # (batch, its kernels' completion event), oldest first
        for _ in range(n):
            cur = api.Batch(reads, p)
            cur.upload(hptr)
            uploaded = torch.cuda.Event()
            uploaded.record(h2d_stream)
            stream.wait_event(uploaded)
            cur.run(sptr)
            done = torch.cuda.Event()
            done.record(stream)
            inflight.append((cur, done))
            if len(inflight) > 2:
                old, old_done = inflight.pop(0)
                d2h_stream.wait_event(old_done)
                old.download(dptr)
                del old
        while inflight:
            old, old_done = inflight.pop(0)
            d2h_stream.wait_event(old_done)
            old.download(dptr)
            del old
        torch.cuda.synchronize()

    pipeline(3)   # untimed: the memory pools then hold the blocks of the three batches in flight
    n_pipe = 8   # a stream of 8 batches, pipeline fill and drain included
    barrier()
    t0 = time.perf_counter()
    pipeline(n_pipe)
    pipe_ms = (time.perf_counter() - t0) * 1e3 / n_pipe
    tp = torch.tensor([pipe_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(tp, op=dist.ReduceOp.MAX)
    e2e_value = cells * world / (float(tp.item()) / 1e3)

    line = None
    if rank == 0:
        peak = api.measure_fp32_peak(local)
        em_ms = statistics.mean(k[0] for k in kern_ms)
        wk_ms = statistics.mean(k[1] for k in kern_ms)
        ga_ms = statistics.mean(k[2] for k in kern_ms)
        achieved = WORKER_FLOP_PER_CELL * cells / (wk_ms / 1e3) / 1e12
        traffic = None
        prof = os.path.join(ROOT, "profiles", "worker_kernel_traffic.json")
        if os.path.exists(prof):
            with open(prof) as fh:
                pj = json.load(fh)
            traffic = pj.get("dram_bytes_per_cell", 0) * cells
        hbm_peak, hbm_src = 6650.0, "fallback"
        mp = os.path.join(ROOT, "MEASURED_PEAKS.json")
        if os.path.exists(mp):
            with open(mp) as fh:
                hbm_peak, hbm_src = float(json.load(fh).get("hbm_gbs", hbm_peak)), "measured"
        em_gbs = EMISSION_BYTES_PER_CELL * cells / (em_ms / 1e3) / 1e9
        # the sequential chain: the longest region's anti-diagonals bound the worker from below.  The
        # bound is measured: the same read alone in a batch (its forward sweep alone on its SM, its
        # windows served by two more CTAs) takes the worker's floor for this batch.
        chain = [len(rd["reference"]) - 5 + len(rd["events"]) for rd in cfg["reads"]]
        longest = max(chain)
        lb = api.Batch([reads[int(np.argmax(chain))]], p)
        lb.upload(sptr)
        alone = []
        for i in range(5):
            lb.run(sptr)
            torch.cuda.synchronize()
            if i >= 2:
                alone.append(lb.kernel_ms()[1])
        alone_ms = min(alone)
        del lb
        # plain FP64 form, one read per launch, on a sample of the batch
        order = np.argsort([len(rd["events"]) for rd in cfg["reads"]])
        sample = [int(i) for i in order[::max(1, len(order) // 8)][:8]]
        sample_cells = 0
        for i in sample:
            rd = cfg["reads"][i]
            L, R = api.band_construct(rd["anchors"], len(rd["reference"]) - 5, len(rd["events"]), 50)
            sample_cells += int(np.sum((R - L) // 2 + 1))
        sm64 = load_product_model(text, device=local)
        api.getAlignedPairsUsingAnchors(sm64, cfg["reads"][sample[0]]["reference"][:300],
                                        cfg["reads"][sample[0]]["events"][:400], [], p)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in sample:
            rd = cfg["reads"][i]
            sm64.set_scaling(rd["scale"], rd["shift"], 1.0)
            api.getAlignedPairsUsingAnchors(sm64, rd["reference"], rd["events"], rd["anchors"], p)
        plain_s = time.perf_counter() - t0
        plain_value = sample_cells / plain_s
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": max(3, args.warmup), "ms_per_step": t_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD, "global_batch": args.reads * world, "regions": b.regions,
                           "launch_config": api.get_launch_config(local, 1),
                           "launch_config_source": launch_source(local),
                           "forward_segments": dict(b.segment_info(), policy=list(api.get_segment_policy())),
                           "cells_per_step_per_gpu": cells, "parallelism": "dp%d (read sharding)" % world,
                           "l2": "flushed between timed steps (256 MiB write); forward store >> L2"},
                "reads_per_sec": reads_per_s,
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "ms_per_step": float(tp.item()),
                        "includes": "host planning (bands, windows, k-mer ids), H2D, launch, D2H of all pairs",
                        "mode": "pipelined through sa_batch_create/upload/run/download, three batches in flight: "
                                "batch k planned on the host and uploaded on an H2D stream while batch k-1's "
                                "kernels run, batch k-2 downloaded on a D2H stream (events order copies and "
                                "kernels)",
                        "sequential": {"value": e2e_seq_value, "ms_per_step": float(te.item()),
                                       "mode": "one synchronous sa_align_batch call per step"}},
                "plain_fp64": {"value": plain_value, "unit": UNIT, "sample": "%d reads, one launch per read" % len(sample),
                               "batched_over_plain": value / world / plain_value},
                "roofline": {"kernel": "worker_kernel", "bound": "fp32", "achieved": achieved, "peak": peak,
                             "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
                             "kernel_ms": wk_ms,
                             "note": "%.0f FP32 FLOP per band cell (transitions of both sweeps + posterior; "
                                     "emissions are emission_kernel's) / worker CUDA-event time; peak = FP32 FMA "
                                     "probe measured in this run; traffic = dram bytes per cell from the ncu capture "
                                     "in profiles/ x cells" % WORKER_FLOP_PER_CELL},
                "kernels_ms": {"emission_kernel": em_ms, "worker_kernel": wk_ms, "gather_pairs": ga_ms},
                "emission_roofline": {"bound": "hbm", "achieved": em_gbs, "peak": hbm_peak, "unit": "GB/s",
                                      "frac": em_gbs / hbm_peak, "peak_source": hbm_src,
                                      "note": "%.0f B written per band cell" % EMISSION_BYTES_PER_CELL},
                "critical_path": {"longest_region_antidiagonals": longest,
                                  "worker_ns_per_antidiagonal": wk_ms * 1e6 / longest,
                                  "alone_worker_ms": alone_ms, "frac": alone_ms / wk_ms,
                                  "note": "a region's forward sweep is sequential over its anti-diagonals unless "
                                          "it is cut into forward segments; alone_worker_ms is the worker kernel "
                                          "on the longest read alone (its segments on separate CTAs), frac = "
                                          "alone / batch worker time"},
                "path_roofline": {"flop_per_cell": PATH_FLOP_PER_CELL, "bound_cells_per_sec": peak * 1e12 / PATH_FLOP_PER_CELL,
                                  "achieved_cells_per_sec": value / world,
                                  "frac": value / world / (peak * 1e12 / PATH_FLOP_PER_CELL),
                                  "note": "all three kernels per band cell against the FP32 FMA probe"},
                "gpu_launches": launches, "clocks": clocks}
    if world > 1:
        dist.barrier()
    if rank == 0 and not args.quick:
        threads = os.cpu_count() or 1
        v, ccells, dt, nr = time_oracle(m, cfg["reads"], 4.0, threads)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": "%d reads (%d cells, smallest bands first), one read per thread, %.1f s"
                                          % (nr, ccells, dt)}
        # accuracy of the batched FP32 form against the FP64 oracle on every read of the batch
        bb = api.align_batch(reads, p, sptr)
        line["accuracy"] = accuracy_vs_oracle(m, cfg["reads"], bb.pairs, bb.log_likelihood, 0.01, threads)
        line["accuracy"]["forward_segments"] = bb.segment_info()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
