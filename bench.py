#!/usr/bin/env python
"""Benchmark of the B200 join engine on the five-way snowflake join.

Workload (seeded synthetic data of the benchmark's shapes; no public dataset):
fact table of 50M rows with four INT32 foreign keys, Zipf(s=1.1) over the
keys of four dimensions of 5M / 1M / 200K / 20K rows; the dimensions arrive
pre-filtered to 1% / 5% / 30% / 60% of their rows and carry a VARCHAR of 1-64
bytes; the plan joins all five and outputs two dimension strings and two
fact keys. The fact's key columns are 206 MB each, far larger than L2, so no
L2 flush is needed between steps.

One step = one execution of the query.
  value : queries/s with the tables resident in HBM (bj_execute_resident,
          result pages left in HBM), timed with CUDA events on the engine's
          stream, max over ranks, all ranks' queries / time.
  e2e   : queries/s through the drop-in path (bj_execute: host pages in,
          host pages out), with the input pages in pinned host memory (read in
          place by the kernels over the host link) and the device->host copy of
          the result pages inside the timed region. e2e_pageable is the same
          with pageable input pages (staged and copied to HBM every step).
  roofline: the scan-side probe stage (the kernel that streams the fact's key
          pages), its page bytes per launch / its CUDA-event duration, against
          the measured HBM copy bandwidth.
  cpu_baseline: the reference CPU engine (oracle/_ref/ref_runner, built from
          the reference's sources) on this host's cores, a bounded sample.

--impl reference times the reference CPU engine alone (rank 0; other ranks
exit at once). --gpus N > 1 runs N independent replicas (the query does not
shard: every rank runs the whole query on its own GPU), launched by torchrun.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "queries/s & p99 latency, learned+batched vs plain GPU path (exact rows); GB/s"
REF_RUNNER = os.path.join(REPO, "oracle", "_ref", "ref_runner")
WORKLOAD_DESC = ("snowflake-5way: fact 50M rows x 4 INT32 FKs (Zipf 1.1); dims 5M/1M/200K/20K rows "
                 "pre-filtered 1%/5%/30%/60%, VARCHAR 1-64 B; output 2 VARCHAR + 2 INT32")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="snowflake")
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--cpu-steps", type=int, default=20, help="0 skips the CPU baseline")
    ap.add_argument("--serve-queries", type=int, default=2000,
                    help="queries per serving measurement (0 skips serving)")
    ap.add_argument("--serve-workers", type=int, default=8)
    ap.add_argument("--serve-large", type=int, default=200,
                    help="large queries in the serving bench's large-only closed loop")
    ap.add_argument("--mode", default="all", choices=["all", "value", "e2e", "serve", "batch"],
                    help="value / e2e run one measurement only (for profiling); all prints the bench line; "
                         "batch runs every query of a batched workload (--workload schema20)")
    return ap.parse_args()


def config(args, world):
    return {"workload": WORKLOAD_DESC if args.workload == "snowflake" else args.workload,
            "name": args.workload, "seed": args.seed, "scale": args.scale,
            "l2": "inputs larger than L2 (each fact key column 206 MB > 126 MB L2); no flush",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


def run_reference(args, steps, warmup):
    """The reference CPU engine: wall-clock per execute(), all host cores."""
    if not os.path.exists(REF_RUNNER):
        return None, "oracle/_ref/ref_runner is not built (the reference sources were not available at build time)"
    p = subprocess.run([REF_RUNNER, "bench", args.workload, str(args.seed), str(args.scale), str(warmup), str(steps)],
                       capture_output=True, text=True, timeout=1800)
    if p.returncode != 0:
        return None, f"ref_runner failed: {p.stderr.strip()[-300:]}"
    line = [l for l in p.stdout.splitlines() if l.startswith("{")][-1]
    return json.loads(line), None


def reference_arm(args, rank):
    if rank != 0:
        return 0
    res, err = run_reference(args, args.steps, args.warmup)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return 0
    times = res["times_ms"]
    mean_ms = statistics.fmean(times)
    qps = 1000.0 / mean_ms
    out = {
        "impl": "reference", "metric": METRIC, "value": qps, "unit": "queries/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": mean_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic", "config": config(args, 1),
        "p50_ms": statistics.median(times), "p99_ms": sorted(times)[min(len(times) - 1, int(0.99 * len(times)))],
        "rows": res["rows"],
        "cpu_baseline": {"value": qps, "unit": "queries/s", "cores": res["threads"], "kind": "reference",
                         "sample": f"{args.steps} timed executions (+{args.warmup} warm-up) of the full query"},
        "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.device), "-lms", "20"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.1)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per launch of the scan-side probe stage from the committed
    ncu summary, if one exists."""
    try:
        with open(os.path.join(REPO, "profiles", "scan_probe_traffic.json")) as f:
            return json.load(f).get("dram_bytes_per_launch")
    except (OSError, ValueError):
        return None


def serve_bench(pkg, args, large):
    """Serving on one GPU: a 9:1 mix of small queries (the 1M-row fact of a
    second snowflake instance joined with 1 or 2 dimensions) and large ones
    (the 5-way snowflake on the 50M-row fact), all over resident tables,
    through a server of 1 worker (the plain path: one query at a time) and of
    `--serve-workers` workers (queries overlap on the device). Closed loop:
    every query submitted at once, queries/s = queries / time to the last
    completion; the same for `--serve-large` large queries alone. Open loop: Poisson arrivals at 50% of the plain path's
    closed-loop rate, p50/p99 of submit-to-completion latency."""
    import random
    import threading

    small = pkg.Workload("snowflake", args.seed + 100, 0.02)
    rng = random.Random(args.seed)
    mix = [("large", None) if i % 10 == 9 else ("small", 1 + rng.randrange(2)) for i in range(args.serve_queries)]
    out = {"mix": "9 small (1M-row fact, 2-3 tables) : 1 large (50M-row fact, 5 tables)", "queries": len(mix)}
    plain_qps = None
    for label, workers in (("plain", 1), ("batched", args.serve_workers)):
        with pkg.Server(0, workers=workers) as srv:
            tabs = {}
            for name, w in (("small", small), ("large", large)):
                plan = w.plan_ptr().contents
                tabs[name] = [srv.upload(plan.inputs[i]) for i in range(plan.num_inputs)]
            plans = {("large", None): large.plan_ptr(), ("small", 1): small.variant_ptr(1),
                     ("small", 2): small.variant_ptr(2)}

            def submit(q):
                p = plans[q]
                return srv.submit(p, tabs[q[0]][:p.contents.num_inputs], pkg.RESULT_DEVICE)

            try:
                # Warm every worker's graph cache for every plan.
                for t in [submit(q) for q in list(plans) * (3 * workers)]:
                    srv.wait(t)[0].free()
                # Closed loop.
                t0 = time.perf_counter()
                tickets = [submit(q) for q in mix]
                for t in tickets:
                    srv.wait(t)[0].free()
                qps = len(mix) / (time.perf_counter() - t0)
                plain_qps = plain_qps or qps
                # Closed loop of large queries only (the bench's own query).
                t0 = time.perf_counter()
                tickets = [submit(("large", None)) for _ in range(args.serve_large)]
                for t in tickets:
                    srv.wait(t)[0].free()
                large_qps = args.serve_large / (time.perf_counter() - t0)
                # Open loop: Poisson arrivals; a waiter thread collects results.
                rate = 0.5 * plain_qps
                lat, issued = [], []
                lock = threading.Lock()

                def waiter():
                    k = 0
                    while k < len(mix):
                        with lock:
                            t = issued[k] if k < len(issued) else None
                        if t is None:
                            time.sleep(0.0001)
                            continue
                        r, ms = srv.wait(t)
                        r.free()
                        lat.append(ms)
                        k += 1

                th = threading.Thread(target=waiter)
                th.start()
                arrivals = random.Random(args.seed + 1)
                t_next = time.perf_counter()
                for q in mix:
                    t_next += arrivals.expovariate(rate)
                    while time.perf_counter() < t_next:
                        pass
                    t = submit(q)
                    with lock:
                        issued.append(t)
                th.join()
                lat.sort()
                out[label] = {"workers": workers, "queries_per_s": qps, "large_only_queries_per_s": large_qps,
                              "arrival_rate_qps": rate,
                              "p50_ms": lat[len(lat) // 2], "p99_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))]}
            finally:
                for xs in tabs.values():
                    for x in xs:
                        x.free()
    out["speedup_closed_loop"] = out["batched"]["queries_per_s"] / out["plain"]["queries_per_s"]
    small.close()
    return out


class Replicas:
    """The ranks of a multi-GPU run: one process per GPU, each running whole
    queries on its own replica of the tables (no data exchange). Timing is the
    max over ranks of each rank's device time, and the job's queries/s counts
    every rank's queries. `dist` is torch.distributed (None for one rank);
    `device` holds the reduction tensor ("cuda" with NCCL, "cpu" with gloo)."""

    def __init__(self, dist=None, device="cuda", sync=None):
        self.dist, self.device, self.sync = dist, device, sync

    @property
    def world(self):
        return self.dist.get_world_size() if self.dist else 1

    def barrier(self):
        if self.dist:
            self.dist.barrier()
        if self.sync:
            self.sync()

    def max_over_ranks(self, x):
        if not self.dist:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def job_rate(self, units_per_rank, elapsed_ms):
        """Whole-job units/s from this rank's units and time (max over ranks)."""
        ms = self.max_over_ranks(elapsed_ms)
        return units_per_rank * self.world / (ms / 1e3) if units_per_rank else 0.0, ms


def batch_bench(args, local):
    """A batched workload (schema20: 256 queries of 2-12 tables over 20 shared
    tables) with its tables resident in HBM: `--warmup` untimed passes over the
    batch (a query's second run captures its CUDA graph), then `--steps` timed
    passes, queries issued one ahead with RESULT_ASYNC. Wall clock from the
    first issue to the last completion (host work included); per-query latency
    issue to completion. The reference engine runs one pass of the same batch."""
    import importlib
    pkg = importlib.import_module("contest-sigmod2025_b200")
    w = pkg.Workload(args.workload, args.seed, args.scale)
    n = w.num_queries()
    queries = [w.query_ptr(k) for k in range(n)]
    ctx = pkg.Context(local)
    inputs = w.plan_ptr().contents
    residents = [ctx.upload(inputs.inputs[i]) for i in range(inputs.num_inputs)]
    for _ in range(args.warmup):
        for q in queries:
            ctx.execute_resident(q, residents, flags=pkg.RESULT_DEVICE).free()
    lat, launches, rows = [], 0, 0

    def complete(entry):
        nonlocal launches, rows
        r, t0 = entry
        r.wait()
        lat.append((time.perf_counter() - t0) * 1e3)
        launches += r.stats().kernel_launches
        rows += r.num_rows
        r.free()

    start = time.perf_counter()
    pending = None
    for _ in range(args.steps):
        for q in queries:
            t0 = time.perf_counter()
            r = ctx.execute_resident(q, residents, flags=pkg.RESULT_DEVICE | pkg.RESULT_ASYNC)
            if pending:
                complete(pending)
            pending = (r, t0)
    if pending:
        complete(pending)
    seconds = time.perf_counter() - start
    for x in residents:
        x.free()
    ctx.close()
    lat.sort()
    out = {"mode": "batch", "workload": args.workload, "seed": args.seed, "scale": args.scale,
           "queries": len(lat), "table_rows": sum(inputs.inputs[i].num_rows for i in range(inputs.num_inputs)),
           "value": len(lat) / seconds, "unit": "queries/s", "p50_ms": lat[len(lat) // 2],
           "p99_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))], "gpu_launches": launches, "rows": rows}
    if args.cpu_steps and os.path.exists(REF_RUNNER):
        p = subprocess.run([REF_RUNNER, "batch", args.workload, str(args.seed), str(args.scale), "1"],
                           capture_output=True, text=True, timeout=1800)
        line = [l for l in p.stdout.splitlines() if l.startswith("{")]
        out["cpu_baseline"] = json.loads(line[-1]) if p.returncode == 0 and line else {"error": p.stderr[-300:]}
    print(json.dumps(out))
    return 0


def serve_schema20(pkg, args, local):
    """Serving the schema20 schema: its 20 tables resident once, a 9:1 mix of
    small queries (2-3 tables) and large ones (8-12 tables; the widest eight
    when fewer) drawn from the 256-query batch, through a server of 1 worker
    (the plain path) and of `--serve-workers` workers. Closed loop (every query
    submitted at once; queries/s to the last completion) and open loop (Poisson
    arrivals at 50% of the plain path's closed-loop rate; p50/p99 of submit to
    completion), as for the snowflake mix."""
    import random
    import threading

    w = pkg.Workload("schema20", args.seed, args.scale)
    n = w.num_queries()
    width = [(w.query_ptr(k).contents.num_nodes + 1) // 2 for k in range(n)]
    small = [k for k in range(n) if width[k] <= 3]
    large = [k for k in range(n) if width[k] >= 8] or sorted(range(n), key=lambda k: (-width[k], k))[:8]
    rng = random.Random(args.seed)
    mix = [rng.choice(large) if i % 10 == 9 else rng.choice(small) for i in range(args.serve_queries)]
    plans = {k: w.query_ptr(k) for k in sorted(set(mix))}
    inputs = w.plan_ptr().contents
    out = {"mode": "serve", "workload": "schema20", "seed": args.seed, "scale": args.scale,
           "mix": f"9 small (2-3 tables, {len(small)} distinct) : 1 large ({min(width[k] for k in large)}-"
                  f"{max(width[k] for k in large)} tables, {len(large)} distinct)", "queries": len(mix)}
    plain_qps = None
    for label, workers in (("plain", 1), ("batched", args.serve_workers)):
        with pkg.Server(local, workers=workers) as srv:
            tabs = [srv.upload(inputs.inputs[i]) for i in range(inputs.num_inputs)]
            try:
                # Warm every worker's graph cache for every plan of the mix.
                for t in [srv.submit(p, tabs, pkg.RESULT_DEVICE) for p in list(plans.values()) * (3 * workers)]:
                    srv.wait(t)[0].free()
                t0 = time.perf_counter()
                tickets = [srv.submit(plans[k], tabs, pkg.RESULT_DEVICE) for k in mix]
                for t in tickets:
                    srv.wait(t)[0].free()
                qps = len(mix) / (time.perf_counter() - t0)
                plain_qps = plain_qps or qps
                rate = 0.5 * plain_qps
                lat, issued = [], []
                lock = threading.Lock()

                def waiter():
                    done = 0
                    while done < len(mix):
                        with lock:
                            t = issued[done] if done < len(issued) else None
                        if t is None:
                            time.sleep(0.0001)
                            continue
                        r, ms = srv.wait(t)
                        r.free()
                        lat.append(ms)
                        done += 1

                th = threading.Thread(target=waiter)
                th.start()
                arrivals = random.Random(args.seed + 1)
                t_next = time.perf_counter()
                for k in mix:
                    t_next += arrivals.expovariate(rate)
                    while time.perf_counter() < t_next:
                        pass
                    t = srv.submit(plans[k], tabs, pkg.RESULT_DEVICE)
                    with lock:
                        issued.append(t)
                th.join()
                lat.sort()
                out[label] = {"workers": workers, "queries_per_s": qps, "arrival_rate_qps": rate,
                              "p50_ms": lat[len(lat) // 2], "p99_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))]}
            finally:
                for x in tabs:
                    x.free()
    out["speedup_closed_loop"] = out["batched"]["queries_per_s"] / out["plain"]["queries_per_s"]
    print(json.dumps(out))
    return 0


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank)
    if args.mode == "batch":
        return batch_bench(args, local) if rank == 0 else 0
    if args.mode == "serve" and args.workload == "schema20":
        import importlib
        return serve_schema20(importlib.import_module("contest-sigmod2025_b200"), args, local) if rank == 0 else 0

    import importlib
    import torch

    pkg = importlib.import_module("contest-sigmod2025_b200")
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    replicas = Replicas(dist, "cuda", torch.cuda.synchronize)
    barrier, max_over_ranks = replicas.barrier, replicas.max_over_ranks

    w = pkg.Workload(args.workload, args.seed, args.scale)
    plan = w.plan_ptr()
    ctx = pkg.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", local))
    inputs = plan.contents
    residents = [ctx.upload(inputs.inputs[i]) for i in range(inputs.num_inputs)]

    if args.mode in ("e2e", "serve"):
        args.steps = 0
    if args.mode == "serve":
        serving = serve_bench(pkg, args, w)
        for x in residents:
            x.free()
        ctx.close()
        if rank == 0:
            print(json.dumps({"mode": "serve", "serving": serving}))
        return 0
    # ---- value: tables resident in HBM ----
    # The timed steps run without instrumentation. A second, shorter pass with
    # the engine's CUDA-event profiling on gives the scan kernel's launch time
    # (the roofline) and the phase split; its event records cost ~35 us per
    # query, so that pass is kept out of `value`.
    for _ in range(args.warmup if args.steps else 0):
        ctx.execute_resident(plan, residents, flags=pkg.RESULT_DEVICE).free()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lat = []
    launches = 0
    rows = 0

    def complete(entry):
        nonlocal launches, rows
        r, t0 = entry
        r.wait()
        lat.append((time.perf_counter() - t0) * 1e3)
        launches += r.stats().kernel_launches
        rows = r.num_rows
        r.free()

    # Queries are issued with RESULT_ASYNC, one ahead: query k+1 is enqueued
    # before query k is waited for, so the host's per-call work overlaps the
    # device's; every result is completed (device checks included) and its
    # latency is issue to completion.
    ev0.record(stream)
    pending = None
    for _ in range(args.steps):
        t0 = time.perf_counter()
        r = ctx.execute_resident(plan, residents, flags=pkg.RESULT_DEVICE | pkg.RESULT_ASYNC)
        if pending:
            complete(pending)
        pending = (r, t0)
    if pending:
        complete(pending)
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    value, elapsed_ms = replicas.job_rate(args.steps, ev0.elapsed_time(ev1))
    # Profiled pass (same query, its own captured graph).
    prof_steps = min(args.steps, 100)
    scan_ms = scan_bytes = scan_n = 0
    phase_sum = [0.0] * 4
    ctx.profile(True)
    for i in range(3 + prof_steps if args.steps else 0):
        r = ctx.execute_resident(plan, residents, flags=pkg.RESULT_DEVICE)
        s = r.stats()
        r.free()
        if i < 3:
            continue
        scan_ms += s.scan_kernel_ms
        scan_bytes += s.scan_kernel_bytes
        scan_n += s.scan_kernel_launches
        for j in range(4):
            phase_sum[j] += s.phase_ms[j]
    ctx.profile(False)
    phases = {name: phase_sum[i] / max(prof_steps, 1) for i, name in
              enumerate(["build_ms", "probe_order_ms", "scan_probe_stages_ms", "output_ms"])}
    if args.mode == "value":
        for x in residents:
            x.free()
        ctx.close()
        if rank == 0:
            scan_gbs = (scan_bytes / scan_n) / (scan_ms / scan_n / 1e3) / 1e9 if scan_n and scan_ms > 0 else None
            print(json.dumps({"mode": "value", "value": value, "unit": "queries/s", "steps": args.steps,
                              "scan_kernel_us": scan_ms / scan_n * 1e3 if scan_n else None,
                              "scan_kernel_gbs": scan_gbs, "p50_ms": statistics.median(lat),
                              "phases": phases}))
        return 0

    # ---- e2e: drop-in path (bj_execute), host pages in and out ----
    e2e_steps = args.e2e_steps or max(3, min(args.steps, 20))

    def e2e_run():
        # Profiling (CUDA events at the executor's phase boundaries) is on, so
        # the line can say where a drop-in call spends its time.
        ctx.profile(True)
        for _ in range(2):
            ctx.execute_raw(plan).free()
        barrier()
        stats, lat_ms = None, []
        split = {"device_ms": 0.0, "phases": [0.0] * 4}
        ev0.record(stream)
        for _ in range(e2e_steps):
            t0 = time.perf_counter()
            r = ctx.execute_raw(plan)
            lat_ms.append((time.perf_counter() - t0) * 1e3)
            stats = r.stats()
            split["device_ms"] += stats.device_ms / e2e_steps
            for i in range(4):
                split["phases"][i] += stats.phase_ms[i] / e2e_steps
            r.free()
        ev1.record(stream)
        torch.cuda.synchronize()
        ctx.profile(False)
        rate, ms = replicas.job_rate(e2e_steps, ev0.elapsed_time(ev1))
        ph = split["phases"]
        split = {"device_ms": split["device_ms"],
                 "inputs_ms": split["device_ms"] - sum(ph),
                 "build_ms": ph[0], "probe_order_ms": ph[1], "scan_probe_stages_ms": ph[2], "output_ms": ph[3]}
        return rate, stats, lat_ms, split

    # (a) pages in pageable memory: gathered into pinned staging and copied.
    pageable_value, pageable_stats, pageable_lat, pageable_split = e2e_run()
    # (b) pages in pinned host memory (registered once, outside the timed
    # region, as a serving process keeps its host tables): read in place.
    registered = []
    for i in range(inputs.num_inputs):
        t = inputs.inputs[i]
        for c in range(t.num_columns):
            col = t.columns[c]
            if col.num_pages:
                ptr, size = col.pages[0], col.num_pages * pkg.PAGE_SIZE
                if torch._C._cudart.cudaHostRegister(ptr, size, 3) == 0:  # portable | mapped
                    registered.append(ptr)
    e2e_value, e2e_stats, e2e_lat, e2e_split = e2e_run()
    for ptr in registered:
        torch._C._cudart.cudaHostUnregister(ptr)
    if args.mode == "e2e":
        for x in residents:
            x.free()
        ctx.close()
        if rank == 0:
            print(json.dumps({"mode": "e2e", "e2e": e2e_value, "e2e_pageable": pageable_value, "unit": "queries/s",
                              "e2e_split": e2e_split, "e2e_pageable_split": pageable_split,
                              "e2e_p50_ms": statistics.median(e2e_lat)}))
        return 0
    h2d = e2e_stats.h2d_bytes + e2e_stats.mapped_input_bytes
    d2h = e2e_stats.d2h_bytes
    # ---- serving: concurrent queries through bj_server (one GPU) ----
    serving = serve_bench(pkg, args, w) if args.serve_queries > 0 and world == 1 else None

    for x in residents:
        x.free()
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0

    peak, peak_kind = measured_peak()
    achieved = (scan_bytes / scan_n) / (scan_ms / scan_n / 1e3) / 1e9 if scan_n and scan_ms > 0 else None
    traffic = profiled_traffic()
    out = {
        "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic", "config": config(args, world),
        "p50_ms": statistics.median(lat), "p99_ms": sorted(lat)[min(len(lat) - 1, int(0.99 * len(lat)))],
        "rows": rows,
        "scan_bytes_per_query": w.scan_bytes(),
        "input_gbs": w.scan_bytes() * value / world / 1e9,
        "e2e": {"value": e2e_value, "unit": "queries/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "p50_ms": statistics.median(e2e_lat),
                "inputs": "pinned host pages read in place by the kernels (h2d = page bytes available to them)",
                "dma_bytes_per_step": e2e_stats.h2d_bytes, "mapped_bytes_per_step": e2e_stats.mapped_input_bytes,
                "split_ms": e2e_split},
        "e2e_pageable": {"value": pageable_value, "unit": "queries/s", "p50_ms": statistics.median(pageable_lat),
                         "h2d_bytes_per_step": pageable_stats.h2d_bytes,
                         "d2h_bytes_per_step": pageable_stats.d2h_bytes,
                         "inputs": "pageable host pages, gathered into pinned staging and copied to HBM",
                         "split_ms": pageable_split},
        "gpu_launches": launches,
        "phases": phases,
        "serving": serving,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if achieved else None, "traffic": traffic,
                     "kernel": "k_scan_probe over the fact's key pages",
                     "launches": scan_n, "bytes_per_launch": scan_bytes / scan_n if scan_n else None,
                     "peak_kind": f"{peak_kind} HBM copy bandwidth"},
        "clocks": clk,
    }
    if world == 1 and args.cpu_steps > 0:
        res, err = run_reference(args, args.cpu_steps, 5)
        if res:
            mean = statistics.fmean(res["times_ms"])
            out["cpu_baseline"] = {"value": 1000.0 / mean, "unit": "queries/s", "cores": res["threads"],
                                   "kind": "reference",
                                   "sample": f"{args.cpu_steps} executions (+5 warm-up) of the full query by the "
                                             f"reference engine, wall clock"}
        else:
            out["cpu_baseline"] = {"value": None, "unit": "queries/s", "cores": None, "kind": "reference",
                                   "sample": err}
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
