"""Benchmark: batched regional SSSP on B200 (queries/s, GTEPS, HBM roofline).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl bfx|reference]

Workload (default c2): 128x128 tiles x 128 nodes (2,097,152 vertices,
16,777,216 edges), float costs base(span) * lognormal(0, 0.5); 256 regional
queries with box sides U[4,64] tiles, one source and one target each; the
planner groups overlapping queries into batches (narrowed to 1/8/16/32
lanes) and one persistent cooperative launch relaxes all of them.

A step is one pass of the hot path over the whole query set: labels reset,
seeded, relaxed to convergence, targets classified.  `value` times the steps
with inputs resident in HBM (device events on the launching stream);
`e2e.value` times the same steps through the C ABI from host buffers
(descriptions H2D from pinned staging, statuses D2H).  Inputs (graph 0.5 GB
+ labels) exceed the 126 MB L2, so no flush is needed between steps.

Multi-GPU (torchrun): replicas -- each rank holds the graph and relaxes its
own query set (weak scaling, no data-path collective); only the timing
max-reduction uses torch.distributed.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
for _p in (REPO, REPO / "bf-new_b200"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

import numpy as np  # noqa: E402

METRIC = "batched SSSP queries/s (256 uneven regional queries, 2.1M V / 16.8M E, one persistent launch)"
METRIC_C3 = "batched SSSP queries/s (64 full-graph sources, 16.8M V / 168M E, one persistent launch)"
METRIC_C5 = "batched SSSP queries/s (4,096 regional + 16 full-graph queries, 16.8M V / 168M E, autotuned)"
METRICS = {"c2": METRIC, "c3": METRIC_C3, "c5": METRIC_C5,
           "c3small": "batched SSSP queries/s (32 full-graph sources, 4.2M V / 42M E, profiling-sized c3)"}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def traffic_estimate(workload: str, relaxations: int, kernel_ms: float, path: Path | None = None):
    """DRAM traffic of one relaxation launch, scaled by relaxations from one
    ncu capture per workload class (profiles/frontier_push_traffic.txt:
    `workload bytes relaxations summary` lines; c2 from the c2 capture, c3 and
    c5 from the c3-shaped capture), and the launch's DRAM rate against the
    random-sector ceiling (`ceiling bytes_per_s summary`).  Returns (bytes or
    None, source text or None, ceiling dict or None)."""
    path = path or REPO / "profiles" / "frontier_push_traffic.txt"
    if not path.exists():
        return None, None, None
    captured, ceiling = {}, None
    for line in path.read_text().splitlines():
        parts = line.split()
        if line.startswith("#"):
            continue
        if len(parts) == 4:
            captured[parts[0]] = (int(parts[1]), int(parts[2]), parts[3])
        elif len(parts) == 3 and parts[0] == "ceiling":
            ceiling = (int(parts[1]), parts[2])
    key = "c2" if workload == "c2" else "c3small"
    if key not in captured or not relaxations:
        return None, None, None
    b, rl, src = captured[key]
    traffic = int(b / rl * relaxations)
    source = f"{src}: {b / rl:.1f} bytes per relaxation x {relaxations:,} relaxations"
    random_ceiling = None
    if ceiling is not None and kernel_ms > 0:
        dram_gbs = traffic / (kernel_ms / 1000) / 1e9
        random_ceiling = {"dram_gbs": dram_gbs, "peak_gbs": ceiling[0] / 1e9, "frac": dram_gbs * 1e9 / ceiling[0],
                          "source": ceiling[1] + " (random 32-byte sectors beyond the L2, 41 G/s)"}
    return traffic, source, random_ceiling


class ClockSampler:
    """nvidia-smi samples (every 50 ms) during the timed region.  Entering
    waits (up to 5 s) for the sampler's first line, so sampling is running
    when the timed region starts; only lines read inside the region count."""

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self._proc = None
        self._first = threading.Event()
        self._keep = False

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                           "--format=csv,noheader,nounits", "-lms", "50"],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            self._first.wait(timeout=5.0)
        except FileNotFoundError:
            self._proc = None
        self._keep = True
        return self

    def _read(self):
        for line in self._proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7:
                self._first.set()
                if self._keep:
                    self.samples.append(parts)

    def __exit__(self, *exc):
        self._keep = False
        if self._proc:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()

    def summary(self) -> dict:
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def cpu_reference_baseline(graph_input, order, queries, sample: int, threads: int):
    """The reference's own CPU engine (oracle/_ref: dijkstra_oracle on each
    query's induced graph, one query per host thread) on a bounded sample."""
    from oracle.oracle import Ref
    if not Ref.available():
        return None
    ref = Ref()
    t0 = time.time()
    h = ref.case_from_input(graph_input, order)
    build_s = time.time() - t0
    idx = []
    for q in queries[:sample]:
        idx.append(ref.query_add(h, q.query_id, q.sources, q.targets, q.selected_tiles))
    r = ref.time_dijkstra(h, idx, threads)
    ref.free(h)
    return {"value": sample / r["wall_s"], "unit": "queries/s", "cores": threads, "kind": "reference",
            "sample": f"first {sample} of the {len(queries)} queries, reference dijkstra_oracle on each induced "
                      f"graph, one query per thread (induced-graph builds, {r['induced_s']:.2f} thread-s, excluded)",
            "wall_s": r["wall_s"], "gteps": r["edges"] / r["wall_s"] / 1e9, "graph_build_s": build_s}


def cpu_port_baseline(layout, queries, sample: int, threads: int):
    """Fallback when the reference build is absent: the oracle's C restatement."""
    from oracle.oracle import Oracle
    orc = Oracle.from_layout(layout)
    t0 = time.time()
    orc.region_sssp_many(queries[:sample], threads)
    wall = time.time() - t0
    return {"value": sample / wall, "unit": "queries/s", "cores": threads, "kind": "port",
            "sample": f"first {sample} of {len(queries)} queries, oracle bounded Dijkstra, one query per thread",
            "wall_s": wall}


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import bfx
    from bfx import workloads
    g, order, _ = bfx.synth_graph(**workloads.GRAPHS["c2"])
    layout = bfx.build_device_graph_layout(g, order)
    grid = (128, 128)
    queries = workloads.box_queries(layout, grid, 256, 4, 64, 202)
    threads = os.cpu_count() or 1
    from oracle.oracle import Ref
    if not Ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU library (oracle/_ref) was not built"}))
        return
    ref = Ref()
    h = ref.case_from_input(g, order)
    idx = [ref.query_add(h, q.query_id, q.sources, q.targets, q.selected_tiles) for q in queries]
    sample = 64
    for _ in range(args.warmup):
        ref.time_dijkstra(h, idx[:8], threads)
    walls = []
    for s in range(args.steps):
        part = [idx[(s * sample + i) % len(idx)] for i in range(sample)]
        walls.append(ref.time_dijkstra(h, part, threads)["wall_s"])
    total = sum(walls)
    v = sample * args.steps / total
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "queries/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "c2: 256 regional queries on 128x128x128 tiles (2.1M V, 16.8M E), f32 lognormal "
                                   "costs; each step a bounded sample of 64 of those queries"},
            "cpu_baseline": {"value": v, "unit": "queries/s", "cores": threads, "kind": "reference",
                             "sample": "64 queries per step, reference dijkstra_oracle on induced graphs"},
            "e2e": {"value": v, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="bfx", choices=["bfx", "reference"])
    ap.add_argument("--engine", default="auto", choices=["auto", "frontier", "jacobi", "dense"])
    ap.add_argument("--workload", default="c2", choices=["c2", "c3", "c5", "c3small"])
    ap.add_argument("--frontier", default="chunked", choices=["groups", "flat", "chunked"],
                    help="frontier-push work layout (sub-warp groups or flat work list)")
    ap.add_argument("--regs", type=int, default=0, choices=[0, 40, 64, 80],
                    help="register budget of the persistent kernel (0: 80 for the chunked layout, else 64)")
    ap.add_argument("--items", type=int, default=2, choices=[2, 3, 4],
                    help="flat layout: work items per thread per iteration")
    ap.add_argument("--policy", default=None,
                    help="planner policy jaccard_num,jaccard_den,inflation_num,inflation_den (default per workload)")
    ap.add_argument("--amin", type=int, default=0, choices=[0, 1],
                    help="flat frontier: 1 = one returning min per relaxation")
    ap.add_argument("--edge-major", type=int, default=0, choices=[0, 1],
                    help="flat/chunked work order: 1 = entry, edge, lane")
    ap.add_argument("--pairs", type=int, default=0, choices=[0, 1],
                    help="chunked frontier: 1 = one (vertex, lane) pair per thread")
    ap.add_argument("--step", type=float, default=None,
                    help="with --engine frontier: near/far threshold step in mean edge weights (0 = plain frontier)")
    ap.add_argument("--tune-policy", action="store_true",
                    help="choose the planner policy by timing each candidate's plan (bfx_autotune_policy)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--queries", type=int, default=None)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference_arm(args)
        return

    rank, world, local = dist_env()
    dist = None
    if world > 1:
        import torch
        import torch.distributed as tdist
        from datetime import timedelta
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=timedelta(seconds=300))
        dist = tdist

    import bfx
    from bfx import replicas, workloads

    t0 = time.time()
    spec = dict(workloads.GRAPHS["c3" if args.workload in ("c5", "c3small") else args.workload])
    if args.workload == "c3small":  # c3 generator on 128x128 tiles: a profiling-sized case of the c3 kernel
        spec["tiles_x"] = spec["tiles_y"] = 128
    g, order, gstats = bfx.synth_graph(**spec)
    layout = bfx.build_device_graph_layout(g, order)
    # query classes: (queries, plain-engine sample size) -- the plain per-query
    # rate is extrapolated class by class from its sample
    if args.workload == "c2":
        grid = (128, 128)
        queries = workloads.box_queries(layout, grid, args.queries or 256, 4, 64, 202 + 1000 * rank)
        classes = [(queries, 64)]
        policy = bfx.BatchPlannerPolicy(32, 1, 8, 2, 1, narrow_lanes=True)
        workload_desc = ("c2: 256 uneven regional queries (box side U[4,64] tiles) on 128x128 tiles x 128 nodes, "
                         "2,097,152 V / 16,777,216 E, f32 lognormal costs")
    elif args.workload == "c3small":
        grid = (128, 128)
        queries = workloads.full_graph_queries(layout, grid, args.queries or 32, 303 + 1000 * rank)
        classes = [(queries, 2)]
        policy = bfx.BatchPlannerPolicy(32, 0, 1, 64, 1)
        workload_desc = ("c3small: 32 full-graph sources in one batch of 32 on 128x128 tiles x 256 nodes, "
                         "4,194,304 V / 41,943,040 E, uint costs U[1,255] (profiling-sized c3)")
    elif args.workload == "c3":
        grid = (256, 256)
        queries = workloads.full_graph_queries(layout, grid, args.queries or 64, 303 + 1000 * rank)
        classes = [(queries, 4)]
        policy = bfx.BatchPlannerPolicy(32, 0, 1, 64, 1)
        workload_desc = ("c3: 64 full-graph sources in batches of 32 on 256x256 tiles x 256 nodes, "
                         "16,777,216 V / 167,772,160 E, uint costs U[1,255]")
    else:
        grid = (256, 256)
        regional = workloads.box_queries(layout, grid, args.queries or 4096, 2, 16, 505 + 1000 * rank)
        full = workloads.full_graph_queries(layout, grid, 16, 506 + 1000 * rank, first_id=len(regional))
        queries = regional + full
        classes = [(regional, 64), (full, 2)]
        policy = bfx.BatchPlannerPolicy(32, 1, 8, 2, 1, narrow_lanes=True)
        workload_desc = ("c5: 4,096 regional queries (box side U[2,16] tiles) + 16 full-graph sources on 256x256 "
                         "tiles x 256 nodes, 16,777,216 V / 167,772,160 E, uint costs U[1,255]")
    if args.policy:
        jn, jd, inn, ind = (int(x) for x in args.policy.split(","))
        policy = bfx.BatchPlannerPolicy(32, jn, jd, inn, ind, narrow_lanes=True)
    t1 = time.time()
    plan = bfx.make_overlapping_batch_plan(layout, queries, policy)
    descs = plan.descriptions()
    t2 = time.time()
    lane_edges = sum(e[3] for e in plan.estimates)
    log(f"[bench] graph+layout {t1 - t0:.1f}s plan {t2 - t1:.1f}s: {plan.batch_count} batches, "
        f"widths {sorted({d.lane_width for d in descs})}, sum selected edges {lane_edges:,}")

    device = local if world > 1 else 0
    resident = bfx.ResidentDeviceGraph.upload_once(layout, device)
    ws = bfx.Workspace(resident)
    ws.set_frontier_layout({"flat": bfx.FRONTIER_FLAT, "groups": bfx.FRONTIER_GROUPS,
                            "chunked": bfx.FRONTIER_CHUNKED}[args.frontier])
    ws.set_register_budget(args.regs)
    # the budget the library applies (blocks of 256 threads)
    eff_regs = args.regs or (80 if args.frontier == "chunked" else 64)
    if args.frontier != "chunked" and eff_regs == 80:
        eff_regs = 64
    ws.set_flat_items(args.items)
    ws.set_relax_atomic(args.amin)
    ws.set_flat_order(args.edge_major)
    ws.set_chunk_pairs(args.pairs)
    engine_id = {"auto": bfx.ENGINE_AUTO, "frontier": bfx.ENGINE_FRONTIER_PUSH, "jacobi": bfx.ENGINE_JACOBI_PULL,
                 "dense": bfx.ENGINE_DENSE_CHAOTIC_PUSH}[args.engine]
    engines_chosen = None
    policy_times = None
    if args.tune_policy:
        # planner / autotuner co-design: the policy whose plan runs fastest
        candidates = [policy] + [bfx.BatchPlannerPolicy(32, *c, narrow_lanes=True)
                                 for c in ((1, 16, 4, 1), (1, 4, 2, 1), (1, 32, 8, 1))]
        t4 = time.time()
        best, policy_times = ws.autotune_policy(layout, queries, candidates)
        policy = candidates[best]
        plan = bfx.make_overlapping_batch_plan(layout, queries, policy)
        descs = plan.descriptions()
        lane_edges = sum(e[3] for e in plan.estimates)
        log(f"[bench] policy tuning {time.time() - t4:.1f}s: times {policy_times}, best {best}, "
            f"{plan.batch_count} batches")
    if engine_id == bfx.ENGINE_AUTO:
        t3 = time.time()
        engines_chosen, measured = ws.autotune(descs)
        log(f"[bench] autotune {time.time() - t3:.1f}s ({measured} batches timed): "
            f"{ {e: engines_chosen.count(e) for e in set(engines_chosen)} } (0 jacobi, 1 dense, 2 frontier)")
    elif args.step is not None:
        # fixed near/far step for every batch (profiling a chosen step)
        wbar = float(np.mean(layout.arrays["csr_weights"]))
        ws.set_batch_deltas([float("inf") if args.step == 0 else args.step * wbar] * len(descs))
    opts = bfx.GpuRunOptions(engine=engine_id)
    opts_instr = bfx.GpuRunOptions(engine=engine_id, instrumentation=1)

    import torch
    torch.cuda.set_device(device)
    stream = torch.cuda.ExternalStream(ws.stream, device=device)

    def barrier():
        torch.cuda.synchronize(device)
        if dist:
            dist.barrier()
        torch.cuda.synchronize(device)

    def max_over_ranks(x: float) -> float:
        return replicas.max_over_ranks(dist, x) if dist else x

    # ---- instrumented pass (untimed): algorithmic work counts + parity spot check
    ws.prepare(descs)
    ws.execute(opts_instr)
    statuses = ws.fetch_statuses()
    work = ws.work_counters()
    engine_work = ws.engine_work()
    assert all(s.stop_reason == bfx.STOP_CONVERGED for s in statuses), "benchmark run did not converge"
    reached = sum(bin(s.reached_target_mask).count("1") for s in statuses)

    # ---- device-resident timing (value)
    for _ in range(args.warmup):
        ws.execute(opts)
    barrier()
    with ClockSampler(device) as clocks:
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        # NVTX range: lets a profiler select the timed launches
        # (ncu --nvtx --nvtx-include "bench_timed/")
        torch.cuda.nvtx.range_push("bench_timed")
        for _ in range(args.steps):
            ws.execute(opts)
        torch.cuda.nvtx.range_pop()
        end.record(stream)
        barrier()
    dev_ms = start.elapsed_time(end)
    # Relaxation-kernel time per launch (library events on the same stream),
    # sampled right after the timed region.
    kernel_ms, execute_ms = [], []
    for _ in range(3):
        ws.execute(opts)
        k, x = ws.last_execute_timing()
        kernel_ms.append(k)
        execute_ms.append(x)
    launches_per_step = ws.last_launch_count()
    dev_ms = max_over_ranks(dev_ms)
    log(f"[bench] device-resident: {dev_ms / args.steps:.3f} ms/step, relaxation kernel {np.mean(kernel_ms):.3f} ms")
    statuses = ws.fetch_statuses()
    assert all(s.stop_reason == bfx.STOP_CONVERGED for s in statuses)
    if dist:  # the job's one exchange: every rank's status records to every rank
        all_statuses = replicas.gather_statuses(dist, statuses)
        assert all(s.stop_reason == bfx.STOP_CONVERGED for part in all_statuses for s in part)

    # ---- end-to-end timing through the C ABI from host buffers (e2e)
    for _ in range(args.warmup):
        ws.prepare(descs)
        ws.execute(opts)
        ws.fetch_statuses()
    barrier()
    s2 = torch.cuda.Event(enable_timing=True)
    e2 = torch.cuda.Event(enable_timing=True)
    s2.record(stream)
    for _ in range(args.steps):
        ws.prepare(descs)
        ws.execute(opts)
        ws.fetch_statuses()
    e2.record(stream)
    barrier()
    e2e_ms = max_over_ranks(s2.elapsed_time(e2))
    log(f"[bench] end-to-end: {e2e_ms / args.steps:.3f} ms/step")
    h2d, d2h = ws.transfer_bytes()

    # ---- plain per-query engine (one query per launch sequence) on a sample
    # of each query class; the whole set's time is extrapolated per class.
    # The baseline is the faster of the frontier layouts for single queries.
    plain_by_layout = {}
    for lname, lid in (("chunked", bfx.FRONTIER_CHUNKED), ("flat", bfx.FRONTIER_FLAT)):
        ws.set_frontier_layout(lid)
        plain_total_s, plain_sampled = 0.0, 0
        for members, n in classes:
            sample_q = members[:n]
            ws.run_query(sample_q[0].sources, sample_q[0].targets, sample_q[0].selected_tiles,
                         bfx.GpuRunOptions(engine=bfx.ENGINE_FRONTIER_PUSH))  # warm-up
            barrier()
            s3 = torch.cuda.Event(enable_timing=True)
            e3 = torch.cuda.Event(enable_timing=True)
            s3.record(stream)
            for q in sample_q:
                ws.run_query(q.sources, q.targets, q.selected_tiles, bfx.GpuRunOptions(engine=bfx.ENGINE_FRONTIER_PUSH))
            e3.record(stream)
            barrier()
            plain_total_s += s3.elapsed_time(e3) / 1000 / len(sample_q) * len(members)
            plain_sampled += len(sample_q)
        plain_by_layout[lname] = len(queries) / plain_total_s
    ws.set_frontier_layout({"flat": bfx.FRONTIER_FLAT, "groups": bfx.FRONTIER_GROUPS,
                            "chunked": bfx.FRONTIER_CHUNKED}[args.frontier])
    plain_layout = max(plain_by_layout, key=plain_by_layout.get)
    plain_qps = plain_by_layout[plain_layout]

    nq = len(queries) * world
    ms_per_step = dev_ms / args.steps
    value = nq / (ms_per_step / 1000)
    e2e_value = nq / (e2e_ms / args.steps / 1000)
    kernel_avg = float(np.mean(kernel_ms))
    # algorithmic bytes per launch, per engine class:
    #   push (frontier, dense): 16 F + 12 S + 8 P + 16 L + 8 N (dense has N = 0)
    #   Jacobi pull:            16 (vertex-lane items) + 12 (in-edge records) + 8 (relaxations)
    pw, jw = engine_work["push"], engine_work["jacobi"]
    F, S, Pp, L, N = (pw[k] for k in ("entries", "records", "active_pairs", "relaxations", "claims"))
    alg_bytes = (16 * F + 12 * S + 8 * Pp + 16 * L + 8 * N +
                 16 * jw["items"] + 12 * jw["records"] + 8 * jw["relaxations"])
    peaks_path = REPO / "MEASURED_PEAKS.json"
    if peaks_path.exists():
        peak = json.loads(peaks_path.read_text())["hbm_gbs"]
        peak_src = "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    achieved = alg_bytes / (kernel_avg / 1000) / 1e9
    traffic, traffic_source, random_ceiling = traffic_estimate(args.workload, work["relaxations"], kernel_avg)

    line = {
        "metric": METRICS[args.workload], "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_desc,
                   "queries_per_gpu": len(queries), "batches": plan.batch_count,
                   "lane_widths": sorted({d.lane_width for d in descs}), "engine": args.engine,
                   "policy_times_ms": policy_times,
                   "planner_policy": [policy.minimum_jaccard_numerator, policy.minimum_jaccard_denominator,
                                      policy.maximum_union_inflation_numerator,
                                      policy.maximum_union_inflation_denominator],
                   "near_far_step": args.step,
                   "frontier_layout": args.frontier, "registers": eff_regs, "flat_items": args.items, "returning_min": args.amin, "edge_major": args.edge_major, "chunk_pairs": args.pairs,
                   "engines_chosen": None if engines_chosen is None else
                   {name: engines_chosen.count(e) for e, name in ((0, "jacobi"), (1, "dense"), (2, "frontier"))},
                   "frontier_steps_chosen": None if engines_chosen is None else
                   {("plain" if not np.isfinite(d) else f"{d:.4g}"): sum(
                       1 for e, x in zip(engines_chosen, ws.tuned_deltas) if e == 2 and x == d)
                    for d in sorted({x for e, x in zip(engines_chosen, ws.tuned_deltas) if e == 2})},
                   "control": "persistent_cooperative", "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2 (graph %s GB + labels), no flush" % (
                       {"c2": "0.54", "c3small": "1.3"}.get(args.workload, "5.4"))},
        "gteps": lane_edges * world / (ms_per_step / 1000) / 1e9,
        "reached_lanes": reached,
        "e2e": {"value": e2e_value, "unit": "queries/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "plain_per_query": {"value": plain_qps, "unit": "queries/s", "sample": plain_sampled,
                            "layout": plain_layout, "by_layout": plain_by_layout,
                            "batched_speedup": value / world / plain_qps},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "traffic_source": traffic_source, "peak_source": peak_src,
                     "random_sector_ceiling": random_ceiling, "kernel": "persistent_kernel (%s frontier, %d registers, %d items%s)" % (
                         args.frontier, eff_regs, args.items if (eff_regs == 64 and args.frontier != "chunked") or (
                             eff_regs == 80 and args.frontier == "chunked" and not args.pairs) else 2,
                         ", mixed engines" if engines_chosen and any(e != 2 for e in engines_chosen) else ""),
                     "kernel_ms": kernel_avg, "execute_ms": float(np.mean(execute_ms)),
                     "algorithmic_bytes_per_launch": alg_bytes, "work": work, "engine_work": engine_work},
        "clocks": clocks.summary(),
        "gpu_launches": launches_per_step * args.steps,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        try:
            cb = cpu_reference_baseline(g, order, queries, 32, threads) if args.workload == "c2" else None
        except Exception as exc:  # reference build unusable here
            log(f"[bench] reference baseline failed: {exc}")
            cb = None
        line["cpu_baseline"] = cb or cpu_port_baseline(layout, queries, 32 if args.workload == "c2" else threads,
                                                       threads)
    if rank == 0:
        print(json.dumps(line))
    ws.close()
    resident.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
