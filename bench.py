"""Benchmark: batched regional SSSP on B200 (queries/s, GTEPS, HBM roofline).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl bfx|reference]
                    [--workload c2|c3|c5|c3small] [--shard] [--no-c3]

Workload (default c2): 128x128 tiles x 128 nodes (2,097,152 vertices,
16,777,216 edges), float costs base(span) * lognormal(0, 0.5); 256 regional
queries with box sides U[4,64] tiles, one source and one target each; the
planner groups overlapping queries into batches (narrowed to 1/8/16/32
lanes) and one persistent cooperative launch relaxes all of them.  On one GPU
the default run also times c3 (64 full-graph sources on 256x256 tiles x 256
nodes, 16.8M V / 168M E, uint costs) and c5 (4,096 regional + 16 full-graph
queries on the same graph) and reports them in the line's `c3` and `c5`
objects, each with its own roofline and plain per-query comparison.

A step is one pass of the hot path over the whole query set: labels reset,
seeded, relaxed to convergence, targets classified.  `value` times the steps
with inputs resident in HBM (device events on the launching stream);
`e2e.value` times the same steps through the C ABI from host buffers
(descriptions H2D from pinned staging, statuses D2H).  The host planner and
the autotuner run before the timed regions; their times are reported as
`host.plan_s` / `host.tune_s`.  Inputs (graph 0.5 GB + labels) exceed the
126 MB L2, so no flush is needed between steps.

The cpu_baseline leg times the reference's own CPU engine (oracle/_ref:
dijkstra_oracle on induced graphs) on a sample of the same queries and
checks the GPU's labels of those queries against it: distances bit for bit
against the reference, predecessors against the oracle's min-eid tight
in-edge (`parity` in the line).

Multi-GPU (torchrun): replicas -- each rank holds the graph and relaxes its
own query set (weak scaling, no data-path collective); with --shard the one
query set is planned once and its batches are split over the ranks by
estimated lane-edges (strong scaling).  Only the timing max-reduction and the
final status gather use torch.distributed.
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

METRICS = {
    "c2": "batched SSSP queries/s (256 uneven regional queries, 2.1M V / 16.8M E, one persistent launch)",
    "c3": "batched SSSP queries/s (64 full-graph sources, 16.8M V / 168M E, one persistent launch)",
    "c5": "batched SSSP queries/s (4,096 regional + 16 full-graph queries, 16.8M V / 168M E, autotuned)",
    "c3small": "batched SSSP queries/s (32 full-graph sources, 4.2M V / 42M E, profiling-sized c3)",
}
GRAPH_GB = {"c2": "0.54", "c3small": "1.3", "c3": "5.4", "c5": "5.4"}
INF_BITS = 0x7F800000


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def traffic_estimate(workload: str, relaxations: int, kernel_ms: float, step: str | None = None,
                     path: Path | None = None):
    """DRAM traffic of one relaxation launch, scaled by relaxations from one
    ncu capture per workload class (profiles/frontier_push_traffic.txt:
    `workload bytes relaxations step summary` lines, one per captured step;
    c2 from the c2 captures, c3 and c5 from the c3-shaped ones), and the
    launch's DRAM rate against the random-sector ceiling (`ceiling
    bytes_per_s summary`).  The near/far step changes the relaxations per
    sector, so only a capture at the launch's own step is scaled (`step` =
    the launch's steps, e.g. "1" or "plain"; None takes the first line).  Returns (bytes or None, source text or None,
    ceiling dict or None)."""
    path = path or REPO / "profiles" / "frontier_push_traffic.txt"
    if not path.exists():
        return None, None, None
    captured, ceiling = {}, None  # workload -> {step: (bytes, relaxations, summary)}
    for line in path.read_text().splitlines():
        parts = line.split()
        if line.startswith("#"):
            continue
        if len(parts) == 5:
            captured.setdefault(parts[0], {})[parts[3]] = (int(parts[1]), int(parts[2]), parts[4])
        elif len(parts) == 3 and parts[0] == "ceiling":
            ceiling = (int(parts[1]), parts[2])
    key = "c2" if workload == "c2" else "c3small"
    if key not in captured or not relaxations:
        return None, None, None
    by_step = captured[key]
    if step is not None and step not in by_step:
        src = next(iter(by_step.values()))[2]
        return None, (f"{src}: captured at step {', '.join(sorted(by_step))}, launch ran at step {step}; "
                      "not scaled"), None
    cstep = step if step is not None else next(iter(by_step))
    b, rl, src = by_step[cstep]
    traffic = int(b / rl * relaxations)
    source = f"{src} (step {cstep}): {b / rl:.1f} bytes per relaxation x {relaxations:,} relaxations"
    random_ceiling = None
    if ceiling is not None and kernel_ms > 0:
        dram_gbs = traffic / (kernel_ms / 1000) / 1e9
        random_ceiling = {"dram_gbs": dram_gbs, "peak_gbs": ceiling[0] / 1e9, "frac": dram_gbs * 1e9 / ceiling[0],
                          "source": ceiling[1] + " (random 32-byte sectors beyond the L2)"}
    return traffic, source, random_ceiling


def step_label(engines, deltas, mean_weight: float) -> str:
    """The near/far step of the launch's frontier batches in mean edge
    weights ("plain" without a threshold, "mixed" when batches differ)."""
    steps = {("plain" if not np.isfinite(d) else f"{d / mean_weight:.3g}")
             for e, d in zip(engines, deltas) if e == 2}
    return steps.pop() if len(steps) == 1 else ("none" if not steps else "mixed")


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


# ---------------------------------------------------------------------------
# Reference arm and CPU baseline (the reference's own CPU engine)
# ---------------------------------------------------------------------------

def reference_case(workload: str, query_count: int | None = None):
    """The reference's own case for a timed workload: the synthetic graph from
    the generator restated in the reference driver, partitioned and laid out
    by the reference, and the query set drawn from the reference's tile table
    by the same samplers as the GPU arm (bfx.workloads is pure Python here:
    libbfx is not loaded)."""
    from bfx import workloads
    from oracle.oracle import Ref
    spec, grid = workloads.bench_graph_spec(workload)
    ref = Ref()
    t0 = time.time()
    h = ref.case_synth(spec)
    build_s = time.time() - t0
    queries, _ = workloads.bench_queries(workload, ref.tiles(h), grid, 0, query_count)
    idx = [ref.query_add(h, q.query_id, q.sources, q.targets, q.selected_tiles) for q in queries]
    return ref, h, queries, idx, build_s


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle.oracle import Ref
    if not Ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU library (oracle/_ref) was not built"}))
        return
    from bfx import workloads
    ref, h, queries, idx, build_s = reference_case(args.workload, args.queries)
    threads = os.cpu_count() or 1
    # Full-graph queries build an induced copy of the whole graph each, so
    # the full-graph workloads time a bounded sample of their queries.
    full_graph = args.workload in ("c3", "c3small")
    timed = idx if not full_graph else idx[:min(len(idx), 4)]
    r = ref.time_dijkstra_steps(h, timed, threads, args.warmup, args.steps)
    total = sum(r["step_s"])
    nq = len(timed)
    v = nq * args.steps / total
    sample = (f"all {nq} queries of the set every step" if nq == len(queries) else
              f"first {nq} of the {len(queries)} queries every step")
    line = {"impl": "reference", "metric": METRICS[args.workload], "value": v, "unit": "queries/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workloads.BENCH_DESCRIPTIONS[args.workload], "queries_per_step": nq},
            "gteps": r["edges"] * args.steps / total / 1e9,
            "host": {"graph_build_s": build_s, "induced_graphs_s": r["induced_wall_s"],
                     "note": "induced graphs are built once before the timed steps (their wall time is "
                             "induced_graphs_s); each step runs dijkstra_oracle over every sampled query"},
            "pipeline": {"value": nq / (r["induced_wall_s"] + total / args.steps), "unit": "queries/s",
                         "what": "induced-graph builds + one step of dijkstra_oracle"},
            "cpu_baseline": {"value": v, "unit": "queries/s", "cores": threads, "kind": "reference",
                             "sample": f"{sample}; reference dijkstra_oracle on each query's induced graph, "
                                       f"one query per host thread"},
            "e2e": {"value": v, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    ref.free(h)
    print(json.dumps(line))


def cpu_baseline_and_parity(wl, lane_images, sample_ids, threads):
    """The reference's own CPU engine timed on a sample of the queries (one
    step, all host threads), and the GPU's labels of those queries checked
    against it: distances bit for bit against the reference's
    dijkstra_oracle, predecessors against the oracle's min-eid tight in-edge.
    `lane_images` maps query index -> (distance bits, predecessors) of the
    GPU run."""
    from oracle.oracle import Oracle, Ref
    checked = dist_bad = pred_bad = 0
    if Ref.available():
        ref, h, queries, idx, build_s = reference_case(wl.name, len(wl.queries))
        r = ref.time_dijkstra_steps(h, [idx[i] for i in sample_ids], threads, 0, 1, want_dist=True)
        wall = r["step_s"][0]
        ref_dist = {q: r["dist"][k].view(np.uint32) for k, q in enumerate(sample_ids)}
        ref.free(h)
        cb = {"value": len(sample_ids) / wall, "unit": "queries/s", "cores": threads, "kind": "reference",
              "sample": f"{len(sample_ids)} of the {len(wl.queries)} queries, reference dijkstra_oracle on each "
                        f"induced graph, one query per thread (induced-graph builds, {r['induced_wall_s']:.2f} s "
                        f"wall, excluded)",
              "wall_s": wall, "gteps": r["edges"] / wall / 1e9, "graph_build_s": build_s}
        checker = "reference dijkstra_oracle distances; oracle min-eid tight predecessors"
    else:
        ref_dist, cb = None, None
        checker = "oracle bounded Dijkstra distances and min-eid tight predecessors"
    orc = Oracle.from_layout(wl.layout)
    t0 = time.time()
    od, op = orc.region_sssp_many([wl.queries[i] for i in sample_ids], threads)
    port_wall = time.time() - t0
    if cb is None:
        cb = {"value": len(sample_ids) / port_wall, "unit": "queries/s", "cores": threads, "kind": "port",
              "sample": f"{len(sample_ids)} of {len(wl.queries)} queries, oracle bounded Dijkstra, one query per thread",
              "wall_s": port_wall}
    for k, q in enumerate(sample_ids):
        bits, pred = lane_images[q]
        want = ref_dist[q] if ref_dist is not None else od[k]
        dist_bad += int(np.count_nonzero(bits != want))
        pred_bad += int(np.count_nonzero(pred != op[k]))
        checked += 1
    parity = {"lanes_checked": checked, "distance_mismatches": dist_bad, "predecessor_mismatches": pred_bad,
              "mismatches": dist_bad + pred_bad, "checker": checker}
    return cb, parity


# ---------------------------------------------------------------------------
# The bfx arm
# ---------------------------------------------------------------------------

def measure(wl, args, *, rank, world, dist, device, steps, warmup, shard=False, sample_ids=(), warm_queries=None):
    """Plans, tunes and times one workload; returns (line dict, lane images of
    the sampled queries)."""
    import bfx
    import torch
    from bfx import replicas

    t0 = time.time()
    plan = bfx.make_overlapping_batch_plan(wl.layout, wl.queries, wl.policy)
    descs = plan.descriptions()
    plan_s = time.time() - t0
    estimates = [e[3] for e in plan.estimates]
    if shard and world > 1:
        mine = replicas.shard_batches(estimates, world)[rank]
        descs = [descs[b] for b in mine]
        estimates = [estimates[b] for b in mine]
    queries_here = sum(bin(d.valid_lane_mask).count("1") for d in descs)
    lane_edges = sum(estimates)
    log(f"[bench] {wl.name}: plan {plan_s:.2f}s: {len(descs)} batches, widths "
        f"{sorted({d.lane_width for d in descs})}, sum selected edges {lane_edges:,}")

    resident = bfx.ResidentDeviceGraph.upload_once(wl.layout, device)
    ws = bfx.Workspace(resident)
    layout_ids = {"flat": bfx.FRONTIER_FLAT, "groups": bfx.FRONTIER_GROUPS, "chunked": bfx.FRONTIER_CHUNKED,
                  "tiled": bfx.FRONTIER_TILED}
    ws.set_frontier_layout(layout_ids[args.frontier])
    ws.set_register_budget(args.regs)
    eff_regs = args.regs or (80 if args.frontier == "chunked" else 64)
    if args.frontier != "chunked" and eff_regs == 80:
        eff_regs = 64
    if args.frontier == "tiled":
        eff_regs = 128  # the tiled kernel's own bound: two 256-thread blocks per SM
        if args.stage_min is not None:
            ws.set_tile_stage_min(args.stage_min)
    ws.set_flat_items(args.items)
    ws.set_relax_atomic(args.amin)
    ws.set_flat_order(args.edge_major)
    ws.set_chunk_pairs(args.pairs)
    if args.pack is not None:
        ws.set_chunk_pack(args.pack)
    engine_id = {"auto": bfx.ENGINE_AUTO, "frontier": bfx.ENGINE_FRONTIER_PUSH, "jacobi": bfx.ENGINE_JACOBI_PULL,
                 "dense": bfx.ENGINE_DENSE_CHAOTIC_PUSH}[args.engine]
    mean_w = float(np.mean(wl.layout.arrays["csr_weights"]))
    engines_chosen, policy_times, tune_s = None, None, 0.0
    if args.tune_policy and not shard:
        candidates = [wl.policy] + [bfx.BatchPlannerPolicy(32, *c, narrow_lanes=True)
                                    for c in ((1, 16, 4, 1), (1, 4, 2, 1), (1, 32, 8, 1))]
        t4 = time.time()
        best, policy_times = ws.autotune_policy(wl.layout, wl.queries, candidates)
        plan = bfx.make_overlapping_batch_plan(wl.layout, wl.queries, candidates[best])
        descs = plan.descriptions()
        lane_edges = sum(e[3] for e in plan.estimates)
        tune_s += time.time() - t4
        log(f"[bench] policy tuning {time.time() - t4:.1f}s: times {policy_times}, best {best}")
    if engine_id == bfx.ENGINE_AUTO:
        t3 = time.time()
        engines_chosen, measured = ws.autotune(descs)
        tune_s += time.time() - t3
        log(f"[bench] autotune {time.time() - t3:.1f}s ({measured} batches timed): "
            f"{ {e: engines_chosen.count(e) for e in set(engines_chosen)} } (0 jacobi, 1 dense, 2 frontier)")
        deltas = list(ws.tuned_deltas)
    else:
        deltas = [float("inf")] * len(descs)
        if args.step is not None:
            deltas = [float("inf") if args.step == 0 else args.step * mean_w] * len(descs)
            ws.set_batch_deltas(deltas)
    # the layout and per-batch mappings the tuner left (it may switch between
    # the chunked and the tiled layout)
    layout_names = {v: k for k, v in layout_ids.items()}
    tuned_layout, tuned_mappings = ws.frontier_mapping(len(descs))
    frontier_used = layout_names[tuned_layout]
    if frontier_used == "tiled":
        eff_regs = 128
    opts = bfx.GpuRunOptions(engine=engine_id)
    opts_instr = bfx.GpuRunOptions(engine=engine_id, instrumentation=1)

    torch.cuda.set_device(device)
    stream = torch.cuda.ExternalStream(ws.stream, device=device)

    def barrier():
        torch.cuda.synchronize(device)
        if dist:
            dist.barrier()
        torch.cuda.synchronize(device)

    def max_over_ranks(x: float) -> float:
        return replicas.max_over_ranks(dist, x) if dist else x

    # ---- instrumented pass (untimed): algorithmic work counts, label bound
    ws.prepare(descs)
    ws.execute(opts_instr)
    statuses = ws.fetch_statuses()
    work = ws.work_counters()
    engine_work = ws.engine_work()
    assert all(s.stop_reason == bfx.STOP_CONVERGED for s in statuses), "benchmark run did not converge"
    reached = sum(bin(s.reached_target_mask).count("1") for s in statuses)
    bound_bits = int(ws.label_bounds().max())
    max_distance = float(np.uint32(bound_bits).view(np.float32))
    if wl.uint_costs:
        # integer costs are exact in float sums only below 2^24
        assert bound_bits < 0x4B800000, f"largest distance {max_distance} is not below 2^24"

    # ---- device-resident timing (value)
    for _ in range(warmup):
        ws.execute(opts)
    barrier()
    with ClockSampler(device) as clocks:
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        # NVTX range: lets a profiler select the timed launches
        torch.cuda.nvtx.range_push("bench_timed")
        for _ in range(steps):
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
    log(f"[bench] {wl.name} device-resident: {dev_ms / steps:.3f} ms/step, relaxation kernel "
        f"{np.mean(kernel_ms):.3f} ms")
    statuses = ws.fetch_statuses()
    assert all(s.stop_reason == bfx.STOP_CONVERGED for s in statuses)
    if dist:  # the job's one exchange: every rank's status records to every rank
        all_statuses = replicas.gather_statuses(dist, statuses)
        assert all(s.stop_reason == bfx.STOP_CONVERGED for part in all_statuses for s in part)

    # ---- end-to-end timing through the C ABI from host buffers (e2e): each
    # step prepares the set (host descriptions, or on the device from the
    # lane -> query assignment), relaxes it and fetches the statuses
    lanes = bfx.QueryLanes.from_descriptions(descs, wl.queries)

    def prepare():
        if args.prepare == "device":
            ws.prepare_from_queries(lanes)
        else:
            ws.prepare(descs)
        if engines_chosen is None and args.step is not None:
            ws.set_batch_deltas(deltas)

    for _ in range(warmup):
        prepare()
        ws.execute(opts)
        ws.fetch_statuses()
    barrier()
    s2 = torch.cuda.Event(enable_timing=True)
    e2 = torch.cuda.Event(enable_timing=True)
    s2.record(stream)
    for _ in range(steps):
        prepare()
        ws.execute(opts)
        ws.fetch_statuses()
    e2.record(stream)
    barrier()
    e2e_ms = max_over_ranks(s2.elapsed_time(e2))
    log(f"[bench] {wl.name} end-to-end: {e2e_ms / steps:.3f} ms/step")
    h2d, d2h = ws.transfer_bytes()

    # ---- the sampled queries' labels from the last launch (checked on the host)
    lane_of = {int(d.query_index_by_lane[l]): (b, l) for b, d in enumerate(descs)
               for l in range(d.lane_width) if (d.valid_lane_mask >> l) & 1}
    lane_images = {q: ws.download_lane(*lane_of[q]) for q in sample_ids if q in lane_of}

    # ---- plain per-query engine (one query per launch sequence) on a sample
    # of each query class; the whole set's time is extrapolated per class.
    # The baseline is the faster of the frontier layouts for single queries.
    plain_by_layout, plain_sampled = {}, 0
    classes = wl.classes if not (shard and world > 1) else []
    for lname, lid in (("chunked", bfx.FRONTIER_CHUNKED), ("flat", bfx.FRONTIER_FLAT)):
        if not classes:
            break
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
        plain_by_layout[lname] = len(wl.queries) / plain_total_s
    ws.set_frontier_layout(tuned_layout)

    nq = (len(wl.queries) if shard else queries_here * world)
    ms_per_step = dev_ms / steps
    value = nq / (ms_per_step / 1000)
    e2e_value = nq / (e2e_ms / steps / 1000)
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
    engines_for_step = engines_chosen or [2 if engine_id == bfx.ENGINE_FRONTIER_PUSH else engine_id] * len(descs)
    step = step_label(engines_for_step, deltas, mean_w)
    if frontier_used == "chunked":
        traffic, traffic_source, random_ceiling = traffic_estimate(wl.name, work["relaxations"], kernel_avg, step)
    else:  # the committed traffic captures are of the chunked kernel
        traffic, traffic_source, random_ceiling = None, f"no capture of the {frontier_used} kernel is scaled", None
    line = {
        "metric": METRICS[wl.name], "value": value, "unit": "queries/s", "n_gpus": world, "steps": steps,
        "warmup": warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "strong" if shard and world > 1 else "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": wl.description, "queries": nq, "batches": len(descs),
                   "lane_widths": sorted({d.lane_width for d in descs}), "engine": args.engine,
                   "policy_times_ms": policy_times,
                   "planner_policy": [wl.policy.minimum_jaccard_numerator, wl.policy.minimum_jaccard_denominator,
                                      wl.policy.maximum_union_inflation_numerator,
                                      wl.policy.maximum_union_inflation_denominator],
                   "near_far_step": step,
                   "frontier_layout": frontier_used,
                   "tile_visit_batches": (sum(1 for m in tuned_mappings if m == bfx.MAPPING_TILE_VISITS)
                                          if frontier_used == "tiled" else 0),
                   "registers": eff_regs, "flat_items": args.items,
                   "returning_min": args.amin, "edge_major": args.edge_major, "chunk_pairs": args.pairs,
                   "chunk_pack": ws.chunk_pack(),
                   "engines_chosen": None if engines_chosen is None else
                   {name: engines_chosen.count(e) for e, name in ((0, "jacobi"), (1, "dense"), (2, "frontier"))},
                   "control": "persistent_cooperative",
                   "parallelism": (f"shards{world}" if shard and world > 1 else f"replicas{world}"),
                   "l2": f"inputs larger than L2 (graph {GRAPH_GB[wl.name]} GB + labels), no flush"},
        "gteps": lane_edges * (1 if shard else world) / (ms_per_step / 1000) / 1e9,
        "reached_lanes": reached,
        "max_finite_distance": max_distance,
        "e2e": {"value": e2e_value, "unit": "queries/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "prepare": args.prepare},
        "host": {"plan_s": plan_s, "tune_s": tune_s,
                 "note": "host planner (batch grouping + descriptions) and autotuner run once per query set, "
                         "before both timed regions"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "traffic_source": traffic_source, "peak_source": peak_src,
                     "random_sector_ceiling": random_ceiling, "kernel": "%s (%s frontier, %d registers%s)" % (
                         "persistent_tiled_kernel" if frontier_used == "tiled" else "persistent_kernel",
                         frontier_used, eff_regs,
                         ", mixed engines" if engines_chosen and any(e != 2 for e in engines_chosen) else ""),
                     "kernel_ms": kernel_avg, "execute_ms": float(np.mean(execute_ms)),
                     "algorithmic_bytes_per_launch": alg_bytes, "work": work, "engine_work": engine_work},
        "clocks": clocks.summary(),
        "gpu_launches": launches_per_step * steps,
    }
    line["pipeline"] = {"value": nq / (plan_s + tune_s + e2e_ms / steps / 1000), "unit": "queries/s",
                        "what": "host plan + autotune + one end-to-end step (a fresh query set, tuned once)"}
    if plain_by_layout:
        plain_layout = max(plain_by_layout, key=plain_by_layout.get)
        plain_qps = plain_by_layout[plain_layout]
        line["plain_per_query"] = {"value": plain_qps, "unit": "queries/s", "sample": plain_sampled,
                                   "layout": plain_layout, "by_layout": plain_by_layout,
                                   "batched_speedup": value / world / plain_qps}
    if warm_queries is not None:
        # A second query set of the same workload (another seed), served by
        # the same workspace: host plan, autotune (its set class is tuned
        # already), device-side preparation, one launch, statuses -- host
        # wall clock around all of it.
        ws.set_frontier_layout(layout_ids[args.frontier])
        torch.cuda.synchronize(device)
        t0 = time.time()
        plan2 = bfx.make_overlapping_batch_plan(wl.layout, warm_queries, wl.policy)
        descs2 = plan2.descriptions()
        t1 = time.time()
        if engine_id == bfx.ENGINE_AUTO:
            ws.autotune(descs2)
        t2 = time.time()
        ws.prepare_from_queries(bfx.QueryLanes.from_descriptions(descs2, warm_queries))
        ws.execute(opts)
        st2 = ws.fetch_statuses()
        t3 = time.time()
        assert all(x.stop_reason == bfx.STOP_CONVERGED for x in st2)
        line["pipeline_warm"] = {"value": len(warm_queries) / (t3 - t0), "unit": "queries/s",
                                 "plan_s": t1 - t0, "tune_s": t2 - t1, "run_s": t3 - t2,
                                 "what": "a second query set of the same workload (another seed) on the same "
                                         "workspace: host plan + autotune (set class already tuned) + device-side "
                                         "preparation + one launch + statuses, host wall clock"}
    ws.close()
    resident.close()
    return line, lane_images


def bfx_policy_regional():
    """The planner policy of the regional workloads (c2, c5)."""
    import bfx
    return bfx.BatchPlannerPolicy(32, 1, 8, 2, 1, narrow_lanes=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="bfx", choices=["bfx", "reference"])
    ap.add_argument("--engine", default="auto", choices=["auto", "frontier", "jacobi", "dense"])
    ap.add_argument("--workload", default="c2", choices=["c2", "c3", "c5", "c3small"])
    ap.add_argument("--frontier", default="chunked", choices=["groups", "flat", "chunked", "tiled"],
                    help="frontier-push work layout (sub-warp groups or flat work list)")
    ap.add_argument("--regs", type=int, default=0, choices=[0, 40, 64, 80],
                    help="register budget of the persistent kernel (0: 80 for the chunked layout, else 64)")
    ap.add_argument("--items", type=int, default=2, choices=[2, 3, 4],
                    help="flat layout: work items per thread per iteration")
    ap.add_argument("--amin", type=int, default=0, choices=[0, 1],
                    help="flat frontier: 1 = one returning min per relaxation")
    ap.add_argument("--edge-major", type=int, default=0, choices=[0, 1],
                    help="flat/chunked work order: 1 = entry, edge, lane")
    ap.add_argument("--pairs", type=int, default=0, choices=[0, 1],
                    help="chunked frontier: 1 = one (vertex, lane) pair per thread")
    ap.add_argument("--pack", type=int, default=None, choices=[1, 2, 4, 8],
                    help="chunked frontier: chunk slots per warp item (default: the library's)")
    ap.add_argument("--step", type=float, default=None,
                    help="with --engine frontier: near/far threshold step in mean edge weights (0 = plain frontier)")
    ap.add_argument("--tune-policy", action="store_true",
                    help="choose the planner policy by timing each candidate's plan (bfx_autotune_policy)")
    ap.add_argument("--prepare", default="device", choices=["host", "device"],
                    help="e2e steps prepare the batch set from host descriptions or on the device from the "
                         "lane -> query assignment")
    ap.add_argument("--stage-min", type=int, default=None,
                    help="tiled layout: lane-edge work from which a tile visit stages its labels")
    ap.add_argument("--shard", action="store_true",
                    help="multi-GPU: split one query set's batches over the ranks (strong scaling)")
    ap.add_argument("--no-c3", action="store_true", help="skip the c3 and c5 objects of the default c2 run")
    ap.add_argument("--c3-steps", type=int, default=3)
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

    from bfx import workloads

    device = local if world > 1 else 0
    t0 = time.time()
    wl = workloads.bench_workload(args.workload, 0 if args.shard else rank, args.queries)
    log(f"[bench] graph+layout {time.time() - t0:.1f}s")
    cpu_leg = rank == 0 and world == 1 and not args.no_cpu_baseline
    threads = os.cpu_count() or 1
    # the cpu_baseline sample: 32 queries spread over the set (regional
    # workloads), or a few full-graph sources
    nsample = 32 if args.workload in ("c2", "c5") else min(2, len(wl.queries))
    sample_ids = sorted(np.random.default_rng(2024).choice(len(wl.queries), nsample, replace=False).tolist()) \
        if cpu_leg else []
    warm = None
    if args.workload == "c2" and world == 1 and args.queries is None:
        warm = workloads.box_queries(wl.layout, wl.grid, 256, 4, 64, 202 + 7)
    line, lane_images = measure(wl, args, rank=rank, world=world, dist=dist, device=device, steps=args.steps,
                                warmup=args.warmup, shard=args.shard, sample_ids=sample_ids, warm_queries=warm)
    if cpu_leg:
        try:
            cb, parity = cpu_baseline_and_parity(wl, lane_images, sample_ids, threads)
        except Exception as exc:  # reference build unusable here
            log(f"[bench] cpu baseline failed: {exc}")
            cb, parity = None, None
        line["cpu_baseline"] = cb
        line["parity"] = parity
    if args.workload == "c2" and world == 1 and not args.no_c3 and args.queries is None:
        # the c3 full-graph configuration and the c5 mixed set on the same
        # graph, timed in the same run (each with its own roofline)
        del wl
        t0 = time.time()
        wl3 = workloads.bench_workload("c3")
        log(f"[bench] c3 graph+layout {time.time() - t0:.1f}s")
        keep = ("metric", "value", "unit", "steps", "warmup", "ms_per_step", "gteps", "e2e", "host", "roofline",
                "clocks", "config", "plain_per_query", "max_finite_distance", "gpu_launches")
        c3, _ = measure(wl3, args, rank=rank, world=world, dist=dist, device=device, steps=args.c3_steps,
                        warmup=3, shard=False)
        line["c3"] = {k: c3[k] for k in keep}
        q5, classes5 = workloads.bench_queries("c5", wl3.layout, wl3.grid)
        wl5 = workloads.BenchWorkload("c5", wl3.graph_input, wl3.order, wl3.layout, wl3.grid, q5, classes5,
                                      bfx_policy_regional(), workloads.BENCH_DESCRIPTIONS["c5"], True)
        c5, _ = measure(wl5, args, rank=rank, world=world, dist=dist, device=device, steps=args.c3_steps,
                        warmup=3, shard=False)
        line["c5"] = {k: c5[k] for k in keep}
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
