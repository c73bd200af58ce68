#!/usr/bin/env python3
"""Benchmark of the batched isolated-route engine (fields + canonical paths).

Workload (default): the congestion board — 512x512x4, 256 nets, directed edge
prices, exact polygon outline, windows by net_window — one "step" routes every
net of the batch (complete u32 fields over every window + canonical paths).
`--workload plain` is the 128x128x2 board with 64 nets and whole-board fields;
`--workload uneven` is 4096 independent one-net instances of log-normal size
and 2-8 layers, staged as one multi-board batch.  The launch sequence is
replayed as a captured CUDA graph (`--no-graph` launches kernel by kernel).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload W]

One JSON line on rank 0.  `value` is whole-job nets/s with the board and nets
resident in HBM (device time from CUDA events on the launching stream, L2
flushed between steps, max over ranks); `e2e` is the same metric through the
public call with host buffers (upload, solve, download of paths and costs).
Under torchrun every rank routes its own net set on the same board (weak
scaling; no collective on the data path).  `--impl reference` times the CPU
restatement of the reference's own isolated search (window A*, full-board
retry) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "metal-route_b200"))

METRIC = "nets routed/sec & HBM GB/s (batched vs per-net, bit-exact); /solve p50/p99 ms"
UNIT = "nets/s"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _profile_figures(kernel: str, workload: str):
    """Figures of one kernel on one workload from the ncu captures summarised in
    profiles/roofline.json (DRAM bytes of one full-size launch, instructions
    per window cell, IPC), or None when that pair was not captured."""
    try:
        with open(os.path.join(ROOT, "profiles", "roofline.json")) as f:
            return json.load(f).get(f"{kernel}/{workload}")
    except (OSError, ValueError):
        return None


def _workload(name: str, rank: int, nets: int = 0):
    from mrcuda import workloads as W

    if name == "uneven":
        s = W.uneven_instances(seed=3 + 1000 * rank, n_instances=nets or 4096)
        return Job(s.instances, s.meta)
    if name == "snapshot":
        wl = W.snapshot_board(n_nets=nets or 3000)
        return Job([wl], wl.meta)
    if name == "plain":
        wl = W.plain_board(seed=1 + 1000 * rank)
    else:
        wl = W.congestion_board(seed=2, net_seed=None if rank == 0 else 2 + 1000 * rank)
    wl = W.scaled(wl, nets) if nets else wl
    return Job([wl], wl.meta)


class Job:
    """One bench step's work: the nets of one or more boards (instances),
    staged as one batch; net i belongs to boards[net_board[i]]."""

    def __init__(self, boards, meta):
        self.boards = boards
        self.meta = meta
        self.nets, self.windows, self.net_board = [], [], []
        for k, wl in enumerate(boards):
            self.nets += wl.nets
            self.windows += wl.windows
            self.net_board += [k] * len(wl.nets)

    def window_cells(self) -> int:
        return sum(wl.window_cells() for wl in self.boards)

    def algorithmic_bytes(self) -> int:
        return sum(wl.window_cells() * wl.bytes_per_cell() for wl in self.boards)

    def bytes_per_cell(self) -> float:
        return self.algorithmic_bytes() / max(self.window_cells(), 1)

    def requests(self):
        return [wl.request() for wl in self.boards]

    def route(self, eng):
        """The public host-buffer call (one request, or many instances in one
        call); returns the result in its CSR form (paths as numpy arrays)."""
        if len(self.boards) == 1:
            return eng.route_isolated_batch(self.boards[0].request())
        return eng.route_instances(self.requests(), split=False)

    def h2d_bytes(self) -> int:
        b = 0
        for wl in self.boards:
            g = wl.grid
            b += (g.cost.nbytes + (g.board_constraint.nbytes if g.board_constraint is not None else 0)
                  + (g.via_forbidden.nbytes if g.via_forbidden is not None else 0)
                  + (wl.directed.nbytes if wl.directed is not None else 0)
                  + 4 * (len(wl.x) + len(wl.y) + len(wl.vias)) + len(wl.vias) + 40 * len(wl.nets)
                  + 16 * len(wl.windows) + 4 * sum(len(nt.passable_pads) + len(nt.via_passable_pads)
                                                   for nt in wl.nets))
        return b


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _cpu_sample_rate(job, n_sample: int, threads: int = 0, mode: str = "astar"):
    """The oracle's alone-path search (window, then full board) on a sample of
    nets, all host threads: nets/s.  mode "astar" is the targeted search with
    early stop (LeeRouter / the rayon alone-path batch); mode "field" expands
    the whole window with h = 0 (the complete field, bfs_distance_field) and
    walks the canonical path.  Oracle code, timed as the CPU baseline; never the
    measured GPU path."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    from mrcuda.types import IsolatedRouteRequest

    o = orc.get()
    if len(job.boards) == 1:
        req = job.boards[0].request()
        sub = IsolatedRouteRequest(req.grid, req.nets[:n_sample], req.windows[:n_sample], req.x_edge_costs,
                                   req.y_edge_costs, req.via_edge_costs, req.directed_in_costs)
        t0 = time.perf_counter()
        o.isolated_batch(sub, retry_full=True, mode=mode, threads=threads)
        dt = time.perf_counter() - t0
        return n_sample / dt, dt
    # instances: one search per instance, spread over the host threads
    from concurrent.futures import ThreadPoolExecutor

    reqs = []
    for wl in job.boards:
        if len(reqs) >= n_sample:
            break
        reqs.append(wl.request())
    n = sum(len(r.nets) for r in reqs)
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads or os.cpu_count() or 1) as ex:
        list(ex.map(lambda r: o.isolated_batch(r, retry_full=True, mode=mode, threads=1), reqs))
    dt = time.perf_counter() - t0
    return n / dt, dt


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    wl = _workload(args.workload, 0, args.nets)
    cores = os.cpu_count() or 1
    # every net of the workload per step (the snapshot board's 3000 nets of
    # up to 1.5 M window cells each would take minutes: a sample there)
    n_sample = min(args.cpu_sample or (48 if args.workload == "snapshot" else len(wl.nets)), len(wl.nets))
    for _ in range(args.warmup):
        _cpu_sample_rate(wl, max(n_sample // 4, 1))
    rates = []
    t_all = time.perf_counter()
    for _ in range(args.steps):
        r, _ = _cpu_sample_rate(wl, n_sample)
        rates.append(r)
    wall = time.perf_counter() - t_all
    value = statistics.median(rates)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * wall / max(args.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": wl.meta["workload"], "windows": wl.meta.get("windows"), "nets": len(wl.nets)},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{n_sample} of {len(wl.nets)} nets per step: A* alone-path search "
                                   f"(window, then full board), {cores} host threads"},
        "same_config": n_sample == len(wl.nets),
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def measure_batch(args, name, eng, rank, world, local, dist, nets=0, steps=None, main=True):
    """One batched workload on the resident engine: autotune, graph capture,
    warm-up, K device-timed steps (L2 flushed between them), the end-to-end
    public call with host buffers, the roofline of the relax kernel.  Returns
    the JSON line (without the plain-form and CPU legs) and the objects the
    caller may still need."""
    import torch

    import mrcuda
    from mrcuda.dist import max_over_ranks
    from mrcuda.workloads import pin_boards

    steps = args.steps if steps is None else steps
    wl = _workload(name, rank, nets)
    boards = [eng.board(b.grid, b.x, b.y, b.vias, b.directed) for b in wl.boards]
    if len(boards) == 1:
        batch = mrcuda.Batch(boards[0], wl.nets, wl.windows, retry_full=True, time_kernels=True)
    else:
        batch = mrcuda.Batch(boards, wl.nets, wl.windows, retry_full=True, time_kernels=True, net_board=wl.net_board)
    # setup, outside the timed region: tile autotune, then capture the launch sequence as a graph
    if args.config and main:
        cfg = [int(v) for v in args.config.split(",")]
        batch.set_config(cfg[0], cfg[1])
        if len(cfg) > 2:
            batch.set_schedule(cfg[2])
        tuned = dict(batch.config(), forced=True)
    else:
        tuned = batch.autotune() if not args.no_autotune else None
    if not args.no_graph:
        batch.capture_graph()
    stream = torch.cuda.Stream()
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")

    # warm-up (also checks that the batch completes without any status error)
    first = None
    for _ in range(max(args.warmup, 1)):
        batch.launch(stream.cuda_stream)
        stream.synchronize()
        if first is None:
            first = batch.finish()
    path_cells = sum(len(p) for p in first.paths if p)
    routed = sum(p is not None for p in first.paths)

    # timed region: barrier + synchronize on both sides, per-step CUDA events
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    step_ms, relax_ms = [], []
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        batch.launch(stream.cuda_stream)
        e.record(stream)
        stream.synchronize()
        step_ms.append(s.elapsed_time(e))
        relax_ms.append(batch.relax_ms())
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    work = batch.stats()
    ms = statistics.fmean(step_ms)
    ms_max = max_over_ranks(ms, device="cuda")
    value = len(wl.nets) * world / (ms_max / 1000.0)

    # end to end through the public call with host buffers: first the caller's
    # ordinary (pageable) arrays, then the same boards in page-locked memory
    e2e_steps = max(1, min(steps, 5))

    def e2e_time():
        wl.route(eng)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            res = wl.route(eng)
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / e2e_steps, res

    e2e_pageable_s, res_pageable = e2e_time()
    pin_boards(eng, wl.boards)
    e2e_s, res = e2e_time()
    out_paths = res.paths  # lists built after the timed calls, for the checks below
    assert res_pageable.paths == out_paths, "page-locked inputs changed the answer"
    e2e_value = len(wl.nets) * world / max_over_ranks(e2e_s, device="cuda")
    e2e_pageable = len(wl.nets) * world / max_over_ranks(e2e_pageable_s, device="cuda")
    h2d = wl.h2d_bytes()
    d2h = int(res.offsets.nbytes + res.costs.nbytes + res.cells.nbytes) + 4  # + the status word
    assert out_paths == first.paths, "end-to-end call disagrees with the resident batch"

    # roofline of the dominant kernel (the relax kernel)
    peak, peak_kind = _peaks()
    alg_bytes = wl.algorithmic_bytes() + 4 * path_cells
    relax_avg = statistics.fmean(relax_ms) if relax_ms and min(relax_ms) > 0 else ms
    achieved = alg_bytes / (relax_avg / 1000.0) / 1e9
    sched = batch.config()
    kname = {0: "relax_rounds_kernel", 1: "relax_async_kernel", 2: "relax_warp_kernel",
             3: "relax_async_kernel"}[sched["schedule"]]
    # the queue kernel's third template argument: step prices staged from the price planes by TMA
    kfull = {0: f"relax_rounds_kernel<{sched['tile_h']},{sched['threads']}>",
             1: f"relax_async_kernel<{sched['tile_h']},{sched['threads']},true>",
             2: "relax_warp_kernel",
             3: f"relax_async_kernel<{sched['tile_h']},{sched['threads']},false>"}[sched["schedule"]]
    # DRAM bytes and instruction counts of one launch, from the ncu capture of this kernel and workload
    prof = _profile_figures(kfull.split("<")[0] + ("_tma" if sched["schedule"] == 1 else ""), name)
    acts = max(work["activations"], 1)
    counters = {"tile_activations": work["activations"], "tiles": work["tiles"],
                "activations_per_tile": work["activations"] / max(work["tiles"], 1),
                "passes_per_activation" if sched["schedule"] == 2 else "sweeps_per_activation": work["sweeps"] / acts,
                "in_tile_sweeps": work["sweeps"]}
    if sched["schedule"] == 2:
        counters["rows_per_activation"] = work["rows"] / acts
    else:
        counters["rounds"] = work["rounds"]

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": wl.meta["workload"], "nets_per_rank": len(wl.nets), "window_cells": wl.window_cells(),
                   "routed": routed, "retried": first.retried, "l2": "flushed between steps (512 MiB write)",
                   "windows": wl.meta.get("windows"), "autotuned": tuned, "graph": not args.no_graph,
                   "instances": len(wl.boards)},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "inputs": "page-locked host arrays", "outputs": "CSR arrays (offsets, cells, costs)",
                "pageable_value": e2e_pageable,
                "vs_device_value": e2e_value / value},
        "gpu_launches": batch.kernel_launches * steps,
        "roofline": dict({"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                          "traffic": None if prof is None else prof.get("dram_bytes_per_launch"),
                          "peak_kind": peak_kind, "kernel": kfull, "kernel_ms": relax_avg,
                          "algorithmic_bytes_per_launch": int(alg_bytes),
                          "bytes_per_cell": round(wl.bytes_per_cell(), 3)}, **counters),
        "clocks": clk,
    }
    if prof is not None:
        # what does bind the kernel: instruction issue (ncu, the same kernel and workload)
        line["roofline"]["issue"] = {k: prof[k] for k in ("ipc_per_sm", "inst_per_cell", "capture") if k in prof}
    return line, wl, batch, boards, first


def _summary(line):
    """The compact form of a workload's line inside `workloads`."""
    out = {"workload": line["config"]["workload"], "value": line["value"], "unit": line["unit"],
           "ms_per_step": line["ms_per_step"], "e2e": line["e2e"]["value"], "clocks": line.get("clocks")}
    r = line.get("roofline")
    if r:
        out["roofline"] = {k: r[k] for k in ("kernel", "kernel_ms", "achieved", "frac", "traffic",
                                             "activations_per_tile", "passes_per_activation",
                                             "sweeps_per_activation", "rows_per_activation") if k in r}
    if "cpu_baseline" in line:
        out["cpu_baseline"] = line["cpu_baseline"]["value"]
    return out


def other_workloads(args, eng, local):
    """The configurations beside the headline one, measured in the same
    invocation on the same GPU: the plain board (config 1), 4096 uneven
    instances in one launch (config 3), snapshot negotiation rounds (config 4)
    and the serving loop (config 5)."""
    out = {}
    for name in ("plain", "uneven"):
        line, _, batch, boards, _ = measure_batch(args, name, eng, 0, 1, local, None, steps=min(args.steps, 10),
                                                  main=False)
        out[name] = _summary(line)
        batch.close()
        for b in boards:
            b.close()
    line = measure_snapshot(args, eng, local, rounds=3, warmup=2, cpu=False)
    out["snapshot"] = _summary(line)
    out["snapshot"]["per_round"] = line["config"]["per_round"]
    rows, clk = measure_serving(args, eng, local, rates=[20.0, 100.0, 400.0], seconds=2.0, max_requests=400,
                                repeats=3)
    out["serving"] = {"workload": "serving, Poisson arrivals (3 rates, 2 s of arrivals each, 3 draws per rate)",
                      "rates": rows, "clocks": clk}
    return out


def run_engine(args):
    import torch

    import mrcuda

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    from mrcuda.dist import init_from_env

    dist = init_from_env("nccl", timeout_s=120.0, device=torch.device("cuda", local))
    eng = mrcuda.Engine(local)
    line, wl, batch, boards, first = measure_batch(args, args.workload, eng, rank, world, local, dist,
                                                   nets=args.nets)
    value = line["value"]

    if rank == 0 and world == 1 and not args.no_plain:
        ps = min(args.plain_sample or (64 if len(wl.boards) > 1 else 8), len(wl.nets))
        t0 = time.perf_counter()
        if len(wl.boards) == 1:
            req = wl.boards[0].request()
            sub = mrcuda.IsolatedRouteRequest(req.grid, req.nets[:ps], req.windows[:ps], req.x_edge_costs,
                                              req.y_edge_costs, req.via_edge_costs, req.directed_in_costs)
            pl_paths = eng.route_isolated_plain(sub).paths
        else:
            pl_paths = [p for b in wl.boards[:ps] for p in eng.route_isolated_plain(b.request()).paths]
        dt = time.perf_counter() - t0
        assert pl_paths == first.paths[:ps], "plain form disagrees with the batched engine"
        line["plain"] = {"value": ps / dt, "unit": UNIT, "sample": f"first {ps} nets, one net per launch sequence"}
        line["vs_plain"] = value / (ps / dt)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # p50 of 7 warm runs on all host threads, and the same single-threaded on
        # a smaller sample (the reference's rayon batch and its LeeRouter loop),
        # for the targeted search (paths) and for complete fields (h = 0)
        n_sample = min(args.cpu_sample or (2048 if len(wl.boards) > 1 else 128), len(wl.nets))
        n_one = max(1, n_sample // 8)
        cores = os.cpu_count() or 1

        def timed(mode):
            _cpu_sample_rate(wl, max(n_sample // 4, 1), mode=mode)
            runs = [_cpu_sample_rate(wl, n_sample, mode=mode) for _ in range(7)]
            one = statistics.median(_cpu_sample_rate(wl, n_one, threads=1, mode=mode)[0] for _ in range(7))
            return statistics.median(r for r, _ in runs), sum(d for _, d in runs), one

        rate, secs, one = timed("astar")
        f_rate, f_secs, f_one = timed("field")
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": f"{n_sample} of {len(wl.nets)} nets, A* alone-path search (window, then "
                                          f"full board), {cores} host threads, p50 of 7 warm runs "
                                          f"({secs:.2f} s in all)",
                                "single_thread": {"value": one, "unit": UNIT,
                                                  "sample": f"{n_one} nets, 1 thread, p50 of 7 warm runs"},
                                "fields": {"value": f_rate, "unit": UNIT, "cores": cores,
                                           "sample": f"{n_sample} nets, complete window field (h = 0 Dijkstra, "
                                                     f"every window cell settled) + canonical path, {cores} host "
                                                     f"threads, p50 of 7 warm runs ({f_secs:.2f} s in all)",
                                           "single_thread": {"value": f_one, "unit": UNIT,
                                                             "sample": f"{n_one} nets, 1 thread, p50 of 7"}}}
    batch.close()
    for b in boards:
        b.close()
    if rank == 0 and world == 1 and not args.no_workloads and args.workload == "congestion":
        line["workloads"] = other_workloads(args, eng, local)
    if rank == 0:
        print(json.dumps(line))
    eng.close()
    if dist:
        dist.destroy_process_group()
    return 0


def run_snapshot(args):
    """Snapshot negotiation: one step = one round (rip-up, price snapshot, route
    the dirty nets, merge, history); `value` = nets routed per second of device
    timeline over the timed rounds; `e2e` = the same through the public calls
    with host buffers, board upload and path download included."""
    import torch

    import mrcuda
    from mrcuda import workloads as W

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1 or args.shards:
        if args.groups:
            raise SystemExit("--groups: connection groups need every path, so they do not run sharded")
        return run_snapshot_sharded(args, rank, world, local)
    eng = mrcuda.Engine(local)
    line = measure_snapshot(args, eng, local, rounds=args.steps, warmup=max(args.warmup, 3),
                            cpu=not args.no_cpu_baseline)
    print(json.dumps(line))
    eng.close()
    return 0


def measure_snapshot(args, eng, local, rounds, warmup, cpu):
    """Snapshot negotiation rounds from a fresh start on the 2048x2048x6 board:
    `rounds` timed rounds (fewer if it converges) after `warmup` rounds of a
    separate negotiation.  Returns the JSON line."""
    import torch

    import mrcuda
    from mrcuda import workloads as W

    wl = W.snapshot_board(n_nets=args.nets or 3000)
    groups = None
    if args.groups:
        # nets renamed into '#'-sibling connection groups of args.groups nets
        wl.nets = [mrcuda.NetEndpoints(f"s{i // args.groups}#{i % args.groups}", nt.src, nt.dst,
                                       nt.passable_pads, nt.via_passable_pads) for i, nt in enumerate(wl.nets)]
        groups = "connections"
    req = wl.request()
    clear = dict(clearance=args.clearance, via_keepout=args.via_keepout)
    warm = eng.negotiation(req, groups=groups, **clear)
    for _ in range(warmup):
        warm.round()
    warm.close()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()
    neg = eng.negotiation(req, groups=groups, **clear)
    n_rounds = rounds
    rounds = []
    for _ in range(n_rounds):
        st = neg.round()
        if not st["dirty"]:
            break
        rounds.append(st)
    paths = neg.paths()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    routed = sum(r["dirty"] for r in rounds)
    dev_ms = sum(r["round_ms"] for r in rounds)
    cells = sum(r["window_cells"] for r in rounds)
    peak, peak_kind = _peaks()
    alg = cells * (wl.bytes_per_cell()) + 4 * sum(len(p) for p in paths if p)
    achieved = alg / (dev_ms / 1000.0) / 1e9
    n = len(wl.grid.dims)
    h2d = wl.grid.cost.nbytes + wl.directed.nbytes + 40 * len(wl.nets) + 16 * len(wl.windows)
    line = {
        "metric": METRIC, "value": routed / (dev_ms / 1000.0), "unit": UNIT, "n_gpus": 1, "steps": len(rounds),
        "warmup": warmup, "ms_per_step": dev_ms / max(len(rounds), 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": wl.meta["workload"], "rounds": len(rounds), "nets_routed": routed,
                   "groups": (f"connection groups: '#'-siblings of {args.groups} nets, plus shared endpoints"
                              if args.groups else "every net its own group"),
                   "clearance": ({"radius_cells": args.clearance, "via_keepout_cells": args.via_keepout,
                                  "rounds": "every net every round, own copper and footprint subtracted"}
                                 if args.clearance or args.via_keepout else None),
                   "window_cells": cells, "l2": "inputs larger than L2 (25M-cell board, 400 MB price planes)",
                   "per_round": [{k: r[k] for k in ("round", "dirty", "routed", "retried", "overused_edges",
                                                     "round_ms")} for r in rounds]},
        "e2e": {"value": routed / wall, "unit": UNIT, "h2d_bytes_per_step": int(h2d / max(len(rounds), 1)),
                "d2h_bytes_per_step": int(4 * sum(len(p) for p in paths if p) / max(len(rounds), 1))},
        "gpu_launches": None,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": peak_kind, "kernel": "whole round (relax + price + merge)",
                     "algorithmic_bytes": int(alg), "bytes_per_cell": wl.bytes_per_cell()},
        "clocks": clk,
    }
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc

        ns = min(args.cpu_sample or 48, len(wl.nets))
        sub = mrcuda.IsolatedRouteRequest(req.grid, req.nets[:ns], req.windows[:ns], req.x_edge_costs,
                                          req.y_edge_costs, req.via_edge_costs, req.directed_in_costs)
        t1 = time.perf_counter()
        orc.get().isolated_batch(sub, retry_full=True, mode="astar")
        dt = time.perf_counter() - t1
        cores = os.cpu_count() or 1
        line["cpu_baseline"] = {"value": ns / dt, "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": f"{ns} nets of round 0 (snapshot = base prices), search with h = 0 "
                                          f"(directed prices), {cores} host threads, {dt:.2f} s"}
    # gpu launches: per round 4 negotiation kernels + the batch sequence (+ a retry batch)
    # with a clearance: the footprint kernels (old out, new in), the override emit and pricing kernels
    line["gpu_launches"] = sum(4 + 4 + (4 if r["retried"] else 0) + (1 if groups else 0)
                               + (4 if args.clearance or args.via_keepout else 0) for r in rounds)
    neg.close()
    return line


def _run_trace(eng, trace, slots, max_batch, boards):
    """Replays a Poisson trace through a server against the resident pool
    boards; returns (latencies ms, nets, makespan s, server stats).  Arrivals
    are submitted on their own thread at their trace times; latency is the
    server's submit -> result-on-host time."""
    import threading

    srv = eng.server(slots=slots, max_batch_requests=max_batch, max_batch_cells=64 << 20)
    for _, wl in trace[:3]:  # warm-up
        srv.wait(srv.submit_resident(boards[wl.meta["board_index"]], wl.nets, wl.windows))
    reqs = [(t, wl) for t, wl in trace]
    tickets = [None] * len(reqs)
    ready = threading.Semaphore(0)
    t0 = time.perf_counter()

    def submitter():
        for i, (t, wl) in enumerate(reqs):
            d = t0 + t - time.perf_counter()
            if d > 0:
                time.sleep(d)
            tickets[i] = srv.submit_resident(boards[wl.meta["board_index"]], wl.nets, wl.windows)
            ready.release()

    th = threading.Thread(target=submitter)
    th.start()
    lat, nets = [], 0
    for i in range(len(reqs)):
        ready.acquire()
        res, info = srv.wait(tickets[i])
        lat.append(info["total_ms"])
        nets += len(res)
    makespan = time.perf_counter() - t0
    th.join()
    st = srv.stats()
    srv.close()
    return lat, nets, makespan, st


def run_snapshot_sharded(args, rank, world, local):
    """The snapshot negotiation split across ranks: rank r routes the nets
    i % world == r of the same board, and the occupancy is all-reduced (NCCL)
    between the phases of every round.  Total work is fixed (strong scaling);
    every rank runs the same rounds until no rank has a dirty net."""
    import torch

    import mrcuda
    from mrcuda import workloads as W
    from mrcuda.dist import init_from_env, max_over_ranks, sharded_negotiation_round

    dist = init_from_env("nccl", timeout_s=300.0, device=torch.device("cuda", local))
    reduce = None if dist else (lambda t: None)  # one rank: the global occupancy is its own
    wl = W.snapshot_board(n_nets=args.nets or 3000)
    req = wl.request()
    owned = [i % world == rank for i in range(len(req.nets))]
    eng = mrcuda.Engine(local)

    def total(v):
        t = torch.tensor([float(v)], dtype=torch.float64, device="cuda")
        if dist:
            dist.all_reduce(t)
        return float(t.item())

    warm = eng.negotiation(req, owned=owned)
    for _ in range(max(args.warmup, 3)):
        sharded_negotiation_round(warm, reduce)
    warm.close()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()
    shard = eng.negotiation(req, owned=owned)
    rounds = []
    for _ in range(args.steps):
        st = sharded_negotiation_round(shard, reduce)
        rounds.append(st)
        if total(st["next_dirty"]) == 0:
            break
    torch.cuda.synchronize()
    wall = max_over_ranks(time.perf_counter() - t0, device="cuda")
    clk = clocks.stop()
    routed = total(sum(r["dirty"] for r in rounds))
    if rank == 0:
        line = {
            "metric": METRIC, "value": routed / wall, "unit": UNIT, "n_gpus": world, "steps": len(rounds),
            "warmup": max(args.warmup, 3), "ms_per_step": 1000.0 * wall / max(len(rounds), 1),
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": wl.meta["workload"] + f", sharded over {world} ranks", "rounds": len(rounds),
                       "nets_routed": int(routed), "exchange": "all-reduce of the occupancy, twice per round",
                       "timing": "wall clock of the synchronised round loop, max over ranks"},
            "e2e": {"value": routed / wall, "unit": UNIT, "h2d_bytes_per_step": None, "d2h_bytes_per_step": None},
            "gpu_launches": None, "clocks": clk,
        }
        print(json.dumps(line))
    shard.close()
    eng.close()
    if dist:
        dist.destroy_process_group()
    return 0


def run_serving(args):
    """Serving: Poisson arrivals of congestion-style boards (side log-uniform
    64-1024, 2-6 layers, 16-512 nets) at several rates through the
    continuous-batching server and through a one-request-at-a-time loop (the
    same server with one launch of one request at a time)."""
    import numpy as np
    import torch

    import mrcuda
    from mrcuda import workloads as W

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if rank != 0:
        return 0
    eng = mrcuda.Engine(local)
    rates = [float(r) for r in args.rates.split(",")]
    rows, clk = measure_serving(args, eng, local, rates, args.serve_seconds, args.serve_max, args.serve_repeats)
    top = rows[-1]["batched"]
    line = {
        "metric": METRIC, "value": top["nets_per_s"], "unit": UNIT, "n_gpus": 1, "steps": len(rates),
        "warmup": 3, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic",
        "config": {"workload": "serving: Poisson arrivals, boards side log-uniform 64-1024, 2-6 layers, "
                               "16-512 nets (log-uniform), generated as the congestion board; 16 boards resident "
                               "in HBM, each request brings its own nets and windows",
                   "slots": args.slots, "hbm_budget": 0.8, "rates": rows},
        "e2e": {"value": top["nets_per_s"], "unit": UNIT, "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                "note": "every request goes through the public submit/wait calls with host buffers"},
        "p50_ms": top["p50_ms"], "p99_ms": top["p99_ms"],
        "vs_one_at_a_time": top["nets_per_s"] / max(rows[-1]["one_at_a_time"]["nets_per_s"], 1e-9),
        "clocks": clk,
    }
    print(json.dumps(line))
    eng.close()
    return 0


# request size classes by window cells (all nets, all layers): the boards span
# 64^2-1024^2 cells and 16-512 nets, so request work spans four decades
SIZE_CLASSES = (("small", 0, 4 << 20), ("medium", 4 << 20, 64 << 20), ("large", 64 << 20, 1 << 62))


def measure_serving(args, eng, local, rates, seconds, max_requests, repeats=1):
    """Each rate's Poisson trace through the continuous-batching server and
    through the one-request-at-a-time loop, `repeats` times (different
    arrival draws); latency percentiles over all repeats, overall and per
    request size class.  Returns (rows, clocks)."""
    import numpy as np

    from mrcuda import workloads as W

    pool = W.serving_pool(n_boards=16)
    boards = [eng.board(b.grid, b.x, b.y, b.vias, b.directed) for b in pool]  # device-resident grids
    rows = []
    clocks = ClockSampler(local)
    clocks.start()

    def pct(v, q):
        return float(np.percentile(v, q)) if len(v) else None

    # warm-up, unmeasured: one short trace through each loop (first-use costs of
    # the process: kernel modules, the engine's memory pool)
    warm = W.serving_trace(pool, rates[0], 20, seed=999)
    _run_trace(eng, warm, args.slots, 64, boards)
    _run_trace(eng, warm, 1, 1, boards)

    for rate in rates:
        n = max(20, min(int(rate * seconds), max_requests))
        traces = [W.serving_trace(pool, rate, n, seed=int(rate) + 1000 * r) for r in range(repeats)]
        row = {"rate_req_s": rate, "requests": n, "repeats": repeats}
        for name, slots, mb in (("batched", args.slots, 64), ("one_at_a_time", 1, 1)):
            lat, cells, runs = [], [], []
            for trace in traces:
                l, nets, span, st = _run_trace(eng, trace, slots, mb, boards)
                lat += l
                cells += [wl.window_cells() for _, wl in trace]
                runs.append({"p50_ms": pct(l, 50), "p99_ms": pct(l, 99), "nets_per_s": nets / span,
                             "req_per_s": n / span, "launches": st["launches"],
                             "largest_launch": st["largest_launch"], "peak_gb": st["peak_bytes"] / 1e9})
            lat, cells = np.array(lat), np.array(cells)
            row[name] = {"p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99),
                         # the median over the repeats of each run's own p99: one host stall in one
                         # run moves the pooled p99 above, not this one
                         "p99_ms_median_run": float(np.median([r["p99_ms"] for r in runs])),
                         "nets_per_s": float(np.mean([r["nets_per_s"] for r in runs])),
                         "req_per_s": float(np.mean([r["req_per_s"] for r in runs])),
                         "by_size": {c: {"requests": int(((cells >= lo) & (cells < hi)).sum()),
                                         "p50_ms": pct(lat[(cells >= lo) & (cells < hi)], 50),
                                         "p99_ms": pct(lat[(cells >= lo) & (cells < hi)], 99)}
                                     for c, lo, hi in SIZE_CLASSES},
                         "runs": runs}
        rows.append(row)
    clk = clocks.stop()
    for b in boards:
        b.close()
    return rows, clk


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--workload", choices=["congestion", "plain", "uneven", "snapshot", "serving"],
                    default="congestion")
    ap.add_argument("--rates", default="20,50,100,200,400", help="serving: offered request rates (req/s)")
    ap.add_argument("--serve-seconds", type=float, default=3.0, help="serving: seconds of arrivals per rate")
    ap.add_argument("--serve-max", type=int, default=600, help="serving: most requests per rate")
    ap.add_argument("--slots", type=int, default=2, help="serving: launches in flight")
    ap.add_argument("--serve-repeats", type=int, default=3, help="serving: arrival draws per rate")
    ap.add_argument("--shards", action="store_true", help="snapshot: run the sharded rounds even on one rank")
    ap.add_argument("--groups", type=int, default=0,
                    help="snapshot: group nets into '#'-sibling connection groups of this size (0 = none)")
    ap.add_argument("--clearance", type=int, default=0,
                    help="snapshot: clearance-halo rounds with this planar radius in cells (0 = off)")
    ap.add_argument("--via-keepout", type=int, default=0, help="snapshot: via keepout radius in cells")
    ap.add_argument("--nets", type=int, default=0, help="route only the first N nets (0 = all)")
    ap.add_argument("--cpu-sample", type=int, default=0, help="nets timed on the CPU (0 = workload default)")
    ap.add_argument("--plain-sample", type=int, default=0, help="nets timed one per launch (0 = workload default)")
    ap.add_argument("--no-graph", action="store_true", help="launch kernel by kernel instead of a CUDA graph")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-workloads", action="store_true",
                    help="measure only the chosen workload (by default the congestion line also carries the "
                         "plain, uneven, snapshot and serving workloads)")
    ap.add_argument("--config", default="",
                    help="force the relax tile height, CTA width and schedule (0 rounds, 1 queue, 2 warp "
                         "tiles), e.g. 8,256,1")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "snapshot":
        return run_snapshot(args)
    if args.workload == "serving":
        return run_serving(args)
    return run_engine(args)


if __name__ == "__main__":
    sys.exit(main())
