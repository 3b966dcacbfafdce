"""Benchmark of the FMM cell-interaction kernels (one JSON line on rank 0).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
                    [--workload amr_polytrope|uniform_level3|amr_binary|single_subgrid]
                    [--precision fp32_split|fp64|fp64_exact]

The default workload is the ragged AMR batch (n = 1.5 polytrope refined to
levels 3-6: multipole, P2P and P2M work items in one solve).

A step is one gravity solve's interaction work list (every work item of the
workload) through one batched launch. ``value`` = cell-interactions / s with the
pool already resident in HBM (device time, CUDA events on the launch stream,
L2 flushed between steps); ``e2e`` = the same through host buffers (pinned
H2D of the pool and work list + launch + D2H of L and L_c inside the timed
region). Under torchrun every rank solves its own copy of the workload
(independent subgrid sets, no data-path collective: weak scaling); timing is
the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from octotiger_b200 import synthetic as syn  # noqa: E402
from octotiger_b200.layout import DRHODT, RHO  # noqa: E402

METRIC = "FMM cell-interactions/s, 1 B200: batched FP32-split vs plain FP64 at ≤1e-6 err"
UNIT = "cell-interactions/s"

# Nominal FLOPs per evaluated pair, counted on the reference's templates
# (compute_kernel_templates.hpp / monopole_kernel_templates.hpp) with every
# add, mul, div and sqrt counted as one.
FLOPS_PER_PAIR = {("m2l", RHO): 406, ("m2l", DRHODT): 272, ("p2p", RHO): 12, ("p2p", DRHODT): 12,
                  ("p2m", RHO): 317, ("p2m", DRHODT): 204}

L2_FLUSH_BYTES = 256 << 20

# DRAM bytes (read + write) of one launch of the multipole-tile kernel, from
# ncu captures (dram__bytes_read.sum + dram__bytes_write.sum) of this command
# on a B200 (the fused split tiles, the FP64 tiles); the algorithmic bytes are
# the pool read once plus L and L_c written (uniform level 3: 50.3 MB + 48.2 MB).
PROFILED_TRAFFIC = {("uniform_level3", "fp32_split"): 48.6e6, ("uniform_level3", "fp64"): 57.9e6,
                    ("amr_polytrope_l6", "fp32_split"): 65.7e6, ("amr_polytrope_l6", "fp64"): 77.4e6}

# Pipe utilisation of one launch of the multipole-tile kernel from ncu --set
# full captures of this command on a B200 (percent of peak while the SMs are
# active), reported beside the nominal-FLOP fraction: the fused split tiles on
# the uniform and AMR batches, the FP64 tiles on the uniform batch.
PROFILED_PIPES = {
    ("uniform_level3", "fp32_split"): {"issue_active": 53.5, "fp64_pipe": 41.6, "fma_pipe": 26.0, "xu_pipe": 15.8,
                                       "warps_per_sm": 8.0},
    ("amr_polytrope_l6", "fp32_split"): {"issue_active": 51.6, "fp64_pipe": 40.8, "fma_pipe": 25.7, "xu_pipe": 15.8,
                                         "warps_per_sm": 8.0},
    ("uniform_level3", "fp64"): {"issue_active": 40.8, "fp64_pipe": 62.1},
}


WORKLOADS = ("uniform_level3", "amr_polytrope", "amr_binary", "single_subgrid")


def make_workload(name: str, theta: float = 0.5):
    if name == "single_subgrid":
        return syn.single_subgrid(theta=theta)
    if name == "uniform_level3":
        return syn.uniform_level(3, theta=theta)
    from octotiger_b200 import amr
    if name == "amr_polytrope":
        return amr.polytrope_batch(theta=theta)
    if name == "amr_binary":
        return amr.binary_batch(theta=theta)
    raise SystemExit(f"unknown workload {name}")


def pair_counts(batch, ctx=None) -> dict:
    """Evaluated cell-interactions of the work list, counted by the library
    (host side); the CPU leg without a GPU context counts with the oracle."""
    if ctx is not None:
        total, per_kind = ctx.count_pairs(batch.pool.is_leaf, batch.items)
    else:
        from oracle.pyoracle import Oracle
        total, per_kind = Oracle().count_pairs(batch.theta, batch.pool, batch.items)
    return {"total": total, "m2l": int(per_kind[0] + per_kind[1]), "p2p": int(per_kind[2]), "p2m": int(per_kind[3])}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
            time.sleep(0.3)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_rate(batch, solve: int, seconds: float = 10.0, nthreads: int | None = None):
    """The reference's own kernel arithmetic (oracle/_ref, SIMD lanes) on the
    host cores, repeated over the workload for about ``seconds``."""
    from oracle.pyoracle import Oracle, RefMath, ref_library_path
    nthreads = nthreads or os.cpu_count() or 1
    counts = pair_counts(batch)
    if ref_library_path() is not None:
        impl, kind = RefMath(), "reference"
        run = lambda: impl.batch(batch.theta, batch.pool, batch.items, rho=(solve == RHO), nthreads=nthreads)
        lanes = impl.simd_width()
    else:
        impl, kind = Oracle(), "port"
        run = lambda: impl.batch(batch.theta, batch.pool, batch.items, rho=(solve == RHO), nthreads=nthreads)
        lanes = 1
    run()   # warm-up
    reps, t0 = 0, time.perf_counter()
    while True:
        run()
        reps += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    rate = counts["total"] * reps / el
    sample = (f"{reps} full passes over the {batch.name} work list ({counts['total']} pairs each), "
              f"{nthreads} host threads, {lanes}-lane SIMD")
    return {"value": rate, "unit": UNIT, "cores": nthreads, "kind": kind, "sample": sample,
            "seconds": round(el, 3)}


def accuracy_report(L, Lc, Lref, Lcref) -> dict:
    """Relative errors per output group against the exact FP64 result:
    max |err| / max |ref| per component (worst component of the group) and the
    relative L2 norm of the group."""
    groups = {"potential_L0": (0, 1), "force_L1_3": (1, 4), "higher_L4_19": (4, 20)}
    out = {}
    for name, (a, b) in groups.items():
        d = (L[:, a:b] - Lref[:, a:b]).double()
        r = Lref[:, a:b].double()
        mx = (d.abs().amax(dim=(0, 2)) / r.abs().amax(dim=(0, 2)).clamp_min(1e-300)).max().item()
        l2 = (d.norm() / r.norm().clamp_min(1e-300)).item()
        out[name] = {"max_rel": mx, "l2_rel": l2}
    d = (Lc - Lcref).double()
    r = Lcref.double()
    if r.abs().max().item() > 0:
        out["L_c"] = {"max_rel": (d.abs().amax(dim=(0, 2)) / r.abs().amax(dim=(0, 2)).clamp_min(1e-300)).max().item(),
                      "l2_rel": (d.norm() / r.norm()).item()}
    return out


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reference_arm(args) -> None:
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    batch = make_workload(args.workload, args.theta)
    solve = RHO if args.gsolve == "rho" else DRHODT
    from oracle.pyoracle import Oracle, RefMath, ref_library_path
    nthreads = os.cpu_count() or 1
    counts = pair_counts(batch)
    if ref_library_path() is not None:
        impl, kind, lanes = RefMath(), "reference", None
        lanes = impl.simd_width()
    else:
        impl, kind, lanes = Oracle(), "port", 1
    run = lambda: impl.batch(batch.theta, batch.pool, batch.items, rho=(solve == RHO), nthreads=nthreads)
    for _ in range(args.warmup):
        run()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        run()
    el = time.perf_counter() - t0
    value = counts["total"] * args.steps / el
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
        "config": {"workload": batch.name, "n_subgrids": batch.pool.n, "n_items": int(len(batch.items)),
                   "pairs_per_step": counts["total"], "theta": batch.theta, "gsolve": args.gsolve},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": kind,
                         "sample": f"the full work list per step, {nthreads} host threads, {lanes}-lane SIMD "
                                   "(reference kernel templates, Kokkos host sweep order)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def gpu_arm(args) -> None:
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    from octotiger_b200.otfmm import BatchSolver, Context, measure_fma_peaks, order_work_list

    batch = make_workload(args.workload, args.theta)
    solve = RHO if args.gsolve == "rho" else DRHODT
    ctx = Context(local, batch.theta)
    counts = pair_counts(batch, ctx)
    solver = BatchSolver(ctx, batch.pool, batch.items)
    stream = torch.cuda.current_stream()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    # every precision is autotuned on this work list, then captured into a
    # CUDA graph (otfmm_plan) and replayed: the production path of a solve
    tunings, tuned, plans = {}, {}, {}

    def prepare(precision: str):
        if precision not in plans:
            tuned[precision] = solver.autotune(solve, precision, repeats=3)
            tunings[precision] = tuned[precision].as_dict()
            plans[precision] = solver.plan(solve, precision)
        return plans[precision]

    def timed_steps(precision: str, steps: int, warmup: int, graph: bool = True):
        plan = prepare(precision)
        step = plan.launch if graph else (lambda: solver.run(solve, precision))
        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        total_ms, per = 0.0, []
        for _ in range(steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            per.append(ms)
            total_ms += ms
        plan.status()
        solver.ctx.batch_status()
        return total_ms, per

    # device-resident timing of the headline precision, clocks sampled meanwhile
    prepare(args.precision)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        total_ms, per = timed_steps(args.precision, args.steps, args.warmup)
    if pg:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * counts["total"] * args.steps / (total_ms * 1e-3)
    direct_ms, _ = timed_steps(args.precision, max(3, args.steps // 2), 3, graph=False)
    direct_ms /= max(3, args.steps // 2)

    # the other precisions on the same workload (device-resident, same method)
    others = {}
    for prec in args.compare:
        if prec == args.precision:
            continue
        ms, _ = timed_steps(prec, max(3, args.steps // 2), 3)
        others[prec] = {"value": counts["total"] * max(3, args.steps // 2) / (ms * 1e-3),
                        "ms_per_step": ms / max(3, args.steps // 2)}

    # the reference's call pattern: one FP64 entry-point call per node (per
    # subgrid), round-robin over a stream pool, halos staged on the device
    # beforehand; the "plain FP64" side of the batched-split comparison
    per_subgrid = None
    if not args.no_per_subgrid:
        from octotiger_b200.otfmm import PerSubgridSolver
        plain = PerSubgridSolver(ctx, batch.pool, batch.items, n_streams=32)
        for _ in range(2):
            plain.run(solve, "fp64")
        torch.cuda.synchronize()
        reps, ms_plain = 3, 0.0
        for _ in range(reps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            plain.run(solve, "fp64")
            e1.record(stream)
            e1.synchronize()
            ms_plain += e0.elapsed_time(e1)
        ms_plain /= reps
        per_subgrid = {"value": counts["total"] / (ms_plain * 1e-3), "ms_per_step": ms_plain, "precision": "fp64",
                       "calls_per_step": plain.n_launches, "streams": 32,
                       "what": "one otfmm_m2l_soa / otfmm_p2p_soa / otfmm_p2m_soa call per node and refined "
                               "neighbour (the reference's per-node call pattern), halos pre-staged on the device"}
        del plain
        torch.cuda.empty_cache()

    # accuracy of the headline form against the exact FP64 form (bit-identical
    # to the reference arithmetic) on this workload
    accuracy = None
    if args.precision != "fp64_exact":
        solver.run(solve, "fp64_exact")
        Le, Lce = solver.L.clone(), solver.Lc.clone()
        plans[args.precision].launch()
        torch.cuda.synchronize()
        accuracy = accuracy_report(solver.L, solver.Lc, Le, Lce)

    # end to end through the library's host-buffer path: pool and work list in
    # pinned host memory, L and L_c back into pinned host memory, all copies
    # inside the timed region (otfmm_batch_host pipelines them with the kernels
    # in chunks of the pool)
    pin = {k: torch.from_numpy(getattr(batch.pool, k)).pin_memory() for k in ("M", "com", "mon", "is_leaf")}
    items_h = order_work_list(batch.items)
    items_pin = torch.from_numpy(items_h.view(np.uint8).reshape(-1).copy()).pin_memory()
    # zeroed once, as node_server::compute_fmm zeroes L before the kernels: the
    # call writes every result but leaves the leaves' L4..L19 (no kernel writes them)
    L_pin = torch.zeros(solver.L.shape, dtype=torch.float64).pin_memory()
    Lc_pin = torch.zeros(solver.Lc.shape, dtype=torch.float64).pin_memory()
    # bytes the call uploads from page-locked buffers: the moments of refined
    # subgrids, the masses of the pool chunks holding leaves (all of it unless no
    # subgrid is a leaf), the centres of mass of refined subgrids and of leaves
    # with a refined neighbour, the leaf and centre-of-mass flags, the work list
    n_ref = int((batch.pool.is_leaf == 0).sum())
    mon_bytes = pin["mon"].numel() * 8 if n_ref < batch.pool.n else 0
    needs_com = batch.pool.is_leaf == 0
    for w in batch.items:
        nb = w["neighbors"][w["neighbors"] >= 0]
        if w["kind"] == 2 and (batch.pool.is_leaf[nb] == 0).any():
            needs_com[w["subgrid"]] = True
    h2d = (n_ref * 20 * 512 * 8 + mon_bytes + int(needs_com.sum()) * 3 * 512 * 8 + 2 * batch.pool.n
           + items_pin.numel())
    n_leaf = int((batch.pool.is_leaf == 1).sum())
    # bytes it downloads: L of refined subgrids, L0..L3 of leaves, L_c where the
    # solve writes it (refined subgrids, leaves with a refined neighbour)
    d2h = L_pin.numel() * 8 - n_leaf * 16 * 512 * 8 + int(needs_com.sum()) * 3 * 512 * 8

    def e2e_step():
        ctx.batch_host(pin["M"], pin["com"], pin["mon"], pin["is_leaf"], batch.pool.n, items_pin, len(items_h),
                       L_pin, Lc_pin, solve, args.precision)

    ctx.set_tuning(tuned[args.precision])
    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    e2e_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e2e_step()
        e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
    ctx.batch_status()
    # the host results equal the resident-pool solve's (outside the timed region)
    plans[args.precision].launch(stream)
    torch.cuda.synchronize()
    leaf = torch.from_numpy(batch.pool.is_leaf == 1)
    Ld = solver.L.cpu()
    e2e_matches = bool(torch.equal(L_pin[~leaf], Ld[~leaf]) and torch.equal(L_pin[leaf, :4], Ld[leaf, :4])
                       and torch.equal(Lc_pin, solver.Lc.cpu()))
    if pg:
        t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = world * counts["total"] * args.steps / (e2e_ms * 1e-3)

    # end to end through the reference's own interfaces: the C++ drop-in adapter
    # (include/otfmm_octotiger.hpp) called once per node from all host threads,
    # as node_server::compute_fmm calls multipole_kernel_interface /
    # monopole_kernel_interface, with AoS inputs; concurrent calls aggregated
    # into batched solves (otfmm_aggregator). Wall time of a whole pass.
    e2e_adapter = None
    if not args.no_adapter:
        from octotiger_b200.otfmm import adapter_pass
        nthr = os.cpu_count() or 8
        # a batch holds up to 8,192 records; every thread keeps up to 512 calls in
        # flight (an HPX task waiting on its call's future is suspended and its
        # worker runs other nodes' tasks: a solve's calls can all be in flight)
        cap = int(min(8192, max(64, batch.pool.n)))
        La, Lca, sec = adapter_pass(ctx, batch.pool, batch.items, solve, args.precision, aggregate=True,
                                    threads=nthr, max_subgrids=cap, max_items=cap, passes=4, calls_in_flight=512)
        leaf_items = batch.items["kind"] == 2
        sub_m = batch.items["subgrid"][~leaf_items]
        sub_l = batch.items["subgrid"][leaf_items]
        adapter_matches = bool(np.array_equal(La[sub_m], Ld.numpy()[sub_m]) and
                               np.array_equal(La[sub_l, :4], Ld.numpy()[sub_l, :4]))
        # the per-node entry points have no FP32-split form: the per-call pass runs FP64
        _, _, sec1 = adapter_pass(ctx, batch.pool, batch.items, solve, "fp64_exact" if args.precision == "fp64_exact"
                                  else "fp64", aggregate=False, threads=nthr, passes=1)
        t_agg = float(np.median(sec[1:]))
        e2e_adapter = {"value": counts["total"] / t_agg, "unit": UNIT, "s_per_pass": t_agg,
                       "host_threads": nthr, "passes_timed": len(sec) - 1,
                       "what": "every node's multipole_kernel_interface / monopole_kernel_interface call through the "
                               "C++ drop-in adapter from all host threads at once (up to 512 calls in flight per "
                               "thread), AoS inputs, calls aggregated into batched solves of up to %d records, results "
                               "added into the grids' cells by the batch (wall time of a pass, first call to last "
                               "return)" % cap,
                       "matches_device_solve": adapter_matches,
                       "per_call_value": counts["total"] / float(sec1[0]), "per_call_s_per_pass": float(sec1[0]),
                       "per_call_what": "the same calls without aggregation: one host-buffer kernel call per node "
                                        "(FP64: the per-node entry points have no FP32-split form)"}

    # a whole gravity solve where the workload is a full octree (upward M2M,
    # the interaction solve replayed from its graph, downward L2L with the
    # leaves' potential and acceleration), device time per solve
    gravity = None
    levels = getattr(batch, "levels", None)
    if levels is not None and len(levels) and int(np.min(levels)) == 0:
        from octotiger_b200.tree import batch_tree
        nodes, level_start = batch_tree(batch)
        nodes_dev = torch.from_numpy(np.ascontiguousarray(nodes).view(np.uint8).reshape(-1).copy()).to(dev)
        com1 = torch.zeros((batch.pool.n, 3, 64), dtype=torch.float64, device=dev)
        G = torch.zeros((batch.pool.n, 4, 512), dtype=torch.float64, device=dev)
        plan = plans[args.precision]

        def gravity_solve(marks):
            marks[0].record(stream)
            ctx.upward(solver.dev, com1, nodes_dev, level_start, solve)
            marks[1].record(stream)
            solver.L.zero_()
            solver.Lc.zero_()
            plan.launch()
            marks[2].record(stream)
            ctx.downward(solver.dev, com1, nodes_dev, level_start, solver.L, solver.Lc, G, 1.0, True, solve)
            marks[3].record(stream)

        marks = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        for _ in range(3):
            gravity_solve(marks)
        parts = []
        for _ in range(max(3, args.steps // 2)):
            flush.zero_()
            gravity_solve(marks)
            marks[3].synchronize()
            parts.append([marks[0].elapsed_time(marks[1]), marks[1].elapsed_time(marks[2]),
                          marks[2].elapsed_time(marks[3])])
        plan.status()
        solver.ctx.batch_status()
        med = np.median(np.array(parts), axis=0)
        gravity = {"ms_per_solve": float(med.sum()), "upward_ms": float(med[0]), "interactions_ms": float(med[1]),
                   "downward_ms": float(med[2]), "n_nodes": int(len(nodes)), "levels": int(len(level_start) - 1),
                   "what": "upward M2M + interaction solve (graph) + downward L2L and leaf potential/acceleration"}

    # roofline of the dominant kernel (the multipole tiles): nominal reference
    # FLOPs of one launch / its device time (CUDA events between the launches
    # of one solve, median of 5, L2 flushed) vs the FMA issue rate measured on
    # this GPU in this run
    ctx.set_tuning(tuned[args.precision])
    kms = []
    for _ in range(5):
        flush.zero_()
        kms.append(solver.profile(solve, args.precision))
    kernel_ms = {k: float(np.median([x[k] for x in kms])) for k in kms[0]}
    flops_m2l = counts["m2l"] * FLOPS_PER_PAIR[("m2l", solve)]
    flops = sum(counts[k] * FLOPS_PER_PAIR[(k, solve)] for k in ("m2l", "p2p", "p2m"))
    achieved = flops_m2l / (kernel_ms["m2l"] * 1e-3) / 1e12
    fp64_peak, fp32_peak = measure_fma_peaks(local)
    peak = fp32_peak if args.precision == "fp32_split" else fp64_peak
    traffic = PROFILED_TRAFFIC.get((batch.name, args.precision))
    traffic_note = None if traffic else (f"no ncu capture of the {args.precision} tile kernel on the {batch.name} "
                                          "workload is recorded in PROFILED_TRAFFIC")
    roof = {"bound": "fp64_fma" if args.precision != "fp32_split" else "fp32_fma", "achieved": achieved,
            "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
            "kernel": "multipole tiles (m2l)", "flops_per_launch": flops_m2l,
            "flops_per_pair": FLOPS_PER_PAIR[("m2l", solve)], "kernel_ms": kernel_ms,
            "step_flops_per_s": flops / (total_ms / args.steps * 1e-3) / 1e12,
            "fp64_equivalent_frac": achieved / fp64_peak,
            "peak_source": "measured in this run: register-resident FMA loop (otfmm_measure_fma_peaks); "
                           "MEASURED_PEAKS.json has no FP64/FP32 figure",
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of the same kernel "
                              "on this workload (tuned variant)" if traffic else traffic_note,
            "fp64_peak_tflops": fp64_peak, "fp32_peak_tflops": fp32_peak}
    pipes = PROFILED_PIPES.get((batch.name, args.precision))
    roof["ncu_pipes_pct"] = dict(pipes, source="ncu --set full, one launch of the same kernel on this workload "
                                              "(sm__pipe_*_cycles_active, smsp__issue_active)") if pipes else None
    if not pipes:
        roof["ncu_pipes_note"] = (f"no ncu capture of the {args.precision} tile kernel on the {batch.name} workload "
                                  "is recorded in PROFILED_PIPES")
    # ncu-free pipe evidence: SM cycles per multipole pair of the tile kernel at
    # the SM clock sampled during the timed region (an FP64 M2L pair needs ~250
    # FP64-pipe instructions = ~3.9 cycles per pair and SM at 64 FP64 lanes)
    clk_summary = clk.summary()
    n_sms = torch.cuda.get_device_properties(local).multi_processor_count
    if clk_summary.get("sm_mhz") and counts["m2l"]:
        roof["tile_sm_cycles_per_pair"] = (kernel_ms["m2l"] * 1e-3 * clk_summary["sm_mhz"] * 1e6 * n_sms
                                           / counts["m2l"])

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision != "fp32_split" else "f32+f64",
        "data": "synthetic (seeded generator)",
        "config": {"workload": batch.name, "n_subgrids": batch.pool.n, "n_items": int(len(batch.items)),
                   "pairs_per_step": counts["total"], "pairs_m2l": counts["m2l"], "pairs_p2p": counts["p2p"],
                   "pairs_p2m": counts["p2m"],
                   "theta": batch.theta, "gsolve": args.gsolve, "precision": args.precision,
                   "l2": "flushed (256 MiB write) before every timed step",
                   "launch": "one CUDA graph replay per step (otfmm_plan: classify + 3 persistent kernels)",
                   "tuning": tunings.get(args.precision),
                   "parallelism": f"{world} independent replicas" if world > 1 else "1 GPU"},
        "precisions": others,
        "direct_launch_ms_per_step": direct_ms,
        "tunings": tunings,
        "per_subgrid_fp64": per_subgrid,
        "gravity_solve": gravity,
        "ratios": {"vs_batched_fp64": (value / world / others["fp64"]["value"]) if "fp64" in others else None,
                   "vs_per_subgrid_fp64": (value / world / per_subgrid["value"]) if per_subgrid else None},
        "accuracy_vs_fp64_exact": accuracy,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "matches_device_solve": e2e_matches},
        "e2e_adapter": e2e_adapter,
        "gpu_launches": 4 * args.steps,
        "roofline": roof,
        "clocks": clk_summary,
        "step_ms": [round(x, 4) for x in per],
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_reference_rate(batch, solve, seconds=args.cpu_seconds)
    if rank == 0:
        print(json.dumps(line), flush=True)
    del solver
    ctx.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def sharded_arm(args) -> None:
    """The solve partitioned over the ranks (one GPU each): Morton ranges of
    the work list, each rank's own records uploaded and the remote neighbour
    records fetched once per solve over NCCL into the rank's own memory
    (octotiger_b200.shard.sharded_problem, the function the gloo tests run),
    then the rank's batched solve replayed from its CUDA graph. Total work is
    fixed as N grows (strong scaling); time = max over ranks."""
    import datetime

    import torch
    import torch.distributed as dist

    from octotiger_b200 import shard
    from octotiger_b200.otfmm import BatchSolver, Context
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        dist.init_process_group("gloo", store=dist.HashStore(), rank=0, world_size=1)
    batch = make_workload(args.workload, args.theta)
    solve = RHO if args.gsolve == "rho" else DRHODT
    ctx = Context(local, batch.theta)
    counts = pair_counts(batch, ctx)
    dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lp = shard.sharded_problem(batch, rank, world, dist, device=dev if world > 1 else None)
    torch.cuda.synchronize()
    exch_s = time.perf_counter() - t0
    solver = BatchSolver.from_device(ctx, lp.pool, lp.items) if world > 1 else BatchSolver(ctx, lp.pool, lp.items)
    is_leaf_local = lp.pool.is_leaf.cpu().numpy() if world > 1 else lp.pool.is_leaf
    local_pairs, _ = ctx.count_pairs(is_leaf_local, lp.items)
    tuned = solver.autotune(solve, args.precision, repeats=3)
    plan = solver.plan(solve, args.precision)
    stream = torch.cuda.current_stream()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        plan.launch()
    plan.status()
    dist.barrier()
    torch.cuda.synchronize()
    total_ms = 0.0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            plan.launch()
            e1.record(stream)
            e1.synchronize()
            total_ms += e0.elapsed_time(e1)
    plan.status()
    dist.barrier()
    t = torch.tensor([total_ms, exch_s, float(local_pairs)], dtype=torch.float64, device=dev if world > 1 else "cpu")
    mx, sm = t.clone(), t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    total_ms, exch_s, pairs_sum = float(mx[0]), float(mx[1]), int(sm[2])
    value = counts["total"] * args.steps / (total_ms * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64" if args.precision != "fp32_split" else "f32+f64", "data": "synthetic (seeded generator)",
        "config": {"workload": batch.name, "n_subgrids": batch.pool.n, "pairs_per_step": counts["total"],
                   "pairs_over_ranks": pairs_sum, "theta": batch.theta, "gsolve": args.gsolve,
                   "precision": args.precision, "l2": "flushed (256 MiB write) before every timed step",
                   "parallelism": f"{world} shards (Morton ranges of the work list, remote neighbour records "
                                  "exchanged once per solve)",
                   "tuning": tuned.as_dict()},
        "exchange_s_max_over_ranks": exch_s,
        "gpu_launches": 4 * args.steps,
        "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    plan.close()
    del solver
    ctx.close()
    dist.barrier()
    dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="amr_polytrope", choices=list(WORKLOADS))
    ap.add_argument("--precision", default="fp32_split", choices=["fp32_split", "fp64", "fp64_exact"])
    ap.add_argument("--compare", nargs="*", default=["fp64", "fp64_exact"])
    ap.add_argument("--gsolve", default="rho", choices=["rho", "drhodt"])
    ap.add_argument("--theta", type=float, default=0.5, help="opening angle (>= 0.34)")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-per-subgrid", action="store_true", help="skip the per-subgrid FP64 comparison")
    ap.add_argument("--no-adapter", action="store_true", help="skip the end-to-end leg through the C++ adapter")
    ap.add_argument("--sharded", action="store_true",
                    help="partition one solve over the ranks (strong scaling) instead of one replica per rank")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.gpus != world:
        if "WORLD_SIZE" in os.environ:
            raise SystemExit(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}")
        # not under a launcher: start one process per GPU ourselves
        import socket
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
               "--master-addr=127.0.0.1", f"--master-port={port}", str(Path(__file__).resolve()), *sys.argv[1:]]
        raise SystemExit(subprocess.run(cmd).returncode)
    if args.impl == "reference":
        reference_arm(args)
    elif args.sharded:
        sharded_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
