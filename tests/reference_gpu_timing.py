"""Times the reference's own CUDA interaction kernels beside this library's
kernels on the same GPU (test infrastructure; run by hand or under a GPU job,
not collected by pytest):

    python tests/reference_gpu_timing.py [uniform_level3|amr_polytrope ...]

The reference's kernels (cuda_multipole_interactions_kernel_rho + its block
sums for refined nodes, cuda_p2p_interactions_kernel + its block sum for
leaves; oracle/build_ref_gpu.sh) run with the reference's launch shapes, one
call per node, round-robin over 32 streams like the reference's stream pool,
on halo buffers staged on the device beforehand. The same per-node pattern
with this library's FP64 entry points, and its batched solves, are timed on
the same work items. Root and P2M calls are left out of every figure (the
reference's CUDA root and P2M kernels are not driven here), so the pair counts
are those of the refined non-root nodes and of the leaves' P2P. One JSON line
per workload; device time by CUDA events, median of 5 after 2 warm-ups."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def main(names):
    import torch

    from octotiger_b200 import amr
    from octotiger_b200 import synthetic as syn
    from octotiger_b200.layout import RHO
    from octotiger_b200.otfmm import BatchSolver, Context, PerSubgridSolver
    from oracle.pyoracle import RefGpu

    make = {"uniform_level3": lambda: syn.uniform_level(3), "amr_polytrope": lambda: amr.polytrope_batch()}
    ctx = Context(0, 0.5)
    ref = RefGpu(0.5)
    dev = torch.device("cuda", 0)

    def timed(fn, reps=5):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    for name in names:
        b = make[name]()
        keep = b.items["kind"] != 1          # root items are left out (see the docstring)
        items = np.ascontiguousarray(b.items[keep])
        _, per = ctx.count_pairs(b.pool.is_leaf, items)
        pairs = int(per[0] + per[2])          # M2L (non-root) + P2P
        plain = PerSubgridSolver(ctx, b.pool, items, n_streams=32)
        ns = len(plain.streams)
        scratch_m = [torch.zeros(ref.m2l_scratch(), dtype=torch.float64, device=dev) for _ in range(ns)]
        scratch_p = [torch.zeros(ref.p2p_scratch(), dtype=torch.float64, device=dev) for _ in range(ns)]

        def fan(launch):
            main = torch.cuda.current_stream()
            start = torch.cuda.Event()
            start.record(main)
            for st in plain.streams:
                st.wait_event(start)
            launch()
            for st in plain.streams:
                ev = torch.cuda.Event()
                ev.record(st)
                main.wait_event(ev)

        def reference_calls():
            for k in range(len(plain.mpole)):
                st = plain.streams[k % ns]
                ref.m2l(plain.m_mon[k], plain.m_com[k], plain.m_M[k], scratch_m[k % ns], plain.m_L[k],
                        plain.m_Lc[k], rho=True, stream=st.cuda_stream)
            off = len(plain.mpole)
            for k, i in enumerate(plain.leaves):
                st = plain.streams[(off + k) % ns]
                ref.p2p(plain.l_mon[k], scratch_p[(off + k) % ns], plain.l_L4[k], float(items[i]["dx"]),
                        stream=st.cuda_stream)

        def library_calls():
            for k, i in enumerate(plain.mpole):
                ctx.m2l_soa(plain.m_mon[k], plain.m_M[k], plain.m_com[k], plain.m_L[k], plain.m_Lc[k], RHO, False,
                            "fp64", plain.streams[k % ns])
            off = len(plain.mpole)
            for k, i in enumerate(plain.leaves):
                ctx.p2p_soa(plain.l_mon[k], float(items[i]["dx"]), plain.l_L4[k], "fp64",
                            plain.streams[(off + k) % ns])

        t_ref = timed(lambda: fan(reference_calls))
        t_lib = timed(lambda: fan(library_calls))
        # the reference kernels' multipole results against the library's exact
        # batched form on the same items (equal to rounding: the reference sums
        # per stencil-column block, then the blocks)
        fan(reference_calls)
        torch.cuda.synchronize()
        ref_L = plain.m_L.cpu().numpy().reshape(len(plain.mpole), 20, -1)[:, :, :512]
        solver = BatchSolver(ctx, b.pool, items)
        solver.run(RHO, "fp64_exact")
        Le, _ = solver.results()
        exp = Le[items["subgrid"][plain.mpole]]
        err = float((np.abs(ref_L - exp).max(axis=(0, 2)) / np.abs(exp).max(axis=(0, 2))).max())
        batched = {}
        for prec in ("fp64", "fp32_split"):
            batched[prec] = timed(lambda: solver.run(RHO, prec))
        print(json.dumps({
            "workload": b.name, "pairs_m2l_nonroot_plus_p2p": pairs, "calls": int(len(items)), "streams": ns,
            "reference_gpu_per_node": {"ms": t_ref, "value": pairs / (t_ref * 1e-3)},
            "library_fp64_per_node": {"ms": t_lib, "value": pairs / (t_lib * 1e-3)},
            "library_batched": {p: {"ms": t, "value": pairs / (t * 1e-3)} for p, t in batched.items()},
            "reference_m2l_max_scaled_diff_vs_library_exact": err,
            "note": "root items and P2M calls left out of every figure; batched solves run the same items "
                    "(their P2M included)"}), flush=True)
        del plain, solver
        torch.cuda.empty_cache()
    ctx.close()


if __name__ == "__main__":
    main(sys.argv[1:] or ["uniform_level3", "amr_polytrope"])
