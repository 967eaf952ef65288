#!/usr/bin/env python
"""Benchmark of the Stratton-Chu field hot path on B200.

Metric: E+H cell x point evaluations per second (one evaluation = one
(observation point, cell, RHS) pair with both the K operator (E) and the R
operator (H) accumulated), mixed form (complex FP32 far cells, FP64 near
cells) at <= 1e-6 relative L2 against the FP64 form, which is itself within
1e-12 of the reference's CPU output.

Workload (one step): the refined PEC sphere, 64 x 128 = 8192 quads, k = 2 pi,
20,000 observation points (18,000 on 2-5 m shells + 2,000 near-field points
0.02-0.1 m above random cells, seed 1), one physical-optics RHS, default
quadrature (n_start 8, p_max 1): 1.64e8 pairs per step, synthetic (seeded).

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

For N > 1 (torchrun, one rank per GPU) every rank evaluates its own 20,000
points against the replicated mesh (the points are independent: no
collective on the data path), so the scaling is weak.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "E+H cell*point evals/s (mixed, <=1e-6 rel-L2 vs FP64)"
UNIT = "pairs/s"
# Algorithmic flops of one far pair with the default 8 x 8 split: 64 nodes x
# 130 real flops for the fused K (F_RotRotSimplePot_H) + R (F_GradSimplePot_H)
# integrand, transcendentals (sqrt, 1/r, sincos) not counted.
FLOPS_PER_NODE = 130
NODES_PER_PAIR = 64
FLOPS_PER_FAR_PAIR = FLOPS_PER_NODE * NODES_PER_PAIR
# Algorithmic flops of one moment contraction per (point, cell, RHS) in the
# batched kernel: (A1 I + T) J is 9 complex multiply-adds (72 flops), G x J
# three components of two complex products and a difference (42 flops).
FLOPS_PER_RHS_CONTRACTION = 114
# moments buffer of the split batched pipeline (the library's default)
SPLIT_MOMENTS_BYTES = 16 << 30


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--fp64-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU-baseline sample time")
    ap.add_argument("--no-batched", action="store_true", help="skip the 256-mesh batched leg")
    ap.add_argument("--batch-meshes", type=int, default=256)
    ap.add_argument("--no-assembly", action="store_true", help="skip the 20,480-triangle assembly leg")
    ap.add_argument("--assembly-level", type=int, default=5, help="icosphere level of the assembly leg (5: 20,480)")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-stream leg")
    ap.add_argument("--no-adaptive", action="store_true", help="skip the adaptive-quadrature (p_max = 2 and 3) leg")
    ap.add_argument("--tensor-cores", action="store_true",
                    help="mixed batches contract on the tensor cores (bielcc_ctx_set_batch_tensor_cores(ctx, 1))")
    ap.add_argument("--small", action="store_true",
                    help="reduced case for profiler captures: 2048-cell sphere x 5000 points (not a bench line)")
    ap.add_argument("--serve-requests", type=int, default=600)
    ap.add_argument("--serve-load", type=float, default=0.9, help="arrival rate / offline capacity")
    ap.add_argument("--serve-slots", type=int, default=4)
    ap.add_argument("--serve-max-batch", type=int, default=64)
    ap.add_argument("--serve-reserve-gb", type=int, default=32, help="device memory the server maps up front")
    ap.add_argument("--serve-persistent", action="store_true", help="persistent far-kernel CTAs in served batches")
    ap.add_argument("--serve-max-batch-pairs", type=float, default=1e10,
                    help="cap on a served batch's (point, cell, RHS) pairs (0: none); 1e10 is ~0.4 s of the GPU")
    ap.add_argument("--serve-asm-max-cells", type=int, default=20000,
                    help="largest mesh an assembly request draws (the config-5 mesh range)")
    ap.add_argument("--serve-asm-host-cells", type=int, default=2000,
                    help="assemblies of larger meshes write a caller-owned device matrix instead of host memory")
    ap.add_argument("--serve-overtake", action="store_true",
                    help="smaller batches overtake larger running ones on a high-priority stream "
                         "(bielcc_server_set_overtake(sv, 1)); default: every served batch at one priority")
    ap.add_argument("--serve-priority-pairs", type=float, default=0.0,
                    help="served batches of at most this many pairs run at high priority (0: none)")
    ap.add_argument("--serve-trace", default=None,
                    help="write the served batches (bielcc_server_trace) and every request's latency to this JSON file")
    ap.add_argument("--serve-p99-target-ms", type=float, default=1000.0,
                    help="stated p99 latency objective of the serving stream")
    return ap.parse_args()


def workload(small=False):
    from bielcc_b200 import workloads as W

    return W.config2(4500, 500, 32) if small else W.config2()


def dist_init(args):
    from bielcc_b200 import replicas

    ws, rank, local = replicas.env()
    replicas.init(ws, local)  # NCCL when a GPU is visible, gloo otherwise (the CPU reference arm)
    return ws, rank, local


def barrier(ws):
    from bielcc_b200 import replicas

    replicas.barrier(ws)


def max_over_ranks(ws, v, local):
    from bielcc_b200 import replicas

    return replicas.max_over_ranks(ws, v, local)


class Clocks:
    """nvidia-smi samples (200 ms) during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, text=True)
        except FileNotFoundError:
            self.p = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.p:
            self.p.terminate()
            try:
                self.out = self.p.communicate(timeout=5)[0]
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        rows = [r.split(", ") for r in getattr(self, "out", "").strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        pw = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows), "power_w_max": max(pw) if pw else None}


# ---------------------------------------------------------------- CPU legs
def cpu_sample(which, wl, target_s, threads):
    """Times the CPU path (reference build or oracle port) on a bounded sample
    of the workload's points (far and near in the workload's proportion)."""
    import oracle

    cells, J, k, pts = wl["cells"], wl["J"], wl["k"], wl["pts"]
    n_far = 18000
    # probe: 8 far + 1 near point
    probe = np.concatenate([pts[:8], pts[n_far:n_far + 1]])
    t0 = time.perf_counter()
    oracle.field_EH(cells, J, k, probe, n_threads=threads, which=which)
    dt = max(time.perf_counter() - t0, 1e-3)
    per_pt = dt / len(probe)
    m = int(max(18, min(4000, target_s / per_pt)))
    m_near = max(2, m // 10)
    sample = np.concatenate([pts[: m - m_near], pts[n_far: n_far + m_near]])
    t0 = time.perf_counter()
    oracle.field_EH(cells, J, k, sample, n_threads=threads, which=which)
    dt = time.perf_counter() - t0
    pairs = len(sample) * len(cells) * J.shape[0]
    return pairs / dt, dt, f"{len(sample)} points ({m_near} near-field) x {len(cells)} cells x {J.shape[0]} RHS"


def run_reference(args, ws, rank):
    """CPU reference arm: the reference's own CPU implementation (compiled from
    its sources into oracle/_ref) with every host thread, on bounded samples."""
    if rank != 0:
        return
    import oracle

    which = "ref" if oracle.available("ref") else "port"
    kind = "reference" if which == "ref" else "port"
    wl = workload()
    threads = os.cpu_count() or 1
    vals = []
    for _ in range(max(0, args.warmup)):
        cpu_sample(which, wl, 1.0, threads)
    t_steps = []
    sample = ""
    for _ in range(args.steps):
        v, dt, sample = cpu_sample(which, wl, 4.0, threads)
        vals.append(v)
        t_steps.append(dt)
    value = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(t_steps)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wl["name"], "cells": 8192, "points": 20000, "rhs": 1, "k": "2pi",
                       "sample_per_step": sample},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- batched leg
def run_batched(args, ctx, torch, dev, stream, flush, fp64_single_rhs_value, peak32):
    """256 meshes of uneven sizes (spheroids, rounded cubes, tori; 200-20,000
    cells log-uniform; k log-uniform in [0.5, 20]; 1-64 PO right-hand sides;
    2,000 far points each, seed 3) in one persistent launch, mixed precision,
    after autotuning the work-item size. Throughput counts (point, cell, RHS)."""
    from bielcc_b200 import workloads as W

    jobs_np = W.batch_meshes(n_meshes=args.batch_meshes, seed=3)
    keep, specs, outs = [], [], []
    geo_pairs = rhs_pairs = 0
    for j in jobs_np:
        m = ctx.mesh(j["cells"])
        S, P = j["J"].shape[0], len(j["pts"])
        Jd = torch.from_numpy(np.ascontiguousarray(j["J"])).to(dev)
        Pd = torch.from_numpy(np.ascontiguousarray(j["pts"])).to(dev)
        Ed = torch.empty((S, P, 3), dtype=torch.complex128, device=dev)
        Hd = torch.empty_like(Ed)
        keep.append((m, Jd, Pd))
        outs.append((Ed, Hd))
        specs.append(dict(mesh=m, n_rhs=S, n_pts=P, J=Jd.data_ptr(), pts=Pd.data_ptr(), E=Ed.data_ptr(),
                          H=Hd.data_ptr(), k=j["k"]))
        geo_pairs += P * len(j["cells"])
        rhs_pairs += P * len(j["cells"]) * S
    jobs = ctx.make_jobs(specs)
    sc = stream.cuda_stream
    item_cost = ctx.batch_autotune(jobs, precision="mixed", stream=sc)
    ctx.field_EH_batch(jobs, precision="mixed", stream=sc)  # warm-up
    torch.cuda.synchronize()
    ctx.stats(reset=True)
    total = 0.0
    steps = max(1, min(args.steps, 3))
    for _ in range(steps):
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rep = ctx.field_EH_batch(jobs, precision="mixed", stream=sc)
        b.record(stream)
        b.synchronize()
        total += a.elapsed_time(b)
    st = ctx.stats(reset=True)
    ms = total / steps
    est_rel_l2 = rep.est_rel_l2
    mixed = [(E.clone(), H.clone()) for E, H in outs]

    def time_batch(n, **kw):
        t = 0.0
        for _ in range(n):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            ctx.field_EH_batch(jobs, precision="mixed", stream=sc, **kw)
            b.record(stream)
            b.synchronize()
            t += a.elapsed_time(b)
        return t / n

    # the same batch without the error report (no FP64 sample), and with the
    # other form of the contraction (tensor cores <-> CUDA cores)
    ms_no_est = time_batch(steps, report=False)
    ctx.set_batch_tensor_cores(not args.tensor_cores)
    ctx.field_EH_batch(jobs, precision="mixed", stream=sc, report=False)  # warm-up of the other kernel
    ctx.stats(reset=True)
    ms_other = time_batch(max(1, min(steps, 2)), report=False)
    ctas_other = ctx.stats(reset=True)["far_ctas"]
    other = [(E.clone(), H.clone()) for E, H in outs]
    ctx.set_batch_tensor_cores(args.tensor_cores)
    # the same batch through the split pipeline (the moments of each wave of
    # work items into a device buffer, then their contraction), without the
    # error report; the library runs one-shot batches through the fused kernel
    ctx.set_batch_split(SPLIT_MOMENTS_BYTES, all_batches=True)
    ctx.field_EH_batch(jobs, precision="mixed", stream=sc, report=False)  # warm-up of the split pipeline
    ms_split = time_batch(max(1, min(steps, 2)), report=False)
    split_identical = all(bool(torch.equal(E, Ef) and torch.equal(H, Hf)) for (E, H), (Ef, Hf) in zip(mixed, outs))
    ctx.set_batch_split(SPLIT_MOMENTS_BYTES)
    # the batch planned once and replayed from its CUDA graph (fixed geometry, currents in place)
    plan = ctx.batch_plan(jobs, precision="mixed", stream=sc)
    torch.cuda.synchronize()
    plan.launch(stream=sc)  # warm-up
    g_total = 0.0
    for _ in range(steps):
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        plan.launch(stream=sc)
        b.record(stream)
        b.synchronize()
        g_total += a.elapsed_time(b)
    plan.close()
    ms_graph = g_total / steps
    kept = run_plan_moments_kept(ctx, torch, stream, flush, jobs_np, specs, outs, steps)
    # the same jobs one call at a time through the single-job path (no batching;
    # no error report, compared with the batch without its report)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    flush.zero_()
    a.record(stream)
    for sp in specs:
        ctx.field_EH_device(sp["mesh"], sp["J"], sp["k"], sp["pts"], sp["E"], sp["H"], sp["n_rhs"], sp["n_pts"],
                            precision="mixed", stream=sc, report=False)
    b.record(stream)
    b.synchronize()
    ms_seq = a.elapsed_time(b)
    # the same batch in FP64 (the plain form, batched the same way): the
    # like-for-like reference for the mixed batch's speed and error
    ctx.field_EH_batch(jobs, precision="fp64", stream=sc)  # warm-up; also the error reference
    torch.cuda.synchronize()
    ms64 = 0.0
    steps64 = max(1, min(args.steps, 2))
    for _ in range(steps64):
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ctx.field_EH_batch(jobs, precision="fp64", stream=sc)
        b.record(stream)
        b.synchronize()
        ms64 += a.elapsed_time(b)
    ms64 /= steps64
    den = 0.0
    for E6, H6 in outs:
        den += float(torch.sum(torch.abs(E6) ** 2) + torch.sum(torch.abs(H6) ** 2))
    for m, _, _ in keep:
        m.close()
    value = rhs_pairs / (ms * 1e-3)
    # Roofline of the whole launch against the measured FP32 FMA peak: 8320
    # flops per (point, cell) quadrature (the moments) plus 114 per (point,
    # cell, RHS) for the contraction on the CUDA cores. The tensor-core form
    # runs the moments on the FP32 pipe and the contraction as 2 M = 128 MMAs
    # of K = 6 and N = 2 min(16, S8 - 16 g) (S8 = S rounded up to 8) per 32-point
    # tile, cell and group of 16 RHS, three TF32 products each. Times without the
    # error report (no FP64 sample).
    ms_cc, ms_tc = (ms_other, ms_no_est) if args.tensor_cores else (ms_no_est, ms_other)
    ctas_cc, ctas_tc = (ctas_other, st["far_ctas"]) if args.tensor_cores else (st["far_ctas"], ctas_other)
    out_cc, out_tc = (other, mixed) if args.tensor_cores else (mixed, other)
    tc_flops = 0.0
    for j in jobs_np:
        S = j["J"].shape[0]
        s8 = (S + 7) // 8 * 8
        n_sum = sum(2 * min(16, s8 - 16 * g) for g in range((S + 15) // 16))
        tiles = (len(j["pts"]) + 31) // 32
        tc_flops += tiles * len(j["cells"]) * 2 * 128 * 6 * n_sum * 3 * 2
    peak_tf32 = None
    try:
        mp = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak_tf32 = mp["bf16_tflops"] / 2.0
    except Exception:
        pass
    cc_achieved = (geo_pairs * FLOPS_PER_FAR_PAIR + rhs_pairs * FLOPS_PER_RHS_CONTRACTION) / (ms_cc * 1e-3) / 1e12
    tc_moments = geo_pairs * FLOPS_PER_FAR_PAIR / (ms_tc * 1e-3) / 1e12
    tc_achieved = tc_flops / (ms_tc * 1e-3) / 1e12

    def rel_vs_fp64(outs_m):
        num = 0.0
        for (Em, Hm), (E6, H6) in zip(outs_m, outs):
            num += float(torch.sum(torch.abs(Em - E6) ** 2) + torch.sum(torch.abs(Hm - H6) ** 2))
        return (num / den) ** 0.5

    roofline = {"bound": "fp32 CUDA-core pipe (the moments and, in the default form, the contraction)",
                "kernel": "batch_far_tc_kernel (whole batch, one launch)" if args.tensor_cores
                else "batch_far_kernel<MIXED=1> (whole batch, one launch)",
                "achieved": tc_moments if args.tensor_cores else cc_achieved, "peak": peak32, "unit": "TFLOP/s",
                "frac": (tc_moments if args.tensor_cores else cc_achieved) / peak32,
                "flops": f"{FLOPS_PER_FAR_PAIR} per (point, cell) quadrature" + (
                    "" if args.tensor_cores else f" + {FLOPS_PER_RHS_CONTRACTION} per (point, cell, RHS)"),
                "peak_source": "measured FMA loop (bielcc_measure_fma_peak)"}
    forms = {"cuda_cores": {"ms": ms_cc, "ctas": ctas_cc, "rel_l2_vs_fp64": rel_vs_fp64(out_cc),
                            "achieved_tflops": cc_achieved, "frac_of_fp32_peak": cc_achieved / peak32},
             "tensor_cores": {"ms": ms_tc, "ctas": ctas_tc, "rel_l2_vs_fp64": rel_vs_fp64(out_tc),
                              "moments_tflops": tc_moments, "moments_frac_of_fp32_peak": tc_moments / peak32,
                              "tensor_tflops_issued": tc_achieved, "tensor_peak": peak_tf32,
                              "tensor_frac": tc_achieved / peak_tf32 if peak_tf32 else None,
                              "tensor_peak_source": "half the measured dense bf16 rate (MEASURED_PEAKS.json)",
                              "kernel": "batch_far_tc_kernel: tcgen05.mma kind::tf32, TF32 hi + lo, "
                                        "two 8-warp groups per CTA"},
             "tensor_core_speedup": ms_cc / ms_tc}
    return {"workload": f"{len(jobs_np)} meshes (spheroids, rounded cubes, tori), 200-20000 cells, k 0.5-20, "
                        f"1-64 PO RHS, 2000 far points each, seed 3",
            "value": value, "unit": "(point, cell, RHS) pairs/s", "geometry_pairs_per_s": geo_pairs / (ms * 1e-3),
            "ms_per_step": ms, "steps": steps, "rhs_pairs_per_step": rhs_pairs, "geometry_pairs_per_step": geo_pairs,
            "rel_l2_vs_fp64": rel_vs_fp64(mixed), "autotuned_item_cost": item_cost, "roofline": roofline,
            "fp64_ms_per_step": ms64, "fp64_value": rhs_pairs / (ms64 * 1e-3),
            "mixed_over_fp64_batched": ms64 / ms,
            "est_rel_l2_reported": est_rel_l2, "ms_without_error_report": ms_no_est,
            "contraction": "tensor cores (tcgen05 kind::tf32, TF32 hi+lo)" if args.tensor_cores else "CUDA cores",
            "contraction_forms": forms, "far_ctas": st["far_ctas"],
            "split_pipeline": {"moments_buffer_bytes": SPLIT_MOMENTS_BYTES, "ms": ms_split,
                               "fused_kernel_ms": ms_no_est, "fused_over_split": ms_no_est / ms_split,
                               "bit_identical_to_fused": split_identical},
            "over_plain_fp64_single_rhs": value / fp64_single_rhs_value,
            "sequential_single_job_ms": ms_seq, "batched_over_sequential": ms_seq / ms_no_est,
            "graph_replay_ms": ms_graph, "graph_replay_value": rhs_pairs / (ms_graph * 1e-3),
            "plan_moments_kept": kept, "gpu_launches_per_step":
                st["kernel_launches"] / steps, "near_pairs": int(rep.n_near_pairs)}


def run_plan_moments_kept(ctx, torch, stream, flush, jobs_np, specs, outs, steps):
    """The batch plan with its far moments kept in HBM: the largest prefix of
    the batched workload's jobs whose moments (80 B per (point, cell) pair, in
    blocks of 8 cells x 32 points) fit the 16 GiB buffer is planned once; each
    replay writes new currents' fields (the contraction and the finalize
    only). Timed against a fresh batch of the same jobs; the replay's result
    is checked against that fresh batch (bit-identical)."""
    block = 8 * 20 * 32 * 4
    used, n = 0, 0
    for j in jobs_np:
        tiles = (len(j["pts"]) + 31) // 32
        need = tiles * ((len(j["cells"]) + 7) // 8 + 6) * block  # + one partial block per cell range
        if used + need > SPLIT_MOMENTS_BYTES:
            break
        used += need
        n += 1
    if n == 0:
        return None
    sub = specs[:n]
    jobs = ctx.make_jobs(sub)
    sc = stream.cuda_stream
    rhs_pairs = sum(len(j["pts"]) * len(j["cells"]) * j["J"].shape[0] for j in jobs_np[:n])

    def timed(fn):
        fn()  # warm-up
        t = []
        for _ in range(steps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            t.append(a.elapsed_time(b))
        return sum(t) / len(t)

    ms_fresh = timed(lambda: ctx.field_EH_batch(jobs, precision="mixed", stream=sc, report=False))
    fresh = [(E.clone(), H.clone()) for E, H in outs[:n]]
    plan = ctx.batch_plan(jobs, precision="mixed", stream=sc)
    torch.cuda.synchronize()
    for E, H in outs[:n]:
        E.zero_()
        H.zero_()
    ms_replay = timed(lambda: plan.launch(stream=sc))
    identical = all(bool(torch.equal(E, Ef) and torch.equal(H, Hf)) for (E, H), (Ef, Hf) in zip(outs[:n], fresh))
    plan.close()
    return {"jobs": n, "moments_bytes": used, "rhs_pairs_per_step": rhs_pairs, "fresh_batch_ms": ms_fresh,
            "replay_ms": ms_replay, "replay_value": rhs_pairs / (ms_replay * 1e-3), "unit": "(point, cell, RHS) pairs/s",
            "replay_speedup": ms_fresh / ms_replay, "replay_identical_to_fresh_batch": identical,
            "what": "plan of the first jobs whose far moments fit 16 GiB; a replay contracts the kept moments "
                    "with the currents in place and finalizes"}


def run_adaptive(ctx, torch, dev, stream, flush, wl, cpu_threads):
    """Adaptive quadrature (the reference's refinement loop) on the headline
    geometry: the 8192-quad sphere, k = 2 pi, every 10th point of the headline
    set (1800 far, 200 near-field), 1 RHS, at p_max = 2 and 3 (n_start 8,
    n_start_seg 10, p_max_seg 2). With p_max = 2 a far pair's result is the pass
    at 2 n_start (table-driven far kernels at n = 16); with p_max = 3 every far
    pair's convergence test runs on the passes at 8 and 16 and the failing pairs
    take the whole loop in the refinement kernel. Near pairs take the full
    schedule. GPU FP64 and mixed are timed with CUDA events on device buffers;
    the compiled reference times a 22-point sample on the host cores, and the
    GPU's FP64 result is checked against it there."""
    import oracle
    from bielcc_b200 import abi

    cells, J, k, pts_all = wl["cells"], wl["J"], wl["k"], wl["pts"]
    pts = np.ascontiguousarray(np.concatenate([pts_all[:18000:10], pts_all[18000::10]]))
    mesh = ctx.mesh(cells)
    P, S, N = len(pts), J.shape[0], len(cells)
    Jd = torch.from_numpy(np.ascontiguousarray(J)).to(dev)
    Pd = torch.from_numpy(pts).to(dev)
    Ed = torch.empty((S, P, 3), dtype=torch.complex128, device=dev)
    Hd = torch.empty_like(Ed)
    sc = stream.cuda_stream
    which = "ref" if oracle.available("ref") else "port"
    idx = list(range(20)) + [1800, 1801]  # 20 far + 2 near-field points
    pairs = P * N * S

    def rel(a, b, c, d):
        return float(np.sqrt((np.sum(np.abs(a - c) ** 2) + np.sum(np.abs(b - d) ** 2)) /
                             (np.sum(np.abs(c) ** 2) + np.sum(np.abs(d) ** 2))))

    out = {"workload": f"sphere{N}_k2pi, {P} points (1800 far, 200 near-field), 1 RHS, n_start 8, n_start_seg 10, "
                       "p_max_seg 2", "unit": "pairs/s"}
    for p_max in (2, 3):
        npm = abi.NumParam.default(p_max=p_max, p_max_seg=2)

        def timed(prec, n):
            def call():
                ctx.field_EH_device(mesh, Jd.data_ptr(), k, Pd.data_ptr(), Ed.data_ptr(), Hd.data_ptr(), S, P,
                                    numparam=npm, precision=prec, stream=sc, report=False)
            call()  # warm-up (and the node tables)
            t = 0.0
            for _ in range(n):
                flush.zero_()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                call()
                b.record(stream)
                b.synchronize()
                t += a.elapsed_time(b)
            return t / n

        ms64 = timed("fp64", 3)
        E64, H64 = Ed.cpu().numpy(), Hd.cpu().numpy()
        msmx = timed("mixed", 3)
        Em, Hm = Ed.cpu().numpy(), Hd.cpu().numpy()
        t0 = time.perf_counter()
        Eo, Ho = oracle.field_EH(cells, J, k, pts[idx], npm, n_threads=cpu_threads, which=which)
        dt = time.perf_counter() - t0
        out[f"p_max_{p_max}"] = {
            "value": pairs / (msmx * 1e-3), "ms": msmx, "rel_l2_vs_fp64": rel(Em, Hm, E64, H64),
            "fp64_value": pairs / (ms64 * 1e-3), "fp64_ms": ms64,
            "fp64_rel_l2_vs_cpu_reference": rel(E64[:, idx], H64[:, idx], Eo, Ho),
            "cpu_reference": {"value": len(idx) * N * S / dt, "unit": "pairs/s", "cores": cpu_threads,
                              "kind": "reference" if which == "ref" else "port",
                              "sample": f"{len(idx)} points (2 near-field) x {N} cells x {S} RHS, {dt:.1f} s"}}
    mesh.close()
    out["far_pass"] = ("p_max = 2: table-driven far kernels at n = 16 (the pass the loop returns); p_max = 3: "
                       "convergence test on the passes at 8 and 16 for every far pair, the pass at 16 where it "
                       "holds, the whole loop for the rest")
    return out


def run_assembly(args, ctx, torch, dev, stream, flush):
    """Collocation assembly of K on the perturbed icosphere (level 5, 20,480
    triangles, seed 2), k = 4 pi: the TAU2 matrix (40,960^2 complex64 entries,
    13.4 GB) with FP64 near / self entries, timed on device-resident output;
    its error is the relative L2 against the FP64 assembly (complex128) of the
    same matrix, which is timed too."""
    from bielcc_b200 import workloads as W

    wl = W.config3(args.assembly_level)
    cells, k = wl["cells"], wl["k"]
    N = len(cells)
    mesh = ctx.mesh(cells)
    n = 2 * N
    sc = stream.cuda_stream
    A = torch.empty((n, n), dtype=torch.complex64, device=dev)

    def timed(prec, out, steps):
        total, rep = 0.0, None
        for _ in range(steps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            rep = ctx.assemble_K_device(mesh, k, out.data_ptr(), c64=out.dtype == torch.complex64, precision=prec,
                                        stream=sc)
            b.record(stream)
            b.synchronize()
            total += a.elapsed_time(b)
        return total / steps, rep

    timed("mixed", A, 1)  # warm-up: node tables, workspaces
    steps = max(1, min(args.steps, 3))
    ms, rep = timed("mixed", A, steps)
    A64 = torch.empty((n, n), dtype=torch.complex128, device=dev)
    ms64, _ = timed("fp64", A64, 1)
    num = den = 0.0
    for r0 in range(0, n, 4096):
        d = A[r0:r0 + 4096].to(torch.complex128) - A64[r0:r0 + 4096]
        num += float(torch.sum(d.real ** 2 + d.imag ** 2))
        den += float(torch.sum(A64[r0:r0 + 4096].real ** 2 + A64[r0:r0 + 4096].imag ** 2))
    del A64
    torch.cuda.empty_cache()
    # the step after assembly: LU solve of this complex64 system (cuSOLVER, bielcc_solve_dense)
    b = torch.randn(n, dtype=torch.complex64, device=dev)
    a0 = torch.cuda.Event(enable_timing=True)
    a1 = torch.cuda.Event(enable_timing=True)
    a0.record(stream)
    info = ctx.solve_dense(n, 1, True, A.data_ptr(), b.data_ptr(), stream=sc)
    a1.record(stream)
    a1.synchronize()
    lu_ms = a0.elapsed_time(a1)
    del A, b
    torch.cuda.empty_cache()
    mesh.close()
    return {"workload": f"{wl['name']}: TAU2 {n}x{n} complex64, FP64 near/self entries",
            "lu_solve": {"n": n, "dtype": "c64", "ms": lu_ms, "info": info,
                         "tflops": 8.0 * n ** 3 / 3.0 / (lu_ms * 1e-3) / 1e12, "library": "cuSOLVER getrf/getrs"},
            "value": N * N / (ms * 1e-3), "unit": "(collocation point, cell) pairs/s", "ms": ms, "steps": steps,
            "fp64_ms": ms64, "mixed_over_fp64": ms64 / ms, "rel_l2_vs_fp64": (num / den) ** 0.5,
            "near_pairs": int(rep.n_near_pairs), "matrix_gb": n * n * 8 / 1e9,
            "write_gbs": n * n * 8 / (ms * 1e-3) / 1e9}


def _pct(v, q):
    """Nearest-rank percentile."""
    if not v:
        return None
    v = sorted(v)
    return v[min(len(v) - 1, max(0, int(np.ceil(q * len(v))) - 1))]


def run_serving(args, ctx, torch, dev, stream, item_cost):
    """Serving stream: Poisson arrivals of field and assembly requests over 24
    resident meshes drawn like the batched workload (seed 4); field requests
    carry 100-50,000 points (log-uniform, 10% near-field) and 1-16 PO current
    sets, complex64 E and H with FP64 near pairs; assembly requests build the
    TAU2 complex64 matrix of a mesh of the same distribution (matrices of
    meshes above --serve-asm-host-cells cells go to caller-owned device
    memory, as a solver on the GPU would take them). The same requests
    first run offline (device-resident inputs, field requests in batches of
    64 through bielcc_field_EH_batch, assembly through
    bielcc_assemble_K_device) to give the offline throughput; the stream then
    arrives at --serve-load x that rate through bielcc_server_* with host
    buffers, and its throughput, p50/p99 latency, agreement with the offline
    results and the stated objective (p99 <= --serve-p99-target-ms while
    serving >= 0.8 x the offline throughput) are reported."""
    import threading

    from bielcc_b200 import abi, gpu
    from bielcc_b200 import workloads as W

    meshes, reqs = W.serving_stream(n_requests=args.serve_requests, seed=4,
                                    max_assembly_cells=args.serve_asm_max_cells)
    mh = [ctx.mesh(m["cells"]) for m in meshes]
    Jd = [torch.from_numpy(m["J"]).to(dev) for m in meshes]
    Pd = [torch.from_numpy(m["pts"]).to(dev) for m in meshes]
    field = [r for r in reqs if r["type"] == "field"]
    asm = [r for r in reqs if r["type"] == "assemble"]
    # assemblies of large meshes write a caller-owned device matrix (one per mesh,
    # shared by its requests: they write the same values), small ones host memory
    big_asm = {r["mesh"] for r in asm if mh[r["mesh"]].n_cells > args.serve_asm_host_cells}
    asm_dev = {i: torch.empty((2 * mh[i].n_cells, 2 * mh[i].n_cells), dtype=torch.complex64, device=dev)
               for i in sorted(big_asm)}
    ROWS = 128  # rows of a device-held matrix compared with the offline run
    pairs = sum(r["P"] * len(meshes[r["mesh"]]["cells"]) * r["S"] for r in field)
    sc = stream.cuda_stream
    # ---- offline
    sample = set(range(0, len(reqs), max(1, len(reqs) // 16)))
    ref = {}

    def offline(keep_ref):
        t = 0.0
        for c0 in range(0, len(reqs), 64):
            chunk = [(i, reqs[i]) for i in range(c0, min(len(reqs), c0 + 64))]
            specs, outs = [], []
            for i, r in chunk:
                if r["type"] != "field":
                    continue
                E = torch.empty((r["S"], r["P"], 3), dtype=torch.complex128, device=dev)
                H = torch.empty_like(E)
                outs.append((i, E, H))
                specs.append(dict(mesh=mh[r["mesh"]], n_rhs=r["S"], n_pts=r["P"], J=Jd[r["mesh"]].data_ptr(),
                                  pts=Pd[r["mesh"]].data_ptr(), E=E.data_ptr(), H=H.data_ptr(),
                                  k=meshes[r["mesh"]]["k"]))
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            if specs:
                ctx.field_EH_batch(ctx.make_jobs(specs), precision="mixed", stream=sc)
            for i, r in chunk:
                if r["type"] == "assemble":
                    n = 2 * mh[r["mesh"]].n_cells
                    A = asm_dev.get(r["mesh"])
                    if A is None:
                        A = torch.empty((n, n), dtype=torch.complex64, device=dev)
                    ctx.assemble_K_device(mh[r["mesh"]], meshes[r["mesh"]]["k"], A.data_ptr(), c64=True,
                                          precision="mixed", stream=sc)
                    if keep_ref and i in sample:
                        outs.append((i, A[:ROWS] if r["mesh"] in asm_dev else A, None))
            b.record(stream)
            b.synchronize()
            t += a.elapsed_time(b) * 1e-3
            if keep_ref:
                for i, E, H in outs:
                    if i in sample:
                        ref[i] = (E.cpu().numpy(), None if H is None else H.cpu().numpy())
        return t

    offline(False)  # warm-up: node tables, allocations
    t_off = offline(True)
    off_pairs_per_s = pairs / t_off
    # arrival times scaled so that the whole stream arrives over t_off / load
    rate = reqs[-1]["t"] * args.serve_load / t_off  # requests/s
    # ---- serving: the clients' output buffers are allocated and touched up
    # front (a client reuses its buffers; first-touch page faults are not the
    # server's cost)
    outs = []
    for r in reqs:
        if r["type"] == "field":
            E = np.ones((r["S"], r["P"], 3), np.complex64)
            outs.append((E, np.ones_like(E)))
        elif r["mesh"] in asm_dev:
            outs.append(None)
        else:
            n = 2 * mh[r["mesh"]].n_cells
            outs.append(np.ones((n, n), np.complex64))
    sv = gpu.Server(ctx, n_slots=args.serve_slots, precision="mixed", item_cost=item_cost,
                    preemptible=not args.serve_persistent, max_batch=args.serve_max_batch,
                    reserve=(args.serve_reserve_gb << 30, 4 << 30),
                    max_batch_pairs=int(args.serve_max_batch_pairs) or None, overtake=args.serve_overtake,
                    priority_pairs=int(args.serve_priority_pairs))

    def submit_asm(i, r):
        if r["mesh"] in asm_dev:
            return sv.submit_assemble(mh[r["mesh"]], meshes[r["mesh"]]["k"], layout="tau2", out_c64=True,
                                      A_dev=asm_dev[r["mesh"]].data_ptr())
        return sv.submit_assemble(mh[r["mesh"]], meshes[r["mesh"]]["k"], layout="tau2", out_c64=True, out=outs[i])
    # a long-running server is warm: one pass over every 8th request before the timed stream
    warm = [i for i in range(0, len(reqs), 8)]
    for i in warm:
        r, m = reqs[i], meshes[reqs[i]["mesh"]]
        if r["type"] == "field":
            sv.wait(sv.submit_field(mh[r["mesh"]], m["J"][:r["S"]], m["pts"][:r["P"]], m["k"], out_c64=True,
                                    out=outs[i]))
        else:
            sv.wait(submit_asm(i, r))
    sv.stats(reset=True)
    res = [None] * len(reqs)
    tickets = [None] * len(reqs)
    ready = threading.Semaphore(0)

    def collect():
        for i in range(len(reqs)):
            ready.acquire()
            st_, lat_, out_ = sv.wait(tickets[i], timeout=600.0)
            res[i] = (st_, lat_, out_ if i in sample else None)  # keep only the compared outputs

    th = threading.Thread(target=collect)
    th.start()
    with Clocks(dev.index or 0) as clk:
        t0 = time.perf_counter()
        for i, r in enumerate(reqs):
            due = t0 + r["t"] / rate
            now = time.perf_counter()
            if due > now:
                time.sleep(due - now)
            m = meshes[r["mesh"]]
            if r["type"] == "field":
                tickets[i] = sv.submit_field(mh[r["mesh"]], m["J"][:r["S"]], m["pts"][:r["P"]], m["k"],
                                             out_c64=True, out=outs[i])
            else:
                tickets[i] = submit_asm(i, r)
            ready.release()
        th.join()
    st = sv.stats()
    if args.serve_trace:
        with open(args.serve_trace, "w") as fh:
            json.dump({"batches": sv.trace(), "rate_per_s": rate,
                       "requests": [{"request": i, "type": r["type"], "mesh": r["mesh"], "P": r.get("P"),
                                     "S": r.get("S"), "arrival_s": r["t"] / rate, "latency_ms": res[i][1]}
                                    for i, r in enumerate(reqs)]}, fh)
    sv.close()
    lat_f = [res[i][1] for i, r in enumerate(reqs) if r["type"] == "field"]
    lat_a = [res[i][1] for i, r in enumerate(reqs) if r["type"] == "assemble"]
    bad = sum(1 for x in res if x[0] != 0)
    # served complex64 results against the offline run (complex128 rounded)
    same, worst, bad_idx = 0, 0.0, []
    for i in sorted(ref):
        o = res[i][2]
        if reqs[i]["type"] == "field":
            pairs_cmp = [(o["E"], ref[i][0].astype(np.complex64)), (o["H"], ref[i][1].astype(np.complex64))]
        elif reqs[i]["mesh"] in asm_dev:
            pairs_cmp = [(asm_dev[reqs[i]["mesh"]][:ROWS].cpu().numpy(), ref[i][0])]
        else:
            pairs_cmp = [(o["A"], ref[i][0])]
        ok = all(np.array_equal(a, b) for a, b in pairs_cmp)
        same += int(ok)
        if not ok:
            bad_idx.append(i)
            worst = max(worst, max(float(np.max(np.abs(a.astype(np.complex128) - b))) /
                                   max(float(np.max(np.abs(b))), 1e-300) for a, b in pairs_cmp))
    served = pairs / st["wall_s"]
    for m in mh:
        m.close()
    asm_dev.clear()
    est = [res[i][2].get("est") for i in sorted(ref) if reqs[i]["type"] == "field" and res[i][2] is not None]
    p99 = _pct(lat_f + lat_a, 0.99)

    # the slowest requests, with their size (pairs; N^2 for an assembly) and arrival time
    def req_pairs(r):
        n = len(meshes[r["mesh"]]["cells"])
        return r["P"] * n * r["S"] if r["type"] == "field" else n * n

    slowest = [{"request": i, "type": reqs[i]["type"], "cells": len(meshes[reqs[i]["mesh"]]["cells"]),
                "points": reqs[i].get("P"), "rhs": reqs[i].get("S"), "pairs": req_pairs(reqs[i]),
                "arrival_s": round(reqs[i]["t"] / rate, 4), "latency_ms": round(res[i][1], 1)}
               for i in sorted(range(len(reqs)), key=lambda i: -res[i][1])[:8]]
    slo = {"p99_target_ms": args.serve_p99_target_ms, "p99_ms": p99, "p99_met": p99 <= args.serve_p99_target_ms,
           "throughput_target": 0.8, "served_over_offline": served / off_pairs_per_s,
           "throughput_met": served / off_pairs_per_s >= 0.8,
           "met": p99 <= args.serve_p99_target_ms and served / off_pairs_per_s >= 0.8,
           "statement": f"p99 latency <= {args.serve_p99_target_ms:.0f} ms (submission to result in the caller's "
                        f"buffer) over all requests while serving >= 0.8 x the offline batched throughput at "
                        f"{args.serve_load} x the offline rate"}
    return {
        "workload": f"{len(reqs)} requests ({len(field)} field, {len(asm)} assembly) over 24 resident meshes "
                    f"(spheroids, rounded cubes, tori, quads or triangles; 200-20000 cells; k 0.5-20; seed 4); "
                    f"field: 100-50000 points log-uniform, 1-16 PO current sets, complex64 E+H, FP64 near pairs; "
                    f"assembly: TAU2 complex64 on meshes <= {args.serve_asm_max_cells} cells (device matrices "
                    f"above {args.serve_asm_host_cells}); Poisson arrivals",
        "arrival_rate_per_s": rate, "load": args.serve_load, "slots": args.serve_slots,
        "hbm_budget_gb": st["budget"] / 2**30,
        "offline_pairs_per_s": off_pairs_per_s, "offline_s": t_off,
        "served_pairs_per_s": served, "served_wall_s": st["wall_s"],
        "served_over_offline": served / off_pairs_per_s,
        "p50_ms": _pct(lat_f + lat_a, 0.50), "p99_ms": _pct(lat_f + lat_a, 0.99),
        "field_p50_ms": _pct(lat_f, 0.50), "field_p99_ms": _pct(lat_f, 0.99),
        "assembly_p50_ms": _pct(lat_a, 0.50), "assembly_p99_ms": _pct(lat_a, 0.99),
        "max_ms": max(lat_f + lat_a), "batches": st["batches"], "max_batch": st["max_batch"],
        "priority_batches": st["priority_batches"], "peak_reserved_gb": st["peak_bytes_reserved"] / 2**30,
        "host_stage_in_s": st["stage_in_s"], "host_copy_out_s": st["copy_out_s"], "gpu_busy_s": st["gpu_busy_s"],
        "host_stage_parts_s": {k: st["stage_" + k + "_s"] for k in ("alloc", "copy", "plan", "launch")},
        "pool_mapped_gb": st["pool_mapped_bytes"] / 2**30, "pinned_gb": st["pinned_bytes"] / 2**30,
        "arrival_window_s": reqs[-1]["t"] / rate, "offered_pairs_per_s": pairs / (reqs[-1]["t"] / rate),
        "failed": bad, "sampled_identical_to_offline": f"{same}/{len(ref)}",
        "sampled_mismatch": {"requests": bad_idx, "max_diff_over_max": worst},
        "unit": "(point, cell, RHS) pairs/s", "clocks": clk.summary(), "slo": slo,
        "max_batch_pairs": args.serve_max_batch_pairs, "overtake": args.serve_overtake,
        "priority_pairs": args.serve_priority_pairs,
        "assembly_meshes": {"max_cells": args.serve_asm_max_cells, "device_output_above_cells":
                            args.serve_asm_host_cells, "largest_assembled": max([mh_n for mh_n in
                            [len(meshes[r["mesh"]]["cells"]) for r in asm]] or [0])},
        "served_est_rel_l2_max": max(est) if est else None,
        "slowest": slowest,
    }


# ---------------------------------------------------------------- GPU arm
def run_ours(args, ws, rank, local):
    import torch

    from bielcc_b200 import abi, gpu

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    wl = workload(args.small)
    cells, J, k = wl["cells"], wl["J"], wl["k"]
    pts = wl["pts"]
    if ws > 1 and rank > 0:  # each rank: its own far points, same distribution (weak scaling)
        from bielcc_b200 import replicas

        pts = replicas.rank_points(cells, rank)
    kv, e0, hs = wl["inc"]
    inc = abi.PlaneWave.make(kv, e0, hs, True, True)
    S, N, P = J.shape[0], len(cells), len(pts)
    pairs_per_step = S * N * P

    ctx = gpu.Context(local)
    if args.tensor_cores:
        ctx.set_batch_tensor_cores(True)
    mesh = ctx.mesh(cells)
    Jd = torch.from_numpy(np.ascontiguousarray(J)).to(dev)
    Pd = torch.from_numpy(np.ascontiguousarray(pts)).to(dev)
    Ed = torch.empty((S, P, 3), dtype=torch.complex128, device=dev)
    Hd = torch.empty_like(Ed)
    E64 = torch.empty_like(Ed)
    H64 = torch.empty_like(Ed)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2
    stream = torch.cuda.current_stream(dev)

    last = {}

    def step(prec, E, H, report=True):
        r = ctx.field_EH_device(mesh, Jd.data_ptr(), k, Pd.data_ptr(), E.data_ptr(), H.data_ptr(), S, P,
                                inc=inc, precision=prec, stream=stream.cuda_stream, report=report)
        if r is not None:
            last["rep"] = r

    def timed(prec, E, H, n, report=True):
        total = 0.0
        for _ in range(n):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step(prec, E, H, report)
            b.record(stream)
            b.synchronize()
            total += a.elapsed_time(b)
        return total

    # FP64 form: reference values for the error of the mixed form, and its own speed
    step("fp64", E64, H64)
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        step("mixed", Ed, Hd)
    torch.cuda.synchronize()
    barrier(ws)
    ctx.stats(reset=True)
    ctx.set_timing(True)
    with Clocks(local) as clk:
        torch.cuda.synchronize()
        t_mixed = timed("mixed", Ed, Hd, args.steps)
        torch.cuda.synchronize()
    ctx.set_timing(False)
    st = ctx.stats(reset=True)
    est_step = last["rep"].est_rel_l2
    barrier(ws)
    t_mixed = max_over_ranks(ws, t_mixed, local)
    ms_step = t_mixed / args.steps
    value = ws * pairs_per_step / (ms_step * 1e-3)
    # the same step without the error report (no FP64 sample beside it)
    t_noest = timed("mixed", Ed, Hd, max(1, min(args.steps, 5)), report=False) / max(1, min(args.steps, 5))
    ctx.stats(reset=True)

    rel = float(torch.sqrt((torch.sum(torch.abs(Ed - E64) ** 2) + torch.sum(torch.abs(Hd - H64) ** 2)) /
                           (torch.sum(torch.abs(E64) ** 2) + torch.sum(torch.abs(H64) ** 2))).item())

    # FP64 form timing (same step, FP64 far cells)
    ctx.set_timing(True)
    t64 = timed("fp64", E64, H64, args.fp64_steps)
    ctx.set_timing(False)
    st64 = ctx.stats(reset=True)
    t64 = max_over_ranks(ws, t64, local)
    value64 = ws * pairs_per_step / (t64 / args.fp64_steps * 1e-3)

    # end to end through the host-buffer C-ABI call (pinned host memory)
    Jh = torch.from_numpy(np.ascontiguousarray(J)).pin_memory().numpy()
    Ph = torch.from_numpy(np.ascontiguousarray(pts)).pin_memory().numpy()
    Eh = torch.empty((S, P, 3), dtype=torch.complex128).pin_memory().numpy()
    Hh = torch.empty((S, P, 3), dtype=torch.complex128).pin_memory().numpy()
    ctx.field_EH(mesh, Jh, k, Ph, inc=inc, precision="mixed", out=(Eh, Hh))
    barrier(ws)
    e2e_total = 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.field_EH(mesh, Jh, k, Ph, inc=inc, precision="mixed", out=(Eh, Hh))
        e2e_total += time.perf_counter() - t0
    e2e_total = max_over_ranks(ws, e2e_total, local)
    e2e_value = ws * pairs_per_step / (e2e_total / args.steps)

    # roofline of the dominant kernel (the mixed far kernel)
    peak32 = ctx.measure_fma_peak(False)
    peak64 = ctx.measure_fma_peak(True)
    far_ms = st["far_ms"] / max(1, st["far_launches"])
    far_flops = FLOPS_PER_FAR_PAIR * st["far_pairs"] / max(1, st["far_launches"])
    achieved = far_flops / (far_ms * 1e-3) / 1e12
    far64_ms = st64["far_ms"] / max(1, st64["far_launches"])
    achieved64 = FLOPS_PER_FAR_PAIR * st64["far_pairs"] / max(1, st64["far_launches"]) / (far64_ms * 1e-3) / 1e12
    # DRAM bytes per far-kernel launch: a constant read from the ncu capture
    # summarised in profiles/ (ncu does not run inside the bench)
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "far_kernel_traffic_sphere8192.md")
    if os.path.exists(tpath):
        import re

        m = re.search(r"traffic_bytes_per_launch \| (\d+)", open(tpath).read())
        traffic = int(m.group(1)) if m else None

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline and not args.small:
        import oracle

        which = "ref" if oracle.available("ref") else "port"
        threads = os.cpu_count() or 1
        v, dt, sample = cpu_sample(which, wl, args.cpu_seconds, threads)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "reference" if which == "ref" else "port",
               "sample": sample + f", {dt:.1f} s"}

    batched = None
    if not args.no_batched:
        batched = run_batched(args, ctx, torch, dev, stream, flush, value64, peak32)
    assembly = None
    if not args.no_assembly:
        assembly = run_assembly(args, ctx, torch, dev, stream, flush)
    adaptive = None
    if not args.no_adaptive and not args.small and rank == 0:
        adaptive = run_adaptive(ctx, torch, dev, stream, flush, wl, os.cpu_count() or 1)
    serving = None
    if not args.no_serving and rank == 0:
        serving = run_serving(args, ctx, torch, dev, stream, batched["autotuned_item_cost"] if batched else None)
    launches = st["kernel_launches"]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c64 far / c128 near (f32 / f64)", "data": "synthetic (seeded)",
        "config": {"workload": wl["name"], "cells": N, "points_per_gpu": P, "rhs": S, "k": "2pi",
                   "quadrature": "n_start=8, n_start_seg=10, p_max=1", "parallelism": f"replicas x{ws}",
                   "l2": "flushed (256 MB write) between timed steps"},
        "rel_l2_vs_fp64": rel,
        "est_rel_l2_reported": est_step,
        "error_report": "each timed step reports its error against FP64 on 256 sampled points (evaluated "
                        "beside the step, inside the timed region)",
        "ms_per_step_without_error_report": t_noest,
        "fp64": {"value": value64, "unit": UNIT, "ms_per_step": t64 / args.fp64_steps,
                 "roofline": {"bound": "fp64 CUDA-core pipe", "achieved": achieved64, "peak": peak64,
                              "unit": "TFLOP/s", "frac": achieved64 / peak64 if peak64 else None,
                              "peak_source": "measured FMA loop (bielcc_measure_fma_peak)"}},
        "mixed_over_fp64": value / value64,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(Jh.nbytes + Ph.nbytes),
                "d2h_bytes_per_step": int(Eh.nbytes + Hh.nbytes)},
        "roofline": {"bound": "fp32 CUDA-core pipe (no tensor-core or HBM bound: compute-only kernel)",
                     "kernel": "far_kernel<1,false,true>", "achieved": achieved, "peak": peak32, "unit": "TFLOP/s",
                     "frac": achieved / peak32 if peak32 else None, "traffic": traffic,
                     "traffic_source": "one-pass ncu capture of the same full-size launch summarised in "
                                       "profiles/far_kernel_traffic_sphere8192.md (a constant from that capture, "
                                       "not measured in this run)",
                     "algorithmic_flops_per_launch": far_flops, "far_ms_per_launch": far_ms,
                     "peak_source": "measured FMA loop (bielcc_measure_fma_peak); MEASURED_PEAKS.json has no FP32 "
                                    "CUDA-core figure"},
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "gpu_launches": launches,
        "near_pairs_per_step": int(last["rep"].n_near_pairs),
        "batched": batched,
        "assembly": assembly,
        "adaptive": adaptive,
        "serving": serving,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    mesh.close()
    ctx.close()


def main():
    args = parse()
    ws, rank, local = dist_init(args)
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        else:
            run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
