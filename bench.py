#!/usr/bin/env python
"""FoF throughput on B200: Mparticles/s on the 256^3 periodic box (default).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one pass of the hot path (ingest + images, keys, sort, cells,
befriending, groups, property sums, ownership, catalog) over the seeded
synthetic 256^3 box (16.8M particles, L = 1000 Mpc/h, FP32 positions,
10,000 Plummer clumps holding 60 % of the particles, linking parameter 0.2,
Boundarysize 10).  The headline form is FP32 pair tests with FP64 re-check of
the band; the plain FP64 form is measured on the same box and reported
beside it.  With N GPUs (torchrun) every rank runs its own box (weak
scaling; the boxes are independent domains, there is no exchange).
Before timing, the plan's autotuner picks the cell-size scale and the
dense-top threshold on the same box (--no-autotune keeps the defaults).

Other workloads: --config c1 (64^3, FP64 positions), c3 (50M-particle
lightcone with a variable linking length), c4 (64 batched boxes, 61M
particles in one run), c5 (1024^3, generated on the device); --scale
shrinks any of them.

Timing: CUDA events on the launching stream, W untimed warm-up steps, K timed
steps between barriers + synchronize; inputs (400 MB) exceed L2.
`e2e` repeats the measurement through the public API with pinned host
inputs: every step copies its inputs host->device inside the timed region
(the copy of step i + 1 is started before step i runs and overlaps it:
Plan.prefetch), runs, and reads its catalog back.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "FoF Mparticles/s at 256^3: FP32+FP64-recheck vs plain; exact groups"
UNIT = "Mparticles/s"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def make_workload(args, rank):
    from cm_halofinder_b200 import synth
    if args.config == "c2":
        return synth.config2(seed=2 + rank, scale=args.scale)
    if args.config == "c1":
        return synth.config1(seed=1 + rank, scale=args.scale)
    if args.config == "c3":
        return synth.config3(seed=3 + rank, scale=args.scale)
    if args.config == "c5":
        return synth.config5(seed=5 + rank, scale=args.scale)
    raise SystemExit(f"unknown config {args.config}")


def describe(args, w, dtype, n):
    dt = "FP32" if dtype == np.float32 else "FP64"
    if getattr(w, "varlink", None):
        tab = w.varlink["table"]
        return (f"{args.config}: lightcone, sphere of radius {w.hi[0]:.1f} Mpc/h around the "
                f"observer, N={n}, {dt} positions, {w.meta['n_clumps']} clumps, mean density "
                f"falling 3x outwards, l(r) from {tab.min():.4f} to {tab.max():.4f} on a "
                f"{w.cells}^3 grid, non-periodic, Boundarysize={w.boundary}")
    return (f"{args.config}: periodic box L={w.hi[0]:.1f} Mpc/h, N={n}, {dt} positions, "
            f"{w.meta['n_clumps']} clumps, l={w.linklength:.6f}, Boundarysize={w.boundary}")


# DRAM bytes per processed particle of the befriending launches (ncu
# dram__bytes_read.sum + dram__bytes_write.sum of the stage's six launches,
# 256^3 box at scale 1/2: 431.9 MB for 8,971,801 processed particles)
BEFRIEND_DRAM_PER_PROC = 431.88e6 / 8971801

# the launches behind each stage's CUDA-event interval
KERNELS = {
    "befriend": "befriending stage: k_befriend_dense + k_befriend_simple + 2 x k_befriend "
                "(near, far) + 2 x k_compress",
    "sort": "radix sort: k_rs_upfront + one k_rs_scatter per digit pass (4 for 34-bit keys)",
    "ingest": "k_ingest_count + 2 scans + k_ingest_emit",
}


def stage_bytes(st, pos_bytes):
    """Algorithmic bytes per stage: the data each stage must move in this
    design (processed particles npr, fine cells R, position record rec)."""
    n, npr, R = st["n_in"], st["n_proc"], st["n_cells"]
    bits = st["key_bits"]
    # passes reading 64-bit keys (the last of them writes 32-bit key words),
    # then 32-bit passes, 9-bit digits where that saves a pass
    wide = min((bits + 7) // 8, max(1, -(-(bits - 32) // 8)))
    rest = max(0, bits - 8 * wide)
    passes = wide + min((rest + 7) // 8, (rest + 8) // 9)
    rec = 16 if pos_bytes == 4 else 32
    return {
        "ingest": 2 * 3 * pos_bytes * n + npr * (8 + 4 + rec),
        "sort": npr * (8 + (wide - 1) * 24 + 20 + (passes - wide) * 16),
        "cells": npr * (4 + rec + rec + 8 + 4) + R * 12,
        "befriend": npr * rec + R * (8 + 4 + 4),
        "groups": npr * (4 + 4 + 4) + R * 12,
        "sums": npr * (4 + 4 + rec + 12),
    }


def run_ours(args):
    import torch
    from cm_halofinder_b200 import FofConfig, Plan, synth

    from cm_halofinder_b200.replicas import Replicas
    rep = Replicas("nccl")
    rank, world, local = rep.rank, rep.world, rep.local
    dev = torch.device("cuda", local)
    if args.config == "c5":
        # 1024^3: drawn on the device (host generation would take minutes)
        w = synth.config5_device(seed=5 + rank, scale=args.scale, device=local)
        pos, vel = w.pos, w.vel
        w.pos = w.vel = None
    else:
        w = make_workload(args, rank)
        pos = torch.from_numpy(w.pos).to(dev)
        vel = torch.from_numpy(w.vel).to(dev)
    n = int(pos.shape[0])
    n_all = rep.sum(n)  # particles of all ranks' boxes
    np_dtype = np.float32 if pos.dtype == torch.float32 else np.float64
    in_bytes = pos.numel() * pos.element_size() + vel.numel() * vel.element_size()
    stream = torch.cuda.current_stream(dev)

    barrier, max_ranks = rep.barrier, rep.max

    def timed(plan, steps, warmup):
        for _ in range(warmup):
            plan.run(pos, vel, out="device", stream=stream)
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        launches = 0
        e0.record(stream)
        for _ in range(steps):
            cat = plan.run(pos, vel, out="device", stream=stream)
            st = cat.stats.as_dict()
            launches += st["n_launches"]
        e1.record(stream)
        barrier()
        return max_ranks(e0.elapsed_time(e1) / steps), st, launches

    def stage_breakdown(plan):
        # one eager (non-graph) step: the library records CUDA events between
        # its stages on this stream
        plan.set_graph(False)
        cat = plan.run(pos, vel, out="device", stream=stream)
        plan.set_graph(not args.no_graph)
        return cat.stats.as_dict()["stage_ms"]

    # the chosen form; each plan is closed after its leg so that the largest
    # workload holds one plan's buffers at a time
    cfg_fast = FofConfig.from_workload(w, precision=args.precision)
    plan = Plan(cfg_fast, pos_dtype=np_dtype, device=local)
    plan.set_graph(not args.no_graph)
    tune = None
    if not args.no_autotune:
        tune = plan.autotune([cfg_fast], [pos], [vel], repeats=2, stream=stream)
    clocks = ClockSampler(local)
    for _ in range(args.warmup):
        plan.run(pos, vel, out="device", stream=stream)
    clocks.start()
    ms, st, launches = timed(plan, args.steps, 0)
    clk = clocks.stop()
    stages = stage_breakdown(plan)
    value = n_all / (ms * 1e-3) / 1e6
    cat_fast = plan.run(pos, vel, out="host", stream=stream)
    plan.close()
    cpu_boxes = None
    if args.config == "c5" and rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the reference's sample sub-domains, cut on the device while the
        # box is there (its host copy is not kept)
        cpu_boxes = subbox_sample(DeviceBox(w, pos, vel), subbox_split(n), 24)

    plain = None
    if not args.no_plain and args.precision != "fp64":
        cfg_p = FofConfig.from_workload(w, precision="fp64")
        plan_p = Plan(cfg_p, pos_dtype=np_dtype, device=local)
        plan_p.set_graph(not args.no_graph)
        if tune is not None:
            plan_p.set_tuning(tune)
        ms_p, st_p, _ = timed(plan_p, max(1, args.steps), args.warmup)
        stages_p = stage_breakdown(plan_p)
        cat_p = plan_p.run(pos, vel, out="host", stream=stream)
        plan_p.close()
        # size-independent parity at full size: the two forms give the same
        # halos (heads, member counts) and properties within 1e-6
        same = (cat_p.nhalos == cat_fast.nhalos and
                np.array_equal(cat_p.head, cat_fast.head) and
                np.array_equal(cat_p.props[:, 0], cat_fast.props[:, 0]))
        rel = 0.0
        if same and cat_p.nhalos:
            a = cat_p.props[:, 1:4].astype(np.float64)
            b = cat_fast.props[:, 1:4].astype(np.float64)
            rel = float(np.max(np.abs(a - b) / np.maximum(np.abs(a), 1e-30)))
        plain = {"value": n_all / (ms_p * 1e-3) / 1e6, "ms_per_step": ms_p,
                 "n_pair_tests": st_p["n_pair_tests"],
                 "stage_ms": {k: round(v, 4) for k, v in stages_p.items()},
                 "speedup_of_chosen_form": ms_p / ms,
                 "same_halos_as_chosen_form": bool(same), "max_rel_diff_com": rel}

    # end to end through the public API: pinned host inputs, catalog back
    pin_pos = torch.empty(tuple(pos.shape), dtype=pos.dtype, pin_memory=True)
    pin_vel = torch.empty(tuple(vel.shape), dtype=vel.dtype, pin_memory=True)
    pin_pos.copy_(pos)
    pin_vel.copy_(vel)
    if args.config == "c5":
        pos = vel = None          # the plan copies the host inputs into its own buffers
        torch.cuda.empty_cache()
    pin_pos, pin_vel = pin_pos.numpy(), pin_vel.numpy()
    plan = Plan(cfg_fast, pos_dtype=np_dtype, device=local)
    plan.set_graph(not args.no_graph)
    if tune is not None:
        plan.set_tuning(tune)
    # a second input buffer does not fit beside the 1024^3 box's workspace:
    # there the next step's copies go into the same buffer once this step
    # has read it (positions after ingest, velocities after the sums)
    if args.config == "c5":
        plan.set_input_buffers(1)

    def e2e_steps(k):
        # every step's inputs are copied from pinned host memory; the copy of
        # step i + 1 is started (prefetch) before step i runs, so that it
        # overlaps step i's work on the GPU
        nbytes = 0
        plan.prefetch(pin_pos, pin_vel, stream=stream)
        for i in range(k):
            if i + 1 < k:
                plan.prefetch(pin_pos, pin_vel, stream=stream)
            hc = plan.run(pin_pos, pin_vel, out="host", stream=stream)
            nbytes = hc.props.nbytes + hc.head.nbytes
        return nbytes

    e2e_steps(max(3, args.warmup))
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    d2h = e2e_steps(args.steps)
    e1.record(stream)
    barrier()
    plan.close()
    ms_e2e = max_ranks(e0.elapsed_time(e1) / args.steps)
    e2e = {"value": n_all / (ms_e2e * 1e-3) / 1e6, "unit": UNIT,
           "h2d_bytes_per_step": int(in_bytes), "d2h_bytes_per_step": int(d2h)}

    peak, peak_kind = peaks()
    pos_bytes = np.dtype(np_dtype).itemsize
    sb = stage_bytes(st, pos_bytes)
    dominant = max(sb, key=lambda k: stages.get(k, 0.0))
    ach = sb[dominant] / (stages[dominant] * 1e-3) / 1e9
    traffic, traffic_src = args.traffic, "--traffic" if args.traffic else None
    if traffic is None and dominant == "befriend" and args.config in ("c2", "c5"):
        # DRAM bytes of the befriending launches per processed particle, from
        # an ncu capture of the 256^3 box at scale 1/2
        traffic = int(BEFRIEND_DRAM_PER_PROC * st["n_proc"])
        traffic_src = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the stage's six "
                       "launches on the 256^3 box at scale 1/2, scaled by processed particles")
    roofline = {"bound": "hbm", "kernel": KERNELS.get(dominant, dominant),
                "achieved": round(ach, 1),
                "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                "frac": round(ach / peak, 4), "traffic": traffic, "traffic_source": traffic_src,
                "algorithmic_bytes_per_launch": int(sb[dominant]),
                "timing": "CUDA events around the stage's launches on the caller's stream, "
                          "eager step after the timed region",
                "stage_gbs": {k: round(sb[k] / (stages[k] * 1e-3) / 1e9, 1)
                              for k in sb if stages.get(k, 0) > 0}}
    if stages.get("befriend", 0) > 0:
        # the befriending stage's work rates beside its GB/s: particle-pair
        # tests (about 9 FP32 operations each) and candidate fine-cell pairs
        # (most of them ended by a union-find check, no pair test)
        sec = stages["befriend"] * 1e-3
        roofline["befriend_rates"] = {
            "pair_tests_per_s": round(st["n_pair_tests"] / sec, 1),
            "pair_test_gflops_fp32": round(9 * st["n_pair_tests"] / sec / 1e9, 2),
            "cell_pairs_per_s": round(st["n_cell_pairs"] / sec, 1),
            "root_skips_per_s": round(st["n_root_skips"] / sec, 1)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(w, args.cpu_seconds, boxes=cpu_boxes,
                           ndiv=subbox_split(n) if cpu_boxes is not None else None)
    rep.close()
    if rank != 0:
        return
    line = {
        "metric": METRIC.replace("256^3", "1024^3") if args.config == "c5" else METRIC,
        "value": round(value, 3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64-recheck" if args.precision == "fp32" else "f64",
        "data": "synthetic (seeded Plummer clumps + uniform background)",
        "config": {"workload": describe(args, w, np_dtype, n),
                   "n_particles": n, "n_processed": st["n_proc"], "n_images": st["n_images"],
                   "n_halos": st["nhalos"], "n_groups": st["n_groups"],
                   "n_fine_cells": st["n_cells"], "cell_factor": st["cell_factor"],
                   "pair_tests": st["n_pair_tests"], "rechecks": st["n_rechecks"],
                   "cell_pairs": st["n_cell_pairs"], "root_skips": st["n_root_skips"],
                   "unions": st["n_unions"], "find_steps": st["n_find_steps"],
                   "scan_iters": st["n_scan_iters"], "window_iters": st["n_window_iters"],
                   "dense_tops": st["n_dense_tops"], "queued_cells": st["n_queued"],
                   "big_tops": st["n_big_tops"], "autotune": tune,
                   "precision": args.precision, "parallelism": f"replicas x{world}",
                   "l2": f"inputs ({in_bytes / 1e6:.0f} MB) larger than L2; no flush"},
        "stage_ms": {k: round(v, 4) for k, v in stages.items()},
        "stage_ms_note": "per-stage CUDA-event times of one eager step after the timed graph replays",
        "plain_fp64": plain,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": clk,
        "e2e": e2e,
        "gpu_launches": int(launches),
    }
    print(json.dumps(line), flush=True)


def run_batched(args):
    """64 independent periodic boxes of uneven size in one batched run per
    step (one sort, one befriending pass, one reduction over all boxes),
    replayed from a captured CUDA graph, after the autotuner has picked the
    cell-size scale and the dense-top threshold."""
    import torch
    from cm_halofinder_b200 import FofConfig, Plan, synth

    from cm_halofinder_b200.replicas import Replicas
    rep = Replicas("nccl")
    rank, world, local = rep.rank, rep.world, rep.local
    boxes = synth.config4(seed=4 + 1000 * rank, scale=args.scale)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    cfgs = [FofConfig.from_workload(w, precision=args.precision) for w in boxes]
    pos = [torch.from_numpy(w.pos).to(dev) for w in boxes]
    vel = [torch.from_numpy(w.vel).to(dev) for w in boxes]
    n = sum(w.n for w in boxes)
    n_all = rep.sum(n)  # particles of all ranks' boxes

    barrier, max_ranks = rep.barrier, rep.max

    def timed(plan, steps, warmup, inputs):
        for _ in range(warmup):
            plan.run_batch(cfgs, *inputs(), stream=stream)
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        nh = 0
        for _ in range(steps):
            cats = plan.run_batch(cfgs, *inputs(), stream=stream)
            nh = sum(c.nhalos for c in cats)
        e1.record(stream)
        barrier()
        return max_ranks(e0.elapsed_time(e1) / steps), cats, nh

    resident = lambda: (pos, vel)  # noqa: E731
    plan = Plan(cfgs[0], pos_dtype=boxes[0].pos.dtype, device=local)
    plan.set_graph(not args.no_graph)
    tune = plan.autotune(cfgs, pos, vel, repeats=2, stream=stream) if not args.no_autotune else None
    clocks = ClockSampler(local)
    for _ in range(args.warmup):
        plan.run_batch(cfgs, pos, vel, stream=stream)
    clocks.start()
    ms, cats, nh = timed(plan, args.steps, 0, resident)
    clk = clocks.stop()
    st = cats[0].stats
    value = n_all / (ms * 1e-3) / 1e6

    plain = None
    if not args.no_plain and args.precision != "fp64":
        cfg_p = [FofConfig.from_workload(w, precision="fp64") for w in boxes]
        plan_p = Plan(cfg_p[0], pos_dtype=boxes[0].pos.dtype, device=local)
        plan_p.set_graph(not args.no_graph)
        if tune is not None:
            plan_p.autotune(cfg_p, pos, vel, repeats=2, stream=stream)
        for _ in range(args.warmup):
            plan_p.run_batch(cfg_p, pos, vel, stream=stream)
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(max(1, args.steps)):
            plan_p.run_batch(cfg_p, pos, vel, stream=stream)
        e1.record(stream)
        barrier()
        ms_p = max_ranks(e0.elapsed_time(e1) / max(1, args.steps))
        plain = {"value": n_all / (ms_p * 1e-3) / 1e6, "ms_per_step": ms_p,
                 "speedup_of_chosen_form": ms_p / ms}
        plan_p.close()

    # end to end: the boxes' pinned host arrays given to run_batch, which
    # copies them to the device in every step; the copy of step i + 1 is
    # started (prefetch_batch) before step i runs, so that it overlaps step
    # i's work on the GPU; catalogs read back
    hpos = [torch.from_numpy(w.pos).pin_memory().numpy() for w in boxes]
    hvel = [torch.from_numpy(w.vel).pin_memory().numpy() for w in boxes]

    def e2e_steps(k):
        plan.prefetch_batch(hpos, hvel, stream=stream)
        for i in range(k):
            if i + 1 < k:
                plan.prefetch_batch(hpos, hvel, stream=stream)
            out = plan.run_batch(cfgs, hpos, hvel, stream=stream)
        return out

    e2e_steps(max(3, args.warmup))
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    cats_e2e = e2e_steps(args.steps)
    e1.record(stream)
    barrier()
    ms_e2e = max_ranks(e0.elapsed_time(e1) / args.steps)
    d2h = sum(c.props.nbytes + c.head.nbytes for c in cats_e2e)
    e2e = {"value": n_all / (ms_e2e * 1e-3) / 1e6, "unit": UNIT,
           "h2d_bytes_per_step": int(sum(w.pos.nbytes + w.vel.nbytes for w in boxes)),
           "d2h_bytes_per_step": int(d2h)}
    rep.close()
    if rank != 0:
        return
    ns = [w.n for w in boxes]
    print(json.dumps({
        "metric": "FoF Mparticles/s, 64 batched boxes: FP32+FP64-recheck vs plain; exact groups",
        "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64-recheck" if args.precision == "fp32" else "f64",
        "data": "synthetic (seeded Plummer clumps + uniform background, per box)",
        "config": {"workload": f"c4: {len(boxes)} periodic boxes, N log-uniform in "
                               f"[{min(ns)}, {max(ns)}], total {n}, constant mean density, "
                               "b uniform in [0.15, 0.25], Boundarysize 8",
                   "n_particles": n, "n_halos": int(nh),
                   "n_processed": int(sum(c.stats["n_proc"] for c in cats)),
                   "n_fine_cells": st["n_cells"], "autotune": tune,
                   "graph": not args.no_graph, "precision": args.precision,
                   "parallelism": f"replicas x{world}",
                   "l2": f"inputs ({n * 24 / 1e9:.2f} GB) larger than L2; no flush"},
        "plain_fp64": plain, "clocks": clk, "e2e": e2e,
        "gpu_launches": int(st["n_launches"]) * args.steps,
    }), flush=True)


class DeviceBox:
    """A workload's run parameters with its particles as device tensors."""

    def __init__(self, w, pos, vel):
        self.__dict__.update({k: v for k, v in vars(w).items() if k not in ("pos", "vel")})
        self.pos, self.vel = pos, vel


def subbox_split(n):
    """Ranks per axis of the reference's domain split for a CPU sample: about
    4096 particles per rank's domain (16^3 for the 256^3 box)."""
    return max(1, int(round((n / 4096) ** (1.0 / 3.0))))


def subbox_sample(w, ndiv, count, seed=0):
    """The first `count` sub-domains of a seeded order of the ndiv^3 split."""
    from oracle import reference
    order = np.random.default_rng(seed).permutation(ndiv ** 3)
    return [reference.SubBox(w, ndiv, int(i)) for i in order[:count]]


def cpu_baseline(w, seconds, ndiv=None, timeout=None, procs=1, seed=0, boxes=None):
    """The reference's own FoF (oracle/_ref) on host cores, on sub-boxes of
    the same box (one rank's domain of an ndiv^3 decomposition each, or the
    given ones)."""
    from oracle import reference
    if not reference.available("cmh_ref_f32_timing"):
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "reference binary not built (oracle/_ref missing)"}
    if boxes is None:
        if ndiv is None:
            ndiv = subbox_split(w.n)
        order = np.random.default_rng(seed).permutation(ndiv ** 3)
    timeout = timeout or max(5.0, seconds / 2)
    done_n, spent, ok, to = 0, 0.0, 0, 0
    t_end = time.perf_counter() + seconds
    k = 0
    limit = len(boxes) if boxes is not None else len(order)
    while time.perf_counter() < t_end and k < limit:
        sb = boxes[k] if boxes is not None else reference.SubBox(w, ndiv, int(order[k]))
        k += 1
        dt, wall = reference.time_subbox(sb, timeout=min(timeout, max(1.0, t_end - time.perf_counter() + 1)))
        spent += wall
        if dt is None:
            to += 1
        else:
            ok += 1
            done_n += sb.n_owned
    value = done_n / spent / 1e6 if spent > 0 else None
    note = ""
    if getattr(w, "varlink", None):
        note = ("; the reference's variable linking length does not compile (VARLINK), so it "
                f"runs with the constant l = {w.linklength:.4f}, the table's largest value")
    return {"value": value, "unit": UNIT, "cores": procs, "kind": "reference",
            "sample": f"{ok} of {ndiv}^3 sub-box domains (one rank each, ghost shell "
                      f"{w.boundary}{'' if w.periodic else ', no periodic wrap'}) of this "
                      f"box run to completion, {to} stopped at the per-domain time limit and "
                      f"counted with zero particles; {spent:.1f} s of one core" + note}


def _ref_worker(argv):
    from oracle import reference
    w_args, index, ndiv, timeout = argv
    import pickle
    w = pickle.loads(w_args)
    sb = reference.SubBox(w, ndiv, index)
    dt, wall = reference.time_subbox(sb, timeout=timeout)
    return (sb.n_owned if dt is not None else 0), wall, dt is None


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    from oracle import reference
    if not reference.available("cmh_ref_f32_timing"):
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference binaries (oracle/_ref) were not built"}))
        return
    import multiprocessing as mp
    import pickle
    w = make_workload(args, 0)
    cores = os.cpu_count() or 1
    ndiv = subbox_split(w.n)
    order = np.random.default_rng(0).permutation(ndiv ** 3)
    blob = pickle.dumps(w)
    ctx = mp.get_context("spawn")
    per_step = cores
    timeout = args.ref_timeout
    res = []
    k = 0
    with ctx.Pool(cores) as pool:
        for step in range(args.warmup + args.steps):
            jobs = [(blob, int(order[(k + j) % len(order)]), ndiv, timeout) for j in range(per_step)]
            k += per_step
            t0 = time.perf_counter()
            out = pool.map(_ref_worker, jobs)
            dt = time.perf_counter() - t0
            if step >= args.warmup:
                res.append((sum(o[0] for o in out), dt, sum(o[2] for o in out)))
    nsum = sum(r[0] for r in res)
    tsum = sum(r[1] for r in res)
    tos = sum(r[2] for r in res)
    value = nsum / tsum / 1e6
    ms = tsum / len(res) * 1e3
    sample = (f"each step: {per_step} sub-box domains of a {ndiv}^3 decomposition of the "
              f"box, one reference process per core; {tos} of {per_step * len(res)} domains "
              f"hit the {timeout:.0f} s limit and count zero particles")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        # MEMORY_MODE: float coordinate differences, double d^2 (FOF.c:351-357)
        "dtype": "f32+f64" if w.pos.dtype == np.float32 else "f64",
        "data": "synthetic (seeded Plummer clumps + uniform background)",
        "config": {"workload": describe(args, w, w.pos.dtype, w.n),
                   "reference_run": "sampled sub-domains of the box (see cpu_baseline.sample)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-graph", action="store_true", help="issue every step eagerly")
    ap.add_argument("--no-autotune", action="store_true",
                    help="skip the autotuner (default cell-size factor and dense-top threshold)")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--ref-timeout", type=float, default=20.0)
    ap.add_argument("--traffic", type=float, default=None,
                    help="dram bytes of the dominant kernel from an ncu capture")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.config == "c4":
        run_batched(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
