#!/usr/bin/env python
"""Benchmark of the B200 rule x scenario evaluator.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one step): the evaluation of one GP generation -- 1024 rules (the
initial ramped half-and-half population of a GP run over the 29-terminal
menu, depth 2-8) on 500 stochastic scenarios of a clustered 100-customer
synthetic instance (8 Gaussian clusters, H=1000, m=3): 512,000 bit-exact
(rule, scenario) route simulations.  Synthetic data stands in for the
benchmark's own instances (the reference ships no generator).

value      : evaluations/s with rules and scenarios resident in HBM, kernel time
             by CUDA events on the launching stream, L2 flushed between steps.
e2e        : the same metric through the reference-shaped host call
             (sidr_evaluate: host rules/scenarios in, host scores out, all
             copies inside the timed region), wall clock.
roofline   : the evaluator is bound by the FP64 pipe / issue rate, not HBM or
             tensor cores; achieved = op-model FP64 operations per launch
             (counted by the kernel's counting instantiation) / kernel time,
             peak = the FP64 pipe throughput measured on this GPU; traffic =
             the launch's DRAM bytes from bench_traffic.json (an ncu capture of
             this command), used only while the kernel sources hash to the
             value recorded there.
evolved    : the same measurements on generation 49 of the benchmark GP run
             (same instance and scenarios): the populations a GP spends most of
             its generations on, several times costlier per evaluation.
cpu_baseline: the reference's CPU simulator (compiled from its own headers,
             oracle/_ref) or else the C oracle, on all host threads, on a
             bounded sample of the same workload (--full-parity: all of it),
             compared bit for bit with the GPU's scores.

Multi-GPU: pairs are independent, so each rank evaluates its own generation
(weak scaling, no collective on the data path); the timing is the maximum over
ranks of the device-timed total.
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import os
import statistics
import subprocess
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "solver-informed-dispatching-rules_b200")
sys.path.insert(0, PKG)

METRIC = "bit-exact rule×scenario evals/s"
UNIT = "evals/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--P", type=int, default=1024)
    ap.add_argument("--S", type=int, default=500)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--shape", type=int, default=-1,
                    help="block shape of the benchmark generation (index into sidr.Batch.SHAPES); "
                         "default: tuned on every 16th rule")
    ap.add_argument("--evolved-shape", type=int, default=-1, help="the same for the evolved leg")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--evolved-steps", type=int, default=3,
                    help="timed steps of the evolved-population leg (generation 49 of the "
                         "benchmark GP run on the same instance and scenarios); 0 skips it")
    ap.add_argument("--full-parity", action="store_true",
                    help="compare every (rule, scenario) pair of the workload with the CPU "
                         "simulator on all host threads, instead of a bounded sample: about "
                         "five minutes per 512,000 pairs on 16 threads")
    ap.add_argument("--gp", action="store_true",
                    help="also run the GP loop of the workload (50 generations of 1024 rules x "
                         "500 scenarios + held-out evaluation) and report its wall time")
    ap.add_argument("--gp-generations", type=int, default=50)
    ap.add_argument("--multi", action="store_true",
                    help="also time the uneven multi-instance batch (40 instances of 25-288 "
                         "customers) in one autotuned, graph-captured launch")
    ap.add_argument("--sgp", action="store_true",
                    help="also run the surrogate-assisted GP against plain GP on the benchmark "
                         "instance (population 1024, 500 training scenarios, screening 8192 "
                         "offspring per generation) and report wall clock to equal held-out fitness")
    ap.add_argument("--sgp-generations", type=int, default=50)
    ap.add_argument("--sgp-seed", type=int, default=0, help="with --sgp: the GP seed of every arm")
    ap.add_argument("--sgp-ablation", action="store_true",
                    help="with --sgp: also run the surrogate arms that change one screening "
                         "setting each (about 3 minutes per arm)")
    ap.add_argument("--campaign", action="store_true",
                    help="also time the reference campaign's c101 generation trace (30 seeds x "
                         "1024 rules x 51 generations + held-out) and its vocabulary GA's first "
                         "batch (13 genomes x 16 seeds x 51 generations), both checked against "
                         "the reference's own artefacts in tests/golden/campaign.npz")
    ap.add_argument("--multi-shape", type=int, default=-1,
                    help="with --multi: use this block shape (index into sidr.Multi.SHAPES) "
                         "instead of autotuning, e.g. at full size (--multi-rules 1000 --multi-S 500), "
                         "where each autotuning launch takes about a minute")
    ap.add_argument("--sharded", action="store_true",
                    help="instead of one independent generation per GPU, run the benchmark GP with "
                         "every generation's rules sharded over the ranks (fitness all_gather, "
                         "strong scaling): W untimed generations, then K timed ones")
    ap.add_argument("--sampling", action="store_true",
                    help="also time scenario sampling on the GPU (sidr_gen_durations_device) against "
                         "the host sampler on the benchmark's block and the large run's block")
    ap.add_argument("--large", action="store_true",
                    help="also run the large combined run's driver (sidr_sgp_run_multi): 10 instances "
                         "of 288 customers x 30 GP seeds x 4096 rules, surrogate screening 16384 "
                         "offspring per seed-generation, for --large-generations generations of "
                         "--large-S training scenarios")
    ap.add_argument("--large-S", type=int, default=4)
    ap.add_argument("--large-generations", type=int, default=2)
    ap.add_argument("--multi-rules", type=int, default=100)
    ap.add_argument("--multi-S", type=int, default=100)
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload_for(rank: int, P: int, S: int):
    """Rank 0 evaluates the GP's initial generation; other ranks evaluate the
    same instance with populations of their own seed (same sizes)."""
    from sidr import workload as W
    if rank == 0:
        return W.gp_generation(P=P, S=S)
    return W.build("gp_generation", 100, "clustered", 1000.0, 3, 2, P, 2, 8, rank, S, 1)


def config_of(P, S, world):
    return {"workload": f"gp_generation: {P} rules x {S} scenarios, clustered synthetic "
                        f"instance n=100 (8 clusters), H=1000, m=3, 29-terminal menu, "
                        f"RHH depth 2-8",
            "rules": P, "scenarios": S, "customers": 100, "vehicles": 3, "horizon": 1000,
            "terminals": 29, "parallelism": f"{world} independent generations (one per GPU)",
            "l2": "flushed between timed steps outside the events: a 256 MiB device write, then a "
                  "256 MiB read that moves the written lines out of L2"}


# --------------------------------------------------------------- clocks

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=10)
        except Exception:
            self.proc.kill()
            out = ""
        rows = [r for r in csv.reader(io.StringIO(out)) if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows]
        mx = max(float(r[2]) for r in rows)
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows)}


def gpu_uuid(dev: int) -> str:
    import torch
    u = str(torch.cuda.get_device_properties(dev).uuid)
    return u if u.startswith("GPU-") else "GPU-" + u


# ---------------------------------------------------------- CPU baseline

def cpu_sample(P, S, stride_rules=16, chunk=8):
    rule_idx = list(range(0, P, stride_rules))
    chunks = [(s, min(S, s + chunk)) for s in range(0, S, chunk)]
    return rule_idx, chunks


def cpu_checker():
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    if O.reference_available():
        return O.Reference(), "reference"
    return O.Oracle(), "port"


def cpu_baseline(w, zp, seconds, gpu_out=None, full=False):
    """The CPU simulator on all host threads over a bounded, strided sample of
    the workload (full: every rule and scenario); returns the baseline record
    and, when the GPU's scores are given, their parity with the CPU's."""
    import numpy as np
    chk, kind = cpu_checker()
    threads = os.cpu_count() or 1
    if full:
        idx, chunks = list(range(w.rules.P)), [(0, w.S)]
        sub = w.rules
    else:
        idx, chunks = cpu_sample(w.rules.P, w.S)
        sub = w.rules.subset(idx)
    evals, t_used, cmp, bad = 0, 0.0, 0, 0
    for s0, s1 in chunks:
        t0 = time.perf_counter()
        out = chk.eval_pairs(w.sd, zp, sub, w.sampled[s0:s1], s1 - s0, w.mask, nthreads=threads)
        t_used += time.perf_counter() - t0
        evals += out.size
        if gpu_out is not None:
            g = gpu_out[idx][:, s0:s1]
            cmp += g.size
            bad += int(np.count_nonzero(g.view(np.uint64) != out.view(np.uint64)))
        if not full and t_used >= seconds:
            break
    sample = (f"all {len(idx)} rules x {w.S} scenarios = {evals} evaluations in {t_used:.1f} s"
              if full else
              f"every 16th rule ({len(idx)} rules) x first {evals // len(idx)} scenarios "
              f"= {evals} evaluations in {t_used:.1f} s")
    rec = {"value": evals / t_used, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample}
    if gpu_out is not None:
        rec["parity"] = {"pairs": cmp, "mismatches": bad}
    return rec


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU simulator on the host cores, each
    step a bounded sample of the workload."""
    if rank != 0:
        return
    from sidr import workload as W
    import sidr.rules  # noqa: F401
    w = W.gp_generation(P=args.P, S=args.S)
    chk, kind = cpu_checker()
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    zp = chk.zp_of(w.sd) if kind == "reference" else chk.zstats(w.sd)
    threads = os.cpu_count() or 1
    idx, _ = cpu_sample(w.rules.P, w.S)
    sub = w.rules.subset(idx)
    per = 16
    nsteps = args.warmup + args.steps
    times, evals = [], 0
    for k in range(nsteps):
        s0 = (k * per) % w.S
        s1 = min(w.S, s0 + per)
        t0 = time.perf_counter()
        out = chk.eval_pairs(w.sd, zp, sub, w.sampled[s0:s1], s1 - s0, w.mask, nthreads=threads)
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            times.append(dt)
            evals += out.size
    tot = sum(times)
    value = evals / tot
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * tot / len(times), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_of(args.P, args.S, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": f"per step {len(idx)} rules (every 16th) x {per} scenarios"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ ours

def kernel_sources_sha():
    """sha256 over the evaluator kernel's sources: the key under which a DRAM
    traffic figure measured by ncu is valid."""
    import hashlib
    h = hashlib.sha256()
    for f in ("sidr_kernel.cuh", "sidr_internal.hpp", "sidr_libm.cuh", "sidr_capi.cu"):
        with open(os.path.join(PKG, "csrc", f), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()


def recorded_traffic(workload_name):
    """Per-launch DRAM bytes (read + write) of eval_kernel on this workload,
    from bench_traffic.json beside this script (written from an ncu capture
    of the same command); None when the record is absent or was measured on
    other kernel sources than the ones built here."""
    p = os.path.join(REPO, "bench_traffic.json")
    try:
        with open(p) as f:
            rec = json.load(f)
    except Exception:
        return None, "no record"
    ent = rec.get(workload_name)
    if not ent:
        return None, "no record for this workload"
    if ent.get("kernel_sources_sha256") != kernel_sources_sha():
        return None, "record measured on other kernel sources"
    return float(ent["bytes_per_launch"]), ent.get("command", "")


def measured_hbm_gbs():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs")), "measured (MEASURED_PEAKS.json)"
    except Exception:
        return 6650.0, "fallback"


def measure(ctx, w, steps, warmup, stream, flush, peak_ops, allmax, barrier, world, e2e_on=True,
            clocks=None, shape=-1):
    """Device time of `steps` evaluations of workload w (resident batch, L2
    flushed between steps), the end-to-end rate through sidr_evaluate with host
    buffers, and the FP64 op-model roofline of the evaluator launch."""
    import numpy as np
    import torch
    import sidr
    batch = ctx.batch(w.rules, w.sampled, w.S, w.mask)
    sh = stream.cuda_stream
    batch.set_counting(True)  # op-model counts: separate, untimed launch
    batch.run(sh)
    torch.cuda.synchronize()
    counts = batch.counts()
    batch.set_counting(False)
    # block shape timed on every 16th rule (untimed) unless given; the same
    # shape for the device-timed steps and the end-to-end calls
    if shape >= 0:
        batch.set_shape(shape)
        shape_ms = None
    else:
        shape, shape_ms = batch.autotune_sampled(stride=16, reps=1)
    ctx.set_shape(shape)
    for _ in range(warmup):
        flush()
        batch.run(sh)
    torch.cuda.synchronize()
    ref_out = batch.read()
    barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
        time.sleep(0.3)
    launches0 = sidr.kernel_launches()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    for e0, e1 in ev:
        flush()
        e0.record(stream)
        batch.run(sh)
        e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    launches = sidr.kernel_launches() - launches0
    clk = clocks.stop() if clocks else None
    step_ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    total_ms = allmax(sum(step_ms))
    evals = w.rules.P * w.S
    value = world * evals * steps / (total_ms / 1e3)
    same = bool(np.array_equal(batch.read().view(np.uint64), ref_out.view(np.uint64)))
    batch.close()
    e2e = None
    if e2e_on:
        ctx.evaluate(w.rules, w.sampled, w.S, w.mask)
        barrier()
        t_e2e = 0.0
        for _ in range(steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = ctx.evaluate(w.rules, w.sampled, w.S, w.mask)
            t_e2e += time.perf_counter() - t0
        t_e2e = allmax(t_e2e)
        h2d, d2h = sidr.last_transfer_bytes()
        same = same and bool(np.array_equal(out.view(np.uint64), ref_out.view(np.uint64)))
        e2e = {"value": world * evals * steps / t_e2e, "unit": UNIT,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": 1e3 * t_e2e / steps}
    avg_s = (sum(step_ms) / len(step_ms)) / 1e3
    achieved = counts["fp64_ops"] / avg_s
    traffic, traffic_src = recorded_traffic(w.name)
    roofline = {"bound": "fp64", "achieved": achieved / 1e12, "peak": peak_ops / 1e12,
                "unit": "Tops/s (FP64 pipe, op model)", "frac": achieved / peak_ops,
                "traffic": traffic, "traffic_source": traffic_src,
                "peak_source": "measured on this GPU by sidr_fp64_peak (DFMA chains over all SMs)",
                "op_model": "sidr_counts.fp64_ops (include/sidr.h)"}
    hbm = None
    if traffic is not None:
        hbm_peak, hbm_src = measured_hbm_gbs()
        hbm = {"achieved": traffic / avg_s / 1e9, "peak": hbm_peak, "unit": "GB/s",
               "frac": traffic / avg_s / 1e9 / hbm_peak, "peak_source": hbm_src,
               "traffic_bytes_per_launch": traffic}
    ctx.set_shape(0)
    return {"value": value, "total_ms": total_ms, "e2e": e2e, "launches": launches,
            "roofline": roofline, "hbm": hbm, "clocks": clk, "counts": counts,
            "repeat_runs_identical": same, "out": ref_out,
            "block_shape": {"warps_per_block": sidr.Batch.SHAPES[shape][0],
                            "blocks_per_sm": sidr.Batch.SHAPES[shape][1],
                            "lanes_per_pair": sidr.Batch.SHAPES[shape][2],
                            "shapes": [list(x) for x in sidr.Batch.SHAPES],
                            "ms_on_sample": shape_ms, "sample": "every 16th rule, all scenarios"}}


def run_ours(args, rank, world, local):
    import torch
    import sidr

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta
        dist_mod.init_process_group("nccl", timeout=timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        dist = dist_mod

    def barrier():
        if dist:
            dist.barrier()

    def allmax(x: float) -> float:
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    w = workload_for(rank, args.P, args.S)
    zp = sidr.zstats(w.sd)
    ctx = sidr.Context(w.sd, zp, device=local)
    stream = torch.cuda.Stream()  # the launching stream: events are recorded on it
    torch.cuda.set_stream(stream)
    peak_ops = sidr.fp64_peak(local)
    flush_w = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    flush_r = torch.ones(256 << 20, dtype=torch.uint8, device="cuda")

    def flush():
        # the write evicts the workload's lines from L2; the read then replaces the
        # written (dirty) lines with clean ones, so their write-back falls here
        # and not inside the next step
        flush_w.zero_()
        flush_r.sum()

    r = measure(ctx, w, args.steps, args.warmup, stream, flush, peak_ops, allmax, barrier, world,
                e2e_on=not args.no_e2e, clocks=ClockSampler(gpu_uuid(local)), shape=args.shape)
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["total_ms"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config_of(args.P, args.S, world),
            "e2e": r["e2e"], "gpu_launches": r["launches"], "roofline": r["roofline"],
            "hbm": r["hbm"], "clocks": r["clocks"], "counts": r["counts"],
            "block_shape": r["block_shape"], "repeat_runs_identical": r["repeat_runs_identical"]}
    if args.evolved_steps > 0:
        # the same instance and scenarios with generation 49 of the benchmark GP run: the
        # populations a GP spends 49 of its 50 generations on
        from sidr import workload as W
        we = W.evolved(49, P=args.P, S=args.S)
        re = measure(ctx, we, args.evolved_steps, 3, stream, flush, peak_ops, allmax, barrier,
                     world, e2e_on=not args.no_e2e, shape=args.evolved_shape)
        line["evolved"] = {"workload": f"evolved_gen49: generation 49 of the benchmark GP run "
                                       f"(seed 0), {args.P} rules x {args.S} scenarios, same "
                                       f"instance and scenarios", "value": re["value"],
                           "unit": UNIT, "steps": args.evolved_steps, "warmup": 3,
                           "ms_per_step": re["total_ms"] / args.evolved_steps, "e2e": re["e2e"],
                           "roofline": re["roofline"], "counts": re["counts"],
                           "block_shape": re["block_shape"],
                           "repeat_runs_identical": re["repeat_runs_identical"]}
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            # a bounded sample: the evolved rules cost the CPU simulator about 3x more per pair
            line["evolved"]["cpu_baseline"] = cpu_baseline(we, zp, args.cpu_seconds / 2,
                                                           gpu_out=re["out"])
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(w, zp, args.cpu_seconds, gpu_out=r["out"],
                                            full=args.full_parity)
    if args.gp and rank == 0:
        line["gp"] = gp_leg(ctx, w, args)
    if args.multi and rank == 0:
        line["multi"] = multi_leg(args, stream)
    if args.sgp and rank == 0:
        line["sgp"] = sgp_leg(ctx, w, args)
    if args.campaign and rank == 0:
        line["campaign"] = campaign_leg()
    if args.large and rank == 0:
        line["large"] = large_leg(args)
    if args.sampling and rank == 0:
        line["sampling"] = sampling_leg()
    ctx.close()
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def multi_leg(args, stream):
    """The uneven batch (40 instances: 25/50/100/288 customers, three layouts,
    m 2-4, H 230/1000, rules of log-uniform length 3-255): one persistent
    launch per instance-size class, each class's block shape (warps, blocks,
    lanes per pair) autotuned on a sample of the class (every 16th rule of its
    longest-first order) unless --multi-shape is given, all captured in one
    CUDA graph, device-timed.  Then, per size class, the same instances in a
    launch of their own (at the chosen shape and at a warp per pair) and one
    by one through the single-instance path, which shows where the batch's
    time goes."""
    import numpy as np
    import torch
    import sidr
    from sidr import workload

    def timed(run, reps=2):
        run()
        torch.cuda.synchronize()
        best = None
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run()
            e1.record(stream)
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1) / 1e3
            best = t if best is None else min(best, t)
        return best

    t0 = time.perf_counter()
    mw = workload.batched_uneven(K=40, rules_per_instance=args.multi_rules, S=args.multi_S)
    zps = [sidr.zstats(sd) for sd in mw.sds]
    m = sidr.Multi(mw.sds, zps, mw.rules, mw.sampled, mw.S, mw.masks)
    prep = time.perf_counter() - t0
    t_tune = time.perf_counter()
    if args.multi_shape >= 0:
        chosen, ms = [args.multi_shape] * len(sidr.Multi.CLASSES), None
        m.set_shape(args.multi_shape)
    else:
        chosen, ms = m.autotune_classes(stride=16, reps=1)
    t_tune = time.perf_counter() - t_tune
    m.capture()
    t = timed(lambda: m.run(stream.cuda_stream))
    P = sum(r.P for r in mw.rules)
    res = m.read()
    m.close()
    # spot check: every 125th rule of instances 3 (288 customers) and 38 by the single-instance path
    mism, pairs = 0, 0
    for k in (3, 38):
        ctx = sidr.Context(mw.sds[k], zps[k])
        idx = list(range(0, mw.rules[k].P, 125))
        want = ctx.evaluate(mw.rules[k].subset(idx), mw.sampled[k], mw.S, mw.masks[k])
        mism += int((res[k][idx].view(np.uint64) != want.view(np.uint64)).sum())
        pairs += want.size
        ctx.close()
    classes = {}
    for n in sorted({sd.n for sd in mw.sds}):
        ks = [k for k, sd in enumerate(mw.sds) if sd.n == n]
        c = next(i for i, (lo, hi) in enumerate(sidr.Multi.CLASSES) if lo <= n <= hi)
        mc = sidr.Multi([mw.sds[k] for k in ks], [zps[k] for k in ks], [mw.rules[k] for k in ks],
                        [mw.sampled[k] for k in ks], mw.S, [mw.masks[k] for k in ks])
        mc.set_shape(chosen[c])
        tc = timed(lambda: mc.run(stream.cuda_stream), reps=1)
        tw = tc
        if sidr.Multi.SHAPES[chosen[c]][2] != 32:
            mc.set_shape(0)
            tw = timed(lambda: mc.run(stream.cuda_stream), reps=1)
        mc.close()
        t_one = 0.0
        for k in ks:
            ctx = sidr.Context(mw.sds[k], zps[k])
            b = ctx.batch(mw.rules[k], mw.sampled[k], mw.S, mw.masks[k])
            t_one += timed(lambda: b.run(stream.cuda_stream), reps=1)
            b.close()
            ctx.close()
        ev = sum(mw.rules[k].P for k in ks) * mw.S
        classes[str(n)] = {"instances": len(ks), "evaluations": ev,
                           "shape": list(sidr.Multi.SHAPES[chosen[c]]), "own_launch_seconds": tc,
                           "own_launch_evals_per_s": ev / tc,
                           "own_launch_warp_per_pair_seconds": tw, "one_by_one_seconds": t_one,
                           "one_by_one_evals_per_s": ev / t_one}
    return {"workload": f"40 instances x {args.multi_rules} rules x {args.multi_S} scenarios",
            "evaluations": P * mw.S, "seconds": t, "evals_per_s": P * mw.S / t,
            "shapes": [list(x) for x in sidr.Multi.SHAPES],
            "class_shapes_ms_on_sample": ms, "tuning_seconds": t_tune,
            "chosen_shape_per_class": [list(sidr.Multi.SHAPES[x]) if x >= 0 else None for x in chosen],
            "host_prep_seconds": prep,
            "spot_check_pairs": pairs, "spot_check_mismatches": mism, "per_size_class": classes}


def sampling_leg():
    """Scenario sampling (gen_durations) on one host core against the GPU
    sampler, which is bit-identical: the benchmark's block (500 scenarios x
    100 customers) and one block of the large combined run (2000 scenarios x
    288 customers).  Host: wall clock of sidr_gen_durations; GPU: wall clock of
    sidr_gen_durations_device with the result in host memory (transfers and the
    host's recomputation of unsettled pairs included) and in device memory."""
    import numpy as np
    import torch
    from sidr import gp as GP
    from sidr import workload as W
    res = {}
    for name, sd, S in (("benchmark_block", W.gp_generation(P=1, S=1).sd, 500),
                        ("large_run_block", W.large_combined(K=1, seeds=1, rules_per_seed=1, S=1).sds[0], 2000)):
        d = sd.durations
        GP.gen_durations_device(d, 0.2, 8, 1)  # warm-up
        t0 = time.perf_counter()
        host = GP.gen_durations(d, 0.2, S, 1)
        t_host = time.perf_counter() - t0
        t0 = time.perf_counter()
        dev, st = GP.gen_durations_device(d, 0.2, S, 1)
        t_dev = time.perf_counter() - t0
        out = torch.empty((S, len(d)), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        GP.gen_durations_device(d, 0.2, S, 1, out_ptr=out.data_ptr())
        t_dres = time.perf_counter() - t0
        same = bool(np.array_equal(host.view(np.uint64), dev.view(np.uint64))) and \
            bool(np.array_equal(host.view(np.uint64), out.cpu().numpy().view(np.uint64)))
        res[name] = {"scenarios": S, "customers": len(d), "host_ms": 1e3 * t_host,
                     "gpu_to_host_ms": 1e3 * t_dev, "gpu_resident_ms": 1e3 * t_dres,
                     "pairs": st["pairs"], "pairs_left_to_host": st["host_pairs"],
                     "bit_identical": same}
    return res


def large_leg(args):
    """The large combined run's driver (sidr_sgp_run_multi) at its full
    population shape -- 10 instances of 288 customers (12-cluster and uniform
    layouts, m = 4, H = 1000) x 30 GP seeds x 4096 rules, 16384 offspring
    screened per seed-generation -- for a few generations with fewer training
    scenarios than the benchmark's 2000.  Every generation simulates all
    1.2 M rules of the populations in one multi-instance launch; the
    evaluation time scales with the scenario count, the model and host time
    do not."""
    import sidr
    from sidr import surrogate as SG
    from sidr import workload as W
    mw = W.large_combined(K=10, seeds=1, rules_per_seed=1, S=1)
    zps = [sidr.zstats(sd) for sd in mw.sds]
    G = args.large_generations
    t0 = time.perf_counter()
    r = SG.sgp_run_multi(mw.sds, zps, W.MENU29, mw.masks, 30, first_seed=0, test_seed=1000000,
                         shape=-1, gp=dict(population=4096, generations=G,
                                           train_samples=args.large_S, test_samples=500),
                         screen=16384)
    wall = time.perf_counter() - t0
    pop_evals = 10 * 30 * 4096 * args.large_S
    return {"workload": f"10 instances x 288 customers x 30 seeds x 4096 rules, {G} generations "
                        f"of {args.large_S} training scenarios, screening 16384 per "
                        f"seed-generation, held-out 500",
            "wall_seconds": wall, "eval_seconds": r["eval_seconds"],
            "model_seconds": r["model_seconds"], "host_seconds": r["host_seconds"],
            "evaluations": r["evaluations"], "evals_per_s": r["evaluations"] / r["eval_seconds"],
            "population_evaluations_per_generation": pop_evals,
            "screened": r["screened"], "fallback": r["fallback"],
            "best_held_out_mean": float(r["held_out"][-1].mean())}


def campaign_leg():
    """The reference campaign's c101 workloads on the evaluator: the generation
    trace of s3_generation/gen_trace.cu (compared with the reference's trace
    file seed by seed) and the first batch_score call of s4_selection/ga.cu's
    search (13 genomes of the 18-terminal universe x 16 seeds x 51 generations
    + the 64-scenario TRAIN block; its proxies give the search log's 'gen 0'
    line only with the next batches, so here they are timed)."""
    import numpy as np
    import sidr
    from sidr import campaign
    from sidr import rules as R
    from sidr.instance import SimData
    z = np.load(os.path.join(REPO, "tests", "golden", "campaign.npz"))
    sd = SimData.from_arrays(*[z[f"c101/inst_{k}"] for k in
                               ("x", "y", "score", "open", "close", "dur", "tmax")], m=3)
    km = float(z["c101/km"][0])
    expected = json.loads(str(z["c101/trace"]))
    ctx = sidr.Context(sd, sidr.zstats(sd))
    t0 = time.perf_counter()
    text, _ = campaign.gen_trace(ctx, "c101", expected["vocab_extra"], km, n_seeds=30)
    t_trace = time.perf_counter() - t0
    got = json.loads(text)
    same = sum(1 for s in range(30) if got["trace"][s] == expected["trace"][s]
               and got["finals"][s] == expected["finals"][s])
    trace_evals = 30 * 1024 * 52 + 30 * 500
    # the search's first batch: genomes 0 and the 18 singletons sorted, first 13
    genomes = sorted([0] + [1 << b for b in range(18)])[:13]
    t0 = time.perf_counter()
    _, res = campaign.batch_score(ctx, R.EXTRA, genomes, 16, 51, bmax=13)
    t_batch = time.perf_counter() - t0
    ctx.close()
    return {"trace": {"workload": "c101 gen_trace: 30 seeds x 1024 rules x 51 generations + "
                                  "30 x 500 held-out, 17 terminals",
                      "wall_seconds": t_trace, "evaluations": trace_evals,
                      "evals_per_s": trace_evals / t_trace,
                      "seeds_identical_to_reference_trace": same},
            "ga_batch": {"workload": "c101 batch_score: 13 genomes x 16 seeds x 1024 rules x 51 "
                                     "generations + 64-scenario TRAIN block",
                         "wall_seconds": t_batch, "eval_seconds": res.eval_seconds,
                         "host_seconds": res.host_seconds, "evaluations": res.evaluations,
                         "evals_per_s": res.evaluations / t_batch}}


def sgp_leg(ctx, w, args):
    """Surrogate-assisted GP vs plain GP through the same driver.  The plain
    arm breeds with gp_step every generation; the "surrogate" arm (the
    driver's defaults) trains the model on rank scores and fills the
    non-elite slots of a screened generation with the best-predicted
    offspring, one per ranking of the decision situations.  --sgp-ablation
    adds arms that change one setting each: one child per distinct rule
    ("rule_distinct"), that plus standardised fitness targets
    ("standardised"), the best-predicted of each group of 8 offspring
    ("preselection"), half the slots bred plainly ("half_screened").  Every run records
    each generation's best rule on the held-out 500 scenarios and the wall
    clock; the result is the time each run needs to reach the plain run's
    final held-out score (within 0.5 %), as a ratio to the plain run's own
    time to that score and to the plain run's whole wall clock."""
    from sidr import surrogate as SG
    from sidr.workload import MENU29
    G = args.sgp_generations
    cfg = dict(population=args.P, generations=G, train_samples=args.S, test_samples=500)
    arms = {"plain": dict(use_surrogate=0), "surrogate": dict(use_surrogate=1)}
    if args.sgp_ablation:
        arms.update({"rule_distinct": dict(use_surrogate=1, distinct=0),
                     "standardised": dict(use_surrogate=1, distinct=0, target=0),
                     "preselection": dict(use_surrogate=1, selection=1),
                     "half_screened": dict(use_surrogate=1, screen_fraction=0.5)})
    runs = {k: SG.sgp_run(ctx, MENU29, w.mask, seed=args.sgp_seed, test_seed=1000000, gp=cfg, **kw)
            for k, kw in arms.items()}
    plain = runs["plain"]
    target = plain["held_out"][-1] * (1.0 - 0.005)
    plain_total = float(plain["seconds"][-1])

    def first_time(r):
        for g in range(G):
            if r["held_out"][g] >= target:
                return float(r["seconds"][g]), g
        return None, None

    tp, _ = first_time(plain)
    out = {"generations": G, "population": args.P, "train_scenarios": args.S, "seed": args.sgp_seed,
           "target_held_out": target, "plain_wall_seconds": plain_total}
    for k, r in runs.items():
        t, g = first_time(r)
        out[k] = {"final_held_out": float(r["held_out"][-1]),
                  "best_held_out": float(max(r["held_out"])),
                  "seconds_to_target": t, "generation_at_target": g,
                  "ratio_to_plain_time_to_target": (t / tp) if (t is not None and tp) else None,
                  "ratio_to_plain_wall": (t / plain_total) if t is not None else None,
                  "wall_seconds": float(r["seconds"][-1]), "eval_seconds": r["eval_seconds"],
                  "model_seconds": r["model_seconds"], "screened": r["screened"],
                  "fallback": r["fallback"],
                  "held_out": [float(v) for v in r["held_out"]],
                  "seconds": [float(v) for v in r["seconds"]],
                  "rho": [None if v != v else float(v) for v in r["rho"]]}
    return out


def gp_leg(ctx, w, args):
    """The GP run behind the workload: the reference's GP (engine/gp.hpp) with
    the benchmark's settings -- population 1024, 500 training scenarios per
    generation (base seed seed*10000+gen), 50 generations, the best rule scored
    on 500 held-out scenarios (base seed 1000000) -- evaluated by the B200
    evaluator; host GP in C++."""
    from sidr import gp
    from sidr.workload import MENU29
    t0 = time.perf_counter()
    res = gp.run_batched(ctx, MENU29, w.mask, 1, first_seed=0, test_seed=1000000,
                         population=args.P, generations=args.gp_generations,
                         train_samples=args.S, test_samples=500)
    wall = time.perf_counter() - t0
    return {"population": args.P, "train_scenarios": args.S, "generations": args.gp_generations,
            "wall_seconds": wall, "eval_seconds": res.eval_seconds,
            "host_seconds": res.host_seconds, "evaluations": res.evaluations,
            "held_out_mean_score": float(res.best_test[0]),
            "best_train_first": float(res.best_train[0, 0]),
            "best_train_last": float(res.best_train[-1, 0]), "best_rule": res.best_rules[0]}


def run_sharded(args, rank, world, local):
    """The benchmark GP (1024 rules, 500 training scenarios per generation),
    its rules sharded over the ranks (sidr.dist.sharded_gp): each generation
    evaluates this rank's block on its GPU, all_gathers the fitness and steps
    the same GP on every rank.  A step is one generation, timed on the host
    (evaluation, gather and GP step) and maximised over ranks."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    import sidr
    from sidr import dist as D
    from sidr import workload as W
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    else:
        dist.init_process_group("gloo", init_method="tcp://127.0.0.1:29533", rank=0, world_size=1)
    w = W.gp_generation(P=1, S=1)
    ctx = sidr.Context(w.sd, sidr.zstats(w.sd), device=local)
    times = []
    dev = torch.device("cuda", local) if world > 1 else None
    D.sharded_gp(ctx, W.MENU29, w.mask, seed=0, generations=args.warmup + args.steps,
                 population=args.P, train_samples=args.S, device=dev,
                 on_generation=lambda g, sec: times.append(sec) if g >= args.warmup else None)
    total = D.max_over_ranks(sum(times), device=dev)
    ctx.close()
    dist.destroy_process_group()
    if rank == 0:
        value = args.P * args.S * args.steps / total
        print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                          "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
                          "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                          "data": "synthetic",
                          "config": dict(config_of(args.P, args.S, world),
                                         parallelism=f"rule shards over {world} GPUs, fitness "
                                                     f"all_gather per generation",
                                         step="one GP generation (host wall clock: evaluation, "
                                              "gather and GP step), max over ranks")}),
              flush=True)


def main():
    args = parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.sharded:
        run_sharded(args, rank, world, local)
        return
    run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
