#!/usr/bin/env python3
"""Ply-step throughput of the B200 engine (positions per second).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]
                    [--workload slice|mix] [--path plain|batched]

Workloads (synthetic, seeded; there is no public dataset for this path):
  slice  KRRRvKRRR, king slice 96 (wK c1, bK e6), N = 1,229,490,380
         positions: one slice-ply (W step + L step, tb8gen_b200.plyjob) with
         L_prev/W_prev Bernoulli(0.01) from seed 1, illegal positions cleared.
  mix    96 king slices from seed 2 over KRRRvKRRR, KQRvKRRR and KQRRvKRR
         with p in {0.001, 0.01, 0.05}; neighbour marks go to per-material
         shared bitmaps (see plyjob).

  serve  a seeded Poisson stream (seed 4) of ply jobs (70%) and probe
         batches (30%, 1k-1M positions) served with continuous batching under
         an HBM admission budget, swept over arrival rates, beside one
         request at a time; p50/p99 latency and positions/s.
  fixpoint  the whole generation of a material (default KQRvKRR) by the
         C host driver with the planes in host memory (tbgen -S); per
         half-ply positions/s; the resident run must print the same counts.
  probe  2^28 seeded legal positions (seed 3), half KRRRvKRR, half KQRvKRR,
         probed (WDL) against the synthetic rANS tables of the two
         materials (seed 3, values mod 3); a step is one probe batch of all
         positions, and the index round trip (encode, decode, re-encode) is
         timed beside it.  Metric: probe positions/s.

A step of the ply workloads is one slice-ply of every slice of the workload.  `value` is the
positions of all slices (all ranks) per second of device time, inputs
resident in HBM.  `e2e` is the same metric through the public C ABI with
the inputs copied from pinned host memory and the W/L results copied back
inside the timed region.  With --gpus N (torchrun) every rank runs its own
replica of the workload (the ply step has no exchange between slices of a
step): weak scaling, no collective on the data path.
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
sys.path.insert(0, ROOT)

METRIC = "ply positions/s (bit-exact)"
UNIT = "positions/s"
ALG_BYTES_PER_POS = 0.875  # W step 0.5 B + L step 0.375 B per position


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--workload", default="slice",
                    choices=["slice", "mix", "small", "slice-pool", "probe", "serve",
                             "fixpoint"])
    ap.add_argument("--fix-material", default="KQRvKRR")
    ap.add_argument("--fix-max-ply", type=int, default=0)
    ap.add_argument("--serve-jobs", type=int, default=120)
    ap.add_argument("--serve-rates", default="10,100,500,2000")
    ap.add_argument("--serve-slots", type=int, default=8)
    ap.add_argument("--serve-budget-gb", type=float, default=150.0)
    ap.add_argument("--probe-n", type=int, default=1 << 28,
                    help="probe workload: positions per step (split over the materials)")
    ap.add_argument("--probe-materials", default="KRRRvKRR,KQRvKRR",
                    help="probe workload: materials (a smaller one makes a profiling case)")
    ap.add_argument("--path", default="batched", choices=["plain", "batched"])
    ap.add_argument("--ctas-per-sm", type=int, default=0,
                    help="persistent-kernel CTAs per SM (0: autotune)")
    ap.add_argument("--profile-run", default="none", choices=["none", "plain", "batched"],
                    help="ply workloads: one more step of that path, after all timing, "
                         "between cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    ap.add_argument("--mode", type=int, default=0, choices=[0, 1, 2],
                    help="persistent kernel: 1 block-wide, 2 warp-wide work items (0: autotune)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="probe workload: target CPU time of the reference probe sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mix", action="store_true",
                    help="slice workload: skip the uneven-mix record (batched vs plain)")
    ap.add_argument("--no-probe", action="store_true",
                    help="slice workload: skip the probe record (config 3)")
    ap.add_argument("--no-serve", action="store_true",
                    help="slice workload: skip the serving record (config 4)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload_spec(name):
    if name == "slice":
        return [("KRRRvKRRR", 96, 0.01, 1)]
    if name == "small":  # profiling case: 24 MB bitmaps
        return [("KQRRvKRR", 96, 0.01, 1)]
    if name == "slice-pool":  # profiling case: the slice, neighbours in shared sinks (~1.4 GB)
        return [("KRRRvKRRR", 96, 0.01, 1)]
    import numpy as np

    rng = np.random.default_rng(2)
    mats = ["KRRRvKRRR", "KQRvKRRR", "KQRRvKRR"]
    ps = [0.001, 0.01, 0.05]
    out = []
    for j in range(96):
        out.append((mats[j % 3], int(rng.integers(0, 462)), ps[(j // 3) % 3], 2))
    return out


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.gpu), "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(ms, world, device="cuda"):
    """The largest per-step time over the ranks (one all-reduce; every rank
    calls it at the same point).  One rank: unchanged."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def committed_issue(kernel):
    """Fraction of instruction-issue slots the kernel used in its committed
    ncu capture (profiles/traffic.json), the roofline that binds it."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return float(json.load(f)[kernel]["issue_active_frac"])
    except Exception:
        return None


def committed_inst(kernel):
    """Warp instructions per unit of `kernel` in its committed ncu capture
    (profiles/traffic.json); None if absent."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return float(json.load(f)[kernel]["warp_inst_per_unit"])
    except Exception:
        return None


def issue_roofline(kernel, units, launch_ms, clocks):
    """The instruction-issue roofline of a kernel bound by issue rather than
    by HBM: its warp instructions per launch (the committed capture's count
    per unit times the units of a launch) against the GPU's issue rate, one
    warp instruction per cycle on each of the 4 schedulers of every SM at
    the SM clock sampled during the run."""
    per = committed_inst(kernel)
    if per is None or not launch_ms:
        return None
    import torch

    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mhz = (clocks or {}).get("sm_mhz") or 1965.0
    inst = per * units
    floor_ms = inst / (sms * 4 * mhz * 1e6) * 1e3
    return {"warp_inst_per_launch": int(inst), "issue_rate_per_s": sms * 4 * mhz * 1e6,
            "floor_ms": round(floor_ms, 4), "frac": round(floor_ms / launch_ms, 4),
            "source": "warp instructions per unit of the committed ncu capture "
                      "(profiles/traffic.json) times the units of a launch"}


def committed_traffic(kernel):
    """DRAM bytes per unit (position, or block for the probe decode) of
    `kernel` from profiles/traffic.json, which records one ncu capture of a
    smaller case of the same kernel; None if absent."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            d = json.load(f)
        return float(d[kernel]["bytes_per_unit"])
    except Exception:
        return None


# ----------------------------------------------------------------- engine arm
def run_engine(a, rank, world, local):
    import torch

    import tb8gen_b200 as tbg
    from tb8gen_b200.plyjob import MaterialPool, SlicePly

    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    tbg.init()
    tbg.set_stream(stream)
    spec = workload_spec(a.workload)
    pools = {}
    jobs = []
    for mat, s, p, seed in spec:
        pool = None
        if a.workload in ("mix", "slice-pool"):
            if mat not in pools:
                pools[mat] = MaterialPool(mat, seed)
            pool = pools[mat]
        jobs.append(SlicePly(mat, s, p, seed + 1000 * rank, pool))
    torch.cuda.synchronize()
    positions = sum(j.positions for j in jobs)

    phase_names = SlicePly.PHASES
    ev = {ph: [] for ph in phase_names}

    def direct_step(timed_phases=False):
        # phase order: all W scatters, all epilogues, all L scatters, all verifies
        for ph in phase_names:
            if timed_phases:
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            for j in jobs:
                getattr(j, ph)()
            if timed_phases:
                e1.record(stream)
                ev[ph].append((e0, e1))

    # the same step recorded once; mode 0 = one launch per call, 1 and 2 =
    # persistent (block-wide or warp-wide work items, picked by the autotuner)
    from tb8gen_b200.plyjob import record_step
    nops, nitems = record_step(jobs)

    def time_mode(md, reps):
        return time_batch(tbg, stream, md, reps)

    # autotune the persistent launch on this batch: CTAs per SM x tiles per
    # scatter work item
    tune, best_mode, best_cps, best_gt, nitems = autotune(
        tbg, time_mode, a.ctas_per_sm, (a.mode,) if a.mode else (1, 2))
    mode = best_mode if a.path == "batched" else 0

    def step():
        tbg.batch_run(mode)

    # clocks are sampled from before the warm-up to the end of the timed steps
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(1.0)
    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()

    # device-time throughput, inputs resident in HBM
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    n0 = tbg.launches()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(a.steps):
        step()
    t1.record(stream)
    torch.cuda.synchronize()
    launches = tbg.launches() - n0
    ms = t0.elapsed_time(t1) / a.steps
    clk = clocks.stop()
    ms = max_over_ranks(ms, world)

    # both paths on the same recorded batch, and per-phase device times
    plain_ms = time_mode(0, max(2, a.steps // 2))
    batched_ms = time_mode(best_mode, max(2, a.steps // 2))
    for _ in range(max(3, a.steps // 2)):
        direct_step(timed_phases=True)
    torch.cuda.synchronize()
    phase_ms = {ph: statistics.median(e0.elapsed_time(e1) for e0, e1 in ev[ph])
                for ph in phase_names}

    if a.profile_run != "none":
        # one extra step outside every timed region, bracketed for a profiler
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        tbg.batch_run(0 if a.profile_run == "plain" else best_mode)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()

    counts = [j.counts() for j in jobs[:4]]
    mix = None
    if a.workload == "slice" and not a.no_mix:
        mix = mix_record(a, stream)
        tbg.batch_shape(*best_gt)  # the timed batch's shape for what follows

    # end to end through the C ABI with host buffers
    e2e = None
    if not a.no_e2e:
        e2e = run_e2e(a, jobs, stream, positions, mode)

    value = positions * world / (ms / 1e3)
    peak, peak_kind = measured_peak()
    # roofline of the dominant kernel: the persistent kernel on the batched
    # path (one launch per step), the slowest phase's kernel on the plain path
    per_pos = {"w_scatter": 0.125, "w_epilogue": 0.5, "l_scatter": 0.125, "l_verify": 0.25}
    kname = {"w_scatter": "k_op_w", "w_epilogue": "k_epilogue_W",
             "l_scatter": "k_op_w", "l_verify": "k_op_w"}
    if mode != 0:
        dom = "k_batch" if mode == 1 else "k_batch_w"
        dom_ms, alg = ms, ALG_BYTES_PER_POS * positions
    else:
        ph = max(phase_ms, key=phase_ms.get)
        dom, dom_ms, alg = kname[ph], phase_ms[ph], per_pos[ph] * positions
    achieved = alg / (dom_ms / 1e3) / 1e9
    tr = committed_traffic(dom)
    traffic = int(tr * positions) if tr else None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "alg_bytes_per_launch": int(alg), "traffic": traffic,
                "issue_active_frac": committed_issue(dom),
                "issue": issue_roofline(dom, positions, dom_ms, clk),
                "step_alg_GBps": round(ALG_BYTES_PER_POS * positions / (ms / 1e3) / 1e9, 1),
                "step_frac": round(ALG_BYTES_PER_POS * positions / (ms / 1e3) / 1e9 / peak, 4)}

    cpu, ref_ply = None, None
    if rank == 0 and world == 1 and not a.no_cpu:
        cpu, ref_ply = run_cpu_baseline(a, jobs)
    # bit-exactness of the timed step's outputs (outside the timing)
    parity = slice_parity(jobs, ref_ply)
    del ref_ply

    # configs 3 and 4 beside the timed workload, each its own full record
    probe = serve = None
    if a.workload == "slice" and world == 1:
        if not a.no_probe:
            probe = embedded(run_probe(a, rank, world, local))
            torch.cuda.empty_cache()
        if not a.no_serve:
            serve = embedded(run_serve(a, rank, world, local))
            torch.cuda.empty_cache()

    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded Bernoulli bitmaps, seeded 7-piece stub)",
        "config": slice_config(a.workload, spec, positions),
        "path": a.path,
        "parity": parity,
        "phase_ms": {k: round(v, 4) for k, v in phase_ms.items()},
        "paths_ms": {"plain": round(plain_ms, 4), "batched": round(batched_ms, 4),
                     "batched_speedup": round(plain_ms / batched_ms, 3)},
        "batch": {"calls": nops, "work_items": nitems, "mode": best_mode, "ctas_per_sm": best_cps,
                  "tiles_per_item": {"predecessors": best_gt[0], "candidates": best_gt[1]},
                  "autotune_ms": tune},
        "counts_first_jobs": counts,
        "roofline": roofline, "gpu_launches": launches, "clocks": clk,
        "e2e": e2e, "cpu_baseline": cpu,
        "mix": mix, "probe": probe, "serve": serve,
    }
    return line


def embedded(line):
    """A workload's own bench line, as a record inside the default line."""
    if line is None:
        return None
    drop = ("n_gpus", "higher_is_better", "scaling", "vs_baseline", "data", "gpu_launches")
    return {k: v for k, v in line.items() if k not in drop}


def time_batch(tbg, stream, md, reps):
    """Device time (ms) of one run of the selected recorded batch: mode 0
    one launch per call, mode 1 or 2 the persistent launch."""
    import torch

    tbg.batch_run(md)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        tbg.batch_run(md)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


# the autotuner's grid per persistent mode: CTAs per SM, tiles per work
# item of the W scatter, tiles per work item of the L candidates
TUNE_GRID = {
    1: ((4, 8), (1, 2), (1, 2, 4)),
    2: ((4,), (1, 2), (1, 2, 4)),
}


def autotune(tbg, time_mode, fixed_cps=0, modes=(1, 2)):
    """The persistent launch's shape picked on the recorded batch by its own
    device time: the mode (1: block-wide work items, 2: one part of an item
    per warp) x CTAs per SM (the blocks that take work items at once) x
    tiles per work item of the W step's scatter x tiles per work item of
    the L step's candidates (the sources a block, or a warp, gathers before
    handing them out).  Returns ({"<mode>:<cps>x<w>x<l>": ms}, mode, cps,
    (w, l), work items)."""
    tune = {}
    for md in modes:
        cpss, gws, gls = TUNE_GRID[md]
        for gw in gws:
            for gl in gls:
                tbg.batch_shape(gw, gl)
                for cps in ((fixed_cps,) if fixed_cps > 0 else cpss):
                    tbg.batch_tune(cps)
                    tune[f"{md}:{cps}x{gw}x{gl}"] = round(time_mode(md, 2), 4)
    best = min(tune, key=tune.get)
    md, shape = best.split(":")
    cps, gw, gl = (int(x) for x in shape.split("x"))
    nitems = tbg.batch_shape(gw, gl)
    tbg.batch_tune(cps)
    return tune, int(md), cps, (gw, gl), nitems


def mix_record(a, stream, slot=2):
    """The uneven mix (96 slices of three materials, seed 2) recorded in its
    own batch slot beside the timed workload: the persistent launch against
    one launch per call, each autotuned on the batch, and every slice's
    W and L counts and digests checked against the reference's recorded
    ones (tests/golden/slice_ply.json "mix", made by the reference's
    workers)."""
    import torch

    import tb8gen_b200 as tbg
    from tb8gen_b200.plyjob import MaterialPool, SlicePly, output_digests, record_step

    spec = workload_spec("mix")
    pools, jobs = {}, []
    for mat, s, p, seed in spec:
        if mat not in pools:
            pools[mat] = MaterialPool(mat, seed)
        jobs.append(SlicePly(mat, s, p, seed, pools[mat]))
    positions = sum(j.positions for j in jobs)
    tbg.batch_select(slot)
    try:
        nops, _ = record_step(jobs)
        tm = lambda md, reps: time_batch(tbg, stream, md, reps)
        tune, md, cps, gt, nitems = autotune(tbg, tm)
        reps = max(2, min(a.steps, 5))
        plain = tm(0, reps)
        batched = tm(md, reps)
        tbg.sync()
    finally:
        tbg.batch_select(0)
    golden = {}
    try:
        with open(GOLDEN_SLICE) as f:
            golden = json.load(f).get("mix", {})
    except OSError:
        pass
    checked, bad = 0, []
    for j in jobs:
        g = golden.get(f"{j.material}/{j.s}/{j.p}/{j.seed}/shared")
        if g is None:
            continue
        checked += 1
        if list(j.counts()) != g["counts"] or output_digests(j.outputs()) != g["sha256"]:
            bad.append(f"{j.material}/{j.s}/{j.p}")
    rec = {"slices": len(jobs), "positions_per_step": positions,
           "materials": sorted(pools), "plain_ms": round(plain, 3),
           "batched_ms": round(batched, 3), "batched_speedup": round(plain / batched, 3),
           "value_batched": round(positions / (batched / 1e3), 1),
           "calls": nops, "work_items": nitems, "mode": md, "ctas_per_sm": cps,
           "tiles_per_item": {"predecessors": gt[0], "candidates": gt[1]},
           "autotune_ms": tune,
           "parity": {"golden": ("differ" if bad else "equal") if checked else "not recorded",
                      "slices_checked": checked, "mismatches": bad}}
    del jobs, pools
    torch.cuda.empty_cache()
    return rec


def run_e2e(a, jobs, stream, positions, mode):
    """Same steps through the C ABI with the inputs in pinned host memory:
    per step the H2D copy of L_prev and W_prev of every slice, the ply (the
    "wins" bitmaps stay resident in HBM, as the tables of a generation do)
    and the D2H copy of the results W(s) and L(s).  Steps alternate between
    two device buffer sets, each recorded in its own batch slot, so that
    step i+1's inputs go in and step i's results come out on the library's
    copy streams (ordered by tickets) while the kernels of the step between
    them run.  The host results of the last step are checked against the
    device buffers."""
    import torch

    import tb8gen_b200 as tbg
    from tb8gen_b200.plyjob import record_step

    names = ("L_prev", "W_prev", "T", "X")
    sets = [[tuple(getattr(j, n) for n in names) for j in jobs]]
    sets.append([(j.L_prev.clone(), j.W_prev.clone(), torch.zeros_like(j.T), torch.zeros_like(j.X))
                 for j in jobs])
    # the second set's step, recorded in batch slot 1
    for j, bufs in zip(jobs, sets[1]):
        for n, t in zip(names, bufs):
            setattr(j, n, t)
    tbg.batch_select(1)
    try:
        record_step(jobs)
    finally:
        tbg.batch_select(0)
        for j, bufs in zip(jobs, sets[0]):
            for n, t in zip(names, bufs):
                setattr(j, n, t)
    pin = lambda t: torch.empty(t.numel(), dtype=torch.uint8, pin_memory=True)
    host_in = []
    for j in jobs:
        hi = [pin(j.L_prev), pin(j.W_prev)]
        hi[0].copy_(j.L_prev)
        hi[1].copy_(j.W_prev)
        host_in.append(hi)
    host_out = [[(pin(j.T), pin(j.X)) for j in jobs] for _ in range(2)]
    torch.cuda.synchronize()
    h2d = sum(j.B * 2 for j in jobs)

    def run(nsteps):
        start = tbg.mark()
        in_t, mk, out_t = {}, {}, {}

        def put(i):
            b = i % 2
            after = mk[i - 2] if i >= 2 else start  # set b last read by step i-2
            t = 0
            for k, (hi, bufs) in enumerate(zip(host_in, sets[b])):
                tbg.copy_in(bufs[0], hi[0], after if k == 0 else 0)
                t = tbg.copy_in(bufs[1], hi[1], ticket=True)
            in_t[i] = t

        put(0)
        for i in range(nsteps):
            b = i % 2
            if i + 1 < nsteps:
                put(i + 1)
            tbg.join(in_t[i])
            if i >= 2:
                tbg.join(out_t[i - 2])  # set b's results of step i-2 are out
            tbg.batch_select(b)
            tbg.batch_run(mode)
            mk[i] = tbg.mark()
            t = 0
            for k, (ho, bufs) in enumerate(zip(host_out[b], sets[b])):
                tbg.copy_out(ho[0], bufs[2], mk[i] if k == 0 else 0)
                t = tbg.copy_out(ho[1], bufs[3], ticket=True)
            out_t[i] = t
        tbg.join(out_t[nsteps - 1])
        tbg.batch_select(0)
        return (nsteps - 1) % 2

    run(2)
    torch.cuda.synchronize()
    steps = max(2, a.steps)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    last = run(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    for ho, bufs in zip(host_out[last], sets[last]):
        assert torch.equal(ho[0], bufs[2].cpu()) and torch.equal(ho[1], bufs[3].cpu()), \
            "host results differ from the device's"
    return {"value": round(positions / (ms / 1e3), 1), "unit": UNIT, "ms_per_step": round(ms, 3),
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d, "steps": steps,
            "pipeline": "two buffer sets in two batch slots; copies on the library's copy "
                        "streams overlap the other set's kernels"}


def cpu_oracle(material, nthreads):
    from oracle import oracle as orc

    if orc.ref_available():
        return orc.Ref(material, nthreads), "reference"
    return orc.Port(material), "port"


def run_cpu_baseline(a, jobs, inputs=None, oracle=None):
    """The reference's CPU ply (oracle/_ref, all host cores) on one whole
    slice-ply of the first job (no sampling): the W step, the epilogue, the
    L step and the verify over all N positions of the slice.  Returns the
    baseline record and the finished CPU ply (its outputs() are compared
    with the engine's)."""
    from oracle.plyjob_cpu import CpuSlicePly

    cores = os.cpu_count() or 1
    job = inputs if inputs is not None else jobs[0]
    material = job["material"] if isinstance(job, dict) else job.material
    if oracle is None:
        O, kind = cpu_oracle(material, cores)
    else:
        O, kind = oracle
    O.set_stub(1, 3)
    threads = getattr(O, "nthreads", 1)
    c = CpuSlicePly(O, job, 1.0)
    t = c.step()
    return {"value": round(c.N / t, 1), "unit": UNIT, "cores": threads,
            "kind": kind, "seconds_measured": round(t, 3),
            "sample": (f"one whole slice-ply of {material} slice {c.s} ({c.N} positions, "
                       f"no sampling): W step, epilogue, L step and verify"),
            "phase_s": {k: round(v, 4) for k, v in c.times.items()}}, c


GOLDEN_SLICE = os.path.join(ROOT, "tests", "golden", "slice_ply.json")


def golden_slice(material, s, p, seed):
    """The reference's recorded outputs of one slice-ply
    (tests/golden/slice_ply.json, made by tests/golden/make_slice_golden.py
    with the reference's workers), or None."""
    try:
        with open(GOLDEN_SLICE) as f:
            return json.load(f).get(f"{material}/{s}/{p}/{seed}")
    except OSError:
        return None


def compare_outputs(eng: dict, ref: dict) -> list:
    """Names of the bitmaps that differ between the engine's outputs
    (device tensors) and the reference's (numpy arrays)."""
    import numpy as np

    bad = [k for k in sorted(set(eng) | set(ref)) if k not in eng or k not in ref]
    for k in sorted(set(eng) & set(ref)):
        if not np.array_equal(eng[k].cpu().numpy(), ref[k]):
            bad.append(k)
    return bad


def slice_parity(jobs, ref_ply=None):
    """Bit-exactness of the workload's slice-plies: the digests and counts
    of the recorded reference outputs where the golden file has the job,
    and a byte-for-byte comparison with a reference ply run in this process
    on the same inputs (ref_ply, for the first job)."""
    from tb8gen_b200.plyjob import output_digests

    out = {"golden": "not recorded", "jobs_checked": 0}
    bad = []
    for j in jobs:
        g = golden_slice(j.material, j.s, j.p, j.seed)
        if g is None or j.pool is not None:
            continue
        counts = list(j.counts())
        dig = output_digests(j.outputs())
        out["jobs_checked"] += 1
        if counts != g["counts"] or dig != g["sha256"]:
            bad.append(f"{j.material}/{j.s}: counts {counts} vs {g['counts']}, digests differ "
                       f"in {[k for k in dig if dig[k] != g['sha256'].get(k)]}")
        if out["jobs_checked"] == 1:
            out["counts"] = counts
            out["digests"] = {k: v[:16] for k, v in dig.items()}
    if out["jobs_checked"]:
        out["golden"] = "differ" if bad else "equal"
    if ref_ply is not None:
        diff = compare_outputs(jobs[0].outputs(), ref_ply.outputs())
        out["vs_reference"] = "differ" if diff else "equal"
        out["vs_reference_bitmaps"] = len(ref_ply.outputs())
        if diff:
            bad.append(f"{jobs[0].material}/{jobs[0].s} differs from the reference ply in {diff}")
    out["mismatches"] = bad
    return out


def slice_config(workload, spec, positions):
    """The `config` of a ply workload, the same dict in both arms."""
    mats = sorted({m for m, _, _, _ in spec})
    cfg = {"workload": workload, "slices": len(spec), "materials": mats,
           "positions_per_step": positions,
           "p": sorted({p for _, _, p, _ in spec}), "seed": spec[0][3],
           "l2": "inputs larger than L2 (>=16 MB bitmaps, many per step)"}
    if len(spec) == 1:
        cfg["slice"] = spec[0][1]
    return cfg


def run_reference(a, rank, world, local, spec=None):
    """Reference arm: the reference's own CPU workers (oracle/_ref) on all
    host cores, inputs built on the CPU by the same workers (no engine).
    A step is one whole slice-ply of the workload's first slice (for the
    slice workload, the whole workload); the first step's outputs are
    checked against the recorded reference digests."""
    if rank != 0:
        return None
    from oracle.plyjob_cpu import CpuSlicePly, inputs_from_oracle
    from tb8gen_b200.plyjob import output_digests

    cores = os.cpu_count() or 1
    full_spec = [spec] if spec else workload_spec(a.workload)
    mat, s, p, seed = full_spec[0]
    O, kind = cpu_oracle(mat, cores)
    O.set_stub(1, 3)
    t0 = time.time()
    inputs = inputs_from_oracle(O, mat, s, p, seed)
    prep = time.time() - t0
    per_step = []
    parity = {"golden": "not recorded"}
    ply = CpuSlicePly(O, inputs, 1.0)
    for i in range(a.warmup + a.steps):
        per_step.append(ply.step())
        if i == 0:
            g = golden_slice(mat, s, p, seed)
            counts = list(ply.counts())
            dig = output_digests(ply.outputs())
            parity = {"counts": counts, "digests": {k: v[:16] for k, v in dig.items()}}
            if g is not None:
                parity["golden"] = "equal" if (counts == g["counts"] and dig == g["sha256"]) \
                    else "differ"
    ts = per_step[a.warmup:] or per_step
    tm = statistics.median(ts)
    v = inputs["N"] / tm
    threads = getattr(O, "nthreads", 1)
    cfg = slice_config(a.workload, [(mat, s, p, seed)], inputs["N"])
    if len(full_spec) > 1:
        cfg["note"] = (f"the reference arm runs the first of the workload's {len(full_spec)} "
                       "slices per step")
    sample = (f"one whole slice-ply of {mat} slice {s} ({inputs['N']} positions, no "
              f"sampling) per step")
    return {
        "metric": METRIC, "value": round(v, 1), "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(tm * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded Bernoulli bitmaps, seeded 7-piece stub)",
        "config": cfg,
        "impl": "reference",
        "cpu_baseline": {"value": round(v, 1), "unit": UNIT, "cores": threads,
                         "kind": kind, "sample": sample},
        "e2e": {"value": round(v, 1), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "parity": parity,
        "phase_s": {k: round(x, 4) for k, x in ply.times.items()},
        "input_prep_s": round(prep, 1),
        "seconds_timed": round(sum(ts), 1),
    }


# ------------------------------------------------------------ probe workload
PROBE_METRIC = "probe positions/s (bit-exact)"
PROBE_MATS = ("KRRRvKRR", "KQRvKRR")
PROBE_SEED = 3
PROBE_BLOCK = 65536


class ProbeSet:
    """The probe workload on the device: the synthetic table and the seeded
    positions (and result buffer) of each material."""

    def __init__(self, n_total, rank=0, materials=PROBE_MATS):
        import torch

        import tb8gen_b200 as tbg

        self.items = []
        self.materials = tuple(materials)
        per = n_total // len(self.materials)
        for m in self.materials:
            t = tbg.DeviceTable(m, PROBE_SEED, 3)
            q = torch.empty(per * 16, dtype=torch.uint8, device="cuda")
            failed = tbg.gen_positions(m, PROBE_SEED + 1000 * rank, q)
            if failed:
                raise RuntimeError(f"{failed} draws found no legal {m} position")
            out = torch.empty(per, dtype=torch.int8, device="cuda")
            self.items.append((m, t, q, out))
        # the workload's queries: the engine's compact 8-byte form (squares
        # 0-6, side to move); the 16-byte tbg_query form is timed beside it
        self.q8 = [tbg.compact_queries(q) for _, _, q, _ in self.items]
        self.positions = per * len(self.materials)
        self.table_bytes = sum(t.bytes for _, t, _, _ in self.items)

    def probe(self):
        for (_, t, _, out), q8 in zip(self.items, self.q8):
            t.probe8(q8, out, 0)

    def probe16(self):
        for _, t, q, out in self.items:
            t.probe(q, out, 0)

    def close(self):
        for _, t, _, _ in self.items:
            t.close()


def probe_roundtrip(m, t, q):
    """encode -> decode -> re-encode of every query on the device; returns
    the number of indices that did not come back.  Both sides of these
    tables list their pieces in one order, so side 0's decode serves both;
    the decoded squares are re-encoded with the side to move of the table
    side (a symmetric table keeps black-to-move positions colour-flipped)."""
    import torch

    import tb8gen_b200 as tbg

    n = q.numel() // 16
    idx = torch.empty(n, dtype=torch.int64, device="cuda")
    side = torch.empty(n, dtype=torch.uint8, device="cuda")
    t.encode(q, idx, side)
    sq = torch.empty((n, 8), dtype=torch.uint8, device="cuda")
    t.decode(0, idx, sq)
    cols = tbg.table_to_query_columns(m)
    q2 = torch.zeros((n, 16), dtype=torch.uint8, device="cuda")
    q2[:, :len(cols)] = sq[:, cols]
    q2[:, 8] = side
    idx2 = torch.empty_like(idx)
    t.encode(q2.view(-1), idx2)
    return int((idx2 != idx).sum().item())


def write_sparse_tables(ps, per_mat, directory):
    """Table files for the reference's reader holding what a sample of the
    first `per_mat` queries of each material reads: the front of the image
    (header, code, index and size tables) and the touched blocks; the rest
    of each file is a hole.  Returns the host queries of the samples."""
    import torch

    import tb8gen_b200 as tbg
    from oracle import probe_ref as PR

    samples = []
    for m, t, q, _ in ps.items:
        qs = q[: per_mat * 16]
        n = qs.numel() // 16
        idx = torch.empty(n, dtype=torch.int64, device="cuda")
        side = torch.empty(n, dtype=torch.uint8, device="cuda")
        t.encode(qs, idx, side)
        img = t.image()
        path = os.path.join(directory, PR.table_file_name(m) + ".rtbw")
        sides = [0]
        try:
            t.layout(1)
            sides.append(1)
        except tbg.TbgError:
            pass  # a symmetric material: one side
        with open(path, "wb") as f:
            f.truncate(t.bytes)
            off0 = t.layout(0)[0]
            f.seek(0)
            f.write(img[:off0].cpu().numpy().tobytes())
            for b in sides:
                off, nb, _ = t.layout(b)
                blk = torch.unique((idx[side == b] >> 16))
                if blk.numel() == 0:
                    continue
                data = img[off: off + nb * PROBE_BLOCK].view(nb, PROBE_BLOCK)
                rows = data.index_select(0, blk).cpu().numpy()
                for k, row in zip(blk.cpu().numpy().tolist(), rows):
                    f.seek(off + k * PROBE_BLOCK)
                    f.write(row.tobytes())
        samples.append((m, qs.cpu().numpy().reshape(n, 16)))
    return samples


def time_reference_probe(directory, samples, seconds, threads):
    """The reference's probe_table (oracle/_ref/libtbprobe.so) over the
    samples on `threads` host threads, repeated until `seconds` pass;
    returns (positions/s, passes, results of the first pass)."""
    import threading

    import numpy as np

    from oracle import probe_ref as PR

    ref = PR.RefProbe(directory)
    if ref.found != len(samples):
        raise RuntimeError(f"reference found {ref.found} tables")
    first = {m: ref.probe(m, q) for m, q in samples}  # maps the tables, warms the page cache
    chunks = []
    for m, q in samples:
        pt = np.array(PR.material_pieces(m), dtype=np.uint8)
        for part in np.array_split(np.arange(len(q)), threads):
            if len(part):
                chunks.append((pt, np.ascontiguousarray(q[part]), np.zeros(len(part), np.int8)))
    import ctypes as C
    L = PR.probe_lib()
    total = sum(len(c[1]) for c in chunks)
    passes, t0 = 0, time.perf_counter()
    while True:
        per_thread = [chunks[i::threads] for i in range(threads)]

        def work(lst):
            for pt, qq, oo in lst:
                L.refp_probe(C.c_void_p(pt.ctypes.data), len(pt), C.c_void_p(qq.ctypes.data),
                             len(qq), C.c_void_p(oo.ctypes.data))
        ths = [threading.Thread(target=work, args=(lst,)) for lst in per_thread]
        for th in ths:
            th.start()
        for th in ths:
            th.join()
        passes += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    return total * passes / el, passes, first


def probe_cpu_baseline(ps, seconds, per_mat=8192):
    import shutil
    import tempfile

    threads = os.cpu_count() or 1
    d = tempfile.mkdtemp(prefix="tbprobe_")
    try:
        samples = write_sparse_tables(ps, per_mat, d)
        v, passes, first = time_reference_probe(d, samples, seconds, threads)
    finally:
        shutil.rmtree(d, ignore_errors=True)
    # the engine's answers for the same positions, bit for bit
    match = all(bool((first[m] == out[:per_mat].cpu().numpy()).all())
                for m, _, _, out in ps.items)
    return {"value": round(v, 1), "unit": "positions/s", "cores": threads, "kind": "reference",
            "sample": (f"the first {per_mat} positions of each material ({len(samples) * per_mat} "
                       f"probes) through the reference's probe_table on {threads} threads, "
                       f"{passes} passes; tables as sparse files holding the touched blocks"),
            "sample_bit_exact": match}


def run_probe(a, rank, world, local):
    import torch

    import tb8gen_b200 as tbg

    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    tbg.init()
    tbg.set_stream(stream)
    t0 = time.time()
    ps = ProbeSet(a.probe_n, rank, a.probe_materials.split(","))
    torch.cuda.synchronize()
    build_s = time.time() - t0

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(1.0)
    for _ in range(a.warmup):
        ps.probe()
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    n0 = tbg.launches()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    phases = []
    for _ in range(a.steps):
        ps.probe()
        phases.append([t.phase_ms() for _, t, _, _ in ps.items])
    e1.record(stream)
    torch.cuda.synchronize()
    launches = tbg.launches() - n0
    ms = e0.elapsed_time(e1) / a.steps
    clk = clocks.stop()
    ms = max_over_ranks(ms, world)
    value = ps.positions * world / (ms / 1e3)
    # the same batches in the 16-byte query form
    q0 = torch.cuda.Event(enable_timing=True)
    q1 = torch.cuda.Event(enable_timing=True)
    ps.probe16()
    q0.record(stream)
    for _ in range(a.steps):
        ps.probe16()
    q1.record(stream)
    torch.cuda.synchronize()
    ms16 = q0.elapsed_time(q1) / a.steps

    # dominant kernel: the block decode (k_probe_decode): a touched block's
    # stream is read once, from its start (found at open) to the block's
    # end; its device time from the library's events
    dec_ms = statistics.median(sum(p[0][1] for p in step) for step in phases)
    touched = sum(p[1] for p in phases[-1])

    def mean_stream(t):
        sb = nb = 0
        for side in (0, 1):
            try:
                sb += t.stream_bytes(side)
                nb += t.layout(side)[1]
            except tbg.TbgError:
                break
        return sb / max(nb, 1)

    alg = int(sum(phases[-1][i][1] * mean_stream(t) for i, (_, t, _, _) in enumerate(ps.items)))
    peak, peak_kind = measured_peak()
    achieved = alg / (dec_ms / 1e3) / 1e9
    tr = committed_traffic("k_probe_decode")
    roofline = {"bound": "hbm", "kernel": "k_probe_decode", "achieved": round(achieved, 1),
                "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "peak_source": peak_kind, "alg_bytes_per_launch": alg,
                "traffic": int(tr * touched) if tr else None,
                "issue_active_frac": committed_issue("k_probe_decode"),
                "issue": issue_roofline("k_probe_decode", touched, dec_ms, clk),
                "note": "algorithmic bytes = touched blocks x their tables' mean stream "
                        "bytes per block (each stream read once; the zero padding in front "
                        "of a stream is skipped); the rANS steps, not HBM, bound this kernel"}
    phase = {m: {"locate_ms": round(statistics.median(s[i][0][0] for s in phases), 3),
                 "decode_ms": round(statistics.median(s[i][0][1] for s in phases), 3),
                 "answer_ms": round(statistics.median(s[i][0][2] for s in phases), 3),
                 "touched_blocks": phases[-1][i][1]}
             for i, (m, _, _, _) in enumerate(ps.items)}

    # index round trip (encode, decode, re-encode) of every position
    r0 = torch.cuda.Event(enable_timing=True)
    r1 = torch.cuda.Event(enable_timing=True)
    r0.record(stream)
    bad = sum(probe_roundtrip(m, t, q) for m, t, q, _ in ps.items)
    r1.record(stream)
    torch.cuda.synchronize()
    rt_ms = r0.elapsed_time(r1)

    e2e = None
    if not a.no_e2e:
        e2e = run_probe_e2e(a, ps, stream, compact=True)
        e16 = run_probe_e2e(a, ps, stream, compact=False)
        e2e["value_query16"] = e16["value"]
        e2e["h2d_bytes_per_step_query16"] = e16["h2d_bytes_per_step"]
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        cpu = probe_cpu_baseline(ps, min(a.cpu_seconds, 20.0))
    line = {
        "metric": PROBE_METRIC, "value": round(value, 1), "unit": "positions/s", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (seeded legal positions, seeded synthetic rANS tables)",
        "config": {"workload": "probe", "materials": list(ps.materials),
                   "positions_per_step": ps.positions, "table_bytes": ps.table_bytes,
                   "block_bytes": PROBE_BLOCK, "seed": PROBE_SEED, "query_bytes": 8,
                   "l2": f"inputs larger than L2 ({ps.table_bytes / 1e9:.1f} GB of tables, "
                         f"{ps.positions * 8 / 1e9:.1f} GB of positions)"},
        "value_query16": round(ps.positions * world / (ms16 / 1e3), 1),
        "ms_per_step_query16": round(ms16, 4),
        "phases": phase, "table_build_s": round(build_s, 2),
        "index_roundtrip": {"ms": round(rt_ms, 3),
                            "positions_per_s": round(ps.positions / (rt_ms / 1e3), 1),
                            "mismatches": bad},
        "roofline": roofline, "gpu_launches": launches, "clocks": clk, "e2e": e2e,
        "cpu_baseline": cpu,
    }
    ps.close()
    return line


def run_probe_e2e(a, ps, stream, compact=True):
    """Probe batches through the C ABI from pinned host memory: per step the
    H2D copy of every query (8-byte compact form, or the 16-byte tbg_query
    form) and the D2H copy of every result.  Steps alternate between two
    device sets of queries and results, so that step i+1's queries go in and
    step i's results come out on the library's copy streams while the probes
    between them run.  The host results of the last step are checked against
    the device's."""
    import torch

    import tb8gen_b200 as tbg

    qs = ps.q8 if compact else [q for _, _, q, _ in ps.items]
    hq = [torch.empty(q.numel(), dtype=torch.uint8, pin_memory=True) for q in qs]
    for h, q in zip(hq, qs):
        h.copy_(q)
    outs = [out for _, _, _, out in ps.items]
    sets = [list(zip(qs, outs)),
            [(torch.empty_like(q), torch.empty_like(o)) for q, o in zip(qs, outs)]]
    ho = [[torch.empty(o.numel(), dtype=torch.int8, pin_memory=True) for o in outs]
          for _ in range(2)]
    tables = [t for _, t, _, _ in ps.items]
    torch.cuda.synchronize()

    def run(nsteps):
        start = tbg.mark()
        in_t, mk, out_t = {}, {}, {}

        def put(i):
            b = i % 2
            after = mk[i - 2] if i >= 2 else start  # set b's queries last read by step i-2
            t = 0
            for k, (h, (q, _)) in enumerate(zip(hq, sets[b])):
                t = tbg.copy_in(q, h, after if k == 0 else 0, ticket=True)
            in_t[i] = t

        put(0)
        for i in range(nsteps):
            b = i % 2
            if i + 1 < nsteps:
                put(i + 1)
            tbg.join(in_t[i])
            if i >= 2:
                tbg.join(out_t[i - 2])  # set b's results of step i-2 are out
            for t, (q, out) in zip(tables, sets[b]):
                if compact:
                    t.probe8(q, out, 0)
                else:
                    t.probe(q, out, 0)
            mk[i] = tbg.mark()
            t = 0
            for k, (r, (_, out)) in enumerate(zip(ho[b], sets[b])):
                t = tbg.copy_out(r, out, mk[i] if k == 0 else 0, ticket=True)
            out_t[i] = t
        tbg.join(out_t[nsteps - 1])
        return (nsteps - 1) % 2

    run(2)
    torch.cuda.synchronize()
    steps = max(2, a.steps)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    last = run(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    for r, (_, out) in zip(ho[last], sets[last]):
        assert torch.equal(r, out.cpu()), "host results differ from the device's"
    return {"value": round(ps.positions / (ms / 1e3), 1), "unit": "positions/s",
            "ms_per_step": round(ms, 3), "h2d_bytes_per_step": sum(h.numel() for h in hq),
            "d2h_bytes_per_step": sum(r.numel() for r in ho[0]), "steps": steps,
            "query_bytes": 8 if compact else 16,
            "pipeline": "two query/result sets; copies on the library's copy streams "
                        "overlap the other set's probes"}


def run_probe_reference(a, rank, world, local):
    """Reference arm of the probe workload: the reference's probe_table on
    all host cores.  The tables and positions are made on the device (the
    reference has no table writer); only the reference's CPU probe is timed,
    one pass over a 16,384-position sample per step."""
    if rank != 0:
        return None
    import shutil
    import tempfile

    import torch

    import tb8gen_b200 as tbg

    torch.cuda.set_device(local)
    tbg.init()
    ps = ProbeSet(a.probe_n, 0, a.probe_materials.split(","))
    per_mat = 8192
    threads = os.cpu_count() or 1
    d = tempfile.mkdtemp(prefix="tbprobe_")
    try:
        samples = write_sparse_tables(ps, per_mat, d)
        per_step = []
        for _ in range(a.warmup + a.steps):
            v, _, _ = time_reference_probe(d, samples, 0.0, threads)
            per_step.append(v)
    finally:
        shutil.rmtree(d, ignore_errors=True)
        ps.close()
    v = statistics.median(per_step[a.warmup:] or per_step)
    n = per_mat * len(ps.materials)
    return {
        "metric": PROBE_METRIC, "value": round(v, 1), "unit": "positions/s", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(n / v * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (seeded legal positions, seeded synthetic rANS tables)",
        "config": {"workload": "probe", "materials": list(ps.materials),
                   "positions_per_step": n, "note": "a step is one pass over the sample"},
        "impl": "reference",
        "cpu_baseline": {"value": round(v, 1), "unit": "positions/s", "cores": threads,
                         "kind": "reference",
                         "sample": f"{per_mat} positions of each material per step, "
                                   f"probe_table on {threads} threads"},
        "e2e": {"value": round(v, 1), "unit": "positions/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


# ------------------------------------------------------------ serving loop
SERVE_METRIC = "serving positions/s (continuous batching), p50/p99 latency"
SERVE_PLY = ("KRRRvKRRR", "KQRvKRRR", "KQRRvKRR")


def run_serve(a, rank, world, local):
    """A seeded Poisson stream (seed 4) of 70% single-slice ply jobs on the
    mix materials and 30% probe batches of 1k-1M positions on the probe
    tables, served with continuous batching under an HBM admission budget
    (pinned-host spill), at each rate of the sweep; beside it the same
    stream served one request at a time (plain serial launches)."""
    import torch

    import tb8gen_b200 as tbg
    from tb8gen_b200.serve import GpuExecutor, Scheduler, make_requests, summarize

    torch.cuda.set_device(local)
    tbg.init()
    tbg.set_stub(1)
    pool_n = 1 << 20
    tables, pools = {}, {}
    for m in PROBE_MATS:
        tables[m] = tbg.DeviceTable(m, PROBE_SEED, 3)
        q = torch.empty(pool_n * 16, dtype=torch.uint8, device="cuda")
        tbg.gen_positions(m, 4, q)
        pools[m] = tbg.compact_queries(q).cpu().pin_memory()  # 8-byte queries
        del q
    ex = GpuExecutor(SERVE_PLY, tables, pools, slots=a.serve_slots,
                     budget_bytes=int(a.serve_budget_gb * 1e9), probe_max=1_000_000,
                     query_bytes=8)
    rates = [float(r) for r in a.serve_rates.split(",")]
    base = make_requests(a.serve_jobs, 1.0, SERVE_PLY, PROBE_MATS, seed=4, pool_n=pool_n)

    def at_rate(rate):
        return [type(r)(**{**r.__dict__, "arrival": r.arrival / rate}) for r in base]

    # warm-up: every table bitmap the stream touches is built once, probe
    # scratch grows to its largest batch
    for m, t in tables.items():
        q = torch.empty(1_000_000 * 8, dtype=torch.uint8, device="cuda")
        q.copy_(pools[m][:1_000_000 * 8])
        o = torch.empty(1_000_000, dtype=torch.int8, device="cuda")
        tbg.set_stream(torch.cuda.current_stream())
        t.probe8(q, o, 0)
        del q, o
    torch.cuda.synchronize()
    t0 = time.time()
    Scheduler(ex, a.serve_slots).run(at_rate(1e9))
    torch.cuda.synchronize()
    warm_s = time.time() - t0

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(1.0)
    n0 = tbg.launches()
    sweep = []
    for rate in rates:
        reqs = at_rate(rate)
        recs, mk = Scheduler(ex, a.serve_slots).run(reqs)
        cb = summarize(recs, mk)
        recs1, mk1 = Scheduler(ex, 1).run(reqs)
        se = summarize(recs1, mk1)
        sweep.append({"rate_per_s": rate, "continuous": cb, "serial": se,
                      "speedup": round(cb["positions_per_s"] / se["positions_per_s"], 3)})
    launches = tbg.launches() - n0
    clk = clocks.stop()
    top = sweep[-1]
    ply = [r for r in base if r.kind == "ply"]
    prb = [r for r in base if r.kind == "probe"]
    ply_pos = sum(ex.mpools[r.material].m.size for r in ply)
    h2d = sum(r.n * 8 for r in prb)  # compact 8-byte queries
    d2h = sum(2 * ex.mpools[r.material].m.bytes for r in ply) + sum(r.n for r in prb)
    value = top["continuous"]["positions_per_s"]
    peak, peak_kind = measured_peak()
    alg = ALG_BYTES_PER_POS * ply_pos
    achieved = alg / top["continuous"]["makespan_s"] / 1e9
    line = {
        "metric": SERVE_METRIC, "value": value, "unit": "positions/s", "n_gpus": world,
        "steps": len(rates), "warmup": 1,
        "ms_per_step": round(1e3 * top["continuous"]["makespan_s"], 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32/u64",
        "data": "synthetic (seeded Poisson request stream, seeded inputs and tables)",
        "config": {"workload": "serve", "jobs": len(base), "ply_jobs": len(ply),
                   "probe_jobs": len(prb), "ply_materials": list(SERVE_PLY),
                   "probe_materials": list(PROBE_MATS), "slots": a.serve_slots,
                   "budget_gb": a.serve_budget_gb, "rates_per_s": rates, "seed": 4,
                   "l2": "inputs larger than L2 (slice bitmaps and tables of GBs)"},
        "sweep": sweep,
        "p50_ms": top["continuous"]["p50_ms"], "p99_ms": top["continuous"]["p99_ms"],
        "serial_positions_per_s": top["serial"]["positions_per_s"],
        "memory": {"peak_gb": round(ex.peak / 1e9, 2), "spills": ex.spills,
                   "reloads": ex.reloads, "builds": ex.builds},
        "warmup_s": round(warm_s, 2),
        "roofline": {"bound": "hbm", "kernel": "ply and probe mix",
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 5), "peak_source": peak_kind,
                     "traffic": None,
                     "note": "ply algorithmic bytes (0.875 B/position) over the top-rate makespan"},
        "gpu_launches": launches, "clocks": clk,
        "e2e": {"value": value, "unit": "positions/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "note": "every request moves its payload and result through pinned host memory"},
        "cpu_baseline": None,
    }
    for t in tables.values():
        t.close()
    return line


# ------------------------------------------------------------ fixpoint
FIX_METRIC = "fixpoint ply positions/s (streamed, host tier)"


def parse_tbgen(stderr):
    times, stats = [], {}
    for line in stderr.splitlines():
        if line.startswith("time "):
            f = line.split()
            kind = f[1]
            kv = dict(x.split("=") for x in f[2:])
            times.append((kind, float(kv["ms"]), int(kv["positions"])))
        elif line.startswith("stats "):
            stats = {k: int(v) for k, v in (x.split("=") for x in line.split()[1:])}
    return times, stats


def fixpoint_parity(material, counts):
    """The generation's count lines against the reference program's run of
    the same material and stub (tests/golden/fixpoint_<material>.json, made
    by tests/golden/make_fixpoint_golden.py from the reference's whole
    generation): every line, or the leading lines of a generation cut short
    by --fix-max-ply."""
    path = os.path.join(ROOT, "tests", "golden", f"fixpoint_{material}.json")
    if not os.path.exists(path):
        return {"vs_reference": "not recorded"}
    with open(path) as f:
        ref = json.load(f)["counts"]
    mine = [c for c in counts if not c.startswith("sum ")]
    n = min(len(mine), len(ref))
    same = n > 0 and mine[:n] == ref[:n] and len(mine) <= len(ref)
    return {"vs_reference": "equal" if same else "differ", "count_lines_compared": n,
            "reference_lines": len(ref),
            "source": "the reference program's whole generation (tb8gen_stub, stub seed 1 mod 3)"}


def run_fixpoint(a, rank, world, local):
    """The whole generation of one material (calc_sub, illegal and mate,
    then calc_L_n / calc_W_n until no bitmap changes) by the C host driver
    in streamed mode: planes in host memory, a device window of slices.
    The same generation in resident mode must print the same counts."""
    import torch

    from tb8gen_b200 import build

    if rank != 0:
        return None
    tbgen = build.build_host()
    mat = a.fix_material
    # -c 16: a digest of 16 seeded slices of every half-ply's output, so
    # that the streamed and the resident run are compared slice-exactly
    base = [tbgen, "-s", "1", "-m", "3", "-p", "-c", "16"]
    if a.fix_max_ply:
        base += ["-n", str(a.fix_max_ply)]
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(1.0)
    t0 = time.time()
    r = subprocess.run(base + ["-S", mat], capture_output=True, text=True, timeout=3000)
    wall = time.time() - t0
    clk = clocks.stop()
    if r.returncode != 0:
        raise RuntimeError("tbgen failed: " + r.stderr[-2000:])
    times, stats = parse_tbgen(r.stderr)
    counts = [l.strip() for l in r.stdout.splitlines() if " = " in l]
    r2 = subprocess.run(base + [mat], capture_output=True, text=True, timeout=3000)
    counts2 = [l.strip() for l in r2.stdout.splitlines() if " = " in l]
    t2, _ = parse_tbgen(r2.stderr)
    ms = sum(t for _, t, _ in times)
    pos = sum(p for _, _, p in times)
    alg = sum((0.5 if k.startswith("w") else 0.375) * p for k, _, p in times)
    value = pos / (ms / 1e3)
    peak, peak_kind = measured_peak()
    achieved = alg / (ms / 1e3) / 1e9
    cpu = None
    if not a.no_cpu:
        from oracle.plyjob_cpu import inputs_from_oracle

        O, kind = cpu_oracle(mat, os.cpu_count() or 1)
        O.set_stub(1, 3)
        cpu, _ = run_cpu_baseline(a, None, inputs=inputs_from_oracle(O, mat, 96, 0.01, 1),
                                  oracle=(O, kind))
    plies = stats.get("plies", 0)
    return {
        "metric": FIX_METRIC, "value": round(value, 1), "unit": "positions/s", "n_gpus": world,
        "steps": len(times), "warmup": 0, "ms_per_step": round(ms / max(len(times), 1), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded 7-piece stub; the generation itself is deterministic)",
        "config": {"workload": "fixpoint", "material": mat, "mode": "streamed",
                   "plies": plies, "half_plies": len(times),
                   "note": "a step is one half-ply (calc_W_n or calc_L_n) over all 462 slices; "
                           "the W, L, X and capture planes stream through page-locked host "
                           "memory, the two wins planes stay in HBM",
                   "l2": "slice planes of the whole material stream through the device"},
        "total_s": round(wall, 2), "half_ply_ms_total": round(ms, 1),
        "resident_half_ply_ms_total": round(sum(t for _, t, _ in t2), 1),
        "counts_match_resident": counts == counts2 and r2.returncode == 0,
        "parity": fixpoint_parity(mat, counts),
        "count_lines": len(counts), "last_counts": counts[-4:],
        "slice_digests_compared": sum(1 for c in counts if c.startswith("sum ")),
        "slices_per_digest": 16,
        "roofline": {"bound": "hbm", "kernel": "half-ply (all kernels)",
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 5), "peak_source": peak_kind,
                     "traffic": None,
                     "note": "0.5 B (W) / 0.375 B (L) per position over the half-ply time; "
                             "host-tier copies included"},
        "gpu_launches": stats.get("launches"), "clocks": clk,
        "e2e": {"value": round(value, 1), "unit": "positions/s",
                "h2d_bytes_per_step": stats.get("h2d_bytes", 0) // max(len(times), 1),
                "d2h_bytes_per_step": stats.get("d2h_bytes", 0) // max(len(times), 1),
                "note": "streamed mode: the W, L, X and capture planes of every slice move "
                        "through host memory"},
        "cpu_baseline": cpu,
    }


def main():
    a = parse()
    rank, world, local = dist_env()
    if world > 1:
        import datetime

        import torch.distributed as dist
        import torch
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        if a.workload == "fixpoint":
            line = None
            if a.impl == "reference":
                # a whole generation by the reference takes hours on the host
                # cores: its arm times the reference's slice-ply of the same
                # material (slice 96, sources Bernoulli(0.01))
                line = run_reference(a, rank, world, local, (a.fix_material, 96, 0.01, 1))
                if line:
                    line["metric"] = FIX_METRIC
            else:
                line = run_fixpoint(a, rank, world, local)
        elif a.workload == "serve":
            line = None if a.impl == "reference" else run_serve(a, rank, world, local)
            if a.impl == "reference" and rank == 0:
                line = {"impl": "reference",
                        "unavailable": "the reference has no serving loop; its per-job CPU "
                                       "costs are the slice and probe reference arms"}
        elif a.workload == "probe":
            line = (run_probe_reference if a.impl == "reference" else run_probe)(a, rank, world,
                                                                                  local)
        elif a.impl == "reference":
            line = run_reference(a, rank, world, local)
        else:
            line = run_engine(a, rank, world, local)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
            par = line.get("parity") or {}
            mixpar = ((line.get("mix") or {}).get("parity") or {}).get("golden")
            probe_ok = ((line.get("probe") or {}).get("cpu_baseline") or {}).get(
                "sample_bit_exact", True)
            if "differ" in (par.get("golden"), par.get("vs_reference"), mixpar) or \
                    probe_ok is False:
                sys.stderr.write("bench: outputs differ from the reference: "
                                 f"{par.get('mismatches')}\n")
                sys.exit(1)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
