#!/usr/bin/env python
"""Benchmark of the SPEEDY column physics on B200.

Metric: physics columns/s (higher is better).  One step = one physics-tendency pass over the
workload's columns with inputs resident in HBM.  Default workload: the ragged ensemble
(32xT21, 16xT31, 8xT42, 4xT85, 1xT170 = 466,944 columns, half-ish at 16 levels), seeded
synthetic fields.  Inputs plus outputs of one step (~200 MB) exceed the 126 MB L2.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--workload ensemble|t425|t31] [--mode batched|plain]

Under torchrun each rank runs its own copy of the workload (weak scaling, no collective on the
data path); the timing is the max over ranks.  ``--impl reference`` times the CPU port of the
reference physics (the oracle) on the host cores on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# DRAM bytes (read + write) per column of the dominant kernel (ensemble_fused) and its warp
# instructions per launch, from one ncu capture each (the summaries under profiles/ give the
# commands): T425 from a --set full capture of one plain call (196.8 MB read + 174.2 MB
# written, 216.9 M warp instructions); the ensemble from the dram__bytes / inst_executed
# metrics of one fused launch of the benchmark's step (96.2 MB read + 60.4 MB written, 103.8 M
# warp instructions; one block per tile, the autotuner's pick); the adjoint (ensemble_adjoint, T170
# with 16 levels) from a --set full capture of one VJP.  Part of each launch's writes is still
# in L2 when the kernel ends, so the write share reads low.
NCU_TRAFFIC_PER_COLUMN = {"ensemble": (96.215296e6 + 60.369920e6) / 466944,
                          "t425": (196.767232e6 + 174.180096e6) / 819200}
NCU_WARP_INSTRUCTIONS = {"ensemble": 103782785.0, "t425": 216850069.0,
                         "adjoint_t170": 129642118.0}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="ensemble", choices=["ensemble", "t425", "t31"])
    ap.add_argument("--mode", default="batched", choices=["batched", "plain"])
    ap.add_argument("--no-plain", action="store_true", help="skip timing the plain path")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--sections", default="t425,adjoint,serving,held_suarez",
                    help="extra single-GPU sections: t425, adjoint, serving, held_suarez "
                         "(comma list, or none)")
    ap.add_argument("--serving-requests", type=int, default=400)
    return ap.parse_args()


def workload_members(pkg, name, rank=0):
    syn = pkg.synthetic
    if name == "ensemble":
        return syn.ensemble_members(base_seed=1000 + 1000 * rank)
    if name == "t425":
        return [syn.t425_instance(seed=425 + rank)]
    return [syn.config0_instance(seed=rank, lfluxland=True)]


def workload_config(name, members, mode):
    cols = sum(m.columns for m in members)
    c8 = sum(m.columns for m in members if m.kx == 8)
    desc = {"ensemble": "ragged ensemble 32xT21+16xT31+8xT42+4xT85+1xT170, 8/16 levels",
            "t425": "T425 1280x640, 16 levels", "t31": "T31 96x48 aquaplanet, 8 levels"}[name]
    return {"workload": desc, "members": len(members), "columns": cols, "columns_kx8": c8,
            "columns_kx16": cols - c8, "mode": mode,
            "l2": "inputs+outputs per step exceed the 126 MB L2" if cols > 100000 else
                  "L2 flushed between steps"}


# ---------------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while it runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
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
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------------------------
def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def max_over_ranks(ms, dist, device):
    """The slowest rank's time (every rank takes this collective at the same point)."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([float(ms)], device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def pcie_copy_ms(h2d, d2h, dev, reps=10):
    """Time of one pinned host->device copy of h2d bytes and one device->host copy of d2h bytes
    running at once on two streams (CUDA events, after three warm-up rounds)."""
    import torch
    h_up = torch.empty(h2d, dtype=torch.uint8, pin_memory=True)
    h_dn = torch.empty(d2h, dtype=torch.uint8, pin_memory=True)
    d_up = torch.empty(h2d, dtype=torch.uint8, device=dev)
    d_dn = torch.empty(d2h, dtype=torch.uint8, device=dev)
    s_up, s_dn = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    cur = torch.cuda.current_stream(dev)

    def both():
        s_up.wait_stream(cur)
        s_dn.wait_stream(cur)
        with torch.cuda.stream(s_up):
            d_up.copy_(h_up, non_blocking=True)
        with torch.cuda.stream(s_dn):
            h_dn.copy_(d_dn, non_blocking=True)
        cur.wait_stream(s_up)
        cur.wait_stream(s_dn)

    for _ in range(3):
        both()
    torch.cuda.synchronize(dev)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(cur)
    for _ in range(reps):
        both()
    b.record(cur)
    torch.cuda.synchronize(dev)
    return a.elapsed_time(b) / reps


def run_b200(args):
    import torch
    pkg = importlib.import_module("jax-gcm_b200")

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)

    members = workload_members(pkg, args.workload, rank)
    cols = sum(m.columns for m in members)
    bytes_path = sum(pkg.synthetic.path_bytes(m.kx, m.columns) for m in members)
    bytes_min = sum(pkg.synthetic.fwd_bytes(m.kx, m.columns) for m in members)
    bytes_lvl = sum(pkg.synthetic.levelset_bytes(m.kx, m.columns) for m in members)

    # device-resident inputs and preallocated outputs
    runs = []
    for m in members:
        state, forcing, geom, date = pkg.instance_to_device(m, dev)
        phys = pkg.SpeedyPhysics(diagnostics=False)
        e3 = lambda: torch.empty((m.kx, m.ix, m.il), dtype=torch.float32, device=dev)
        e2 = lambda: torch.empty((m.ix, m.il), dtype=torch.float32, device=dev)
        out = dict(u_wind=e3(), v_wind=e3(), temperature=e3(), specific_humidity=e3(),
                   precnv=e2(), precls=e2())
        runs.append((m, state, forcing, geom, date, phys, out))

    def step_plain():
        for (_, state, forcing, geom, date, phys, out) in runs:
            phys.compute_tendencies(state, forcing, geom, date, out=out)

    ens = None
    if args.mode == "batched":
        ens = pkg.Ensemble([pkg.Member(st, fo, ge, out) for (_, st, fo, ge, _, _, out) in runs],
                           runs[0][4])
        ens.autotune()

        def step(marker=None):
            ens.forward(marker=marker)

        launches_per_step = 2
    else:
        def step(marker=None):
            step_plain()

        launches_per_step = 2 * len(runs)

    def barrier():
        if dist is not None:
            dist.barrier()

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1), dist, dev)

    # The timed region: K steps between two events.  A second pass records a marker event
    # between the two launches of every step (batched mode) so that each launch is timed alone;
    # a third runs steps back to back for at least a second while nvidia-smi samples the clocks
    # (the K-step region is a few milliseconds, shorter than one clock sample).
    marks = [(primed_event(), primed_event(), primed_event()) for _ in range(args.steps)]
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier()
    spec = ens is not None and ens.speculate
    redone0 = ens.redone() if spec else None
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    barrier()
    redone_timed = ens.redone() - redone0 if spec else None
    total_ms = max_over_ranks(e0.elapsed_time(e1), dist, dev)
    ms_step = total_ms / args.steps
    clocks = ClockSampler(dev.index)
    clocks.start()
    time.sleep(0.3)
    reps_1s = max(args.steps, int(1000.0 / max(ms_step, 1e-3)) + 1)
    c0 = torch.cuda.Event(enable_timing=True)
    c1 = torch.cuda.Event(enable_timing=True)
    c0.record()
    for _ in range(reps_1s):
        step()
    c1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms_step_1s = c0.elapsed_time(c1) / reps_1s
    if clk is not None:
        clk["window"] = f"{reps_1s} steps back to back, {c0.elapsed_time(c1):.0f} ms"
    barrier()
    # the two launches timed apart, in a separate pass of as many steps (a marker event between
    # them serialises them in plain stream order; the timed steps above overlap them)
    if ens is not None:
        for (a, m, b) in marks:
            a.record()
            step(marker=m)
            b.record()
        torch.cuda.synchronize()
    fused_ms = other_ms = None
    if ens is not None:
        first = sum(a.elapsed_time(m) for (a, m, b) in marks) / args.steps
        second = sum(m.elapsed_time(b) for (a, m, b) in marks) / args.steps
        # speculating: the fused launch, then the fixup; otherwise the level-set launch first
        fused_ms, other_ms = (first, second) if ens.speculate else (second, first)
    value = cols * world / (ms_step / 1e3)
    grid_blocks = ens.grid_blocks if ens is not None else None
    plain = None
    if args.mode == "batched" and not args.no_plain:
        pms = timed(step_plain, args.steps, args.warmup) / args.steps
        plain = {"value": round(cols * world / (pms / 1e3), 1), "ms_per_step": round(pms, 4),
                 "launches_per_step": 2 * len(runs),
                 "batched_over_plain": round(pms / ms_step, 2)}

    # Roofline of the dominant kernel, ensemble_fused (every column whole): the path's
    # algorithmic bytes, 4 (9 kx + 12) per column (u and v at every level read, the four
    # tendency planes and the precipitation written, once each), over its own event-timed
    # duration.  Beside it: the same over the whole step (both launches), the bytes the kernel
    # must move at least (4 (7 kx + 14): the physics reads u and v at the lowest level only),
    # and the level-set launch, whose reads of T, q, phi and psa repeat the fused launch's.
    peak, peak_kind = load_peaks()
    kern_ms = fused_ms if fused_ms is not None else ms_step
    two = fused_ms is not None
    achieved = bytes_path / (kern_ms / 1e3) / 1e9
    traffic = NCU_TRAFFIC_PER_COLUMN.get(args.workload)
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                "kernel": ("ensemble_fused" if two
                           else "ensemble_fused + ensemble_fixup (one forward per member)"),
                "kernel_ms": round(kern_ms, 4),
                "algorithmic_bytes_per_launch": bytes_path,
                "bytes_per_column": "4 (9 kx + 12)",
                "traffic": (round(traffic * cols) if traffic else None),
                "traffic_over_algorithmic": (round(traffic * cols / bytes_path, 3)
                                             if traffic else None),
                "kernel_minimum_bytes": bytes_min,
                "kernel_minimum_frac": round(bytes_min / (kern_ms / 1e3) / 1e9 / peak, 4),
                "step": {"ms": round(ms_step, 4),
                         "achieved_gbs": round(bytes_path / (ms_step / 1e3) / 1e9, 1),
                         "frac": round(bytes_path / (ms_step / 1e3) / 1e9 / peak, 4)}}
    if two and ens.speculate:
        roofline["fixup_launch"] = {
            "kernel": "ensemble_fixup", "ms": round(other_ms, 4),
            "members_redone_in_timed_steps": redone_timed,
            "note": "each member's cloud-top level set is predicted from the previous step "
                    "and checked on the device; the fixup redoes the members whose prediction "
                    "missed and returns at once when none did"}
    elif two:
        roofline["levelset_launch"] = {
            "kernel": "ensemble_levelset", "ms": round(other_ms, 4), "bytes_read": bytes_lvl,
            "achieved_gbs": round(bytes_lvl / (other_ms / 1e3) / 1e9, 1)}
    # the issue bound: one warp instruction per scheduler per cycle, with the instruction count
    # of the ncu capture and the SM clock sampled here
    insts = NCU_WARP_INSTRUCTIONS.get(args.workload)
    issue = None
    if insts and clk and world == 1:
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        peak_issue = sms * 4 * clk["sm_mhz"] * 1e6
        ach = insts / (kern_ms / 1e3)
        issue = {"bound": "issue", "unit": "warp instructions/s", "achieved": round(ach, 1),
                 "peak": round(peak_issue, 1), "frac": round(ach / peak_issue, 4),
                 "warp_instructions_per_launch": insts, "sm_mhz": clk["sm_mhz"]}

    # end to end through the public API with host buffers (pinned), H2D + D2H timed
    e2e = None
    if not args.no_e2e and ens is not None:
        # batched: HostPipeline, one packed upload and one packed download per step,
        # double-buffered so that uploads, compute and downloads of consecutive steps overlap
        pipe = pkg.batched.HostPipeline(
            [pkg.Member(st, fo, ge) for (_, st, fo, ge, _, _, _) in runs], runs[0][4])
        for i, r in enumerate(runs):
            pipe.set_state(i, r[1])
        h2d, d2h = pipe.h2d_bytes, pipe.d2h_bytes
        nsteps = max(3, args.steps // 2)

        def pipe_steps(k):
            pipe.begin()
            for _ in range(k):
                pipe.submit()
            pipe.end()

        pipe_steps(max(3, args.warmup))
        torch.cuda.synchronize()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        pipe_steps(nsteps)
        e1.record()
        torch.cuda.synchronize()
        barrier()
        e2e_ms = max_over_ranks(e0.elapsed_time(e1), dist, dev) / nsteps
        del pipe
    elif not args.no_e2e:
        host = []
        h2d = d2h = 0
        for (m, state, forcing, geom, date, phys, out) in runs:
            hs = {}
            for name, t in [("u", state.u_wind), ("v", state.v_wind), ("t", state.temperature),
                            ("q", state.specific_humidity), ("phi", state.geopotential),
                            ("psa", state.normalized_surface_pressure)]:
                hs[name] = torch.empty(t.shape, dtype=t.dtype, pin_memory=True).copy_(t.cpu())
                h2d += t.numel() * 4
            ho = {k: torch.empty(v.shape, dtype=v.dtype, pin_memory=True)
                  for k, v in out.items() if k in ("temperature", "specific_humidity",
                                                   "u_wind", "v_wind", "precnv", "precls")}
            d2h += sum(v.numel() * 4 for v in ho.values())
            host.append((hs, ho))

        def e2e_step():
            for (hs, ho), (m, state, forcing, geom, date, phys, out) in zip(host, runs):
                state.u_wind.copy_(hs["u"], non_blocking=True)
                state.v_wind.copy_(hs["v"], non_blocking=True)
                state.temperature.copy_(hs["t"], non_blocking=True)
                state.specific_humidity.copy_(hs["q"], non_blocking=True)
                state.geopotential.copy_(hs["phi"], non_blocking=True)
                state.normalized_surface_pressure.copy_(hs["psa"], non_blocking=True)
                if ens is None:
                    phys.compute_tendencies(state, forcing, geom, date, out=out)
            if ens is not None:
                ens.forward()
            for (hs, ho), (m, state, forcing, geom, date, phys, out) in zip(host, runs):
                for k, v in ho.items():
                    v.copy_(out[k], non_blocking=True)
            torch.cuda.current_stream().synchronize()

        e2e_ms = (timed(e2e_step, max(3, args.steps // 2), max(3, args.warmup)) /
                  max(3, args.steps // 2))
    if not args.no_e2e:
        copy_ms = pcie_copy_ms(h2d, d2h, dev)
        e2e = {"value": cols * world / (e2e_ms / 1e3), "unit": "columns/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": round(e2e_ms, 4),
               # the bus bound: the step's upload and download bytes alone, as one pinned copy
               # each on two streams at once (no compute)
               "pcie_copy_ms": round(copy_ms, 4),
               "frac_of_pcie_copy": round(copy_ms / e2e_ms, 3),
               "path": ("batched.HostPipeline: one packed upload, spd_ensemble_fwd and one packed "
                        "download per step, consecutive steps overlapped" if ens is not None
                        else "per-member copies and spd_fwd calls")}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(members)

    sections = {}
    wanted = [x for x in args.sections.split(",") if x and x != "none"]
    if world == 1:
        del runs, ens
        torch.cuda.empty_cache()
        if "t425" in wanted:
            sections["t425"] = t425_section(pkg, dev, peak, peak_kind,
                                            clk["sm_mhz"] if clk else None)
        if "adjoint" in wanted:
            sections["adjoint"] = adjoint_section(pkg, dev, peak, peak_kind,
                                                  clk["sm_mhz"] if clk else None)
        if "serving" in wanted:
            sections["serving"] = serving_section(pkg, dev, args.serving_requests)
        if "held_suarez" in wanted:
            sections["held_suarez"] = held_suarez_section(pkg, dev, peak, peak_kind)

    if rank == 0:
        line = {"metric": "physics columns/s", "value": round(value, 1), "unit": "columns/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(ms_step, 4), "ms_per_step_1s_loop": round(ms_step_1s, 4),
                "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded generators with the workload's shapes and distributions)",
                "config": workload_config(args.workload, members, args.mode),
                "roofline": roofline, "issue_roofline": issue, "cpu_baseline": cpu, "e2e": e2e,
                "clocks": clk,
                "plain": plain, "grid_blocks": grid_blocks,
                "gpu_launches": launches_per_step * args.steps,
                "gpu_launches_note": "launches of this library's kernels in the K timed steps"}
        line.update(sections)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def primed_event():
    """A timing event whose CUDA event exists (torch creates it on the first record)."""
    import torch
    e = torch.cuda.Event(enable_timing=True)
    e.record()
    return e


def event_ms(fn, reps, warmup=3):
    """Mean device milliseconds of fn() over reps calls (events on the current stream)."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def held_suarez_section(pkg, dev, peak, peak_kind):
    """Held-Suarez forcing (spd_held_suarez) on T425 with 16 levels: one element-wise launch,
    HBM-bound; its bytes are u, v, T read and four tendency planes written per level and column
    plus psa once per column, 4 (7 kx + 1) B per column (370 MB per call, above the L2)."""
    import torch
    inst = pkg.synthetic.t425_instance()
    st, fo, ge, da = pkg.instance_to_device(inst, dev)
    hs = pkg.HeldSuarezPhysics()
    out = {k: torch.empty_like(st.temperature) for k in ("u_wind", "v_wind", "temperature",
                                                          "specific_humidity")}
    call = lambda: hs.compute_tendencies(st, fo, ge, da, out=out)
    ms = event_ms(call, 20, warmup=5)
    cols = inst.columns
    nbytes = 4 * (7 * inst.kx + 1) * cols
    bw = nbytes / (ms / 1e3) / 1e9
    return {"workload": "T425 1280x640, 16 levels, one instance", "columns": cols,
            "ms_per_call": round(ms, 4), "columns_per_s": round(cols / (ms / 1e3), 1),
            "algorithmic_bytes_per_call": nbytes, "hbm_gbs": round(bw, 1), "peak_gbs": peak,
            "peak_kind": peak_kind, "hbm_frac": round(bw / peak, 4), "kernel": "hs_vec4"}


def t425_section(pkg, dev, peak, peak_kind, sm_mhz=None):
    """T425 (1280x640, 16 levels): the plain drop-in call, its two launches timed apart, and 24
    consecutive calls captured in one CUDA graph."""
    import torch
    inst = pkg.synthetic.t425_instance()
    st, fo, ge, da = pkg.instance_to_device(inst, dev)
    phys = pkg.SpeedyPhysics(diagnostics=False)
    e3 = lambda: torch.empty((inst.kx, inst.ix, inst.il), dtype=torch.float32, device=dev)
    e2 = lambda: torch.empty((inst.ix, inst.il), dtype=torch.float32, device=dev)
    out = dict(u_wind=e3(), v_wind=e3(), temperature=e3(), specific_humidity=e3(),
               precnv=e2(), precls=e2())
    call = lambda marker=None: phys.compute_tendencies(st, fo, ge, da, out=out, marker=marker)
    reps = 24
    marks = [(primed_event(), primed_event(), primed_event()) for _ in range(reps)]
    for _ in range(3):
        call()
    torch.cuda.synchronize()
    for (a, m, b) in marks:
        a.record()
        call(marker=m)
        b.record()
    torch.cuda.synchronize()
    marked_ms = sum(a.elapsed_time(b) for (a, m, b) in marks) / reps
    call_ms = event_ms(call, reps)  # the drop-in call as used: the two launches overlapped
    first = sum(a.elapsed_time(m) for (a, m, b) in marks) / reps
    second = sum(m.elapsed_time(b) for (a, m, b) in marks) / reps
    spec = phys.speculating()
    col_ms, first_ms = (first, second) if spec else (second, first)
    # 24 calls in one graph
    s = torch.cuda.Stream(dev)
    s.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(s):
        call()
    torch.cuda.current_stream(dev).wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for _ in range(24):
            call()
    graph_ms = event_ms(g.replay, 5, warmup=3) / 24
    cols = inst.columns
    nbytes = pkg.synthetic.path_bytes(inst.kx, cols)
    nmin = pkg.synthetic.fwd_bytes(inst.kx, cols)
    bw = nbytes / (col_ms / 1e3) / 1e9
    out_d = {"workload": "T425 1280x640, 16 levels, one instance", "columns": cols,
             "path_algorithmic_bytes_per_call": nbytes,
             "plain_call_ms": round(call_ms, 4),
             "plain_call_launches_apart_ms": round(marked_ms, 4),
             ("fixup_launch_ms" if spec else "levelset_launch_ms"): round(first_ms, 4),
             "fused_launch_ms": round(col_ms, 4),
             "graph_24_calls_ms_per_call": round(graph_ms, 4),
             "columns_per_s_plain": round(cols / (call_ms / 1e3), 1),
             "columns_per_s_graph": round(cols / (graph_ms / 1e3), 1),
             "speculating": spec,
             "fused_launch_hbm_gbs": round(bw, 1), "peak_gbs": peak, "peak_kind": peak_kind,
             "fused_launch_hbm_frac": round(bw / peak, 4),
             "fused_launch_kernel_minimum_frac": round(nmin / (col_ms / 1e3) / 1e9 / peak, 4),
             "plain_call_hbm_frac": round(nbytes / (call_ms / 1e3) / 1e9 / peak, 4),
             "graph_call_hbm_frac": round(nbytes / (graph_ms / 1e3) / 1e9 / peak, 4)}
    t = NCU_TRAFFIC_PER_COLUMN.get("t425")
    if t:
        out_d["fused_launch_traffic"] = round(t * cols)
    if sm_mhz and NCU_WARP_INSTRUCTIONS.get("t425"):
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        peak_issue = sms * 4 * sm_mhz * 1e6
        ach = NCU_WARP_INSTRUCTIONS["t425"] / (col_ms / 1e3)
        out_d["fused_launch_issue_frac"] = round(ach / peak_issue, 4)
        out_d["issue_roofline_note"] = ("warp instructions per launch from ncu over one "
                                        "instruction per scheduler per cycle at the sampled "
                                        "SM clock")
    del g
    return out_d


def adjoint_section(pkg, dev, peak=None, peak_kind=None, sm_mhz=None):
    """Adjoint at T42 (128x64 = 8,192 columns, 8 levels): one VJP call beside one forward call,
    and the 48-step rollout VJP with checkpoints every 8 steps; plus the VJP at T170x16 with
    its place against HBM (B_vjp = 4 (10 kx + 15) bytes per column) and instruction issue."""
    import torch
    res = {}
    for label, (ix, il, kx) in (("t42_k8", (128, 64, 8)), ("t170_k16", (512, 256, 16))):
        inst = pkg.synthetic.land_instance(42, ix, il, kx)
        st, fo, ge, da = pkg.instance_to_device(inst, dev)
        phys = pkg.SpeedyPhysics(diagnostics=False)
        gen = torch.Generator(device=dev).manual_seed(0)
        ct = pkg.PhysicsTendency(*(torch.randn(st.temperature.shape, generator=gen, device=dev)
                                   for _ in range(4)))
        vjp_ms = event_ms(lambda: pkg.adjoint.vjp(phys, st, fo, ge, da, ct), 20)
        fwd_ms = event_ms(lambda: phys.compute_tendencies(st, fo, ge, da), 20)
        r = {"columns": inst.columns, "vjp_ms": round(vjp_ms, 4), "forward_ms": round(fwd_ms, 4),
             "vjp_columns_per_s": round(inst.columns / (vjp_ms / 1e3), 1),
             "vjp_over_forward": round(vjp_ms / fwd_ms, 2)}
        if label == "t42_k8":
            roll_ms = event_ms(lambda: pkg.rollout.rollout_vjp(None, st, fo, ge, da, ct,
                                                               nsteps=48, checkpoint_every=8),
                               2, warmup=3)
            r["rollout48_vjp_ms"] = round(roll_ms, 2)
            r["rollout48_checkpoint_every"] = 8
        else:
            nbytes = 4 * (10 * kx + 15) * inst.columns
            r["algorithmic_bytes"] = nbytes
            if peak:
                r["hbm_frac_of_call"] = round(nbytes / (vjp_ms / 1e3) / 1e9 / peak, 4)
                r["peak_kind"] = peak_kind
            if sm_mhz:
                sms = torch.cuda.get_device_properties(dev).multi_processor_count
                ach = NCU_WARP_INSTRUCTIONS["adjoint_t170"] / (vjp_ms / 1e3)
                r["issue_frac_of_call"] = round(ach / (sms * 4 * sm_mhz * 1e6), 4)
        res[label] = r
    return res


def serving_section(pkg, dev, n_requests):
    """The request stream (Poisson, 200 req/s, 80/20 tendency/VJP, 1-32 members at T21-T170,
    8 or 16 levels) under a 120 GB budget: continuous batching against the plain per-request
    drop-in, and both at saturation (every request arriving at once)."""
    import gc
    import torch
    S = pkg.serving
    src = S.synthetic_source()
    reqs = S.poisson_stream(seed=1, rate=200.0, n=n_requests)
    sat = S.poisson_stream(seed=2, rate=0.0, n=max(50, n_requests // 4))
    for r in reqs + sat:
        for k in r.members:
            src(k)
    budget = 120 << 30
    out = {"workload": "Poisson 200 req/s, 80/20 tendency/VJP, 1-32 members, T21-T170, 8/16 "
                       "levels, 120 GB budget; member state resident before the stream",
           "requests": n_requests}
    for mode in ("batched", "plain"):
        # the device pool is reserved once at startup, the size of the admission budget less
        # the adjoint and forward scratch
        be = S.CudaBackend(dev, mode=mode, reserve_bytes=budget - (1 << 30))
        warm = S.Scheduler(be, src, budget, mode=mode)
        warm.run([S.Request(S.TENDENCY, list(r.members)) for r in reqs[:8]] +
                 [S.Request(S.VJP, list(r.members)) for r in reqs[:2]])
        for label, stream in (("stream", reqs), ("saturation", sat)):
            # one unmeasured pass first: the first batches of a new size grow the pinned host
            # cache (a pinned allocation stalls the loop for milliseconds to tens of them) and
            # the device arena, a one-off cost of a server's warm-up
            pre = S.Scheduler(be, src, budget, mode=mode)
            pre.prefetch([k for r in stream for k in r.members])
            pre.run([S.Request(r.kind, list(r.members), r.arrival, r.seed) for r in stream],
                    timeout_s=600)
            del pre
            sch = S.Scheduler(be, src, budget, mode=mode)
            # member state is resident before traffic arrives (a resident-state service)
            sch.prefetch([k for r in stream for k in r.members])
            fin = sch.run([S.Request(r.kind, list(r.members), r.arrival, r.seed) for r in stream],
                          timeout_s=600)
            st = S.latency_stats(fin)
            st.update({k: round(v, 4) for k, v in S.overlap_stats(sch.items).items()})
            st["launches"] = {k: v for k, v in sch.stats.items() if k.startswith("launches")}
            st["uploads_during_run"] = sch.stats.get("uploads", 0)
            st["prefetched_members"] = sch.stats.get("prefetched", 0)
            st["peak_budget_bytes"] = sch.peak
            # the loop's passes over 5 ms (wall, CPU and context switches), longest first
            st["slow_passes"] = len(sch.slow_passes)
            st["slowest_passes"] = sorted(sch.slow_passes, key=lambda p: -p["wall_ms"])[:4]
            out[f"{mode}_{label}"] = {k: (round(v, 3) if isinstance(v, float) else v)
                                      for k, v in st.items()}
            del sch, fin
        # release this backend's pool before the next one reserves its own
        del be, warm
        gc.collect()
        torch.cuda.empty_cache()
    b, p = out["batched_stream"], out["plain_stream"]
    out["p50_ms"], out["p99_ms"] = b["p50_ms"], b["p99_ms"]
    out["plain_p50_ms"], out["plain_p99_ms"] = p["p50_ms"], p["p99_ms"]
    out["saturation_columns_per_s"] = out["batched_saturation"]["columns_per_s"]
    out["plain_saturation_columns_per_s"] = out["plain_saturation"]["columns_per_s"]
    return out


def cpu_baseline(members, min_seconds=10.0):
    """The compiled CPU restatement of the reference physics (oracle/cpu_port.cpp: float32,
    -O3 without fast-math, OpenMP) over the whole workload on every host core, repeated for at
    least ``min_seconds``; columns/s.  The NumPy port (the oracle) on one core beside it as a
    cross-check."""
    from oracle import cpu_port
    from oracle import speedy_oracle as O
    cores = os.cpu_count() or 1
    batch = cpu_port.Batch(members)
    batch.run(nthreads=cores)
    passes, t0 = 0, time.perf_counter()
    while True:
        batch.run(nthreads=cores)
        passes += 1
        el = time.perf_counter() - t0
        if el >= min_seconds:
            break
    value = passes * batch.columns / el
    # NumPy cross-check: one pass over a sample of members, one core
    sample = members[:: max(1, len(members) // 8)]
    np_cols, np_secs = 0, 0.0
    for m in sample:
        args = m.oracle_args(O.default_parameters())
        t1 = time.perf_counter()
        O.compute_tendencies(*args)
        np_secs += time.perf_counter() - t1
        np_cols += m.columns
    return {"value": round(value, 1), "unit": "columns/s", "cores": cores, "kind": "port",
            "sample": f"{passes} passes of the compiled C++ port of the reference physics "
                      f"(oracle/cpu_port.cpp, float32, -O3, no fast-math, OpenMP) over all "
                      f"{len(members)} members ({batch.columns} columns) on {cores} threads, "
                      f"{el:.1f} s",
            "numpy_port_one_core": {"value": round(np_cols / np_secs, 1),
                                    "sample": f"the NumPy oracle over {len(sample)} of the "
                                              f"members ({np_cols} columns), one core"}}


def run_reference(args):
    """The reference arm: the compiled CPU port of the reference physics on all host cores,
    one step = one pass over the workload's members."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import cpu_port
    pkg = importlib.import_module("jax-gcm_b200")
    members = workload_members(pkg, args.workload, 0)
    cores = os.cpu_count() or 1
    batch = cpu_port.Batch(members)
    for _ in range(max(1, args.warmup)):
        batch.run(nthreads=cores)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        batch.run(nthreads=cores)
    el = time.perf_counter() - t0
    value = args.steps * batch.columns / el
    cols = batch.columns
    line = {"impl": "reference", "metric": "physics columns/s", "value": round(value, 1),
            "unit": "columns/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(el / args.steps * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generators with the workload's shapes and distributions)",
            "config": workload_config(args.workload, members, "reference"),
            "cpu_baseline": {"value": round(value, 1), "unit": "columns/s", "cores": cores,
                             "kind": "port",
                             "sample": f"each step: the compiled C++ port of the reference "
                                       f"physics (oracle/cpu_port.cpp, float32, -O3, no "
                                       f"fast-math, OpenMP) over all {len(members)} members "
                                       f"({cols} columns) on {cores} threads"},
            "e2e": {"value": round(value, 1), "unit": "columns/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
