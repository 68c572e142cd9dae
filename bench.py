"""Benchmark of the plain FP64 FrehdC step on B200.

Workload (one GPU): a 4096 x 4096 subgrid basin at dx = 2 m, dt = 0.5 s, 4 x 4
fine pixels per cell, about 30% of the cells above low tide, Manning n = 0.025,
one scalar, CG to ||r|| < 1e-12 ||b|| from x = 0 (the reference's solver set-up).
Synthetic, seeded deck (frehdc_b200.deck); the state of a 4096^2 domain is far
larger than the 126 MB L2, so no flush is needed between steps.

Printed JSON line (rank 0):
  value        cell-steps/s of all ranks, device time (CUDA events on the
               library's stream) of the K timed steps, inputs resident in HBM
  e2e          the same metric through the C ABI from host buffers: deck upload
               and initialisation, K steps each returning its monitorCFL
               statistics to the host, final state download
  roofline     the CG kernel (the dominant one): algorithmic bytes per launch
               (cg_bytes_per_cell: 48 B/cell set-up + 72 B/cell per iteration)
               over its mean event-timed launch duration, against the measured
               HBM copy peak
  cpu_baseline the reference program itself (oracle/_ref, one core) on a
               256 x 256 window of the same deck
and the other forms of the metric, each a sub-record with its own config:
  mixed        the same 4096^2 deck in mixed precision (FP32 inner CG in FP64
               refinement): device rate, and eta/u/v/scalar/volume errors against
               the FP64 run after 1000 steps
  batched      256 seeded basins, sides 64-1024, 2 scalars, mixed precision, one
               batch (five launches per step, graph-replayed), autotuned packing:
               rate, the same mix stepped one domain at a time in FP64, the
               speed-up, and errors against FP64 after 500 steps
  served       the head of a 2000-request stream (Poisson arrivals 50/s, sides
               64-2048, 100-2000 steps, 1-3 scalars), continuous batching in mixed
               precision: cell-steps/s, p50/p99 latency, errors of a sample of
               requests against FP64
With --gpus N (torchrun) every rank steps its own replica domain (the step does
not shard: one domain lives on one GPU), value sums them, time is the max over
ranks; the batched mix and the request stream are partitioned over the ranks.
--impl reference times the reference program on all host cores.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = ("cell-steps/s plain FP64 vs batched FP32+refine at ≤1e-6 m eta err; "
          "served p50/p99")
UNIT = "cell-steps/s"


SCHEDULES = {"single_sweep": 0, "two_phase": 1}  # FREHD_CG_SINGLE_SWEEP / FREHD_CG_TWO_PHASE


def c2_spec(n: int = 4096, steps: int = 1000, crop=None):
    from frehdc_b200 import deck as D
    return D.DeckSpec(nx=n, ny=n, dx=2.0, dt=0.5, steps=steps, seed=2024, dry_frac=0.3,
                      manning_n=0.025, crop=crop)


def c2_crop_spec(n_full: int, w: int, steps: int):
    """A w x w window of the full deck along its tidal (YP) edge."""
    s = c2_spec(n_full, steps)
    return s.replace(nx=w, ny=w, crop=(0, n_full - w, n_full, n_full))


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- helpers
def measured_hbm_peak():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_baseline_reference(steps: int, n_full: int, w: int = 256):
    """The reference program (oracle/_ref, stock allocator build) on one core."""
    from frehdc_b200 import deck as D
    from oracle import refrun
    if not refrun.available():
        return None
    from oracle import port
    spec = c2_crop_spec(n_full, w, steps)
    d = D.make_deck(spec, host=port)
    tmp = tempfile.mkdtemp(prefix="frehd_cpu_")
    D.write_reference_deck(d, tmp, binary_tables=True, host=port)
    t = refrun.time_run(tmp, steps)
    return {"value": t["cell_steps_per_s"], "unit": UNIT, "cores": 1, "kind": "reference",
            "cg_iters_per_step": t.get("cg_iters_per_step"),
            "sample": f"{w}x{w} window of the {n_full}^2 deck along its tidal edge, "
                      f"{steps} steps, reference program (frehdc5+ + laspack, SSOR-PCG as "
                      f"shipped) on 1 core, {t['seconds']:.1f} s"}


# ---------------------------------------------------------------- reference arm
def run_reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from frehdc_b200 import deck as D
    from oracle import port, refrun
    if not refrun.available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference oracle binaries (oracle/_ref) not built"}))
        return 0
    cores = os.cpu_count() or 1
    w = 256
    sample_steps = 40
    spec = c2_crop_spec(args.n, w, sample_steps)
    # the window's tables and bottoms come from the oracle's pre-processor: this
    # process loads no library of the product
    d = D.make_deck(spec, host=port)
    tmp = tempfile.mkdtemp(prefix="frehd_refarm_")
    D.write_reference_deck(d, tmp, binary_tables=True, host=port)
    total_steps = args.steps + args.warmup
    # every "step" of this arm is a bounded sample: all cores each run the
    # reference program over the window concurrently
    rates, its = [], []
    t_all0 = time.time()
    for s in range(total_steps):
        procs = [subprocess.Popen([refrun.TIMING_BIN, "time", tmp, str(sample_steps)],
                                  stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                 for _ in range(cores)]
        outs = [p.communicate()[0] for p in procs]
        secs = []
        for o in outs:
            for ln in o.splitlines():
                if ln.startswith("{"):
                    rec = json.loads(ln)
                    secs.append(rec["seconds"])
                    its.append(rec.get("cg_iters_per_step", float("nan")))
        if s >= args.warmup and len(secs) == cores:
            # concurrent step loops: all cells of all processes over the slowest loop
            rates.append(cores * w * w * sample_steps / max(secs))
    value = statistics.median(rates)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * (w * w * sample_steps * cores) / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": f"{w}x{w} window of the {args.n}^2 plain FP64 subgrid deck "
                               f"(reference cannot hold a {args.n}-cell tidal row: "
                               f"tideLocP[1000], configuration.h:60)",
                   "parallelism": f"{cores} independent reference processes"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"{cores} concurrent runs of the reference program, "
                                   f"{sample_steps} steps of a {w}^2 window each"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": time.time() - t_all0,
        # the work per cell-step differs from the 4096^2 domain's: the window's
        # SSOR-PCG needs fewer iterations per step than the large domain's
        # Jacobi-PCG (65 at 4096^2), which flatters the CPU rate
        "cg_iters_per_step": statistics.median(its) if its else None,
        "cg_preconditioner": "SSOR (the reference as shipped)",
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- GPU arm
def run_gpu_arm(args):
    import torch

    from frehdc_b200 import deck as D
    from frehdc_b200 import native

    ws, rank, local = dist_env()
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = local
    n = args.n
    extras = args.extras.split(",") if args.extras and args.extras != "none" else []
    spec = c2_spec(n, steps=max(args.steps + args.warmup, args.mixed_steps) + 5)
    t0 = time.time()
    deck = D.make_deck(spec)
    gen_s = time.time() - t0
    cfg = D.config_dict(deck)
    tide = D.tide_series(deck)
    N = n * n

    # ---- value: resident in HBM, device time of K steps
    dom = native.Domain(cfg, dev)
    dom.set_fine_bottoms(deck.zf, deck.r)
    dom.set_tide(tide)
    dom.set_solver(native.X0_ZERO)
    dom.set_cg_schedule(SCHEDULES[args.cg_schedule])
    if args.precision == "mixed":
        dom.set_precision(native.PRECISION_MIXED,
                          args.eps_inner if args.eps_inner is not None else 1e-5)
    dom.init(deck.bottom, deck.bottomXP, deck.bottomYP, deck.surf0, None, None, deck.S0)
    rc = dom.run(1, args.warmup)
    if rc != 0:
        raise RuntimeError(f"warm-up steps returned status {rc}")
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    dom.sync()
    dom.set_profiling(True)
    with ClockSampler(dev) as clk:
        rc = dom.run(1 + args.warmup, args.steps)
    dom.sync()
    if rc != 0:
        raise RuntimeError(f"timed steps returned status {rc}")
    kt = dom.kernel_times()
    st = dom.stats()
    dev_ms = _step_ms(kt)
    t_max = dev_ms
    if ws > 1:
        tt = torch.tensor([dev_ms], device=f"cuda:{dev}", dtype=torch.float64)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        t_max = float(tt.item())
    value = ws * N * args.steps / (t_max / 1e3)
    iters = kt["cg_iters"] / max(kt["steps"], 1)
    dom.set_profiling(False)

    # ---- e2e: through the C ABI from host buffers
    e2e = None if args.no_e2e else run_e2e(args, deck, cfg, tide, dev, ws, N)

    # ---- the other forms of the metric, each its own sub-record
    sub = {}
    if "mixed" in extras and args.precision == "fp64":
        sub["mixed"] = _guard(lambda: measure_mixed_domain(args, deck, cfg, tide, dev, ws, dom))
    dom.close()
    del deck
    if "batched" in extras:
        sub["batched"] = _guard(lambda: measure_batched(
            args, ws, rank, dev, 256, 64, 1024, 2, args.batched_total, "mixed",
            args.batched_steps, args.warmup))
    if "served" in extras:
        sub["served"] = _guard(lambda: measure_served(
            args, ws, rank, dev, 2000, args.served_requests, 64, 2048, 100, 2000, 3, 50.0,
            "mixed", args.served_cells_per_cta, 1e-4, 10))
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank != 0:
        return 0
    return report(args, kt, st, iters, t_max, value, ws, n, spec, gen_s, e2e, clk, sub)


def _guard(fn):
    """A sub-measurement's record, or its error: a failure there must not cost
    the headline line.  (Every rank takes the same collective steps either way:
    the sub-measurements gather only at their end.)"""
    t0 = time.time()
    try:
        rec = fn()
        rec["wall_s"] = round(time.time() - t0, 1)
        return rec
    except Exception as e:  # reported in the JSON line
        import traceback
        traceback.print_exc(file=sys.stderr)
        return {"error": f"{type(e).__name__}: {e}"}


def measure_mixed_domain(args, deck, cfg, tide, dev, ws, ref):
    """The mixed-precision form on the same domain (FP32 inner CG iterations in
    FP64 refinement): device time of K steps after W warm-up steps, then the run
    continued untimed to args.mixed_steps steps and its state compared with the
    FP64 domain `ref` (the plain measurement's, at step W+K) continued to the
    same step."""
    import torch

    from frehdc_b200 import native
    N = cfg["nx"] * cfg["ny"]
    W, K, S = args.warmup, args.steps, args.mixed_steps
    eps_inner = args.eps_inner if args.eps_inner is not None else 1e-5
    g = native.Domain(cfg, dev)
    g.set_fine_bottoms(deck.zf, deck.r)
    g.set_tide(tide)
    g.set_precision(native.PRECISION_MIXED, eps_inner)
    g.init(deck.bottom, deck.bottomXP, deck.bottomYP, deck.surf0, None, None, deck.S0)
    if g.run(1, W) != 0:
        raise RuntimeError("mixed warm-up failed")
    g.sync()
    g.set_profiling(True)
    if g.run(1 + W, K) != 0:
        raise RuntimeError("mixed timed steps failed")
    g.sync()
    kt = g.kernel_times()
    g.set_profiling(False)
    ms = _step_ms(kt)
    if ws > 1:
        t = torch.tensor([ms], device=f"cuda:{dev}", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    if S > W + K:
        if g.run(1 + W + K, S - W - K) != 0 or ref.run(1 + W + K, S - W - K) != 0:
            raise RuntimeError("mixed or FP64 continuation failed")
    names = ["surf", "uuXP", "vvYP", "S"]
    a, r = g.download(names), ref.download(names)
    import numpy as np
    err = _state_errors(a, r, N)
    err["S_max_abs"] = float(np.max(np.abs(a["S"][:N] - r["S"][:N])))
    va, vr = g.stats()["volume"], ref.stats()["volume"]
    err["volume_rel"] = abs(va - vr) / abs(vr)
    err["after_steps"] = max(S, W + K)
    err["against"] = "the FP64 run of the same deck and steps"
    inner = kt["cg_iters"] / max(kt["steps"], 1)
    g.close()
    return {"value": ws * N * K / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / K,
            "steps_timed": K, "warmup": W, "dtype": "f32+f64",
            "config": {"workload": f"{cfg['nx']}x{cfg['ny']} mixed FP32/FP64 (the plain "
                                   "workload's deck)", "eps_inner": eps_inner},
            "per_kernel_ms_per_step": {k: kt[k] / kt["steps"] for k in
                                       ("explicit_ms", "cg_ms", "update_geo_ms",
                                        "update_vel_ms", "finish_ms")},
            "cg_inner_iters_per_step": inner, "errors_vs_fp64": err}


def run_e2e(args, deck, cfg, tide, dev, ws, N):
    """The steps as a host program drives them through the C ABI: before each
    step the host queues the copy of that step's boundary input (its tidal
    level, from pinned host memory: frehd_domain_update_series), and each step
    hands its monitorCFL statistics back to the host (frehd_domain_step waits for
    them).  Host wall clock over the timed steps, after warm-up steps.  The deck's
    one-time upload and initialisation (2.8 GB at 4096^2) are timed on their own
    and reported in `with_setup`."""
    import numpy as np
    import torch

    from frehdc_b200 import native
    zf = np.ascontiguousarray(deck.zf)
    host_fields = [deck.bottom, deck.bottomXP, deck.bottomYP, deck.surf0, deck.S0]
    torch.cuda.synchronize(dev)
    ts0 = time.perf_counter()
    dom2 = native.Domain(cfg, dev)
    dom2.set_fine_bottoms(zf, deck.r)
    dom2.set_tide(tide)
    dom2.set_cg_schedule(SCHEDULES[args.cg_schedule])
    dom2.init(deck.bottom, deck.bottomXP, deck.bottomYP, deck.surf0, None, None, deck.S0)
    dom2.sync()
    setup_s = time.perf_counter() - ts0
    pinned = torch.empty(len(tide), dtype=torch.float64).pin_memory()
    pinned.copy_(torch.from_numpy(np.ascontiguousarray(tide)))
    base = pinned.data_ptr()

    def one(tt):
        dom2.update_series(native.SERIES_TIDE, tt, 1, base + 8 * tt)  # this step's input
        rc = dom2.step(tt)             # the step; its statistics come back to the host
        if rc != 0:
            raise RuntimeError(f"e2e step returned status {rc}")
    for s in range(args.warmup):
        one(1 + s)
    if ws > 1:
        torch.distributed.barrier()
    te0 = time.perf_counter()
    for s in range(args.steps):
        one(1 + args.warmup + s)
    e2e_s = time.perf_counter() - te0
    out = dom2.download(["surf", "uuXP", "vvYP", "S"])
    dom2.close()
    if ws > 1:
        tt = torch.tensor([e2e_s, setup_s], device=f"cuda:{dev}", dtype=torch.float64)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        e2e_s, setup_s = float(tt[0].item()), float(tt[1].item())
    setup_h2d = zf.nbytes + sum(a.nbytes for a in host_fields) + tide.nbytes
    return {"value": ws * N * args.steps / e2e_s, "unit": UNIT,
            "h2d_bytes_per_step": 8, "d2h_bytes_per_step": 72,
            "includes": "per step: the step's tidal level copied from pinned host memory "
                        "(frehd_domain_update_series), frehd_domain_step with its statistics "
                        "read back to the host; host wall clock",
            "with_setup": {"value": ws * N * args.steps / (e2e_s + setup_s), "setup_s": setup_s,
                           "setup_h2d_bytes": setup_h2d,
                           "includes": "the same steps plus domain creation, the deck upload "
                                       "(fine bottoms and fields) and initialisation"},
            "final_state_d2h_bytes": sum(a.nbytes for a in out.values())}


def cg_bytes_per_cell(iters: float, fp64: bool = True) -> float:
    """Compulsory DRAM bytes per cell of one single-sweep solve of `iters`
    iterations: set-up 48 B, then per iteration read r~, p, Hx, Hy, x~ and |Ct|
    and write r~, p and x~ (72 B in FP64; the FP32 inner iteration of the mixed
    form moves r~, p, d~, Hx, Hy in FP32, 32 B)."""
    return 48.0 + (72.0 if fp64 else 32.0) * iters


def report(args, kt, st, iters, t_max, value, ws, n, spec, gen_s, e2e, clk, sub=None):
    N = n * n
    peak, peak_kind = measured_hbm_peak()
    cg_launch_ms = kt["cg_ms"] / kt["steps"]
    fp64 = args.precision == "fp64"
    cg_cell = cg_bytes_per_cell(iters, fp64)
    cg_bytes = N * cg_cell
    achieved = cg_bytes / (cg_launch_ms / 1e3) / 1e9
    kname = {"single_sweep": "k_cg1 (persistent single-sweep Jacobi-PCG, one launch per step)",
             "two_phase": "k_cg (persistent two-phase Jacobi-PCG, one launch per step)"}
    roof = {"kernel": kname[args.cg_schedule], "bound": "hbm",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_kind": peak_kind, "traffic": None,
            "bytes_model": ("48 B/cell set-up + 72 B/cell per CG iteration" if fp64 else
                            "48 B/cell set-up + 32 B/cell per FP32 inner iteration (FP64 "
                            "refinement sweeps not counted)"),
            "bytes_per_cell": cg_cell,
            "cg_iters_per_step": iters, "launch_ms": cg_launch_ms}
    # DRAM traffic of one launch from the committed ncu summary (scaled from a
    # smaller capture; it describes the 4096^2 single-sweep solve only)
    prof = os.path.join(REPO, "profiles", "k_cg1_2048x2048_fp64.md")
    if args.cg_schedule == "single_sweep" and n == 4096 and args.precision == "fp64" and os.path.exists(prof):
        import re
        m = re.search(r"traffic_bytes_per_4096_launch:\s*([0-9.eE+]+)", open(prof).read())
        if m:
            roof["traffic"] = float(m.group(1))
            roof["traffic_source"] = "profiles/k_cg1_2048x2048_fp64.md (ncu, scaled by cells x iterations)"
    # the step: explicit + assembly 200 B, post-solve + scalar 208 B per cell, and the solve
    step_cell = 408.0 + cg_cell
    step_bytes = N * step_cell
    whole = step_bytes * args.steps / (t_max / 1e3) / 1e9
    cpu = None if args.no_cpu else cpu_baseline_reference(args.cpu_steps, n)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32+f64", "data": "synthetic",
        "config": {"workload": f"{n}x{n} {'plain FP64' if args.precision == 'fp64' else 'mixed FP32/FP64'}"
                               " subgrid basin (dx 2 m, dt 0.5 s, 4x4 fine, "
                               f"~30% dry at low tide, n 0.025, 1 scalar), CG eps 1e-12 from x=0",
                   "precision": args.precision,
                   "nx": n, "ny": n, "parallelism": f"{ws} replica domain(s), one per GPU",
                   "l2": "no flush: the domain state (>2 GB) exceeds the 126 MB L2",
                   "deck_seed": spec.seed, "deck_gen_s": round(gen_s, 1),
                   "cg_schedule": args.cg_schedule},
        "e2e": e2e,
        "roofline": roof,
        "step_roofline": {"bytes_per_cell_step": step_cell, "achieved": whole,
                          "peak": peak, "unit": "GB/s", "frac": whole / peak},
        "per_kernel_ms_per_step": {k: kt[k] / kt["steps"] for k in
                                   ("explicit_ms", "cg_ms", "update_geo_ms", "update_vel_ms",
                                    "finish_ms")},
        "gpu_launches": 5 * args.steps + 1,
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
        "last_step": st,
    }
    for k, v in (sub or {}).items():
        line[k] = v
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- batched / served forms
def mix_specs(n: int, seed: int, smin: int, smax: int, steps: int, scalars=(1, 1)):
    """Seeded mix of basins: sides log-uniform in [smin, smax] (multiples of 8),
    square or 1:4 (fair coin), depth 0.3-8 m, 0-40 % dry at low tide, tide
    amplitude 0.1-0.5 m, Manning n 0.02-0.04, dt 1 s, dx 10 m, 4x4 subgrid;
    each basin carries a number of scalars uniform in scalars = (lo, hi)."""
    import numpy as np

    from frehdc_b200 import deck as D
    rng = np.random.default_rng(seed)
    n_sc = np.random.default_rng(seed + 1).integers(scalars[0], scalars[1] + 1, size=n)
    out = []
    for k in range(n):
        side = float(np.exp(rng.uniform(np.log(smin), np.log(smax))))
        a = int(max(8, round(side / 8) * 8))
        if rng.random() < 0.5:
            nx = ny = a
        else:  # 1:4, same cell count scale
            nx, ny = max(8, (a // 2) // 8 * 8), max(8, (a * 2) // 8 * 8)
        out.append(D.DeckSpec(nx=nx, ny=ny, dx=10.0, dt=1.0, steps=steps, seed=seed * 1000 + k,
                              depth_min=0.3, depth_max=8.0,
                              dry_frac=float(rng.uniform(0.0, 0.4)) or None,
                              tide_amp=float(rng.uniform(0.1, 0.5)),
                              manning_n=float(rng.uniform(0.02, 0.04)),
                              n_scalars=int(n_sc[k])))
    return out


def _dist_init():
    """(world size, rank, device) of this process; under torchrun one process
    per GPU with an NCCL group used only for host-side gathers of metrics."""
    ws, rank, local = dist_env()
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def _dist_done(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def _step_ms(kt) -> float:
    return sum(kt[k] for k in ("explicit_ms", "cg_ms", "update_geo_ms", "update_vel_ms",
                               "finish_ms"))


def _state_errors(a: dict, ref: dict, n: int) -> dict:
    """Errors of a state against a reference state (both in the reference
    layout): eta absolute (m), face velocities relative to the reference's max."""
    import numpy as np

    def rel(f):
        sc = max(float(np.max(np.abs(ref[f][:n]))), 1e-300)
        return float(np.max(np.abs(a[f][:n] - ref[f][:n]))) / sc
    return {"eta_max_abs_m": float(np.max(np.abs(a["surf"][:n] - ref["surf"][:n]))),
            "u_max_rel": rel("uuXP"), "v_max_rel": rel("vvYP")}


def _worst(errs: list) -> dict | None:
    errs = [e for e in errs if e]
    return {k: max(e[k] for e in errs) for k in errs[0]} if errs else None


def _fp64_batch_run(decks, dev, budget, packing, cpc, steps):
    """Fresh FP64 domains of `decks` stepped `steps` times in one batch; the
    domains (released from the batch, still open) are returned."""
    from frehdc_b200 import native
    doms = [native.domain_from_deck(dk, device=dev) for dk in decks]
    b = native.Batch(budget, cpc, dev)
    b.set_cg_packing(packing)
    for g in doms:
        b.admit(g, 1)
    for _ in range(steps):
        b.step()
    b.sync()
    for sl in list(b.members):
        b.release(sl)
    b.close()
    return doms


def measure_batched(args, ws, rank, dev, n_mix, smin, smax, scalars, total_steps, precision,
                    K, W):
    """A mix of basins stepped as one batch (one launch per sub-step for all of
    them, replayed from a CUDA graph), against the same mix stepped one domain
    at a time through the single-domain API in FP64.

    Under torchrun the mix is partitioned across ranks by cell count
    (frehdc_b200.shard.balance); each rank batches its share on its own GPU and
    the slowest rank's device time sets the whole-job rate.  The batch runs W
    warm-up steps, K timed steps (device time, CUDA events on the batch's
    stream) and the rest of total_steps untimed; in the mixed form every basin's
    state after total_steps is compared with an FP64 run of the same steps (the
    FP64 domains of the plain-form timing, continued in an FP64 batch)."""
    import torch

    from frehdc_b200 import deck as D
    from frehdc_b200 import native, shard
    specs_all = mix_specs(n_mix, 77, smin, smax, total_steps + 5, (scalars, scalars))
    mine = shard.balance([sp.nx * sp.ny for sp in specs_all], ws)[rank]
    specs = [specs_all[i] for i in mine]
    t0 = time.time()
    decks = D.make_decks(specs)
    gen_s = time.time() - t0
    cells = [sp.nx * sp.ny for sp in specs]
    prec = native.PRECISION_MIXED if precision == "mixed" else native.PRECISION_FP64
    budget = args.budget_gb << 30
    # plain form: each domain alone (FP64), device time of its K steps
    ref = [native.domain_from_deck(dk, device=dev) for dk in decks]
    plain_ms = 0.0
    for g in ref:
        g.run(1, W)
        g.sync()
        g.set_profiling(True)
        g.run(1 + W, K)
        g.sync()
        plain_ms += _step_ms(g.kernel_times())
        g.set_profiling(False)
    # packing of the solve and inner tolerance from the autotuner, tuned on rank
    # 0's share and used by every rank (a given cells_per_cta selects CTA groups)
    tuning = None
    cpc, eps_inner = args.cells_per_cta, args.eps_inner
    packing = "cta_groups" if cpc > 0 else "tile_list"
    if cpc <= 0:
        from frehdc_b200 import autotune
        if rank == 0:
            tuning = autotune.tune(decks, budget, prec, device=dev)
        tuning = shard.broadcast(tuning, ws)
        cpc = tuning["best"]["cells_per_cta"]
        eps_inner = tuning["best"]["eps_inner"]
        packing = tuning["best"]["packing"]
        tpb = tuning["best"]["tiles_per_block"]
    else:
        tpb = args.tiles_per_block
    if eps_inner is None:
        eps_inner = 1e-4
    pk = native.BATCH_TILE_LIST if packing == "tile_list" else native.BATCH_CTA_GROUPS
    doms = [native.domain_from_deck(dk, device=dev, precision=prec, eps_inner=eps_inner)
            for dk in decks]
    b = native.Batch(budget, cpc if cpc > 0 else 1.0, dev)
    b.set_cg_packing(pk)
    b.set_stencil_tiles(tpb)
    for g in doms:
        b.admit(g, 1)
    for _ in range(W):
        b.step()
    b.sync()
    if ws > 1:
        torch.distributed.barrier()
    st = torch.cuda.ExternalStream(b.stream(), device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        e0.record(st)
        for _ in range(K):
            b.step()
        e1.record(st)
        e1.synchronize()
    batch_ms = e0.elapsed_time(e1)
    for _ in range(total_steps - W - K):
        b.step()
    b.sync()
    info = b.info()
    for sl in list(b.members):
        b.release(sl)
    b.close()
    errors = None
    if precision == "mixed":
        import numpy as np
        fb = native.Batch(budget, cpc if cpc > 0 else 1.0, dev)
        fb.set_cg_packing(pk)
        for g in ref:
            fb.admit(g, W + K + 1)
        for _ in range(total_steps - W - K):
            fb.step()
        fb.sync()
        for sl in list(fb.members):
            fb.release(sl)
        fb.close()
        # two noise floors of the FP64 run itself: the same steps with the
        # solve's sums added in the other packing's order (rounding only), and
        # with the CG tolerance tightened tenfold (another solution that meets
        # the same residual bound); wet/dry branches amplify either difference
        other = native.BATCH_CTA_GROUPS if pk == native.BATCH_TILE_LIST else native.BATCH_TILE_LIST
        names = ["surf", "uuXP", "vvYP"]
        ref_state = [(r.download(names), r.stats()["volume"]) for r in ref]

        def spread(run):  # each floor run's domains compared, then closed
            out = []
            for h, (rs, vr), dk in zip(run, ref_state, decks):
                f = _state_errors(h.download(names), rs, dk.spec.nx * dk.spec.ny)
                f["volume_rel"] = abs(h.stats()["volume"] - vr) / abs(vr)
                out.append(f)
                h.close()
            return out

        per = []
        for g, r, (rs, vr), dk in zip(doms, ref, ref_state, decks):
            n_ = dk.spec.nx * dk.spec.ny
            e = _state_errors(g.download(names), rs, n_)
            e["scalar_max_abs"] = max(float(np.max(np.abs(
                g.download_scalar(s_)[:n_] - r.download_scalar(s_)[:n_])))
                for s_ in range(1 + len(dk.tracers)))
            e["volume_rel"] = abs(g.stats()["volume"] - vr) / abs(vr)
            per.append(e)
        floor = spread(_fp64_batch_run(decks, dev, budget, other, 393216.0, total_steps))
        tight_decks = [dataclasses.replace(dk, spec=dataclasses.replace(dk.spec, eps=dk.spec.eps / 10))
                       for dk in decks]
        tfloor = spread(_fp64_batch_run(tight_decks, dev, budget, pk, cpc if cpc > 0 else 1.0,
                                        total_steps))
        over = lambda es: sum(1 for e in es if e["eta_max_abs_m"] > 1e-6)  # noqa: E731
        errors = {"mixed": _worst(per), "fp64_other_order": _worst(floor),
                  "fp64_tighter_eps": _worst(tfloor),
                  "domains_eta_over_1e-6": over(per), "domains_fp64_eta_over_1e-6": over(floor),
                  "domains_tight_eta_over_1e-6": over(tfloor),
                  "over_1e-6_both": sum(1 for a, c in zip(per, tfloor)
                                        if a["eta_max_abs_m"] > 1e-6 and c["eta_max_abs_m"] > 1e-6)}
    for g in doms + ref:
        g.close()
    parts = shard.gather({"batch_ms": batch_ms, "plain_ms": plain_ms, "cells": int(sum(cells)),
                          "domains": len(decks), "errors": errors, "clocks": clk.summary(),
                          "info": info, "gen_s": gen_s}, ws)
    t_batch = max(p["batch_ms"] for p in parts)
    t_plain = max(p["plain_ms"] for p in parts)
    total_cells = sum(p["cells"] for p in parts)
    total = float(total_cells) * K
    rec = {"value": total / (t_batch / 1e3), "unit": UNIT, "ms_per_step": t_batch / K,
           "steps_timed": K, "warmup": W, "steps_total": total_steps,
           "dtype": "f64" if precision == "fp64" else "f32+f64",
           "config": {"precision": precision,
                      "workload": f"{n_mix} seeded basins, sides log-uniform {smin}-{smax} "
                                  "(square or 1:4), dx 10 m, dt 1 s, depth 0.3-8 m, 0-40% dry, "
                                  "tide 0.1-0.5 m, n 0.02-0.04, 4x4 subgrid, "
                                  f"{scalars} scalar(s)",
                      "cells": int(total_cells), "packing": packing,
                      "cells_per_cta": cpc if packing == "cta_groups" else None,
                      "eps_inner": eps_inner if precision == "mixed" else None,
                      "stencil_tiles_per_block": tpb,
                      "sharding": "by cell count over ranks" if ws > 1 else None,
                      "deck_gen_s": round(max(p["gen_s"] for p in parts), 1)},
           "plain_form_same_mix": {"value": total / (t_plain / 1e3), "unit": UNIT,
                                   "note": "each domain stepped alone in FP64, device time of "
                                           "its kernels summed over the mix"},
           "batch": parts[0]["info"] if ws == 1 else [p["info"] for p in parts],
           "gpu_launches_timed": 5 * K, "clocks": parts[0]["clocks"]}
    rec["speedup_vs_plain_form"] = rec["value"] / rec["plain_form_same_mix"]["value"]
    if ws > 1:
        rec["per_rank"] = [{"domains": p["domains"], "cells": p["cells"],
                            "batch_ms": p["batch_ms"]} for p in parts]
    if tuning is not None:
        rec["autotune"] = tuning
    if precision == "mixed":
        errs = [p["errors"] for p in parts if p["errors"]]
        if errs:
            rec["errors_vs_fp64"] = {**_worst([e["mixed"] for e in errs]), "after_steps": total_steps,
                                     "domains_over_1e-6_m": sum(e["domains_eta_over_1e-6"] for e in errs)}
            rec["fp64_vs_fp64_other_sum_order"] = {
                **_worst([e["fp64_other_order"] for e in errs]),
                "domains_over_1e-6_m": sum(e["domains_fp64_eta_over_1e-6"] for e in errs),
                "note": "the same FP64 steps with the solve's partial sums added in the other "
                        "packing's order: the spread any rounding difference grows to"}
            rec["fp64_vs_fp64_tighter_eps"] = {
                **_worst([e["fp64_tighter_eps"] for e in errs]),
                "domains_over_1e-6_m": sum(e["domains_tight_eta_over_1e-6"] for e in errs),
                "domains_over_1e-6_m_in_both": sum(e["over_1e-6_both"] for e in errs),
                "note": "the same FP64 steps with the CG tolerance 1e-13 instead of 1e-12: the "
                        "spread between two solutions that both meet the FP64 residual bound; "
                        "in_both counts domains over 1e-6 m here and in the mixed run"}
    return rec


def measure_served(args, ws, rank, dev, n_stream, n_req, smin, smax, steps_lo, steps_hi,
                   scalars_max, rate, precision, cells_per_cta, eps_inner, check_every):
    """The first n_req requests of a seeded stream of n_stream (Poisson
    arrivals at `rate`/s, sides log-uniform smin-smax, steps uniform in
    steps_lo..steps_hi, 1..scalars_max scalars), served by continuous batching
    (the native server).  Under torchrun each request goes to the rank with the
    least work assigned so far, in arrival order (frehdc_b200.shard.assign_stream).
    Every check_every-th request (mixed precision) is run again alone in FP64
    afterwards and its final state compared with the served one."""
    import numpy as np

    from frehdc_b200 import deck as D
    from frehdc_b200 import native, serve, shard
    rng = np.random.default_rng(5)
    specs = mix_specs(n_stream, 91, smin, smax, 10, (1, scalars_max))[:n_req]
    steps = rng.integers(steps_lo, steps_hi + 1, size=n_stream)[:n_req]
    arr = serve.poisson_arrivals(n_stream, rate, 17)[:n_req]
    owner = shard.assign_stream(arr, [sp.nx * sp.ny * int(k) for sp, k in zip(specs, steps)], ws)
    mine = [i for i in range(n_req) if owner[i] == rank]
    t0 = time.time()
    gen = D.make_decks([specs[i].replace(steps=int(steps[i]) + 5) for i in mine])
    decks = dict(zip(mine, gen))
    gen_s = time.time() - t0
    reqs = [serve.Request(i, decks[i], int(steps[i]), float(arr[i])) for i in mine]
    prec = native.PRECISION_MIXED if precision == "mixed" else native.PRECISION_FP64
    check = [i for i in mine if i % check_every == 0] if precision == "mixed" else []
    served_state = {}

    def build(req):
        return native.domain_from_deck(req.deck, device=dev, precision=prec, eps_inner=eps_inner)

    def done(req):
        if req.rid in check:
            served_state[req.rid] = req.domain.download(["surf", "uuXP", "vvYP"])

    if ws > 1:
        import torch
        torch.distributed.barrier()
    with ClockSampler(dev) as clk:
        res = serve.serve(reqs, args.budget_gb << 30, cells_per_cta, device=dev, build=build,
                          on_done=done)
    per = []
    for i in check:
        g = native.domain_from_deck(decks[i], device=dev)
        g.run(1, int(steps[i]))
        n_ = decks[i].nx * decks[i].ny
        per.append(_state_errors(served_state[i], g.download(["surf", "uuXP", "vvYP"]), n_))
        g.close()
    parts = shard.gather({**res, "clocks": clk.summary(), "gen_s": gen_s,
                          "errors": _worst(per), "checked": len(per)}, ws)
    merged = shard.merge_served(parts)
    rec = {"value": merged["cell_steps_per_s"], "unit": UNIT,
           "p50_latency_s": merged["p50_s"], "p99_latency_s": merged["p99_s"],
           "dtype": "f64" if precision == "fp64" else "f32+f64",
           "config": {"workload": f"the first {n_req} requests of a {n_stream}-request stream: "
                                  f"Poisson arrivals {rate}/s, sides log-uniform {smin}-{smax} "
                                  f"(square or 1:4), steps {steps_lo}-{steps_hi}, "
                                  f"1-{scalars_max} scalars, {precision}",
                      "requests": n_req, "cells_per_cta": cells_per_cta,
                      "eps_inner": eps_inner if precision == "mixed" else None,
                      "sharding": "least assigned work, arrival order" if ws > 1 else None,
                      "deck_gen_s": round(max(p["gen_s"] for p in parts), 1)},
           "serving": merged, "clocks": parts[0]["clocks"],
           "gpu_launches": 5 * sum(int(p.get("batch_steps", 0)) for p in parts)}
    if precision == "mixed":
        rec["errors_vs_fp64"] = _worst([p["errors"] for p in parts])
        rec["errors_checked_requests"] = int(sum(p["checked"] for p in parts))
    return rec


def run_batched_form(args):
    """--form batched: the batched measurement alone, as its own JSON line."""
    ws, rank, dev = _dist_init()
    rec = measure_batched(args, ws, rank, dev, args.mix, args.mix_min, args.mix_max,
                          args.scalars, args.steps + args.warmup, args.precision, args.steps,
                          args.warmup)
    _dist_done(ws)
    if rank == 0:
        print(json.dumps({"metric": METRIC, "form": "batched", "n_gpus": ws,
                          "higher_is_better": True, "scaling": "weak", "data": "synthetic",
                          **rec}), flush=True)
    return 0


def run_served_form(args):
    """--form served: the served measurement alone, as its own JSON line."""
    ws, rank, dev = _dist_init()
    eps = args.eps_inner if args.eps_inner is not None else 1e-4
    cpc = args.cells_per_cta if args.cells_per_cta > 0 else 65536.0
    rec = measure_served(args, ws, rank, dev, args.requests, args.requests, args.mix_min,
                         args.mix_max, args.req_steps_min, args.req_steps_max, args.scalars_max,
                         args.rate, args.precision, cpc, eps, 10)
    _dist_done(ws)
    if rank == 0:
        print(json.dumps({"metric": METRIC, "form": "served", "n_gpus": ws,
                          "higher_is_better": True, "scaling": "weak", "data": "synthetic",
                          **rec}), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--cpu-steps", type=int, default=300,
                    help="steps of the reference program on one core for cpu_baseline (about 13 s)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU reference baseline")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end C-ABI leg")
    ap.add_argument("--cg-schedule", default="single_sweep", choices=list(SCHEDULES),
                    help="CG schedule: one sweep and one reduction per iteration, or the "
                         "textbook two-phase ordering")
    ap.add_argument("--form", default="plain", choices=["plain", "batched", "served"],
                    help="plain: one 4096^2 domain; batched: a mix of domains as one batch; "
                         "served: Poisson request stream with continuous batching")
    ap.add_argument("--mix", type=int, default=64, help="batched form: domains in the mix")
    ap.add_argument("--mix-min", type=int, default=64)
    ap.add_argument("--mix-max", type=int, default=512)
    ap.add_argument("--cells-per-cta", type=float, default=0.0,
                    help="batched/served: cells per CTA of a domain's CG (<= 0: batched form "
                         "autotunes it on the mix; served form uses 32768)")
    ap.add_argument("--tiles-per-block", type=int, default=4,
                    help="batched form with a given --cells-per-cta: 32x8 stencil tiles per "
                         "block of the batched stencil kernels (1..8)")
    ap.add_argument("--budget-gb", type=int, default=120)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="mixed: FP32 inner CG iterations inside FP64 iterative refinement")
    ap.add_argument("--eps-inner", type=float, default=None,
                    help="mixed precision: inner FP32 tolerance (default: plain 1e-5, batched "
                         "autotuned, served 1e-4)")
    ap.add_argument("--scalars", type=int, default=2, help="batched form: scalars per basin")
    ap.add_argument("--scalars-max", type=int, default=3,
                    help="served form: scalars per request uniform in 1..this")
    ap.add_argument("--extras", default="mixed,batched,served",
                    help="plain form: the other forms measured into the same JSON line "
                         "(comma list of mixed, batched, served; 'none' for none)")
    ap.add_argument("--mixed-steps", type=int, default=1000,
                    help="mixed sub-record: steps after which its state is compared with FP64")
    ap.add_argument("--batched-steps", type=int, default=20,
                    help="batched sub-record: timed batch steps")
    ap.add_argument("--batched-total", type=int, default=500,
                    help="batched sub-record: steps after which the errors are taken")
    ap.add_argument("--served-requests", type=int, default=100,
                    help="served sub-record: requests taken from the head of the 2000-request "
                         "stream")
    ap.add_argument("--served-cells-per-cta", type=float, default=65536.0)
    ap.add_argument("--requests", type=int, default=120)
    ap.add_argument("--rate", type=float, default=50.0)
    ap.add_argument("--req-steps-min", type=int, default=50)
    ap.add_argument("--req-steps-max", type=int, default=400)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.form == "batched":
        return run_batched_form(args)
    if args.form == "served":
        return run_served_form(args)
    return run_gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
