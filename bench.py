#!/usr/bin/env python
"""Benchmark of the Monte Carlo hot path on B200.

Workload (one "step"): the Heston European strike strip - kappa=2, theta=0.04,
xi=0.5, rho=-0.7, v0=0.04, S0=100, r=0.03, q=0, T=1; 41 call strikes 80..120
priced from one shared set of 2^20 paths x 256 Euler steps (the reference's
Heston Euler step, variance floored after each step), FP32 Philox4x32-10
paths, compensated FP32 -> FP64 sums, seed 7 (+ rank for replicas).

value  = path-steps/s of the device kernels (inputs resident, CUDA events on
         the engine's stream, L2 flushed between timed iterations), summed over
         ranks / max rank time.
e2e    = the same metric through the public API (openferric_b200.price_strike_strip),
         host wall clock, including the strike upload and the result readback.
cpu_baseline / --impl reference = the CPU restatement of the reference's
         Monte Carlo (xoshiro256++ + Acklam, FP64, OpenMP over all host
         cores) on a bounded sample of the same workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "path-steps/s & priced+Greeks options/s at SE≤1e-4: FP32+adjoint vs FP64 plain"
UNIT = "path-steps/s"
HESTON = dict(mu=0.03, kappa=2.0, theta=0.04, xi=0.5, rho=-0.7, v0=0.04)
S0, RATE, T = 100.0, 0.03, 1.0
STRIKES = [80.0 + k for k in range(41)]
PATHS, STEPS, SEED = 1 << 20, 256, 7
PATH_STEPS = float(PATHS) * STEPS
# Declared algorithmic work of one Heston Euler path-step in the FP32 kernel:
# one Box-Muller pair (u1 2, radius constant 1, angle fma 2, r cos / r sin 2:
# 7 flops; lg2, sqrt, sin, cos on the MUFU unit; sqrt(dt) rides in the radius
# constant) and the step (correlation 3, log-spot 5, variance 5, floors 2: 15
# flops; one sqrt): 22 FP32 flops (FMA = 2) and 5 MUFU operations.  The
# Philox rounds (integer multiply and xor, ~20 instructions per step) use
# neither pipe's budget in this count.
FLOPS_PER_STEP = 22.0
SFU_PER_STEP = 5.0
# Issued thread instructions per path-step of the strip kernel, Philox
# included, from ncu captures (smsp__inst_executed.sum x 32 / path-steps) of
# the bench's kernel at 2^20 paths, by samples in flight per thread.  With the
# sampled SM clock they give the issue fraction: warp instructions per second
# over 148 SMs x 4 schedulers x 1 instruction per cycle.
INSTR_PER_STEP = {1: 48.8, 2: 45.7}
INSTR_SOURCE = "ncu smsp__inst_executed.sum of strip_kernel at 2^20 paths (profiles/strip_kernel_heston_euler_*)"
# DRAM bytes (read + write) of one strip launch from an ncu capture of the
# kernel; the kernel reads no input from HBM, so the figure does not grow
# with the path count.
STRIP_DRAM_BYTES = 31488
STRIP_DRAM_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of strip_kernel<ILP=2> at 2^20 paths "
                     "(the kernel reads no HBM input; the figure does not grow with paths)")
CONFIG = {"workload": "heston_euler_strike_strip", "paths": PATHS, "steps": STEPS, "strikes": 41,
          "strike_range": [80, 120], "kappa": 2.0, "theta": 0.04, "xi": 0.5, "rho": -0.7, "v0": 0.04, "s0": S0,
          "r": RATE, "q": 0.0, "T": T, "seed": SEED, "rng": "philox4x32-10", "path_dtype": "fp32",
          "sum_dtype": "kahan-fp32->fp64",
          "l2": "flushed between timed iterations (256 MiB write); the kernel reads no HBM input"}


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ["index", "clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + ",".join(self.FIELDS),
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1])]
        mx = [num(r[2]) for r in rows if num(r[2])]
        pw = [num(r[3]) for r in rows if num(r[3])]
        load = [s for s, w in zip(sm, pw) if w and w > 250.0] or sm
        reasons = set()
        for r in rows:
            for name, v in zip(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"], r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows), "power_w_max": max(pw) if pw else None}


def cpu_sample(threads, target_s, max_paths=PATHS):
    """Times the oracle strip (CPU restatement of the reference MC) on a
    sample sized to about target_s seconds; returns (path-steps/s, sample)."""
    from oracle import oracle as orc
    from openferric_b200 import _abi as A
    from openferric_b200.engines import Heston, HestonPathGenerator
    gen = HestonPathGenerator(Heston(**HESTON), S0, T, STEPS).to_abi()
    df = math.exp(-RATE * T)

    def run(paths):
        cfg = A.OfMcConfig(num_paths=paths, seed=SEED, discount_factor=df)
        t0 = time.perf_counter()
        orc.mc_strip(gen, A.OF_CALL, STRIKES, cfg, threads=threads)
        return time.perf_counter() - t0

    probe = 1 << 12
    dt = run(probe)
    paths = int(min(max_paths, max(probe, probe * target_s / max(dt, 1e-6))))
    dt = run(paths)
    return paths * STEPS / dt, {"paths": paths, "steps": STEPS, "strikes": 41, "seconds": round(dt, 3)}


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    per_step = max(2.0, min(10.0, 150.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_sample(threads, per_step / 4)
    vals, sample = [], None
    for _ in range(args.steps):
        v, sample = cpu_sample(threads, per_step)
        vals.append(v)
    value = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * PATH_STEPS / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": CONFIG,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{sample['paths']} paths x {STEPS} steps x 41 strikes per step (bounded)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "oracle/of_oracle.c: C restatement of openferric's MonteCarloEngine::run with the Heston "
                    "Euler generator (no Rust toolchain to build the reference); OpenMP over all host cores"}
    print(json.dumps(line), flush=True)


def fp64_strip_check(paths, strip_prices):
    """The strip's FP32 Philox prices against the FP64 engine on the
    reference's own stream (xoshiro256++ + Acklam, MonteCarloEngine::run's
    arithmetic) for the same Heston Euler workload: per strike
    z = (FP32 - FP64) / sqrt(se32^2 + se64^2).  Both are unbiased estimates of
    the same discretised price from independent streams, so |z| is a standard
    normal; run outside the timed region."""
    import openferric_b200 as of
    gen = of.HestonPathGenerator(of.Heston(**HESTON), S0, T, STEPS)
    eng = of.MonteCarloEngine(paths, SEED)
    df = math.exp(-RATE * T)
    zs, ms, k100 = [], 0.0, None
    for k, (p32, s32) in zip(STRIKES, strip_prices):
        r = eng.run_full(gen, of.VanillaOption.european_call(k, T), df)
        ms += r.kernel_ms
        z = (p32 - r.price) / math.sqrt(s32 * s32 + r.stderr_ * r.stderr_)
        zs.append(z)
        if k == 100.0:
            k100 = {"fp64_price": r.price, "fp64_stderr": r.stderr_, "fp32_price": p32, "fp32_stderr": s32, "z": z}
    return {"engine": "FP64 reference-stream MonteCarloEngine (xoshiro256++ seed 7, Acklam), same paths/steps",
            "strikes": len(zs), "max_abs_z": max(abs(z) for z in zs),
            "within_3_combined_se": sum(1 for z in zs if abs(z) <= 3.0), "K100": k100,
            "fp64_kernel_ms_total": ms}


ADJ_HESTON = dict(spot=100.0, rate=0.03, v0=0.04, kappa=2.0, theta=0.04, xi=0.5, rho=-0.7)


def greeks_comparison(paths=PATHS, steps=512, reps=3):
    """Priced + full-Greeks options/s for one Heston arithmetic Asian call
    (K=100, T=2, daily fixings at all 512 steps, the parameters of the strip):
    FP32 QE + checkpointed adjoint (one call) against the plain FP64 engine
    (the reference-stream Euler engine) with the 7 Greeks by central bumps
    with common random numbers (15 runs).  Both at the same path count; the
    standard error of both is below 1e-4 S0 = 0.01."""
    import openferric_b200 as of
    from openferric_b200.adjoint import HestonAdjointSpec, heston_adjoint
    spec = HestonAdjointSpec(strike=100.0, expiry=2.0, num_paths=paths, num_steps=steps, seed=SEED, asian=True)
    heston_adjoint(spec, **ADJ_HESTON)
    adj = [heston_adjoint(spec, **ADJ_HESTON) for _ in range(reps)]
    t_adj = min(a.kernel_ms for a in adj)
    obs = [2.0 * (j / steps) for j in range(1, steps + 1)]
    opt = of.AsianOption(of.OptionType.Call, 100.0, 2.0, of.AsianSpec(of.Averaging.Arithmetic, of.StrikeType.Fixed, obs))

    def fp64_run(p):
        gen = of.HestonPathGenerator(of.Heston(p["rate"], p["kappa"], p["theta"], p["xi"], p["rho"], p["v0"]),
                                     p["spot"], 2.0, steps)
        eng = of.MonteCarloEngine(paths, SEED)
        r = eng.run_full(gen, opt, math.exp(-2.0 * p["rate"]))
        return r.price, r.stderr_, r.kernel_ms

    fp64_run(ADJ_HESTON)
    t64, base_price, base_se = 0.0, None, None
    for name in [None] + list(ADJ_HESTON):
        for sgn in ((0,) if name is None else (1, -1)):
            p = dict(ADJ_HESTON)
            if name is not None:
                p[name] *= 1.0 + sgn * 1e-4
            price, se, ms = fp64_run(p)
            t64 += ms
            if name is None:
                base_price, base_se = price, se
    return {"workload": "heston_qe_asian_adjoint", "paths": paths, "steps": steps, "strike": 100.0, "T": 2.0,
            "fp32_adjoint_ms": t_adj, "fp32_adjoint_options_per_s": 1e3 / t_adj,
            "fp32_adjoint_price": adj[0].price, "fp32_adjoint_se": adj[0].stderr,
            "fp64_plain_bump_ms": t64, "fp64_plain_bump_options_per_s": 1e3 / t64,
            "fp64_plain_price": base_price, "fp64_plain_se": base_se,
            # QE (FP32) against Euler (FP64) at 512 steps: the two schemes'
            # discretisation biases differ, so this z is not only rounding
            "z_fp32_qe_vs_fp64_euler": (adj[0].price - base_price) / math.sqrt(adj[0].stderr ** 2 + base_se ** 2),
            "speedup": t64 / t_adj, "greeks": adj[0].greeks}


def run_workload(args, local_rank):
    """Single-GPU lines for configurations 3-5 (not the headline)."""
    import torch
    import numpy as np
    import openferric_b200 as of
    torch.cuda.set_device(local_rank)
    if args.workload == "adjoint":
        g = greeks_comparison(args.paths)
        line = {"metric": "priced+Greeks options/s at SE<=1e-4*S0", "value": g["fp32_adjoint_options_per_s"],
                "unit": "options/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
                "config": g}
    elif args.workload == "book":
        from openferric_b200.book import BookPlan, synthetic_book
        plan = BookPlan(synthetic_book(args.book_options), seed=20261203)
        info = plan.info()
        for _ in range(max(1, args.warmup)):
            plan.launch()
        plan.raw_results()
        ctx = of.context(local_rank)
        stream = torch.cuda.ExternalStream(ctx.stream_ptr())
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for s, e in ev:
            s.record(stream)
            plan.launch()
            e.record(stream)
        stream.synchronize()
        ms = statistics.median(s.elapsed_time(e) for s, e in ev)
        plan.close()
        line = {"metric": "path-steps/s", "value": info["path_steps"] / (ms / 1e3), "unit": "path-steps/s",
                "n_gpus": 1, "higher_is_better": True, "dtype": "f32", "data": "synthetic", "ms_per_step": ms,
                "config": {"workload": f"batched_book_{args.book_options}", "tiles": info["tiles"],
                           "block": info["block"],
                           "paths_per_thread": info["paths_per_thread"], "path_steps": info["path_steps"],
                           "options_per_s": args.book_options / (ms / 1e3), "cuda_graph": True}}
    elif args.workload == "book_se":
        # options/s with every option priced to SE <= 1e-4 S0: pilot launch,
        # then launches with the paths each option's pilot SE asks for
        import time
        from openferric_b200.book import BookEntry, price_book_to_stderr, synthetic_book
        from openferric_b200.engines import VarianceReduction
        from openferric_b200.instruments import AsianOption
        book = synthetic_book(4096)[:args.se_options]
        vr_note = "none (plain Monte Carlo)"
        if args.variance_reduction == "mixed":
            # the reference's VarianceReduction per option: the geometric-Asian
            # control variate for the arithmetic Asians; antithetic pairs for
            # the Europeans (whose reference control variate is their own
            # payoff, i.e. the closed form) and the barriers (no control variate)
            book = [BookEntry(e.instrument, e.market, e.num_paths, e.num_steps,
                              VarianceReduction.ControlVariate if isinstance(e.instrument, AsianOption)
                              else VarianceReduction.Antithetic) for e in book]
            vr_note = "geometric-Asian control variate for the Asians; antithetic for Europeans and barriers"
        price_book_to_stderr(book[:8], seed=1)  # warm-up (library load, clocks)
        times, rounds = [], None
        for k in range(max(1, args.steps)):
            t0 = time.perf_counter()
            res, rounds = price_book_to_stderr(book, seed=20261203 + 100 * k)
            times.append(time.perf_counter() - t0)
        s = statistics.median(times)
        ok = sum(1 for e, r in zip(book, res) if r.stderr <= 1e-4 * e.market.spot)
        ps = sum(r.path_steps for r in rounds)
        line = {"metric": "options/s at SE<=1e-4*S0", "value": len(book) / s, "unit": "options/s", "n_gpus": 1,
                "higher_is_better": True, "dtype": "f32", "data": "synthetic", "ms_per_step": s * 1e3,
                "config": {"workload": f"batched_book_se_{len(book)}", "se_target": "1e-4*S0",
                           "variance_reduction": vr_note,
                           "timing": "wall clock of the whole procedure (pilot + follow-up launches, host planning)",
                           "options_meeting_target": ok, "path_steps": ps, "path_steps_per_s": ps / s,
                           "rounds": [r.__dict__ for r in rounds]}}
    else:  # lsm
        from openferric_b200.lsm import LongstaffSchwartzEngine
        rng = np.random.default_rng(20261203)
        items = []
        for i in range(args.contracts):
            vol, T = (0.2, 0.4)[i % 2], (1.0, 2.0)[(i // 2) % 2]
            m = of.Market.builder().spot(rng.uniform(30.0, 50.0)).rate(0.06).flat_vol(vol).build()
            items.append((of.VanillaOption.american_put(40.0, T), m))
        total_ms, alg_bytes = 0.0, 0.0
        for T in (1.0, 2.0):
            sub = [it for it in items if it[0].expiry == T]
            eng = LongstaffSchwartzEngine(args.paths, int(50 * T), SEED).with_precision(
                of.Precision.Fp32Philox).with_basis_degree(3)
            eng.price_batch(sub[:2], with_delta=True)
            eng.price_batch(sub, with_delta=True)
            total_ms += eng.last_kernel_ms
            alg_bytes += len(sub) * float(args.paths) * int(50 * T) * 16.0
        line = {"metric": "LSM contracts/s (price + delta)", "value": args.contracts / (total_ms / 1e3),
                "unit": "contracts/s",
                "n_gpus": 1, "higher_is_better": True, "dtype": "f32", "data": "synthetic", "ms_per_step": total_ms,
                "config": {"workload": f"lsm_american_put_{args.contracts}", "paths": args.paths, "dates_per_year": 50,
                           "basis": "1,x,x^2,x^3 (x=S/K), Cholesky", "algorithmic_bytes": alg_bytes,
                           "algorithmic_GBps": alg_bytes / (total_ms / 1e3) / 1e9}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-greeks", action="store_true", help="skip the adjoint vs FP64-bump comparison")
    ap.add_argument("--workload", default="strip", choices=["strip", "adjoint", "book", "book_se", "lsm"],
                    help="strip is the benchmark line; the others are single-GPU lines for configurations 3-5 "
                         "(book_se: the book's options priced to SE <= 1e-4 S0)")
    ap.add_argument("--se-options", type=int, default=256,
                    help="book_se workload: the first N options of the synthetic book")
    ap.add_argument("--paths", type=int, default=PATHS,
                    help="paths per strip (profiling a smaller case; the benchmark workload is 2^20)")
    ap.add_argument("--book-options", type=int, default=4096,
                    help="book workload: number of options (4096 in the benchmark; fewer for a profiler capture)")
    ap.add_argument("--variance-reduction", default="none", choices=["none", "mixed"],
                    help="book_se workload: none (plain MC), or mixed (geometric-Asian control variate for the "
                         "Asians, antithetic for the Europeans and barriers)")
    ap.add_argument("--contracts", type=int, default=256,
                    help="LSM workload: number of American puts (256 in the benchmark; fewer for a profiler capture)")
    args = ap.parse_args()
    global PATH_STEPS
    PATH_STEPS = float(args.paths) * STEPS
    CONFIG["paths"] = args.paths
    rank, world, local_rank = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload != "strip":
        return run_workload(args, local_rank) if rank == 0 else None

    import torch
    import openferric_b200 as of
    from openferric_b200.engines import StripPlan
    from openferric_b200.replicas import max_over_ranks, replica_seed

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    ctx = of.context(local_rank)
    gen = of.HestonPathGenerator(of.Heston(**HESTON), S0, T, STEPS)
    df = math.exp(-RATE * T)
    seed = replica_seed(SEED, rank)  # independent replica per GPU
    # tile shape (samples in flight per thread) picked by the native autotuner
    # on this GPU, before and outside the timed region
    from openferric_b200 import autotune
    tile_ilp, tune_ms = autotune.tune_strip(gen, STRIKES, args.paths, reps=5, device=local_rank)
    plan = StripPlan(gen, of.OptionType.Call, STRIKES, args.paths, seed, df, tile_ilp=tile_ilp)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=torch.device("cuda", local_rank))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local_rank}")

    for _ in range(max(3, args.warmup)):
        plan.launch()
    prices = plan.results()
    peaks = ctx.device_peaks()  # MUFU and FP32 denominators, measured on this GPU before the timed region

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clocks:
        with torch.cuda.stream(stream):
            for i in range(args.steps):
                flush.zero_()
                starts[i].record(stream)
                plan.launch()
                ends[i].record(stream)
        stream.synchronize()
        torch.cuda.synchronize()
    kernel_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = sum(kernel_ms)
    total_ms = max_over_ranks(total_ms, device=torch.device("cuda", local_rank))
    if dist:
        dist.barrier()
    prices = plan.results()
    clk = clocks.summary()

    # End to end through the public API (host wall clock, sync inside each call).
    for _ in range(2):
        of.price_strike_strip(gen, of.OptionType.Call, STRIKES, args.paths, seed, df, tile_ilp=tile_ilp)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_prices = of.price_strike_strip(gen, of.OptionType.Call, STRIKES, args.paths, seed, df, tile_ilp=tile_ilp)
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, device=torch.device("cuda", local_rank))

    ms_per_step = total_ms / args.steps
    value = world * PATH_STEPS * args.steps / (total_ms / 1e3)
    per_gpu = PATH_STEPS / (ms_per_step / 1e3)
    sm_max = clk.get("sm_max_mhz") or 1965.0
    sfu_peak, fp32_peak = peaks["sfu_ops_per_s"], peaks["fp32_flops_per_s"]
    sfu_frac = per_gpu * SFU_PER_STEP / sfu_peak
    fp32_frac = per_gpu * FLOPS_PER_STEP / fp32_peak
    probe_src = "measured in this run by of_measure_device_peaks"
    fp32_line = {"achieved": per_gpu * FLOPS_PER_STEP / 1e12, "peak": fp32_peak / 1e12, "unit": "TFLOP/s",
                 "frac": fp32_frac, "per_step": FLOPS_PER_STEP,
                 "peak_source": f"{probe_src} (FP32 FMA chains); derived nominal "
                                f"{148 * 128 * 2 * sm_max * 1e6 / 1e12:.1f} TFLOP/s at {sm_max:.0f} MHz"}
    sfu_line = {"achieved": per_gpu * SFU_PER_STEP / 1e12, "peak": sfu_peak / 1e12, "unit": "TOP/s",
                "frac": sfu_frac, "per_step": SFU_PER_STEP,
                "peak_source": f"{probe_src} (MUFU lg2/sqrt/sin/cos chains); derived nominal "
                               f"{148 * 16 * sm_max * 1e6 / 1e12:.2f} TOP/s at 16/clk/SM"}
    bound, main_line, other_name, other_line = (
        ("sfu", sfu_line, "fp32", fp32_line) if sfu_frac >= fp32_frac else ("fp32", fp32_line, "sfu", sfu_line))
    # issue slots: Philox, conversions and control flow included
    sm_run = clk.get("sm_mhz") or sm_max
    ips = INSTR_PER_STEP.get(tile_ilp, INSTR_PER_STEP[1])
    issue_peak = 148 * 4 * sm_run * 1e6
    issue_line = {"achieved": per_gpu * ips / 32.0 / 1e12, "peak": issue_peak / 1e12, "unit": "T warp-inst/s",
                  "frac": per_gpu * ips / 32.0 / issue_peak, "per_step": ips,
                  "peak_source": f"148 SMs x 4 schedulers x 1 warp instruction per cycle at the sampled "
                                 f"{sm_run:.0f} MHz",
                  "per_step_source": INSTR_SOURCE}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": dict(CONFIG, parallelism=f"replicas{world}", tile_ilp=tile_ilp,
                                                          tile_ilp_ms={str(k): v for k, v in tune_ms.items()}),
        "roofline": dict(main_line, bound=bound, traffic=STRIP_DRAM_BYTES, traffic_source=STRIP_DRAM_SOURCE,
                         issue=issue_line, **{other_name: other_line}),
        "e2e": {"value": world * PATH_STEPS * args.steps / e2e_s, "unit": UNIT,
                "h2d_bytes_per_step": 41 * 4, "d2h_bytes_per_step": 41 * 2 * 8},
        "gpu_launches": 2 * args.steps,
        "clocks": clk,
        "kernel_ms": {"min": min(kernel_ms), "median": statistics.median(kernel_ms), "max": max(kernel_ms)},
        "check": {"price_K100": prices[20][0], "stderr_K100": prices[20][1],
                  "e2e_price_K100": e2e_prices[20][0]},
    }
    if rank == 0 and not args.no_greeks:
        # the priced+Greeks part of the metric, and the FP32 strip's error
        # against an FP64 run (both outside the timed region)
        line["greeks"] = greeks_comparison()
        line["check"]["fp64"] = fp64_strip_check(args.paths, prices)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, sample = cpu_sample(os.cpu_count() or 1, 10.0)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
                                "sample": f"{sample['paths']} paths x {STEPS} Heston Euler steps x 41 strikes, "
                                          f"FP64 xoshiro256++/Acklam oracle, {sample['seconds']} s"}
    plan.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
