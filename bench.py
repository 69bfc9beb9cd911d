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

The same line carries one key per other workload, each with its own device
timing, clock samples and roofline (run after the strip's timed region):
  config1     the reference's own MC benchmark (100k x 252 GBM European, FP64
              reference draws, seed 42) with its CPU baseline;
  book        the 4096-option batched book in one persistent launch;
  book_se     its first 256 options priced to SE <= 1e-4 S0;
  book_greeks the same with pathwise delta/vega/rho/theta (the FP32 batched
              adjoint form) against the plain FP64 engine with central bumps;
  greeks      the Heston QE adjoint (configuration 4);
  lsm         256 American puts by Longstaff-Schwartz (configuration 5).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload ...]
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
INSTR_PER_STEP = {1: 48.8, 2: 40.0}
INSTR_SOURCE = ("ncu smsp__inst_executed.sum of strip_kernel at 2^20 paths (profiles/strip_kernel_heston_euler_ilp2_2p20.md "
                "for two samples per thread, profiles/strip_kernel_pipe_mix_2p20.md for one)")
# DRAM bytes (read + write) of one strip launch from an ncu capture of the
# kernel; the kernel reads no input from HBM, so the figure does not grow
# with the path count.
STRIP_DRAM_BYTES = 30720
STRIP_DRAM_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of strip_kernel<ILP=2> at 2^20 paths "
                     "(the kernel reads no HBM input; the figure does not grow with paths)")
CONFIG = {"workload": "heston_euler_strike_strip", "paths": PATHS, "steps": STEPS, "strikes": 41,
          "strike_range": [80, 120], "kappa": 2.0, "theta": 0.04, "xi": 0.5, "rho": -0.7, "v0": 0.04, "s0": S0,
          "r": RATE, "q": 0.0, "T": T, "seed": SEED, "rng": "philox4x32-10", "path_dtype": "fp32",
          "sum_dtype": "kahan-fp32->fp64",
          "l2": "flushed between timed iterations (256 MiB write); the kernel reads no HBM input"}


def _json_default(o):
    """numpy scalars and arrays in a line become plain numbers and lists."""
    if hasattr(o, "item") and getattr(o, "ndim", 0) == 0:
        return o.item()
    if hasattr(o, "tolist"):
        return o.tolist()
    raise TypeError(f"Object of type {type(o).__name__} is not JSON serializable")


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
    config = {k: v for k, v in CONFIG.items() if k not in ("rng", "path_dtype", "sum_dtype", "l2")}
    config.update({
        "rng": "xoshiro256++ per sample, SplitMix64-seeded with seed + i*7919 (the reference's own draws)",
        "normal": "Acklam inverse CDF", "path_dtype": "fp64", "sum_dtype": "fp64",
        "path_set": "the 41 strikes share one path set; the reference's API would run MonteCarloEngine::run once "
                    "per strike (41x the work), so this baseline favours the CPU by up to 41x",
        "precision_note": "FP64 on the reference's streams, where the GPU arm runs FP32 on Philox draws: a "
                          "deliberate difference (the GPU arm's line states its FP32 error against an FP64 run)"})
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * PATH_STEPS / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{sample['paths']} paths x {STEPS} steps x 41 strikes per step (bounded)",
                             **cpu_info()},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "oracle/of_oracle.c: C restatement of openferric's MonteCarloEngine::run with the Heston "
                    "Euler generator (no Rust toolchain on either machine to build the reference); OpenMP over "
                    "all host cores"}
    print(json.dumps(line, default=_json_default), flush=True)


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


# ---------------------------------------------------------------------------
# Shared helpers of the workload legs
# ---------------------------------------------------------------------------
def _find_key(d, key):
    if isinstance(d, dict):
        if key in d and isinstance(d[key], (int, float)):
            return float(d[key])
        for v in d.values():
            r = _find_key(v, key)
            if r is not None:
                return r
    return None


def measured_hbm_gbs():
    """HBM copy bandwidth of this pool's B200s from MEASURED_PEAKS.json (written
    beside this file by the harness), else the recipe's fallback figure."""
    try:
        v = _find_key(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "hbm_gbs")
        if v:
            return v, "measured (MEASURED_PEAKS.json hbm_gbs, STREAM-style copy)"
    except Exception:
        pass
    return 6650.0, "fallback 6650 GB/s (MEASURED_PEAKS.json absent)"


def cpu_info():
    model = None
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count()}


def device_timed(stream, fn, steps, flush=None):
    """Median and all device times (ms) of `steps` calls of fn() between CUDA
    events on `stream`; the L2 flush (a write larger than L2) runs outside the
    events."""
    import torch
    ts = []
    for _ in range(steps):
        if flush is not None:
            with torch.cuda.stream(stream):
                flush.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        fn()
        e.record(stream)
        stream.synchronize()
        ts.append(s.elapsed_time(e))
    return statistics.median(ts), ts


# ---------------------------------------------------------------------------
# Configuration 1: the reference's own MC benchmark
# ---------------------------------------------------------------------------
# Declared FP64 work of one sample-step of the reference-stream kernel
# (xoshiro256++ draw, clamp, Acklam central region: 10 FMA + 1 mul + 1 div =
# 22 flops) and of one leg-step (log-Euler growth exp(fma(diff, z, drift)) and
# the spot update: fma + mul = 3 flops; the exp itself is a multi-instruction
# FP64 routine and counts 0 here).
FP64_NORMAL_FLOPS = 22.0
FP64_LEG_FLOPS = 3.0


def leg_config1(steps, warmup, peaks, threads):
    """MonteCarloPricingEngine::new(100_000, 252, 42).price(european_call(100, 1))
    on S0=100, r=0.05, q=0, sigma=0.2 (benches/pricing_bench.rs:89-109, the
    reference's mc_european_call/100000), FP64 reference draws, plus the
    same with 50,000 antithetic pairs.  Device time from the library's CUDA
    events around the simulation kernels; e2e = the public call's wall clock."""
    import openferric_b200 as of
    from openferric_b200.analytic import bs_price
    from oracle import oracle as orc
    from openferric_b200 import _abi as A
    market = of.Market.builder().spot(100.0).rate(0.05).dividend_yield(0.0).flat_vol(0.20).build()
    opt = of.VanillaOption.european_call(100.0, 1.0)
    bs = bs_price(of.OptionType.Call, 100.0, 100.0, 0.05, 0.0, 0.20, 1.0)
    ps = 100_000 * 252.0
    out = {}
    with ClockSampler(0) as clocks:
        for name, vr in (("plain", of.VarianceReduction.None_), ("antithetic", of.VarianceReduction.Antithetic)):
            eng = of.MonteCarloPricingEngine(100_000, 252, 42).with_variance_reduction(vr)
            for _ in range(max(3, warmup)):
                eng.price(opt, market)
            ks = []
            t0 = time.perf_counter()
            for _ in range(steps):
                r = eng.price(opt, market)
                ks.append(eng.last_kernel_ms)
            wall = time.perf_counter() - t0
            ms = statistics.median(ks)
            anti = vr is of.VarianceReduction.Antithetic
            flops = (FP64_NORMAL_FLOPS + 2 * FP64_LEG_FLOPS) / 2.0 if anti else FP64_NORMAL_FLOPS + FP64_LEG_FLOPS
            v = ps / (ms / 1e3)
            out[name] = {
                "value": v, "unit": "path-steps/s", "ms_per_step": ms, "kernel_ms_all": [round(k, 4) for k in ks],
                "e2e": {"value": ps * steps / wall, "unit": "path-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 8 * 8,
                        "note": "public MonteCarloPricingEngine.price, host wall clock; inputs are scalars in the "
                                "launch parameters, the readback is the 5 sums + count"},
                "price": r.price, "stderr": r.stderr, "bs_price": bs, "z_vs_bs": (r.price - bs) / r.stderr,
                "roofline": {"bound": "fp64", "achieved": v * flops / 1e12, "peak": peaks["fp64_flops_per_s"] / 1e12,
                             "unit": "TFLOP/s", "frac": v * flops / peaks["fp64_flops_per_s"], "per_step": flops,
                             "peak_source": "measured in this run by of_measure_device_peaks (FP64 FMA chains)",
                             "note": "declared flops: Acklam central region + log-Euler update per path-step; the "
                                     "FP64 exp/log/div routines are multi-instruction and not counted, so the pipe "
                                     "is busier than this fraction"},
                "gpu_launches_per_step": 2}
    out["clocks"] = clocks.summary()
    out["workload"] = ("european_call_gbm_100k_x_252 (S0=100 K=100 r=0.05 q=0 sigma=0.2 T=1 seed 42; "
                       "benches/pricing_bench.rs:89-109)")
    out["l2"] = "not flushed: the kernel reads no HBM input (streams and path state in registers)"
    # CPU baseline: the oracle's restatement of MonteCarloEngine::run, same config
    gen = of.GbmPathGenerator(of.Gbm(0.05, 0.20), 100.0, 1.0, 252).to_abi()
    from openferric_b200.engines import _payoff_abi
    payoff, _keep = _payoff_abi(opt)
    cfg = A.OfMcConfig(num_paths=100_000, seed=42, discount_factor=math.exp(-0.05))
    t0 = time.perf_counter()
    orc.mc_run(gen, payoff, cfg, threads=threads)
    t_all = time.perf_counter() - t0
    t0 = time.perf_counter()
    orc.mc_run(gen, payoff, cfg, threads=1)
    t_one = time.perf_counter() - t0
    out["cpu_baseline"] = {"value": ps / t_all, "unit": "path-steps/s", "cores": threads, "kind": "port",
                           "single_thread_value": ps / t_one, "single_thread_ms": 1e3 * t_one,
                           "sample": "the full workload (100k x 252, no antithetic), oracle/of_oracle.c restatement "
                                     "of MonteCarloEngine::run, OpenMP over samples", **cpu_info()}
    out["published_reference"] = {"ms": 406.0, "path_steps_per_s": ps / 0.406,
                                   "source": "openferric README.md:33 (mc_european_call/100000, hardware not stated)"}
    return out


# ---------------------------------------------------------------------------
# Configuration 3: the batched book
# ---------------------------------------------------------------------------
# Issued thread instructions per path-step of book_kernel on the synthetic
# mixed book, from the ncu capture of 256 options (profiles/book_kernel_book256.md).
BOOK_INSTR_PER_STEP = 19.0
BOOK_SEED = 20261203


def book_mufu_per_step(entry):
    """MUFU operations per path-step of the book's GBM step loops: half a
    Box-Muller pair (lg2, sqrt, sin, cos) per step, plus ex2 for an
    arithmetic average's fixing; a European's loop takes each pair as its
    sum (lg2, sqrt, sin: 1.5 per step)."""
    from openferric_b200.instruments import AsianOption, VanillaOption
    if isinstance(entry.instrument, AsianOption):
        return 3.0
    return 1.5 if isinstance(entry.instrument, VanillaOption) else 2.0


def leg_book(stream, flush, steps, warmup, peaks, n=4096, greeks=False):
    """The synthetic book in one persistent launch at its fixed path counts:
    prices (greeks=False, the configuration-3 line), or prices with the
    pathwise delta/vega/rho/theta (greeks=True, plan mode OF_BOOK_GREEKS)."""
    from openferric_b200.analytic import bs_price
    from openferric_b200.book import BookPlan, synthetic_book
    from openferric_b200 import _abi as A
    import openferric_b200 as of
    book = synthetic_book(n)
    plan = BookPlan(book, seed=BOOK_SEED, mode=A.OF_BOOK_GREEKS if greeks else A.OF_BOOK_PRICE)
    info = plan.info()
    for _ in range(max(3, warmup)):
        plan.launch()
    res = plan.results()
    with ClockSampler(0) as clocks:
        ms, all_ms = device_timed(stream, plan.launch, steps, flush)
    plan.close()
    clk = clocks.summary()
    mufu = sum(e.num_paths * e.num_steps * book_mufu_per_step(e) for e in book)
    ps = info["path_steps"]
    v = ps / (ms / 1e3)
    sm = clk.get("sm_mhz") or 1965.0
    issue_peak = 148 * 4 * sm * 1e6
    z = []
    for e, r in zip(book, res):
        if isinstance(e.instrument, of.VanillaOption):
            m = e.market
            bs = bs_price(of.OptionType.Call, m.spot, e.instrument.strike, m.rate, 0.0,
                          m.vol_for(m.spot, e.instrument.expiry), e.instrument.expiry)
            z.append((r.price - bs) / r.stderr)
    if greeks:  # the price-mode instruction count does not apply; MUFU per step differs for barriers
        return {"workload": f"batched_book_{n} with pathwise Greeks (plan mode OF_BOOK_GREEKS; barriers by "
                            f"one-step survival)",
                "value": v, "unit": "path-steps/s", "ms_per_step": ms, "kernel_ms_all": [round(t, 3) for t in all_ms],
                "options_per_s": n / (ms / 1e3), "path_steps": ps, "tiles": info["tiles"],
                "check": {"european_calls": len(z), "max_abs_z_vs_bs": max(abs(x) for x in z),
                          "within_5_se": sum(1 for x in z if abs(x) <= 5.0)},
                "clocks": clk, "gpu_launches_per_step": 4}  # three kind-group kernels and the reduction
    return {"workload": f"batched_book_{n} (1/3 each European / daily arithmetic Asian / up-and-out call; "
                        f"synthetic_book seed {BOOK_SEED})",
            "value": v, "unit": "path-steps/s", "ms_per_step": ms, "kernel_ms_all": [round(t, 3) for t in all_ms],
            "options_per_s": n / (ms / 1e3), "path_steps": ps, "tiles": info["tiles"], "block": info["block"],
            "paths_per_thread": info["paths_per_thread"], "cuda_graph": True,
            "l2": "flushed between timed launches (256 MiB write); the kernel reads only its option and tile tables",
            "roofline": {"bound": "sfu", "achieved": mufu / (ms / 1e3) / 1e12, "peak": peaks["sfu_ops_per_s"] / 1e12,
                         "unit": "TOP/s", "frac": mufu / (ms / 1e3) / peaks["sfu_ops_per_s"],
                         "per_step": mufu / ps, "peak_source": "measured in this run by of_measure_device_peaks",
                         "issue": {"frac": v * BOOK_INSTR_PER_STEP / 32.0 / issue_peak,
                                   "per_step": BOOK_INSTR_PER_STEP,
                                   "per_step_source": "ncu smsp__inst_executed.sum of book_kernel "
                                                      "(profiles/book_kernel_book256.md)",
                                   "peak": f"148 SMs x 4 schedulers x 1 warp instruction per cycle at {sm:.0f} MHz"},
                         "traffic": None},
            "check": {"european_calls": len(z), "max_abs_z_vs_bs": max(abs(x) for x in z),
                      "within_5_se": sum(1 for x in z if abs(x) <= 5.0)},
            "clocks": clk, "gpu_launches_per_step": 2}  # the book kernel and the reduction


def mixed_book(entries):
    """The reference's VarianceReduction per option: the geometric-Asian
    control variate for the arithmetic Asians, antithetic pairs for the
    Europeans (whose reference control variate is their own payoff) and for
    the barriers (no control variate)."""
    from openferric_b200.book import BookEntry
    from openferric_b200.engines import VarianceReduction
    from openferric_b200.instruments import AsianOption
    return [BookEntry(e.instrument, e.market, e.num_paths, e.num_steps,
                      VarianceReduction.ControlVariate if isinstance(e.instrument, AsianOption)
                      else VarianceReduction.Antithetic) for e in entries]


def leg_book_se(steps, n=256):
    from openferric_b200.book import price_book_to_stderr, synthetic_book
    book = mixed_book(synthetic_book(4096)[:n])
    # warm-up: the whole procedure once, so that the context's cached buffers
    # reach their working sizes before the timed runs (the first call of a
    # process at this size pays their one-time device allocation)
    price_book_to_stderr(book, seed=1)
    times, rounds, res = [], None, None
    with ClockSampler(0) as clocks:
        for k in range(max(1, steps)):
            t0 = time.perf_counter()
            res, rounds = price_book_to_stderr(book, seed=BOOK_SEED + 100 * k)
            times.append(time.perf_counter() - t0)
    s = statistics.median(times)
    ps = sum(r.path_steps for r in rounds)
    dev = sum(r.kernel_ms for r in rounds)
    return {"workload": f"batched_book_se_{n} (the first {n} options of the 4096-option book)",
            "metric": "options/s at SE<=1e-4*S0", "value": n / s, "unit": "options/s", "ms_per_step": s * 1e3,
            "variance_reduction": "geometric-Asian control variate for the Asians; antithetic for Europeans and "
                                  "barriers",
            "timing": "wall clock of the whole procedure (pilot + follow-up launches, host planning)",
            "options_meeting_target": sum(1 for e, r in zip(book, res) if r.stderr <= 1e-4 * e.market.spot),
            "path_steps": ps, "device_ms": dev, "device_path_steps_per_s": ps / (dev / 1e3) if dev > 0 else None,
            "rounds": [r.__dict__ for r in rounds], "clocks": clocks.summary()}


# ---------------------------------------------------------------------------
# The target form: a book priced to SE <= 1e-4 S0 with its pathwise Greeks,
# against the plain FP64 engine with central bumps (2 x 4 + 1 runs per option)
# ---------------------------------------------------------------------------
GREEK_NAMES = ("delta", "vega", "rho", "theta")
FD_BUMP = 1e-5  # relative bump of the accuracy check's central differences


def _bumped(entry, which, rel):
    """The entry with spot, vol, rate or expiry scaled by (1 + rel); the
    expiry bump keeps the step count and scales the observation times."""
    from openferric_b200.book import BookEntry
    from openferric_b200.core import AsianSpec, BarrierSpec
    from openferric_b200.instruments import AsianOption, BarrierOption, VanillaOption
    import openferric_b200 as of
    inst, m = entry.instrument, entry.market
    spot, vol, rate, T = m.spot, m.vol_for(m.spot, inst.expiry), m.rate, inst.expiry
    if which == "delta":
        spot *= 1.0 + rel
    elif which == "vega":
        vol *= 1.0 + rel
    elif which == "rho":
        rate *= 1.0 + rel
    else:
        T *= 1.0 + rel
    mk = of.Market.builder().spot(spot).rate(rate).dividend_yield(m.dividend_yield).flat_vol(vol).build()
    if isinstance(inst, VanillaOption):
        new = VanillaOption(inst.option_type, inst.strike, T)
    elif isinstance(inst, AsianOption):
        a = inst.asian
        new = AsianOption(inst.option_type, inst.strike, T,
                          AsianSpec(a.averaging, a.strike_type,
                                    [min(t * T / inst.expiry, T) for t in a.observation_times]))  # last fixing at T
    else:
        new = BarrierOption(inst.option_type, inst.strike, T, inst.barrier)
    return BookEntry(new, mk, entry.num_paths, entry.num_steps, entry.variance_reduction)


def _bump_param(entry, which):
    m = entry.market
    return {"delta": m.spot, "vega": m.vol_for(m.spot, entry.instrument.expiry), "rho": m.rate,
            "theta": entry.instrument.expiry}[which]


def fp64_plain_bump_greeks(entry, se_target, seed, bump=1e-4, pilot=8192, max_rounds=4):
    """The plain FP64 GPU engine (MonteCarloPricingEngine on the reference
    draws, the entry's variance reduction): the price to the SE target
    (pilot, then the path count its SE asks for) and the four Greeks by
    central bumps with common random numbers at that path count; wall clock."""
    import openferric_b200 as of
    from openferric_b200.book import paths_for_stderr
    t0 = time.perf_counter()
    paths = pilot
    for _ in range(max_rounds):
        eng = of.MonteCarloPricingEngine(paths, entry.num_steps, seed).with_variance_reduction(entry.variance_reduction)
        base = eng.price(entry.instrument, entry.market)
        if base.stderr <= se_target:
            break
        # margin 1.1: this procedure reruns from scratch when it misses the
        # target (no pooling), and 1.1 measured faster for it than the pooled
        # driver's 1.05 (5.5 against 5.2 options/s on the 24 options)
        paths = paths_for_stderr(paths, base.stderr, se_target, margin=1.1)
    greeks = {}
    for name in GREEK_NAMES:
        up, dn = _bumped(entry, name, bump), _bumped(entry, name, -bump)
        pu = eng.price(up.instrument, up.market).price
        pd = eng.price(dn.instrument, dn.market).price
        d = (pu - pd) / (2.0 * bump * _bump_param(entry, name))
        greeks[name] = -d if name == "theta" else d
    return time.perf_counter() - t0, base, greeks, paths


def leg_book_greeks(n=256, per_kind=8, seed=BOOK_SEED):
    from openferric_b200.book import (BookEntry, price_book_fp64, price_book_greeks, price_book_to_stderr,
                                      synthetic_book)
    from openferric_b200.instruments import AsianOption, BarrierOption, VanillaOption
    book = mixed_book(synthetic_book(4096)[:n])
    price_book_to_stderr(book, seed=1, greeks=True)  # warm-up: the whole procedure once (see leg_book_se)
    with ClockSampler(0) as clocks:
        t0 = time.perf_counter()
        res, rounds = price_book_to_stderr(book, seed=seed, greeks=True)
        t32 = time.perf_counter() - t0
    ok = sum(1 for e, r in zip(book, res) if r.result.stderr <= 1e-4 * e.market.spot)
    # the comparison subset: the first `per_kind` options of each kind
    idx = []
    for cls in (VanillaOption, AsianOption, BarrierOption):
        idx += [i for i, e in enumerate(book) if isinstance(e.instrument, cls)][:per_kind]
    sub = [book[i] for i in idx]
    t0 = time.perf_counter()
    res_sub, _ = price_book_to_stderr(sub, seed=seed + 1, greeks=True)
    t32_sub = time.perf_counter() - t0
    t64, zs = 0.0, []
    for i, e in zip(idx, sub):
        dt, base, g64, _ = fp64_plain_bump_greeks(e, 1e-4 * e.market.spot, seed=42)
        t64 += dt
        r = res[i]
        se = math.hypot(r.result.stderr, base.stderr)
        zs.append(abs(r.result.price - base.price) / se if se > 0.0 else 0.0)
    # accuracy on the same draws: FP32 pathwise Greeks against central differences
    # of FP64 revaluations of the same launch (bumps 1e-5 relative: at 1e-4 the
    # differences' own truncation error reached 1e-3 on the longest-dated
    # barriers, where the FP64 pathwise Greek and a 1e-5 difference agree to 1e-8)
    # the Greeks carry no control variate: revalue the estimator they differentiate
    # (antithetic pairs kept, the Asians' control variate dropped)
    from openferric_b200.engines import VarianceReduction
    fixed = [BookEntry(e.instrument, e.market, int(r.result.diagnostics.get("num_paths")), e.num_steps,
                       e.variance_reduction if e.variance_reduction is VarianceReduction.Antithetic
                       else VarianceReduction.None_) for e, r in zip(sub, res_sub)]
    acc_seed = seed + 7
    g32 = price_book_greeks(fixed, acc_seed)
    worst, misses = {}, []
    within = 0
    for name in GREEK_NAMES:
        pu = price_book_fp64([_bumped(e, name, FD_BUMP) for e in fixed], acc_seed)
        pd = price_book_fp64([_bumped(e, name, -FD_BUMP) for e in fixed], acc_seed)
        errs = []
        for e, a, b, g in zip(fixed, pu, pd, g32):
            fd = (a.price - b.price) / (2.0 * FD_BUMP * _bump_param(e, name))
            fd = -fd if name == "theta" else fd
            v = getattr(g.result.greeks, name)
            errs.append(abs(v - fd) / max(abs(fd), 1e-2))
            hit = abs(v - fd) <= max(1e-3 * abs(fd), 2e-4)
            within += hit
            if not hit:
                misses.append({"greek": name, "kind": type(e.instrument).__name__, "steps": e.num_steps,
                               "paths": e.num_paths, "pathwise": v, "fd": fd})
        worst[name] = max(errs)
    v32, v64 = n / t32, len(sub) / t64
    return {"workload": f"batched_book_greeks_{n} (the first {n} options of the 4096-option book, price + delta, "
                        f"vega, rho, theta, every option to SE<=1e-4*S0)",
            "metric": "priced+Greeks options/s at SE<=1e-4*S0", "value": v32, "unit": "options/s",
            "ms_per_step": t32 * 1e3, "options_meeting_target": ok,
            "timing": "wall clock of the whole procedure (pilot + follow-up launches, host planning)",
            "variance_reduction": "price: geometric-Asian control variate (Asians), antithetic (Europeans), one-step "
                                  "survival (barriers, antithetic); Greeks: pathwise, no control variate",
            "rounds": [r.__dict__ for r in rounds],
            "fp64_plain_bumps": {
                "engine": "MonteCarloPricingEngine FP64 reference draws (xoshiro256++/Acklam), the same variance "
                          "reduction; price to SE<=1e-4*S0 (pilot 8192 paths, then the paths its SE asks for), "
                          "4 Greeks by central bumps of 1e-4 relative with common random numbers (9 runs/option)",
                "options": len(sub), "seconds": t64, "options_per_s": v64,
                "max_abs_z_price_vs_fp32": max(zs)},
            "fp32_same_options": {"options": len(sub), "seconds": t32_sub, "options_per_s": len(sub) / t32_sub},
            "speedup": v32 / v64, "speedup_same_options": (len(sub) / t32_sub) / v64,
            "greeks_vs_crn_fd_same_draws": {
                "max_rel_err": worst, "rel_err_floor": "relative to max(|fd|, 0.01)",
                "within_1e-3_rel_or_2e-4_abs": within, "of": 4 * len(sub), "misses": misses,
                "how": "FP32 pathwise Greeks vs central differences (bump 1e-5 relative) of FP64 revaluations of "
                       "the same launch on the same Philox draws, at each option's SE-target path count"},
            "clocks": clocks.summary()}


# ---------------------------------------------------------------------------
# Configuration 5: Longstaff-Schwartz
# ---------------------------------------------------------------------------
LSM_ALG_BYTES_PER_PATH_DATE = 16.0  # store 4 + reload 4 + cash flow read/write 8


def leg_lsm(paths, contracts, seed=7, batch_contracts=0):
    import numpy as np
    import openferric_b200 as of
    from openferric_b200.lsm import LongstaffSchwartzEngine
    rng = np.random.default_rng(BOOK_SEED)
    items = []
    for i in range(contracts):
        vol, T = (0.2, 0.4)[i % 2], (1.0, 2.0)[(i // 2) % 2]
        m = of.Market.builder().spot(rng.uniform(30.0, 50.0)).rate(0.06).flat_vol(vol).build()
        items.append((of.VanillaOption.american_put(40.0, T), m))
    total_ms, alg_bytes, prices = 0.0, 0.0, []
    with ClockSampler(0) as clocks:
        for T in (1.0, 2.0):
            sub = [it for it in items if it[0].expiry == T]
            eng = LongstaffSchwartzEngine(paths, int(50 * T), seed).with_precision(
                of.Precision.Fp32Philox).with_basis_degree(3).with_batch_contracts(batch_contracts)
            eng.price_batch(sub[:2], with_delta=True)
            out = eng.price_batch(sub, with_delta=True)
            prices += [r.price for r in out]
            total_ms += eng.last_kernel_ms
            alg_bytes += len(sub) * float(paths) * int(50 * T) * LSM_ALG_BYTES_PER_PATH_DATE
    hbm, src = measured_hbm_gbs()
    gbs = alg_bytes / (total_ms / 1e3) / 1e9
    return {"workload": f"lsm_american_put_{contracts} (K=40, S0~U[30,50], sigma in {{0.2,0.4}}, T in {{1,2}}, "
                        f"r=0.06, 50 dates/yr, {paths} FP32 paths, basis 1,x,x^2,x^3 + Cholesky, with delta)",
            "metric": "LSM contracts/s (price + delta)", "value": contracts / (total_ms / 1e3), "unit": "contracts/s",
            "ms_per_step": total_ms, "algorithmic_bytes": alg_bytes,
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                         "peak_source": src, "per_path_date_bytes": LSM_ALG_BYTES_PER_PATH_DATE,
                         "scope": "all kernels of the workload (generation, passes, final), device time from CUDA "
                                  "events around each batch"},
            "batch_contracts": batch_contracts or "automatic (path-store budget)",
            "price_range": [min(prices), max(prices)], "clocks": clocks.summary()}



def run_workload(args, local_rank):
    """Single-GPU lines of one workload leg (the default run prints them all as
    keys of the benchmark line): adjoint (configuration 4), config1, book,
    book_se, book_greeks, lsm."""
    import torch
    import openferric_b200 as of
    torch.cuda.set_device(local_rank)
    ctx = of.context(local_rank)
    if args.workload == "adjoint":
        g = greeks_comparison(args.paths)
        line = {"metric": "priced+Greeks options/s at SE<=1e-4*S0", "value": g["fp32_adjoint_options_per_s"],
                "unit": "options/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
                "config": g}
    elif args.workload == "config1":
        line = leg_config1(args.steps, args.warmup, ctx.device_peaks(), os.cpu_count() or 1)
    elif args.workload == "book":
        stream = torch.cuda.ExternalStream(ctx.stream_ptr())
        flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local_rank}")
        line = leg_book(stream, flush, args.steps, args.warmup, ctx.device_peaks(), args.book_options,
                        greeks=args.book_mode == "greeks")
    elif args.workload == "book_se":
        line = leg_book_se(args.steps, args.se_options)
    elif args.workload == "book_greeks":
        line = leg_book_greeks(args.se_options)
    else:  # lsm
        line = leg_lsm(args.paths, args.contracts, batch_contracts=args.lsm_batch)
    print(json.dumps(line, default=_json_default), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-greeks", action="store_true", help="skip the adjoint vs FP64-bump comparison")
    ap.add_argument("--workload", default="strip",
                    choices=["strip", "adjoint", "config1", "book", "book_se", "book_greeks", "lsm"],
                    help="strip is the benchmark line (it also carries every other leg as a key); the others print "
                         "one leg alone: configuration 1, 3 (book; book_se: priced to SE <= 1e-4 S0; book_greeks: "
                         "with pathwise Greeks against the FP64 engine's bumps), 4 (adjoint) or 5 (lsm)")
    ap.add_argument("--no-legs", action="store_true",
                    help="strip line only (skip the config1 / book / book_se / book_greeks / lsm keys)")
    ap.add_argument("--se-options", type=int, default=256,
                    help="book_se workload: the first N options of the synthetic book")
    ap.add_argument("--paths", type=int, default=PATHS,
                    help="paths per strip (profiling a smaller case; the benchmark workload is 2^20)")
    ap.add_argument("--book-options", type=int, default=4096,
                    help="book workload: number of options (4096 in the benchmark; fewer for a profiler capture)")
    ap.add_argument("--variance-reduction", default="none", choices=["none", "mixed"],
                    help="book_se workload: none (plain MC), or mixed (geometric-Asian control variate for the "
                         "Asians, antithetic for the Europeans and barriers)")
    ap.add_argument("--lsm-batch", type=int, default=0,
                    help="lsm workload: contracts per date loop (0 = automatic)")
    ap.add_argument("--book-mode", default="price", choices=["price", "greeks"],
                    help="book workload: prices only, or prices with the pathwise Greeks")
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
    # the warp-specialised shape (3) is timed too, so that the line shows its cost
    tile_ilp, tune_ms = autotune.tune_strip(gen, STRIKES, args.paths, reps=5, device=local_rank,
                                            candidates=(1, 2, 3))
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
    ips = INSTR_PER_STEP.get(tile_ilp)
    issue_peak = 148 * 4 * sm_run * 1e6
    issue_line = {"achieved": per_gpu * ips / 32.0 / 1e12 if ips else None, "peak": issue_peak / 1e12,
                  "unit": "T warp-inst/s", "frac": per_gpu * ips / 32.0 / issue_peak if ips else None,
                  "per_step": ips,
                  "peak_source": f"148 SMs x 4 schedulers x 1 warp instruction per cycle at the sampled "
                                 f"{sm_run:.0f} MHz",
                  "per_step_source": INSTR_SOURCE if ips else "no ncu instruction count for this tile shape"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": dict(CONFIG, parallelism=f"replicas{world}", tile_ilp=tile_ilp,
                                                          tile_ilp_ms={str(k): v for k, v in tune_ms.items()}),
        "roofline": dict(main_line, bound=bound, traffic=STRIP_DRAM_BYTES, traffic_source=STRIP_DRAM_SOURCE,
                         issue=issue_line, **{other_name: other_line},
                         # the workload's declared algorithmic count: a single-log inverse normal per
                         # draw (2 lg2 per step) + sqrt + ex2 = 4 MUFU per path-step; Box-Muller issues
                         # 5 (lg2, sqrt, sin, cos per pair of normals, sqrt of the variance)
                         frac_at_4_mufu_per_step=per_gpu * 4.0 / sfu_peak),
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
        v1, sample1 = cpu_sample(1, 5.0)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
                                "sample": f"{sample['paths']} paths x {STEPS} Heston Euler steps x 41 strikes, "
                                          f"FP64 xoshiro256++/Acklam oracle, {sample['seconds']} s; the 41 strikes "
                                          f"share one path set (the reference API would run 41 MonteCarloEngine::run "
                                          f"calls, 41x the work)",
                                "single_thread_value": v1,
                                "single_thread_sample": f"{sample1['paths']} paths, {sample1['seconds']} s",
                                **cpu_info()}
    if rank == 0 and world == 1 and not args.no_legs:
        # configurations 1, 3 and 5 and the target form, each with its own
        # device timing, clock samples and roofline (outside the timed region)
        legs = {"config1": lambda: leg_config1(args.steps, args.warmup, peaks, os.cpu_count() or 1),
                "book": lambda: leg_book(stream, flush, min(args.steps, 5), 3, peaks),
                "book_greeks_launch": lambda: leg_book(stream, flush, min(args.steps, 5), 3, peaks, greeks=True),
                "book_se": lambda: leg_book_se(1),
                "book_greeks": lambda: leg_book_greeks(),
                "lsm": lambda: leg_lsm(PATHS, 256)}
        for name, leg in legs.items():
            try:
                line[name] = leg()
            except Exception as exc:  # one failing leg does not take the benchmark line with it
                line[name] = {"error": f"{type(exc).__name__}: {exc}"}
    plan.close()
    if rank == 0:
        print(json.dumps(line, default=_json_default), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
