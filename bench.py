"""Benchmark of the engine's headline workload: path-steps per second of the fused local-vol Phoenix kernel.

Workload (default `lv_phoenix`): Dupire local vol of the SSVI power-law surface (theta_t = 0.04 t, rho -0.6, eta 1,
gamma 0.5) tabulated on 200 log-strikes x 40 expiries; a 3-year Phoenix autocall (quarterly, autocall 100 %, coupon
2 % at 70 % with memory, daily knock-in at 60 % into a put at 100 %); 756 daily steps; 2^20 paths; FP32 path
evolution with FP64 sums. `--workload heston_qe` runs the Heston QE ladder (2^16 paths x 252 steps, FP64).

One step = one launch of the fused kernel over the whole batch (plus the one-block kernel that adds the block totals),
inputs resident on the device; between steps a 512 MB buffer is written to flush L2. `value` is path-steps/s of the
device-timed steps (CUDA events on the launching stream), max over ranks. `e2e` is the same metric through the public
call with host inputs (`optlab_b200.engine.mc_price`: upload, kernel, read-back). Ranks (torchrun) each take their own
range of pairs (first_pair = rank x pairs): weak scaling, no collective in the timed steps, and one FP64 all-reduce
of the sums after them (optlab_b200.shard). `--workload adjoint` times the Greeks of the worst-of autocall (FP32
adjoint against FP64 bump-and-revalue); `--workload batch` the batched revaluation of a 512-trade book;
`--workload leverage` the SLV leverage calibration; `--workload script` the default Phoenix written as a payoff script
and run by the device's script interpreter; `--workload paths` the drop-in path engine's columns; `--workload
callable` a whole issuer-call valuation (pilot, policy fit, pricing, dual bound).

`--impl reference` times the reference's CPU implementation of the same workload instead: its path engine
(optlab::api::paths, compiled from the reference's sources into oracle/_ref) writing the 12 quarterly columns and the
daily knock-in window, then the Phoenix payoff evaluated on those columns, on all host cores.
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "option-pricing-lab_b200"))

PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}

# Executed warp instructions per path-step of the dominant kernel, measured by ncu (smsp__inst_executed.sum of one
# launch divided by its path-steps) and recorded under profiles/. The issue roofline below multiplies it by the live
# path-step rate. A launch's instruction count does not depend on timing, so a profiled launch gives it exactly.
INST_PER_PATH_STEP = {"lv_phoenix": 1.0527, "heston_qe": 20.30, "script": 1.518,
                      # the 11 class kernels of one revaluation of the 32-trade book: 326.2 G over 2.49e11 path-steps
                      "batch": 1.310,
                      # the drop-in path engine's local-vol kernel on the Phoenix model (12 columns + a daily window)
                      "paths": 2.354}
# The ALGORITHM's lane instructions per path-step of the local-vol Phoenix (one name, both legs of a pair share each
# normal), counted from the algorithm, not from the compiled code, so that extra instructions lower the fraction:
#   Philox4x32-10, one call per 4 normals = 4 pair-steps = 8 path-steps: 10 rounds x (2 wide multiplies, 2 three-way
#     xors, 2 key additions) + 4 to set the counter = 64, so 8 per path-step;
#   Box-Muller, per 2 normals = 4 path-steps: 2 conversions and 2 multiply-adds to (0, 1), a logarithm (10 with its
#     range reduction), a square root (2), sin and cos of 2 pi v (10), 2 products = 28, so 7 per path-step;
#   the local-vol step, per path-step: the table coordinate (1 multiply-add), its integer part and back (2), the
#     weight (1), the index clamp (2), the address (1), one 8-byte shared load of the interval (1), the interpolation
#     (1 multiply-add); variance x dt (1), its square root (2), the drift and the diffusion (2 multiply-adds); the
#     knock-in's running minimum (1): 14.
# 29 lane instructions = 0.906 warp instructions per path-step. The observations (12 over 756 steps) add < 1 %.
ALG_INST_PER_PATH_STEP = {"lv_phoenix": (8 + 7 + 14) / 32.0}

# Warp instructions of one leverage calibration at 2^18 particles x 504 steps: one lev_persistent launch
# (ncu smsp__inst_executed.sum).
LEV_INST_PER_CALIBRATION = 2.2436e9
# One grid barrier of 148 blocks (arrival counter with a release, acquiring polls), measured alone on a B200: 1.27 us.
# A leverage step needs three (the particles' range, the step's bins, the leverage row): 3.81 us a step is the floor
# of any calibration that keeps this dependency structure.
LEV_BARRIER_US = 1.27


def issue_roofline(warp_inst_per_s: float | None, note: str) -> dict:
    """The issue roofline of a bench line: achieved warp instructions per second (None: not measured for this size)
    against SMs x 4 schedulers x the measured max SM clock."""
    import torch

    peaks, peak_kind = load_peaks()
    sm_max = float(peaks.get("sm_max_mhz", 1965.0))
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    peak = props.multi_processor_count * 4 * sm_max * 1e6 / 1e9
    achieved = warp_inst_per_s / 1e9 if warp_inst_per_s is not None else None
    return {"bound": "issue", "achieved": achieved, "peak": peak, "unit": "Gwarp-inst/s",
            "frac": achieved / peak if achieved is not None else None, "traffic": None,
            "note": f"{note}; peak = SMs x 4 schedulers x max SM clock ({sm_max:.0f} MHz, {peak_kind})"}


# DRAM bytes (read + written) of one profiled launch of the dominant kernel: the packed inputs, read once from HBM
# and then from L2; the loop keeps its state in registers, so the figure does not grow with the path count.
DRAM_PER_LAUNCH = {"lv_phoenix": 119296, "heston_qe": 44288}


def load_peaks():
    if PEAKS_FILE.exists():
        d = json.loads(PEAKS_FILE.read_text())
        return d, "measured"
    return FALLBACK_PEAKS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the timed region runs."""

    FIELDS = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, device: int):
        self.device, self.rows, self.proc = device, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"],
                stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL,
                text=True,
            )
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) < 9:
                continue
            for name, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(mx) if mx else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def build_workload(name: str, n_paths: int | None, table: str = "builder"):
    from optlab_b200 import workloads

    if name == "lv_phoenix":
        grid = reference_rows() if table == "reference" else None
        return workloads.lv_phoenix(n_paths=n_paths or 2**20, seed=7, grid=grid), "fp32", {
            "workload": "lv_phoenix",
            "model": "Dupire local vol, SSVI power law (rho -0.6, eta 1, gamma 0.5, theta 0.04 t), "
            + ("200 x 40 table" if table == "builder" else "801 x 756 per-step rows (the reference plan's)"),
            "product": "3y Phoenix, quarterly autocall 100%, coupon 2% at 70% with memory, daily KI 60%",
            "n_paths": n_paths or 2**20,
            "n_steps": 756,
            "precision": "fp32 paths, fp64 sums",
        }
    if name == "heston_qe":
        return workloads.heston_qe_ladder(n_paths=n_paths or 2**16, seed=1), "fp64", {
            "workload": "heston_qe",
            "model": "Heston QE-M (S0 100, v0 .04, kappa 1.5, theta .04, xi .5, rho -.7, r .02, q .01)",
            "product": "11 calls K 80..120 + daily up-and-out call K 100 B 130",
            "n_paths": n_paths or 2**16,
            "n_steps": 252,
            "precision": "fp64",
        }
    raise SystemExit(f"unknown workload {name}")


def input_bytes(held) -> int:
    return int(sum(a.nbytes for a in held.keep if isinstance(a, np.ndarray)))


# ---------------------------------------------------------------------------------------------------- CPU baseline


def reference_rows():
    """The default surface tabulated as the reference's plan() does it: one 801-point row for each of the 756 daily
    steps of three years (4.8 MB of float intervals, beyond the kernels' shared-memory stage)."""
    from optlab_b200 import workloads

    return workloads.LocalVarGrid.from_surface(workloads.lv_surface(horizon=3.0), 3.0 * np.arange(1, 757) / 756, 801)


def phoenix_paths_request(n_paths: int, seed: int = 7, table: str = "builder", model: str = "lv"):
    """The local-vol Phoenix's model as a drop-in paths request (the reference's `run()`): the 12 quarterly columns
    and one daily window (lowest, highest) of the name, for n_paths paths; returns (request, Phoenix, market). table:
    "builder" (200 points x 40 expiries) or "reference" (801 points x 756 per-step rows); model: "lv", "heston"
    (v0 .04, kappa 1.5, theta .04, xi .5, rho -.7, Euler) or "slv" (the same Heston with the local variance over 0.04
    as its leverage-squared table)."""
    from optlab_b200 import workloads
    from optlab_b200.requests import paths_request

    held, _, _ = build_workload("lv_phoenix", n_paths)
    s = held.struct
    ph = workloads.Phoenix()
    obs_step, _ = ph.schedule(252)
    n_steps = s.n_steps
    all_obs = np.arange(0, n_steps + 1, dtype=np.int32)  # every step end (and t = 0) for the daily window
    col_of = np.full(len(all_obs), -1, np.int32)
    col_of[obs_step] = np.arange(len(obs_step), dtype=np.int32)
    m = workloads.FlatMarket(100.0, 0.02, 0.01)
    dt = np.ctypeslib.as_array(s.dt, shape=(n_steps,)).copy()
    t_end = np.concatenate([[0.0], np.cumsum(dt)])
    g = workloads.lv_grid() if table == "builder" else reference_rows()
    t0 = t_end[:-1]
    kind = {"lv": 1, "heston": 2, "slv": 3}[model]
    rq = paths_request(
        dt=dt, t0=t0, obs_step=all_obs, root=[[1.0]], kind=[kind], cvar=[0.04],
        heston=[0.0, 1, 1, 0, 0] if kind == 1 else [0.04, 1.5, 0.04, 0.5, -0.7], same=1, fwd=m.F(t_end)[None, :],
        n_pairs=n_paths // 2, seed=seed, step_row=g.row_of(t0), lo=g.lo, inv_dx=g.inv_dx,
        table=g.rows / 0.04 if kind == 3 else g.rows, n_x=g.n_x, col_of=col_of, n_keep=len(obs_step), win_lo=[0],
        win_hi=[n_steps],
    )
    return rq, ph, m


def cpu_reference_sample(name: str, n_paths: int, threads: int):
    """Time the reference's CPU implementation of the workload on n_paths paths: (seconds, kind, cores, detail)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle import Oracle, Reference, reference_available

    from optlab_b200 import workloads

    held, _, _ = build_workload("lv_phoenix" if name == "paths" else name, n_paths)
    kind = "reference" if reference_available() else "port"
    if name == "heston_qe":
        if kind == "reference":
            R = Reference()
            lt = np.ones(12, np.int32)
            ks = np.append(np.arange(80.0, 121.0, 4.0), 100.0)
            up = np.zeros(12, np.int32)
            up[-1] = 1
            lv = np.zeros(12)
            lv[-1] = 130.0
            t = time.perf_counter()
            R.qe_ladder(100.0, 0.02, 0.01, 1.0, 252, workloads.HESTON_CFG0, n_paths // 2, 1, lt, ks, up, lv,
                        threads=threads)
            return time.perf_counter() - t, kind, threads, "reference QE-M step on the reference Philox stream"
        t = time.perf_counter()
        Oracle().mc_price(held, threads)
        return time.perf_counter() - t, kind, threads, "oracle port (C, double)"
    # local-vol Phoenix: the reference's path engine writes the quarterly columns and the daily window, then the
    # payoff is evaluated on the columns (the reference's structured engine does this in NumPy); the paths workload
    # is the path engine alone.
    rq, ph, m = phoenix_paths_request(n_paths)
    n_obs = len(ph.schedule(252)[0])
    t = time.perf_counter()
    if kind == "reference":
        Reference().paths(rq, threads)
    else:
        Oracle().paths(rq, threads)
    if name == "paths":
        return time.perf_counter() - t, kind, threads, "reference path engine (12 columns + daily window)"
    out = next(a for a in rq.keep if isinstance(a, np.ndarray) and a.ndim == 3)[0]
    phoenix_payoff(out[:n_obs].T / 100.0, out[n_obs] / 100.0, ph, m)
    return time.perf_counter() - t, kind, threads, "reference path engine (columns + daily window) + payoff on columns"


def phoenix_payoff(perf, low, ph, market):
    """Pair-averaged Phoenix value from observation performances (paths x obs) and the window lows (paths)."""
    n, n_obs = perf.shape
    _, obs_t = ph.schedule(252)
    D = market.D(obs_t)
    pv, missed, alive = np.zeros(n), np.zeros(n), np.ones(n, bool)
    for j in range(n_obs):
        p = perf[:, j]
        hit = alive & (p >= ph.coupon_barrier)
        pv += np.where(hit, D[j] * ph.coupon * (1 + missed), 0.0)
        missed = np.where(hit, 0.0, np.where(alive, missed + 1, missed))
        if j < n_obs - 1:
            call = alive & (p >= ph.trigger)
            pv += np.where(call, D[j], 0.0)
            alive &= ~call
        else:
            ki = low < ph.ki_barrier
            pv += np.where(alive, D[j] * np.where(ki, 1 - np.maximum(ph.put_strike - p, 0), 1.0), 0.0)
    h = n // 2
    y = 0.5 * (pv[:h] + pv[h:])
    return float(y.mean()), float(y.std(ddof=1) / np.sqrt(h))


# ---------------------------------------------------------------------------------------------------- main


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="lv_phoenix",
                    choices=["lv_phoenix", "heston_qe", "adjoint", "batch", "leverage", "script", "paths", "callable"])
    ap.add_argument("--trades", type=int, default=512, help="batch workload: trades in the book")
    ap.add_argument("--paths", type=int, default=None)
    ap.add_argument("--table", default="builder", choices=["builder", "reference"],
                    help="lv_phoenix and paths: the builder's 200 x 40 grid or the reference plan's 801-point "
                    "per-step rows")
    ap.add_argument("--model", default="lv", choices=["lv", "heston", "slv"],
                    help="paths workload: the name's model (Heston and SLV with the Heston parameters of heston_qe)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="default workload: skip the nested FP64 error, Heston QE and adjoint figures")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, world, rank)
    if args.workload == "adjoint":
        return run_adjoint(args, world, rank)
    if args.workload == "batch":
        return run_batch(args, world, rank)
    if args.workload == "leverage":
        return run_leverage(args, world, rank)
    if args.workload == "script":
        return run_script(args, world, rank)
    if args.workload == "paths":
        return run_paths(args, world, rank)
    if args.workload == "callable":
        return run_callable(args, world, rank)

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    from optlab_b200 import engine
    from optlab_b200.workloads import path_steps

    held, prec, config = build_workload(args.workload, args.paths, args.table)
    n_pairs = held.struct.n_pairs
    first = rank * n_pairs
    units = path_steps(held)
    stream = torch.cuda.current_stream()
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    plan = engine.McPlan(held, prec)

    def step():
        plan.run(n_pairs, first, held.struct.seed, stream.cuda_stream)

    for _ in range(args.warmup):
        flush.zero_()
        step()
    warm = plan.result()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        t_wall = time.perf_counter()
        for k in range(args.steps):
            flush.zero_()
            starts[k].record(stream)
            step()
            ends[k].record(stream)
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t_wall
    if dist:
        dist.barrier()
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    ms_t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    res = plan.result()
    price, se = list(res.price[: res.n_out]), list(res.se[: res.n_out])
    if dist:  # the one exchange: every rank's FP64 sums into the job's price and SE
        from optlab_b200.shard import allreduce_result

        p, e = allreduce_result(res, device="cuda")
        price, se = list(p), list(e)
    per_step = ms_max / args.steps
    value = units * world * args.steps / (ms_max / 1e3)

    # end to end through the public call: host arrays in, prices out, each rank its own shard of the pairs; the job's
    # rate is every rank's path-steps over the slowest rank's median call
    held.struct.first_pair = first
    e2e_ms = []
    for _ in range(max(3, min(args.steps, 10))):
        t = time.perf_counter()
        r_e2e = engine.mc_price(held, prec)
        e2e_ms.append((time.perf_counter() - t) * 1e3)
    e2e_call_ms = statistics.median(e2e_ms)
    if dist:
        e2e_t = torch.tensor([e2e_call_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
        e2e_call_ms = float(e2e_t.item())
    e2e_value = units * world / (e2e_call_ms / 1e3)

    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return
    # the rest of the headline metric, on one GPU (each timed on its own after the headline's timed region): the
    # result's error against an FP64 run of the same request, the Heston QE ladder (path-steps/s) and the adjoint
    # Greeks ladder against FP64 bump-and-revalue (Greeks/s)
    extras = {}
    if world == 1 and not args.no_extras and args.workload == "lv_phoenix" and args.table == "builder":
        extras["error_vs_fp64"] = precision_gap(held, r_e2e)
        extras["heston_qe"] = fused_summary("heston_qe", args.steps, args.warmup, local)
        extras["adjoint"] = adjoint_summary(2**19, min(args.steps, 5), 3, local)

    peaks, peak_kind = load_peaks()
    props = torch.cuda.get_device_properties(local)
    sm_max = float(peaks.get("sm_max_mhz", 1965.0))
    issue_peak = props.multi_processor_count * 4 * sm_max * 1e6 / 1e9  # G warp-instructions/s
    ipu = INST_PER_PATH_STEP.get(args.workload) if args.table == "builder" else None  # counted on the builder grid
    alg = ALG_INST_PER_PATH_STEP.get(args.workload)
    per_gpu = value / world
    executed = {"achieved": ipu * per_gpu / 1e9 if ipu else None,
                "frac": ipu * per_gpu / 1e9 / issue_peak if ipu else None, "inst_per_path_step": ipu,
                "note": "warp instructions the compiled kernel executes per path-step (ncu) x live rate"}
    roofline = {
        "bound": "issue",
        "achieved": (alg * per_gpu / 1e9) if alg else executed["achieved"],
        "peak": issue_peak,
        "unit": "Gwarp-inst/s",
        "frac": (alg * per_gpu / 1e9 / issue_peak) if alg else executed["frac"],
        "traffic": DRAM_PER_LAUNCH.get(args.workload) if args.table == "builder" else None,
        "algorithmic_inst_per_path_step": alg,
        "executed": executed,
        "executed_over_algorithmic": (ipu / alg) if (alg and ipu) else None,
        "note": ("FP32/SFU issue-bound kernel" if prec == "fp32" else "FP64 kernel bound by its dependent FP64 chain")
        + " (no HBM or tensor-core bound applies); peak = SMs x 4 schedulers x "
        f"max SM clock ({sm_max:.0f} MHz, {peak_kind}); achieved = the algorithm's warp instructions per path-step "
        "(frozen in bench.py from the algorithm's operation count) x live rate"
        + ("" if alg else " (no algorithmic count for this workload: the executed count stands in)"),
    }
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        n_s = 2**18
        threads = os.cpu_count() or 1
        secs, kind, cores, detail = cpu_reference_sample(args.workload, n_s, threads)
        n_units = n_s * config["n_steps"]
        cpu = {"value": n_units / secs, "unit": "path-steps/s", "cores": cores, "kind": kind,
               "sample": f"{n_s} paths x {config['n_steps']} steps of the same workload ({detail})"}
    clk = clocks.summary()
    line = {
        "metric": "path-steps/s",
        "value": value,
        "unit": "path-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32" if prec == "fp32" else "f64",
        "data": "synthetic (seeded SSVI surface and Heston parameters; no market data)",
        "config": dict(config, l2="flushed between steps (512 MB write)", parallelism=f"pairs sharded over {world}"),
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": {
            "value": e2e_value,
            "unit": "path-steps/s",
            "h2d_bytes_per_step": input_bytes(held),
            "d2h_bytes_per_step": 2 * 32 * 8,
            "ms_per_call": e2e_call_ms,
        },
        "gpu_launches": 2 * args.steps,
        "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]},
        "wall_s": t_wall,
        # one run's estimate (the e2e call: each pair once); the timed steps repeat the same pairs, so their pooled
        # sums would understate the standard error
        "result": {"price": list(r_e2e.price[: r_e2e.n_out]), "se": list(r_e2e.se[: r_e2e.n_out]),
                   "timed_steps_price": price, "warmup_price": warm.price[0]},
    }
    line.update(extras)
    print(json.dumps(line))


def adjoint_summary(n_paths: int, steps: int, warmup: int, clock_device: int | None = None) -> dict:
    """cfg3: the Greeks ladder of the 3-name worst-of (n_paths paths x 1008 steps) by the FP32 adjoint, against FP64
    bump-and-revalue on the same GPU (central differences: 1 + 2 x (3 + 450) revaluations, each timed as the FP64
    smoothed revaluation of the same request; a bounded number is timed and the ladder's time is their median times
    907). Also the FP32 adjoint against the FP64 adjoint on the same paths: every price and Greek within 4 SE and 1e-4
    relative (vegas relative to the ladder's largest), the north-star criterion."""
    import torch

    from optlab_b200 import workloads
    from optlab_b200.adjoint import AdjointPlan, VegaNodes, autocall_greeks

    w = workloads.worst_of(n_paths=n_paths)
    nodes = VegaNodes(w.row_name, w.row_T, w.row_lo, w.row_inv_dx, w.n_x, w.node_T, w.node_k)
    n_greeks = w.held.struct.n_names * (1 + len(w.node_T) * len(w.node_k))
    s = w.held.struct
    units = 2 * s.n_pairs * s.n_steps * s.n_names
    states = s.n_steps * s.n_names * 2 * s.n_pairs * 4  # FP32 states the forward keeps when it keeps every step
    plan = AdjointPlan(w.held, 0.005, "fp32")
    for _ in range(warmup):
        autocall_greeks(w.held, nodes, 0.005, plan=plan)
    torch.cuda.synchronize()
    times, fwd, bwd = [], [], []
    with ClockSampler(clock_device if clock_device is not None else 0) as clocks:
        for _ in range(steps):
            t = time.perf_counter()
            g32 = autocall_greeks(w.held, nodes, 0.005, plan=plan)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t)
            fwd.append(g32["forward_ms"]), bwd.append(g32["backward_ms"])
    plan.close()
    t_adj = statistics.median(times)
    # FP64 references: the adjoint in double (agreement) and the smoothed revaluation (bump-and-revalue cost)
    p64 = AdjointPlan(w.held, 0.005, "fp64")
    g64 = autocall_greeks(w.held, nodes, 0.005, plan=p64)
    reval = []
    for _ in range(max(3, min(steps, 6))):
        r = p64.run(grad=False)
        reval.append(r.forward_ms / 1e3)
    p64.close()
    t_rev = statistics.median(reval)
    n_reval = 1 + 2 * n_greeks
    vscale = np.abs(g64["vega"]).max()
    dv = np.abs(g32["vega"] - g64["vega"])
    dd = np.abs(g32["delta"] - g64["delta"])
    dp = abs(g32["price"] - g64["price"])
    over_se = {"price": dp / g64["price_se"], "delta": float(np.max(dd / np.maximum(g64["delta_se"], 1e-30))),
               "vega": float(np.max(dv / np.maximum(g64["vega_se"], 1e-30)))}
    rel = {"price": dp / abs(g64["price"]), "delta": float(np.max(dd / np.maximum(np.abs(g64["delta"]), 1e-30))),
           "vega": float(dv.max() / vscale)}
    return {
        "config": {"workload": "adjoint_worst_of", "n_paths": 2 * s.n_pairs, "n_steps": s.n_steps, "names": s.n_names,
                   "nodes_per_name": [len(w.node_T), len(w.node_k)], "smoothing": 0.005,
                   "states_kept": "every step" if states <= 24 * 2**30 else "every fourth step",
                   "states_bytes": states},
        "greeks": n_greeks,
        "greeks_per_s": n_greeks / t_adj,
        "ms_per_ladder": t_adj * 1e3,
        "adjoint": {"forward_ms": statistics.median(fwd), "backward_ms": statistics.median(bwd),
                    "path_steps_per_s": 2 * units / t_adj, "price": g32["price"], "price_se": g32["price_se"]},
        "bump_and_revalue_fp64": {"revaluation_ms": t_rev * 1e3, "revaluations": n_reval,
                                   "ladder_s": n_reval * t_rev, "greeks_per_s": n_greeks / (n_reval * t_rev),
                                   "timed_revaluations": len(reval)},
        "speedup_vs_fp64_bump": (n_reval * t_rev) / t_adj,
        "fp32_vs_fp64": {"max_diff_over_se": over_se, "max_diff_rel": rel,
                         "within_4se": bool(max(over_se.values()) <= 4.0),
                         "within_1e-4_rel": bool(max(rel.values()) <= 1e-4),
                         "note": "FP32 adjoint against the FP64 adjoint on the same paths; vegas relative to the "
                                 "ladder's largest; the FP64 adjoint is checked against central differences on "
                                 "common random numbers in the tests"},
        "clocks": {k: v for k, v in clocks.summary().items() if k != "samples"},
    }


def run_adjoint(args, world, rank):
    """The cfg3 line: adjoint_summary at 2^19 paths (or --paths)."""
    import torch

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    a = adjoint_summary(args.paths or 2**19, args.steps, args.warmup, int(os.environ.get("LOCAL_RANK", "0")))
    line = {
        "metric": "Greeks/s (delta per name + vega per node, FP32 adjoint)",
        "value": a["greeks_per_s"],
        "unit": "Greeks/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": a["ms_per_ladder"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded SSVI surfaces)",
        "config": a["config"],
        "adjoint": a["adjoint"],
        "bump_and_revalue_fp64": a["bump_and_revalue_fp64"],
        "speedup_vs_fp64_bump": a["speedup_vs_fp64_bump"],
        "fp32_vs_fp64": a["fp32_vs_fp64"],
        "clocks": a["clocks"],
        "gpu_launches": 2 * args.steps,
    }
    print(json.dumps(line))


def fused_summary(workload: str, steps: int, warmup: int, clock_device: int) -> dict:
    """One fused workload (its default size) timed as the headline is: device steps between L2 flushes (CUDA events
    on the launching stream), then the public one-shot call from host arrays; with its issue roofline."""
    import torch

    from optlab_b200 import engine
    from optlab_b200.workloads import path_steps

    held, prec, config = build_workload(workload, None)
    n_pairs = held.struct.n_pairs
    units = path_steps(held)
    stream = torch.cuda.current_stream()
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    plan = engine.McPlan(held, prec)
    for _ in range(warmup):
        flush.zero_()
        plan.run(n_pairs, 0, held.struct.seed, stream.cuda_stream)
    plan.result()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.synchronize()
    with ClockSampler(clock_device) as clocks:
        for a, b in ev:
            flush.zero_()
            a.record(stream)
            plan.run(n_pairs, 0, held.struct.seed, stream.cuda_stream)
            b.record(stream)
        torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    res = plan.result()
    plan.close()
    del flush
    e2e_ms = []
    for _ in range(max(3, min(steps, 10))):
        t = time.perf_counter()
        engine.mc_price(held, prec)
        e2e_ms.append((time.perf_counter() - t) * 1e3)
    value = units * steps / (ms / 1e3)
    ipu = INST_PER_PATH_STEP.get(workload)
    return {
        "metric": "path-steps/s", "value": value, "unit": "path-steps/s", "ms_per_step": ms / steps,
        "dtype": "f32" if prec == "fp32" else "f64", "config": config,
        "roofline": issue_roofline(ipu * value if ipu else None, "achieved = ncu warp instructions per path-step x "
                                   "live rate"),
        "e2e": {"value": units / (statistics.median(e2e_ms) / 1e3), "unit": "path-steps/s",
                "h2d_bytes_per_step": input_bytes(held), "d2h_bytes_per_step": 2 * 32 * 8,
                "ms_per_call": statistics.median(e2e_ms)},
        "result": {"price": list(res.price[: res.n_out]), "se": list(res.se[: res.n_out])},
        "clocks": {k: v for k, v in clocks.summary().items() if k != "samples"},
    }


def precision_gap(held, res32) -> dict:
    """The FP32 result against an FP64 run of the same request (same pairs, same normals up to rounding): per
    output the relative gap and the gap in FP64 standard errors."""
    from optlab_b200 import engine

    plan = engine.McPlan(held, "fp64")
    plan.run(held.struct.n_pairs, held.struct.first_pair, held.struct.seed)
    r64 = plan.result()
    plan.close()
    n = r64.n_out
    p32, p64 = np.array(res32.price[:n]), np.array(r64.price[:n])
    se64 = np.array(r64.se[:n])
    gap = np.abs(p32 - p64)
    return {"fp64_price": list(p64), "fp64_se": list(se64),
            "rel_gap": list(gap / np.maximum(np.abs(p64), 1e-300)), "gap_over_se": list(gap / np.maximum(se64, 1e-300)),
            "max_rel_gap": float(np.max(gap / np.maximum(np.abs(p64), 1e-300))),
            "max_gap_over_se": float(np.max(gap / np.maximum(se64, 1e-300))),
            "fp64_kernel_ms": r64.kernel_ms}


def run_batch(args, world, rank):
    """cfg4: the seeded book (512 trades, 60 scenarios: spot, vol and skew moves) revalued by one replay of the
    captured graph, FP32 paths with FP64 sums; against the same simulations as one launch per trade simulation.
    Units: name-path-steps simulated (2 paths per pair x steps x names, over the base and the vol-scenario
    simulations; spot moves ride on the base simulation). One rank: the book is one job (more GPUs would split its
    trades)."""
    import torch

    from optlab_b200.batch import Batch, sample_book

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if rank != 0:
        return
    book = sample_book(n_trades=args.trades)
    units = book.path_steps()
    t0 = time.perf_counter()
    b = Batch(book, "fp32")
    t_create = time.perf_counter() - t0
    t0 = time.perf_counter()
    b.tune()
    t_tune = time.perf_counter() - t0
    shapes = b.classes()
    b.capture()
    stream = torch.cuda.current_stream()
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(args.warmup):
        flush.zero_()
        b.launch(stream)
        b.result()
    ms = []
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            b.launch(stream)
            ms.append(b.result()[2])
    price, se, _ = b.result()
    per_trade = []
    for _ in range(max(1, min(args.steps, 3))):
        flush.zero_()
        b.run_per_trade(stream)
        per_trade.append(b.result()[2])
    b.close()
    # end to end: the public calls from host arrays (upload, one direct run, read back the values)
    e2e = []
    for _ in range(max(1, min(args.steps, 2))):
        t = time.perf_counter()
        with Batch(book, "fp32") as g:
            g.launch()
            g.result()
        e2e.append(time.perf_counter() - t)
    h2d = sum(getattr(book, k).nbytes for k in ("table", "row_lo", "row_inv_dx", "root", "leg_type", "leg_strike",
                                                  "leg_barrier", "leg_level", "obs_step", "obs_trigger",
                                                  "obs_discount", "spot_shift", "vol_shift", "vol_tilt",
                                                  "carry_rate", "carry_div"))
    h2d += book.n_trades * ctypes_sizeof_trade()
    n_sims = book.simulations()
    t_step = statistics.median(ms) / 1e3
    t_pt = statistics.median(per_trade) / 1e3
    cpu = None
    if not args.no_cpu_baseline:
        n_s = 2**18
        secs, kind, cores, detail = cpu_reference_sample("lv_phoenix", n_s, os.cpu_count() or 1)
        cpu = {"value": n_s * 756 / secs, "unit": "path-steps/s", "cores": cores, "kind": kind,
               "sample": f"{n_s} paths x 756 steps of the local-vol Phoenix, the book's dominant kind of simulation "
               f"({detail})"}
    clk = clocks.summary()
    line = {
        "metric": "path-steps/s",
        "value": units / t_step,
        "unit": "path-steps/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_step * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded book, SSVI surfaces and Heston parameters)",
        "config": {"workload": "batch_revaluation", "trades": book.n_trades, "scenarios": book.n_scenarios - 1,
                   "simulations": n_sims, "revaluations": book.revaluations(), "path_steps": units,
                   "l2": "flushed between steps (512 MB write); the book's paths are far larger than L2"},
        "revaluations_per_s": book.revaluations() / t_step,
        "per_trade_launches": {"ms_per_step": t_pt * 1e3, "path_steps_per_s": units / t_pt,
                               "speedup_of_graph": t_pt / t_step, "launches": n_sims},
        "autotune": {"seconds": t_tune, "create_seconds": t_create, "classes": shapes,
                     "sample_speedup_over_untuned_shapes": (sum(c["untuned_us"] for c in shapes) /
                                                            max(1, sum(c["tuned_us"] for c in shapes)))},
        "roofline": issue_roofline(INST_PER_PATH_STEP["batch"] * units / t_step,
                                   "FP32/SFU issue-bound stepping as the fused kernels; achieved = ncu warp "
                                   "instructions per path-step of the class kernels (32-trade book) x live rate"),
        "cpu_baseline": cpu,
        "e2e": {"value": units / statistics.median(e2e), "unit": "path-steps/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": n_sims * 32 * 2 * 8, "seconds_per_call": statistics.median(e2e)},
        "gpu_launches": args.steps * (1 + len({(t.model, t.n_names, t.product) for t in book.trades})),
        "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]},
        "result": {"mean_base_price": float(price[:, 0].mean()), "median_se": float(np.median(se[:, 0]))},
    }
    print(json.dumps(line))


def run_leverage(args, world, rank):
    """cfg2: the SLV leverage calibration by particles (2^18 particles x 504 steps, 128-point regression grid, 400
    bins), FP32 particles with FP64 bins and regression, through ob_leverage (upload of the 504 x 801 local-variance
    rows, one persistent kernel over the 504 dependent steps, read-back of the two 504 x 128 tables). Units:
    particle-steps. `value` is timed by CUDA events around the call on its stream (the upload of 3.2 MB is inside
    it); `e2e` by the host clock around the same call. The roofline is the latency floor of three grid barriers a
    step, with the issue rate beside it."""
    import torch

    from optlab_b200 import engine, workloads

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if rank != 0:
        return
    n_particles = args.paths or 2**18
    held = workloads.slv_leverage(n_particles=n_particles)
    s = held.struct
    units = 2 * s.n_pairs * s.n_steps
    for _ in range(args.warmup):
        engine.leverage(held, "fp32")
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    wall = []
    with ClockSampler(local) as clocks:
        for a, b in ev:
            t = time.perf_counter()
            a.record()
            engine.leverage(held, "fp32")
            b.record()
            torch.cuda.synchronize()
            wall.append(time.perf_counter() - t)
    ms = statistics.median(a.elapsed_time(b) for a, b in ev)
    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "oracle"))
        from oracle import Reference, reference_available

        if reference_available():
            n_s = 2**16
            small = workloads.slv_leverage(n_particles=n_s)
            threads = os.cpu_count() or 1
            t = time.perf_counter()
            Reference().leverage(small, threads=threads)
            secs = time.perf_counter() - t
            cpu = {"value": n_s * s.n_steps / secs, "unit": "path-steps/s", "cores": threads, "kind": "reference",
                   "sample": f"{n_s} particles x {s.n_steps} steps of the same calibration (optlab::api::leverage, "
                   f"CPU backend, compiled from the reference's sources)"}
    clk = clocks.summary()
    line = {
        "metric": "path-steps/s",
        "value": units / (ms / 1e3),
        "unit": "path-steps/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "us_per_time_step": ms * 1e3 / s.n_steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (SSVI surface, Heston parameters)",
        "config": {"workload": "slv_leverage", "particles": 2 * s.n_pairs, "n_steps": s.n_steps, "n_x": s.n_x,
                   "n_bins": s.n_bins, "n_fine": s.n_fine, "lv_row_points": s.n_lv,
                   "l2": "particles stay in the persistent blocks' shared memory; the calibration is latency-bound"},
        "roofline": {
            "bound": "latency",
            "achieved": s.n_steps / (ms / 1e3),
            "peak": 1e6 / (3 * LEV_BARRIER_US),
            "unit": "time-steps/s",
            "frac": (s.n_steps / (ms / 1e3)) / (1e6 / (3 * LEV_BARRIER_US)),
            "traffic": None,
            "note": f"peak = three grid barriers a step at the measured {LEV_BARRIER_US} us each; achieved includes "
                    "the call's upload and read-back",
            "issue": issue_roofline(
                LEV_INST_PER_CALIBRATION / (ms / 1e3)
                if LEV_INST_PER_CALIBRATION and 2 * s.n_pairs == 2**18 and s.n_steps == 504 else None,
                "achieved = ncu warp instructions of a calibration / its measured time"),
        },
        "cpu_baseline": cpu,
        "e2e": {"value": units / statistics.median(wall), "unit": "path-steps/s",
                "h2d_bytes_per_step": s.n_steps * (s.n_lv + 5) * 8, "d2h_bytes_per_step": 2 * s.n_steps * s.n_x * 8},
        # one persistent kernel a calibration; the three-kernel schedule: lev_init, then per step bin (not at step 0),
        # regress and step
        "gpu_launches": args.steps * (3 * s.n_steps if os.environ.get("OPTLAB_B200_LEVERAGE") == "graphs" else 1),
        "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]},
        "result": {"leverage_at_atm_last_step": float(held.values[-1, s.n_x // 2])},
    }
    print(json.dumps(line))


def phoenix_script(ph, steps_per_year: int) -> str:
    """The local-vol Phoenix of the default workload written in the payoff language."""
    n_obs = int(round(ph.years * ph.obs_per_year))
    lines = ["underlying X", "param S0 = 100", f"param cb = {ph.coupon_barrier!r}", f"param cpn = {ph.coupon!r}",
             f"param call = {ph.trigger!r}", f"param ki = {ph.ki_barrier!r}", f"param K = {ph.put_strike!r}"]
    for j in range(1, n_obs + 1):
        t = j / ph.obs_per_year
        lines.append(f"event t={t!r} pay t={t!r}")
        if j == 1:
            lines.append("  missed = 0")
        lines += ["  perf = X / S0", "  if perf >= cb then", "    pay cpn * (1 + missed) as coupon", "    missed = 0",
                  "  else", "    missed = missed + 1", "  end"]
        if j < n_obs:
            lines += ["  if perf >= call then", "    pay 1 as redemption", "    terminate", "  end"]
        else:
            n_fix = int(round(ph.years * steps_per_year))
            lines += [f"  knocked = lowest(X, t=0, t={t!r}, n={n_fix}) < ki * S0", "  if knocked then",
                      "    pay 1 - max(K - perf, 0) as redemption", "  else", "    pay 1 as redemption", "  end"]
        lines.append("end")
    return "\n".join(lines) + "\n"


def run_script(args, world, rank):
    """The default workload's Phoenix (2^20 paths x 756 steps of local vol, FP32 paths, FP64 sums) written as a payoff
    script and run by the device's script interpreter (ob_script_price), beside the fused Phoenix kernel on the same
    paths: what a general script costs against the specialised kernel. Units: path-steps."""
    import torch

    from optlab_b200 import engine, workloads
    from optlab_b200 import script as sc

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if rank != 0:
        return
    ph = workloads.Phoenix()
    held = workloads.lv_phoenix(n_paths=args.paths or 2**20, phoenix=ph,
                                grid=reference_rows() if args.table == "reference" else None)
    comp = sc.compile_script(phoenix_script(ph, 252))
    req = sc.script_request(comp, held, lambda t: float(np.exp(-0.02 * t)))
    units = workloads.path_steps(held)
    for _ in range(args.warmup):
        sc.run(req, "fp32")
    ms, wall = [], []
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            t = time.perf_counter()
            r = sc.run(req, "fp32")
            wall.append(time.perf_counter() - t)
            ms.append(r.kernel_ms)
    plan = engine.McPlan(held, "fp32")  # the fused kernel on the same pairs, warmed as the script was
    for _ in range(args.warmup):
        plan.run(held.struct.n_pairs, 0, held.struct.seed)
    plan.result()
    fused_ms = []
    for _ in range(args.steps):
        plan.run(held.struct.n_pairs, 0, held.struct.seed)
        fused = plan.result()
        fused_ms.append(fused.kernel_ms)
    t_ms = statistics.median(ms)
    clk = clocks.summary()
    line = {
        "metric": "path-steps/s",
        "value": units / (t_ms / 1e3),
        "unit": "path-steps/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded SSVI surface; the default workload's Phoenix as a script)",
        "config": {"workload": "script_phoenix", "n_paths": 2 * held.struct.n_pairs, "n_steps": held.struct.n_steps,
                   "instructions": int(comp.code.shape[0]), "registers": int(comp.n_regs),
                   "table": f"{held.struct.n_rows} rows x {held.struct.n_x} points ({args.table})",
                   "l2": "no flush: one call holds uploads, kernel and read-back"},
        "fused_kernel": {"ms_per_step": statistics.median(fused_ms), "price": fused.price[0],
                         "script_over_fused_time": t_ms / statistics.median(fused_ms)},
        "roofline": issue_roofline(
            INST_PER_PATH_STEP["script"] * units / (t_ms / 1e3)
            if held.struct.n_pairs == 2**19 and args.table == "builder" else None,
            "the local-vol step plus the interpreter at events; achieved = ncu warp instructions per path-step x "
            "live rate"),
        "cpu_baseline": None,
        "e2e": {"value": units / statistics.median(wall), "unit": "path-steps/s",
                "h2d_bytes_per_step": int(req.struct.n_code * 16 + held.struct.n_rows * held.struct.n_x * 8),
                "d2h_bytes_per_step": 5 * 8},
        "gpu_launches": 2 * args.steps,
        "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]},
        "result": {"price": r.price, "se": r.se, "fused_price": fused.price[0], "fused_se": fused.se[0]},
    }
    print(json.dumps(line))


def ctypes_sizeof_trade() -> int:
    import ctypes

    from optlab_b200._abi import ObBatchTrade

    return ctypes.sizeof(ObBatchTrade)


def run_paths(args, world, rank):
    """The drop-in path engine (the reference's `run()`, `ob_paths`): the local-vol Phoenix's model, 2^20 paths x 756
    steps, its 12 quarterly spot columns and one daily window (lowest and highest spot) written for every path and
    copied back to the host (2^20 x 14 doubles = 117 MB). `value`: path-steps per second of the kernel, timed by CUDA
    events inside the engine (inputs on the device); `e2e`: the whole call from host arrays (upload, kernel, the
    columns back), by the host clock. One rank: the call is one job."""
    import torch

    from optlab_b200 import engine

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if rank != 0:
        return
    n_paths = args.paths or 2**20
    rq, _, _ = phoenix_paths_request(n_paths, table=args.table, model=args.model)
    s = rq.struct
    units = 2 * s.n_pairs * s.n_steps * s.n_names
    for _ in range(args.warmup):
        engine.paths(rq, "fp32")
    kern, wall = [], []
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
        for _ in range(args.steps):
            t = time.perf_counter()
            k_ms, _ = engine.paths(rq, "fp32")
            wall.append(time.perf_counter() - t)
            kern.append(k_ms)
    t_k = statistics.median(kern) / 1e3
    out_bytes = 2 * s.n_pairs * s.n_names * s.n_cols * 8
    in_bytes = input_bytes(rq) - out_bytes
    cpu = None
    if not args.no_cpu_baseline and args.model == "lv":
        n_s = 2**18
        secs, kind, cores, detail = cpu_reference_sample("paths", n_s, os.cpu_count() or 1)
        cpu = {"value": n_s * s.n_steps / secs, "unit": "path-steps/s", "cores": cores, "kind": kind,
               "sample": f"{n_s} paths x {s.n_steps} steps ({detail})"}
    clk = clocks.summary()
    ipu = INST_PER_PATH_STEP.get("paths")
    line = {
        "metric": "path-steps/s",
        "value": units / t_k,
        "unit": "path-steps/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_k * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded SSVI surface)",
        "config": {"workload": "paths", "n_paths": 2 * s.n_pairs, "n_steps": s.n_steps, "columns": s.n_cols,
                   "table": f"{s.n_rows} rows x {s.n_x} points ({args.table})", "model": args.model,
                   "output_bytes": out_bytes, "l2": "each call uploads its inputs and writes 117 MB of columns"},
        "roofline": issue_roofline(ipu * units / t_k
                                   if ipu and n_paths == 2**20 and args.table == "builder" and args.model == "lv"
                                   else None,
                                   "the local-vol step plus the column and window stores; achieved = ncu warp "
                                   "instructions per path-step x live rate"),
        "cpu_baseline": cpu,
        "e2e": {"value": units / statistics.median(wall), "unit": "path-steps/s", "h2d_bytes_per_step": int(in_bytes),
                "d2h_bytes_per_step": int(out_bytes)},
        # outputs of 32 MB or more run in four chunks of pairs, one launch each
        "gpu_launches": args.steps * (4 if out_bytes >= 32 << 20 and s.n_pairs >= 4 else 1),
        "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]},
    }
    print(json.dumps(line))


def run_callable(args, world, rank):
    """The issuer's call: the callable reverse convertible of the reference's issuer-call test (2y, semiannual 3 %
    coupons, callable at par on the first three dates, redemption min(S / S0, 1)) under Black-Scholes as a flat
    local-variance table, FP64. One step is one whole valuation: the device pilot (pilot_paths(2 pairs) paths,
    recorded in device memory), the Longstaff-Schwartz fit on the device (ob_script_pilot_fit), the pricing run
    applying the policy (2^17 pairs), and the
    Andersen-Broadie dual bound from 1000 outer paths x 200 branched continuations at each of the 3 call dates. Timed
    by the host clock around the whole valuation (every stage reads its results back); `value` is valuations per
    second, `e2e` the same figure (the stages take host arrays and return host results)."""
    import torch

    from optlab_b200 import exercise
    from optlab_b200 import script as sc
    from optlab_b200._abi import OB_MODEL_PATHS, OB_PRODUCT_LADDER
    from optlab_b200.models import time_grid
    from optlab_b200.requests import mc_request

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if rank != 0:
        return
    case = json.loads((ROOT / "tests" / "golden" / "script_dual.json").read_text())
    r, q, vol = case["r"], case["q"], case["vol"]
    comp = sc.compile_script(case["script"])

    def disc(t):
        return float(np.exp(-r * t))

    def make_sim(n_pairs, seed):
        grid = time_grid(comp.timeline.sim_times, 1 / 12)
        dt, t0 = np.diff(grid), grid[:-1]
        n_x = 11
        return mc_request(model=OB_MODEL_PATHS, dt=dt, t0=t0, spot=[100.0], n_pairs=n_pairs, seed=seed, root=[[1.0]],
                          kind=np.ones(1, np.int32), cvar=[vol**2], log_fwd=(r - q) * grid[None, :],
                          step_row=np.zeros((1, len(dt)), np.int32), lo=[-5.0], inv_dx=[(n_x - 1) / 10.0],
                          table=np.full((1, n_x), vol**2), n_x=n_x, r=r, q=q, product=OB_PRODUCT_LADDER, leg_type=[1],
                          leg_strike=[1.0])

    n_pairs = (args.paths or 2**18) // 2
    n_outer, n_inner = 1000, 200

    def valuation():
        res, policy = exercise.price(comp, make_sim, n_pairs, 11, disc, "fp64")
        b = exercise.dual_bound(comp, make_sim, policy, res.price, res.se, 11, disc, n_outer=n_outer, n_inner=n_inner,
                                precision="fp64")
        return res, b

    for _ in range(args.warmup):
        valuation()
    wall = []
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t = time.perf_counter()
            res, b = valuation()
            torch.cuda.synchronize()
            wall.append(time.perf_counter() - t)
    t_s = statistics.median(wall)
    clk = clocks.summary()
    n_calls = len(comp.calls)
    line = {
        "metric": "callable valuations/s",
        "value": 1.0 / t_s,
        "unit": "valuations/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_s * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (the reference's callable reverse convertible under Black-Scholes)",
        "config": {"workload": "callable", "pricing_pairs": n_pairs, "pilot_paths": exercise.pilot_paths(2 * n_pairs),
                   "dual_outer": n_outer, "dual_inner": n_inner, "call_dates": n_calls,
                   "l2": "no flush: each stage uploads its inputs and reads its results back"},
        "roofline": None,
        "cpu_baseline": None,
        "e2e": {"value": 1.0 / t_s, "unit": "valuations/s", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None},
        # script runs (kernel and sums, 2 each): pilot, pricing, outer paths, one branched run a call date; the fit:
        # per call date its preparation, moments, order statistics, three normal-equation passes (2 each) and the
        # decisions, then the flows before the first call date (when it is not the first event) and the total
        "gpu_launches": 2 * (3 + n_calls) + 10 * n_calls + (comp.calls[0][0] != 0) + 1,
        "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]},
        "result": {"price": res.price, "se": res.se, "dual_lower": b["lower"], "gap": b["gap"], "gap_se": b["gap_se"],
                   "pde": case["pde"]},
    }
    print(json.dumps(line))


def run_reference(args, world, rank):
    if rank != 0:
        return
    if args.workload not in ("lv_phoenix", "heston_qe", "paths"):
        # the other workloads carry their CPU comparison in their own line (cpu_baseline, or the FP64
        # bump-and-revalue of the adjoint)
        print(json.dumps({"impl": "reference", "unavailable": f"no separate reference arm for --workload "
                          f"{args.workload}: its line from the default arm holds the reference comparison"}))
        return
    threads = os.cpu_count() or 1
    n_s = 2**18
    for _ in range(args.warmup):
        cpu_reference_sample(args.workload, n_s, threads)
    secs = []
    for _ in range(args.steps):
        s, kind, cores, detail = cpu_reference_sample(args.workload, n_s, threads)
        secs.append(s)
    _, _, config = build_workload("lv_phoenix" if args.workload == "paths" else args.workload, None)
    if args.workload == "paths":
        config = dict(config, workload="paths", product="12 quarterly columns + a daily window (no payoff)")
    else:  # the workload exactly as the default arm names it (each timed step is a bounded sample of it)
        config = dict(config, l2="flushed between steps (512 MB write)", parallelism=f"pairs sharded over {world}")
    n_units = n_s * config["n_steps"]
    tot = sum(secs)
    value = n_units * args.steps / tot
    line = {
        "impl": "reference",
        "metric": "path-steps/s",
        "value": value,
        "unit": "path-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": tot / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": config,
        "cpu_baseline": {"value": value, "unit": "path-steps/s", "cores": cores, "kind": kind,
                         "sample": f"{n_s} paths x {config['n_steps']} steps per step ({detail})"},
        "e2e": {"value": value, "unit": "path-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        # what each timed step ran, where it differs from the workload the config names
        "reference_sample": {
            "n_paths": n_s,
            "precision": "fp64 (the reference's CPU engine computes in double)",
            "threads": cores,
            "payoff": ("none: the path engine's columns and window are the output" if args.workload == "paths" else
                       "the Phoenix evaluated on the engine's columns by a vectorised NumPy restatement of the "
                       "reference's script evaluator (cheaper than its Evaluator, so the ratio against this arm is "
                       "conservative)" if args.workload == "lv_phoenix" else
                       "the reference's QE step on its Philox stream with the 11 calls and the up-and-out call"),
        },
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
