"""FMM throughput benchmark: bodies/s of full Laplace FMM solves on one B200 per rank.

Workload (the single large adaptive solve): N = 4,194,304 bodies from a Plummer
sphere (scale 1, truncated at r = 20), equal charges 1/N, P = 8, theta = 0.35,
ncrit tuned in {32, 64, 128}, nspawn = 5000, mixed precision (FP32 M2L/P2P with
compensated accumulation, FP64 root levels).  One step = one complete solve from bodies resident
in device memory to results in device memory: getBounds (with the reference's
drift), tree build, upward pass, dual tree traversal with M2L and P2P, downward
pass, results scattered back to input order.

  value : N * steps / device time of the steps (CUDA events on the solver's stream)
  e2e   : the same through the public API from pinned host buffers: the host->device
          copy of the bodies and the device->host copy of the results are timed
  roofline : the dominant kernel timed live with CUDA events; rooflines: every
             hot-path kernel (P2P against the FP32 FMA peak, M2L and the
             upward / downward passes against the measured HBM bandwidth)
  cpu_baseline : the reference's own CPU FMM (its headers compiled in place),
          all host threads, on a bounded sample of the same workload

Multi-GPU (torchrun): replicas only -- every rank solves its own instance, no
data-path collective; the step time is the max over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "exafmm-beta_b200")

WORKLOAD = dict(name="plummer_4m_p8", n=4_194_304, P=8, theta=0.35, ncrit=64, nspawn=5000, seed=2)
METRIC = "FMM bodies/s (full mixed-precision solve, Plummer N=4,194,304, P=8, theta=0.35)"
CPU_SAMPLE_N = 262_144
# DRAM bytes per M2L pair of the mixed M2L phase at P = 8: the per-class products write each
# pair's contribution (256 B) and the per-target pass reads it back; dram__bytes_read.sum +
# dram__bytes_write.sum of those two kernels in the ncu capture of the 1M-body case (4.43 GB
# for 8,233,680 pairs, profiles/m2l_traffic_plummer_1m_p8_mixed_ncrit128.txt), scaled by pairs
M2L_DRAM_BYTES_PER_PAIR = 538.0


def _package():
    if "exafmm_b200" in sys.modules:
        return sys.modules["exafmm_b200"]
    spec = importlib.util.spec_from_file_location("exafmm_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["exafmm_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), float(p["bf16_tflops"]), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms while running."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        # nvidia-smi start-up is CPU-heavy: let it reach its first sample before timing
        t0 = time.time()
        while self.proc and time.time() - t0 < 5.0:
            try:
                if os.path.getsize(self.path) > 0:
                    break
            except OSError:
                pass
            time.sleep(0.05)
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9 and parts[1].isdigit():
                    rows.append(parts)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [int(r[1]) for r in rows]
        smax = int(rows[0][2])
        power = [float(r[3]) if r[3].replace(".", "", 1).isdigit() else 0.0 for r in rows]
        loaded = [s for s, p in zip(sm, power) if p > 0.35 * max(power)] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": int(statistics.median(loaded)), "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(rows), "power_w_max": max(power)}


def cpu_reference_baseline(n_sample: int, threads: int, steps: int = 1):
    """The reference CPU FMM (oracle/_ref) or, if it was not built, the C restatement,
    on a smaller Plummer system with the workload's parameters."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import bindings
    pkg = _package()
    from exafmm_b200 import datasets
    x = datasets.plummer(n_sample, seed=WORKLOAD["seed"])
    kw = dict(P=WORKLOAD["P"], theta=WORKLOAD["theta"], ncrit=WORKLOAD["ncrit"], nspawn=WORKLOAD["nspawn"])
    if bindings.reference_available():
        impl, kind = bindings.Reference(), "reference"
        run = lambda: impl.solve(x, threads=threads, record_lists=False, **kw)
    else:
        impl, kind = bindings.Oracle(), "port"
        run = lambda: impl.solve(x, **kw)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        run()
        times.append(time.perf_counter() - t0)
    return kind, times, x


def run_reference_arm(args, rank: int):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    kind, _, _ = cpu_reference_baseline(8192, threads, steps=max(1, args.warmup))
    kind, times, x = cpu_reference_baseline(CPU_SAMPLE_N, threads, steps=args.steps)
    total = sum(times)
    value = CPU_SAMPLE_N * len(times) / total
    sample = (f"Plummer N={CPU_SAMPLE_N} (same generator and P/theta/ncrit/nspawn as the {WORKLOAD['n']}-body "
              f"workload; each step one full CPU solve)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "bodies/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD["name"], "n_bodies": WORKLOAD["n"], "P": WORKLOAD["P"],
                   "theta": WORKLOAD["theta"], "ncrit": WORKLOAD["ncrit"], "sample_n": CPU_SAMPLE_N},
        "cpu_baseline": {"value": value, "unit": "bodies/s", "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "bodies/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def replica_value(local_seconds: float, units_per_rank: float, world: int, dist=None, device="cuda"):
    """Replicas only: every rank solves its own systems.  The job's time is the
    slowest rank's (one MAX all-reduce of a scalar, no data-path collective);
    the value is the units all ranks processed over that time."""
    import torch
    t = torch.tensor([float(local_seconds)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    tmax = float(t.item())
    return tmax, units_per_rank * world / tmax


def agree_ncrit(best: int, world: int, dist=None, device="cuda") -> int:
    """Every rank solves on rank 0's tuned ncrit (the same trees everywhere)."""
    import torch
    t = torch.tensor([int(best)], dtype=torch.int64, device=device)
    if world > 1:
        dist.broadcast(t, 0)
    return int(t.item())


def torchrun_command(argv: list[str], gpus: int, port: int) -> list[str]:
    """The launch of `gpus` replica ranks of this script on one node."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}",
            "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + list(argv)


def _free_port() -> int:
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def check_world(gpus: int, env=None) -> str:
    """'spawn' when --gpus N > 1 was given without a rank environment (this
    process then launches the ranks itself), 'run' otherwise; a rank
    environment whose size differs from --gpus is an error."""
    env = os.environ if env is None else env
    if "WORLD_SIZE" not in env:
        return "spawn" if gpus > 1 else "run"
    world = int(env["WORLD_SIZE"])
    if world != gpus:
        raise SystemExit(f"bench.py: --gpus {gpus} but WORLD_SIZE={world}; launch one rank per GPU")
    return "run"


P2P_FLOPS_PER_INTERACTION = 20   # the canonical count for a Laplace potential + gradient pair


def fp32_fma_peak_tflops(sm_mhz: float) -> float:
    """CUDA-core FP32 peak: 148 SMs x 128 FMA lanes x 2 flop per clock (no measured figure exists)."""
    return 148 * 128 * 2 * sm_mhz * 1e6 / 1e12


def kernel_rooflines(P, mixed, n, info, phases, interactions, hbm_peak, peak_kind, sm_mhz):
    """One entry per hot-path kernel of a solve, from its phase time (CUDA events
    over the timed steps) and its algorithmic work:
      p2p      20 flop per pair interaction (sum over the P2P list of n_i n_j, counted
               on the device) against the CUDA-core FP32 FMA peak;
      m2l      per pair the source's expansion (NTERM x 8 B in FP32, 16 B in FP64) and an
               8-byte list entry, per cell the local expansion read and written, against
               the measured HBM copy bandwidth (also its flop rate, 8 NTERM P^2 per pair);
      upward   the bodies read by P2M (32 B each), every cell's multipole written and
               every non-root cell's read by its parent's M2M (NTERM x 16 B each);
      downward every non-root cell's parent local expansion read and its own read and
               written by L2L (3 x NTERM x 16 B), the bodies read and their results read
               and written by L2P (96 B each)."""
    nt = P * (P + 1) // 2
    C, n_m2l = info["ncells"], info["n_m2l"]
    cplx = 8 if mixed else 16
    fp32_peak = fp32_fma_peak_tflops(sm_mhz)
    out = []

    def hbm(kernel, ms, nbytes, note, **extra):
        a = nbytes / (ms / 1e3) / 1e9 if ms > 0 else 0.0
        d = {"kernel": kernel, "bound": "hbm", "achieved": a, "peak": hbm_peak, "unit": "GB/s",
             "frac": a / hbm_peak, "traffic": None, "peak_kind": peak_kind, "ms_per_launch": ms,
             "algorithmic_bytes": int(nbytes), "note": note}
        d.update(extra)
        out.append(d)

    p2p_ms = phases["p2p"]
    flops = P2P_FLOPS_PER_INTERACTION * interactions
    a = flops / (p2p_ms / 1e3) / 1e12 if p2p_ms > 0 else 0.0
    out.append({"kernel": "p2p", "bound": "fp32", "achieved": a, "peak": fp32_peak, "unit": "TFLOP/s",
                "frac": a / fp32_peak, "traffic": None,
                "peak_kind": f"nominal CUDA-core FP32 (148 SMs x 128 lanes x 2 flop x {sm_mhz:.0f} MHz)",
                "ms_per_launch": p2p_ms, "interactions": int(interactions),
                "flops_per_interaction": P2P_FLOPS_PER_INTERACTION,
                "note": "both P2P launches of a solve (FP32 in the mixed form, FP64 in the plain one)"})
    m2l_ms = phases["m2l"]
    alg_flops = n_m2l * 8 * nt * P * P
    hbm("m2l", m2l_ms, n_m2l * (nt * cplx + 8) + C * 2 * nt * cplx,
        "the M2L phase: class hashing and sorting, the per-class products (tensor cores in the mixed "
        "form), their per-target sums, the pair-by-pair FP32 launches and the FP64 root-level pairs",
        algorithmic_flops=int(alg_flops), achieved_tflops=alg_flops / (m2l_ms / 1e3) / 1e12 if m2l_ms else 0.0,
        traffic=(M2L_DRAM_BYTES_PER_PAIR * n_m2l if mixed and P == 8 else None))
    hbm("upward", phases["upward"], n * 32 + C * nt * 16 + max(C - 1, 0) * nt * 16,
        "P2M at the leaves and M2M level by level (FP64)")
    hbm("downward", phases["downward"], 3 * max(C - 1, 0) * nt * 16 + n * 96,
        "L2L level by level and L2P at the leaves (FP64)")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--n", type=int, default=WORKLOAD["n"], help=argparse.SUPPRESS)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--ncrit", type=int, default=0, help="0: pick the fastest of 32, 64, 128 during warm-up")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--m2l-policy", type=int, default=1, help=argparse.SUPPRESS)  # Fmm.set_mixed_policy m2l_fp32
    ap.add_argument("--no-plain", action="store_true", help="skip the FP64 plain-method comparison run")
    ap.add_argument("--workload", default="solve", choices=["solve", "batch", "serve", "periodic"],
                    help="solve: the single large solve (default); batch: 512 independent systems per step; "
                         "serve: Poisson request trace through the request server; periodic: water box "
                         "with images=3 against Ewald")
    ap.add_argument("--workers", type=int, default=16, help="contexts (streams) of the batch / serve runtime")
    ap.add_argument("--buckets", type=int, default=3,
                    help="batch: size groups solved as one forest each (0: one context per system)")
    ap.add_argument("--min-level", type=int, default=None,
                    help="mixed form: lowest target level of the FP32 M2L (default 2: levels 0 and 1 in FP64)")
    ap.add_argument("--orders", default="6,8,10",
                    help="serve: the expansion orders requests draw from (10 alone: a stream of P = 10 requests only)")
    ap.add_argument("--group-max-n", type=int, default=262144,
                    help="serve: requests of at most this many bodies are grouped into forests")
    ap.add_argument("--ncrit-candidates", default="32,64,128",
                    help="batch: the ncrit values the autotuner tries per size group")
    ap.add_argument("--p2p-candidates", default="0,2,3",
                    help="batch: the P2P targets-per-lane settings tried with every ncrit (mixed form)")
    args = ap.parse_args()
    if check_world(args.gpus) == "spawn":
        r = subprocess.run(["timeout", "-k", "60", "3600"] + torchrun_command(sys.argv[1:], args.gpus, _free_port()))
        sys.exit(r.returncode)
    if args.workload != "solve":
        return run_runtime_workload(args)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, rank)
        return

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    pkg = _package()
    pkg.build()
    from exafmm_b200 import datasets

    n = args.n
    wl = dict(WORKLOAD)
    x = datasets.plummer(n, seed=wl["seed"] + rank)
    prec = pkg.FP64 if args.precision == "fp64" else pkg.MIXED
    dx = torch.from_numpy(x).cuda()
    dout = torch.empty_like(dx)
    hx = torch.from_numpy(x).pin_memory()
    hout = torch.empty_like(hx).pin_memory()

    def make(precision, ncrit):
        f = pkg.Fmm(P=wl["P"], theta=wl["theta"], ncrit=ncrit, nspawn=wl["nspawn"], precision=precision,
                    device=local_rank)
        if precision == pkg.MIXED and (args.m2l_policy != 1 or args.min_level is not None):
            f.set_mixed_policy(m2l_fp32=args.m2l_policy, min_level=2 if args.min_level is None else args.min_level)
        return f

    def solve_device(f, out):
        f.set_bodies_device(dx.data_ptr(), n)
        f.solve()
        f.results_device(out.data_ptr())

    # ncrit autotuning (warm-up, untimed): one solve per candidate, keep the fastest.
    tuned = {}
    if args.ncrit:
        ncrit = args.ncrit
    else:
        for cand in (32, 64, 128):
            f = make(prec, cand)
            solve_device(f, dout)
            solve_device(f, dout)
            tuned[cand] = f.phase_times()["total"]
            f.close()
        ncrit = agree_ncrit(min(tuned, key=tuned.get), world, dist)

    fmm = make(prec, ncrit)
    stream = torch.cuda.ExternalStream(fmm.stream())
    for _ in range(args.warmup):
        solve_device(fmm, dout)
    torch.cuda.synchronize()
    info = fmm.info()

    # ---- value: device-resident steps ----
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    phase_acc = {k: 0.0 for k in pkg.Fmm.PHASES}
    launches0 = pkg.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            solve_device(fmm, dout)
            for k, v in fmm.phase_times().items():
                phase_acc[k] += v
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = pkg.launch_count() - launches0
    ms = ev0.elapsed_time(ev1)
    clk = clocks.summary()
    s_max, value = replica_value(ms / 1e3, n * args.steps, world, dist)
    ms_max = 1e3 * s_max
    if world > 1:
        dist.barrier()

    # ---- e2e: public API from pinned host memory ----
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    hx_np, hout_np = hx.numpy(), hout.numpy()
    e0.record(stream)
    for _ in range(args.steps):
        fmm.set_bodies(hx_np)
        fmm.solve()
        fmm.results(out=hout_np)
    e1.record(stream)
    torch.cuda.synchronize()
    _, e2e_value = replica_value(e0.elapsed_time(e1) / 1e3, n * args.steps, world, dist)

    # ---- plain FP64 run of the same input, and the three-way error split ----
    plain = None
    if not args.no_plain and prec == pkg.MIXED:
        f64 = make(pkg.FP64, ncrit)
        dref = torch.empty_like(dx)
        solve_device(f64, dref)
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s64 = torch.cuda.ExternalStream(f64.stream())
        p0.record(s64)
        for _ in range(args.steps):
            solve_device(f64, dref)
        p1.record(s64)
        torch.cuda.synchronize()
        tp_s, _ = replica_value(p0.elapsed_time(p1) / 1e3, n * args.steps, world, dist)
        plain_ms = 1e3 * tp_s / args.steps
        mixed_out, plain_out = dout.cpu().numpy(), dref.cpu().numpy()
        idx = datasets.strided_sample(n, 4096)
        direct = pkg.direct(x[idx], x)
        plain = {"value": n * world / (plain_ms / 1e3), "unit": "bodies/s", "ms_per_step": plain_ms,
                 "speedup_of_mixed": (n * world / (ms_max / args.steps / 1e3)) / (n * world / (plain_ms / 1e3)),
                 "rel_l2": {"mixed_vs_direct_pot": datasets.rel_l2(mixed_out[idx, 0], direct[:, 0]),
                            "plain_vs_direct_pot": datasets.rel_l2(plain_out[idx, 0], direct[:, 0]),
                            "mixed_vs_plain_pot": datasets.rel_l2(mixed_out[:, 0], plain_out[:, 0]),
                            "mixed_vs_direct_acc": datasets.rel_l2(mixed_out[idx, 1:], direct[:, 1:]),
                            "plain_vs_direct_acc": datasets.rel_l2(plain_out[idx, 1:], direct[:, 1:]),
                            "mixed_vs_plain_acc": datasets.rel_l2(mixed_out[:, 1:], plain_out[:, 1:]),
                            "direct_sample": 4096}}
        f64.close()

    # ---- rooflines of the hot-path kernels, from the timed steps; the dominant one is `roofline`
    hbm_peak, bf16_peak, peak_kind = _peaks()
    P = wl["P"]
    phases = {k: v / args.steps for k, v in phase_acc.items()}
    interactions = fmm.p2p_interactions()
    rooflines = kernel_rooflines(P, prec == pkg.MIXED, n, info, phases, interactions, hbm_peak, peak_kind,
                                 clk.get("sm_max_mhz") or 1965.0)
    roofline = max(rooflines, key=lambda r: r["ms_per_launch"])

    line = {
        "metric": METRIC, "value": value, "unit": "bodies/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if prec == pkg.FP64 else "f32+kahan", "data": "synthetic",
        "config": {"workload": wl["name"], "n_bodies": n, "distribution": "plummer(scale=1, rmax=20), q=1/N",
                   "P": P, "theta": wl["theta"], "ncrit": ncrit, "ncrit_tuning_ms": tuned, "nspawn": wl["nspawn"],
                   "precision": args.precision, "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2 (134 MB of bodies per solve)",
                   "cells": info["ncells"], "depth": info["depth"], "m2l_pairs": info["n_m2l"], "p2p_pairs": info["n_p2p"]},
        "phases_ms": phases,
        "roofline": roofline,
        "rooflines": rooflines,
        "e2e": {"value": e2e_value, "unit": "bodies/s", "h2d_bytes_per_step": int(n * 32),
                "d2h_bytes_per_step": int(n * 32)},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if plain is not None:
        line["plain_fp64"] = plain
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        kind, times, _ = cpu_reference_baseline(CPU_SAMPLE_N, threads, steps=1)
        cpu_v = CPU_SAMPLE_N / times[0]
        line["cpu_baseline"] = {"value": cpu_v, "unit": "bodies/s", "cores": threads, "kind": kind,
                                "sample": f"one solve of a Plummer N={CPU_SAMPLE_N} system with the same "
                                          f"P/theta/ncrit/nspawn ({times[0]:.1f} s)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    fmm.close()
    if world > 1:
        dist.destroy_process_group()


# ---------------------------------------------------------------- batched and served workloads
BATCH = dict(name="batch_512_p10", count=512, lo=2000, hi=200_000, P=10, theta=0.4, ncrit=64, nspawn=5000)
SERVE = dict(name="serve_poisson_p6_8_10", count=60, lo=1000, hi=1_000_000, theta=0.4, ncrit=64, nspawn=5000,
             budget=150e9, repeat_frac=0.2, repeat_steps=50, loads=(0.5, 0.8), replays=3)


def _three_way(ex, datasets, xs, mixed, plain, sample=256, take=None):
    """rel-L2 (pot, acc) of mixed vs direct, plain vs direct and mixed vs plain per
    system (every system, or `take` spread over the sizes), direct on `sample`
    strided targets of each; returns the per-system lists and their maxima."""
    order = np.argsort([len(x) for x in xs])
    pick = order if take is None else order[np.linspace(0, len(xs) - 1, min(take, len(xs))).astype(int)]
    per = {k: [] for k in ("mixed_vs_direct", "plain_vs_direct", "mixed_vs_plain")}
    for i in pick:
        x = xs[i]
        if not len(x):
            continue
        idx = datasets.strided_sample(len(x), sample)
        d = ex.direct(x[idx], x)
        for key, a, b in (("mixed_vs_direct", mixed[i][idx], d), ("plain_vs_direct", plain[i][idx], d),
                          ("mixed_vs_plain", mixed[i], plain[i])):
            per[key].append((int(i), datasets.rel_l2(a[:, 0], b[:, 0]), datasets.rel_l2(a[:, 1:], b[:, 1:])))
    out = {}
    for k, vals in per.items():
        pot = np.array([v[1] for v in vals])
        acc = np.array([v[2] for v in vals])
        out[k] = {"pot_max": float(pot.max()), "pot_median": float(np.median(pot)),
                  "acc_max": float(acc.max()), "acc_median": float(np.median(acc)),
                  "pot_worst_system": int(vals[int(pot.argmax())][0])}
    out["systems"] = len(per["mixed_vs_plain"])
    out["direct_sample_per_system"] = sample
    out["per_system_pot"] = {k: [float(v[1]) for v in vals] for k, vals in per.items()}
    return out


def _batch_cpu_baseline(xs, threads):
    """The reference CPU FMM on a bounded sample of the systems (about 10 s)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import bindings
    if not bindings.reference_available():
        return None
    ref = bindings.Reference()
    kw = dict(P=BATCH["P"], theta=BATCH["theta"], ncrit=BATCH["ncrit"], nspawn=BATCH["nspawn"])
    order = np.argsort([len(x) for x in xs])
    pick = order[np.linspace(0, len(xs) - 1, 6).astype(int)]
    t0 = time.perf_counter()
    bodies = 0
    for i in pick:
        ref.solve(xs[i], threads=threads, record_lists=False, **kw)
        bodies += len(xs[i])
    dt = time.perf_counter() - t0
    return {"value": bodies / dt, "unit": "bodies/s", "cores": threads, "kind": "reference",
            "sample": f"{len(pick)} of the systems ({bodies} bodies, smallest to largest), one after another, "
                      f"each with all host threads ({dt:.1f} s)"}


def run_runtime_workload(args):
    import torch
    pkg = _package()
    pkg.build()
    from exafmm_b200 import datasets, workloads
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local_rank)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    prec = pkg.FP64 if args.precision == "fp64" else pkg.MIXED
    if args.workload == "batch":
        line = _run_batch(args, pkg, datasets, workloads, prec, rank, world, local_rank)
    elif args.workload == "periodic":
        line = _run_periodic(args, pkg, datasets, prec, rank, world, local_rank)
    else:
        line = _run_serve(args, pkg, datasets, workloads, prec, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist
        if args.workload in ("batch", "periodic"):  # whole-job bodies/s over the slowest rank's time
            _, line["value"] = replica_value(line["_time"], line["_units"], world, dist)
        else:  # latency: the worst rank's p99
            t = torch.tensor([line["value"]], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            line["value"] = float(t.item())
        dist.barrier()
        dist.destroy_process_group()
    line.pop("_time")
    line.pop("_units")
    if rank == 0:
        print(json.dumps(line), flush=True)


def _run_batch(args, pkg, datasets, workloads, prec, rank, world, local_rank):
    """Batched uneven systems: each step solves all 512 systems, grouped by size
    into `--buckets` forests (one context and stream each, running concurrently).
    value: bodies resident on the device, timed by the batch's own device events
    (from an event every forest's stream waits on to the last forest's copy out);
    e2e: the same call with pinned host buffers, host clock around it."""
    import torch
    cfg = BATCH
    xs = workloads.batch_systems(cfg["count"], cfg["lo"], cfg["hi"], seed0=1000 + 100000 * rank)
    sizes = [len(x) for x in xs]
    nbodies = sum(sizes)
    min_level = 2 if args.min_level is None else args.min_level

    def make(precision):
        b = pkg.Batch(P=cfg["P"], theta=cfg["theta"], ncrit=cfg["ncrit"], nspawn=cfg["nspawn"], precision=precision,
                      device=local_rank, workers=args.workers, forest=args.buckets)
        if precision == pkg.MIXED:
            b.set_mixed_policy(m2l_fp32=args.m2l_policy, min_level=min_level)
        return b

    dev_in = [torch.from_numpy(x).to(f"cuda:{local_rank}") for x in xs]
    dev_out = [torch.empty_like(d) for d in dev_in]
    in_ptrs, out_ptrs = [d.data_ptr() for d in dev_in], [d.data_ptr() for d in dev_out]

    pool_out = [np.zeros_like(x) for x in xs]

    def step(b):
        if args.buckets > 0:
            b.solve_device(sizes, in_ptrs, out_ptrs)
            return b.elapsed_ms()
        b.solve(xs, pool_out)  # one context per system takes host buffers
        for d, o in zip(dev_out, pool_out):
            d.copy_(torch.from_numpy(o))
        return 0.0

    b = make(prec)
    forest = args.buckets > 0
    cands = [int(v) for v in args.ncrit_candidates.split(",") if v]
    p2p_cands = [int(v) for v in args.p2p_candidates.split(",") if v] if prec == pkg.MIXED else [0]
    if forest:  # the tuner tries one configuration per call: untimed tuning calls, then the table is frozen
        b.set_ncrit_candidates(cands)
        b.set_p2p_candidates(p2p_cands)
        b.autotune(True)
        for _ in range(len(cands) * len(p2p_cands)):
            step(b)
        b.autotune(False)
        warm = max(1, args.warmup - len(cands) * len(p2p_cands))
    else:
        b.autotune(True)
        step(b)
        b.autotune(False)
        warm = max(1, args.warmup - 1)
    for _ in range(warm):
        step(b)
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    launches0 = pkg.launch_count()
    dev_ms = 0.0
    with ClockSampler(local_rank) as clocks:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            dev_ms += step(b)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
    clk = clocks.summary()
    launches = pkg.launch_count() - launches0
    if not forest:
        dev_ms = 1e3 * dt  # one context per system: many streams, host clock around each call
    group, group_ncrit = b.buckets(len(xs)) if forest else (np.zeros(len(xs), dtype=int), np.array([]))
    mixed_out = [d.cpu().numpy() for d in dev_out]

    # e2e: the public call from pinned host buffers, copies inside the timed region
    hin = [torch.from_numpy(x).pin_memory() for x in xs]
    hout = [torch.empty_like(h).pin_memory() for h in hin]
    hin_ptrs, hout_ptrs = [h.data_ptr() for h in hin], [h.data_ptr() for h in hout]
    hin_np, hout_np = [h.numpy() for h in hin], [h.numpy() for h in hout]

    def host_call():
        if forest:
            b.solve_device(sizes, hin_ptrs, hout_ptrs)
        else:
            b.solve(hin_np, hout_np)

    host_call()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        host_call()
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    assert all(np.array_equal(m, h) for m, h in zip(mixed_out, hout_np))

    value = nbodies * args.steps / (dev_ms / 1e3)
    line = {
        "metric": "batched FMM bodies/s (512 systems per step, N log-uniform [2e3, 2e5], P=10, theta=0.4)",
        "value": value, "unit": "bodies/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if prec == pkg.FP64 else "f32+kahan", "data": "synthetic",
        "config": {"workload": cfg["name"], "systems": cfg["count"], "bodies_per_step": nbodies,
                   "distribution": "even systems uniform in [-1,1]^3, odd on the unit sphere; q U[-1,1]",
                   "P": cfg["P"], "theta": cfg["theta"], "forest_groups": int(len(group_ncrit)),
                   "group_ncrit": [int(v) for v in group_ncrit], "ncrit_table": b.ncrit_table(),
                   "group_p2p_targets_per_lane": [int(v) for v in b.bucket_p2p()] if forest else None,
                   "tuned": {"ncrit": cands, "p2p_targets_per_lane": p2p_cands},
                   "group_bodies": [int(sum(n for n, gi in zip(sizes, group) if gi == k))
                                    for k in range(len(group_ncrit))],
                   "mixed_min_level": min_level if prec == pkg.MIXED else None,
                   "precision": args.precision, "parallelism": f"replicas{world}",
                   "timing": ("device events of the batch call: an event every forest's stream waits on, to "
                              "the last forest's results copied out" if forest else
                              "host clock around each call, device synchronized on both sides"),
                   "l2": "each step reads 0.7 GB of bodies and writes 0.7 GB of results (larger than L2)"},
        "e2e": {"value": nbodies * args.steps / e2e_s, "unit": "bodies/s", "h2d_bytes_per_step": nbodies * 32,
                "d2h_bytes_per_step": nbodies * 32,
                "timing": "host clock around each call from pinned host buffers, device synchronized on both sides"},
        "gpu_launches": int(launches), "clocks": clk, "roofline": None,
        "_time": dev_ms / 1e3, "_units": nbodies * args.steps,
    }
    if not args.no_plain and prec == pkg.MIXED:
        bp = make(pkg.FP64)
        bp.set_ncrit_table(b.ncrit_table())  # the same trees, so mixed vs plain is precision only
        step(bp)
        torch.cuda.synchronize()
        kp = max(1, min(args.steps, 3))
        tp = 0.0
        t0 = time.perf_counter()
        for _ in range(kp):
            tp += step(bp)
        torch.cuda.synchronize()
        if not forest:
            tp = 1e3 * (time.perf_counter() - t0)
        plain = [d.cpu().numpy() for d in dev_out]
        plain_value = nbodies * kp / (tp / 1e3)
        tw = _three_way(pkg, datasets, xs, mixed_out, plain)
        per = tw.pop("per_system_pot")
        line["plain_fp64"] = {"value": plain_value, "unit": "bodies/s", "ms_per_step": tp / kp,
                              "speedup_of_mixed": value / plain_value, "rel_l2": tw}
        line["per_system_rel_l2_pot"] = {k: [float(f"{v:.3e}") for v in vals] for k, vals in per.items()}
        bp.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = _batch_cpu_baseline(xs, os.cpu_count() or 1)
        if cb:
            line["cpu_baseline"] = cb
    b.close()
    return line


def _request_errors(pkg, datasets, workloads, trace, mixed_samples, plain_samples):
    """Per request (the final step of each job): rel-L2 of the potential on its
    sampled targets, mixed vs an FP64 direct sum over all its bodies, plain vs the
    same, and mixed vs plain."""
    rows = []
    for k, job in enumerate(trace.jobs):
        if k not in mixed_samples:
            continue
        idx, mres, final = mixed_samples[k]
        x = final if final is not None else workloads.job_bodies(job)
        d = pkg.direct(x[idx], x)
        row = {"job": k, "n": job.n, "P": job.P, "kind": job.kind, "steps": job.steps,
               "mixed_vs_direct": datasets.rel_l2(mres[:, 0], d[:, 0])}
        if k in plain_samples:
            pidx, pres, pfinal = plain_samples[k]
            if np.array_equal(pidx, idx) and (pfinal is None) == (final is None) and \
                    (final is None or np.array_equal(pfinal, final)):
                row["plain_vs_direct"] = datasets.rel_l2(pres[:, 0], d[:, 0])
                row["mixed_vs_plain"] = datasets.rel_l2(mres[:, 0], pres[:, 0])
        rows.append(row)
    return rows


def _saturated_replays(srv, trace, precision, cfg, workloads, pinned, samples):
    """The trace with every job queued at once, replayed cfg["replays"] times: the
    medians of bodies/s (whole trace and until its last single solve), capacity and
    latencies, with their ranges; samples from the first replay."""
    reps = []
    for r in range(cfg["replays"]):
        done, wall = workloads.replay(srv, trace, precision=precision, ncrit=cfg["ncrit"], nspawn=cfg["nspawn"],
                                      deadline_s=600.0, samples=samples if r == 0 else None, host_alloc=pinned)
        s = workloads.latency_summary(done, wall)
        s["while_saturated"] = workloads.saturated_throughput(done)
        s["capacity_jobs_per_s"] = len(trace.jobs) / wall
        reps.append(s)
    med = lambda f: float(np.median([f(x) for x in reps]))
    out = {k: med(lambda x, k=k: x[k]) for k in ("p50_ms", "p99_ms", "mean_ms", "bodies_per_s", "wall_s",
                                                  "capacity_jobs_per_s", "device_ms_sum")}
    out["requests"] = reps[0]["requests"]
    out["replays"] = len(reps)
    out["bodies_per_s_range"] = [min(x["bodies_per_s"] for x in reps), max(x["bodies_per_s"] for x in reps)]
    ws = [x["while_saturated"]["bodies_per_s"] for x in reps]
    out["while_saturated"] = {"bodies_per_s": float(np.median(ws)), "range": [min(ws), max(ws)],
                              "window_s": med(lambda x: x["while_saturated"]["window_s"])}
    if "chain_step_p50_ms" in reps[0]:
        out["chain_step_p50_ms"] = med(lambda x: x["chain_step_p50_ms"])
        out["chain_step_p99_ms"] = med(lambda x: x["chain_step_p99_ms"])
    return out


def _run_serve(args, pkg, datasets, workloads, prec, rank, world, local_rank):
    """Served request stream: a saturated replay (everything queued at once) gives
    the capacity; the same trace replayed with the plain FP64 method gives the
    mixed/plain ratio in bodies/s; Poisson traces at 0.5 and 0.8 of capacity,
    three replays each, give p50/p99 as medians with their spread.  Repeat
    chains stay on the device (server sessions)."""
    import torch
    cfg = SERVE
    srv = pkg.Server(device=local_rank, workers=args.workers, hbm_budget_bytes=cfg["budget"])
    if args.min_level is not None:
        srv.set_mixed_policy(min_level=args.min_level)
    srv.set_grouping(max_request_bodies=args.group_max_n)
    # warm-up: one request per order and precision
    for P in sorted(set(int(v) for v in args.orders.split(",") if v)):
        for pr in {prec, pkg.FP64}:
            srv.wait(srv.submit(datasets.cube(20000, seed=P), P=P, theta=cfg["theta"], ncrit=cfg["ncrit"],
                                precision=pr))
    orders = tuple(int(v) for v in args.orders.split(",") if v)
    sat = workloads.make_trace(cfg["count"], rate=1e6, lo=cfg["lo"], hi=cfg["hi"], orders=orders,
                               repeat_frac=cfg["repeat_frac"],
                               repeat_steps=cfg["repeat_steps"], seed=4000 + 1000 * rank, theta=cfg["theta"])
    def pinned(shape):
        return torch.empty(shape, dtype=torch.float64).pin_memory().numpy()

    launches0 = pkg.launch_count()
    mixed_samples, plain_samples = {}, {}
    with ClockSampler(local_rank) as clocks:
        saturated = _saturated_replays(srv, sat, prec, cfg, workloads, pinned, mixed_samples)
        capacity = saturated["capacity_jobs_per_s"]
        rates = {}
        for load in cfg["loads"]:
            reps = []
            for r in range(cfg["replays"]):
                tr = workloads.make_trace(cfg["count"], rate=load * capacity, lo=cfg["lo"], hi=cfg["hi"], orders=orders,
                                          repeat_frac=cfg["repeat_frac"], repeat_steps=cfg["repeat_steps"],
                                          seed=5000 + int(100 * load) + 10 * r + 1000 * rank, theta=cfg["theta"])
                d, w = workloads.replay(srv, tr, precision=prec, ncrit=cfg["ncrit"], nspawn=cfg["nspawn"],
                                        deadline_s=300.0, host_alloc=pinned)
                reps.append(workloads.latency_summary(d, w))
            med = lambda key: float(np.median([x[key] for x in reps]))
            rates[f"{load:.2f}"] = {"rate_jobs_per_s": load * capacity, "replays": len(reps),
                                    "p50_ms": med("p50_ms"), "p99_ms": med("p99_ms"), "mean_ms": med("mean_ms"),
                                    "bodies_per_s": med("bodies_per_s"),
                                    "p50_ms_range": [min(x["p50_ms"] for x in reps), max(x["p50_ms"] for x in reps)],
                                    "p99_ms_range": [min(x["p99_ms"] for x in reps), max(x["p99_ms"] for x in reps)],
                                    "requests": reps[0]["requests"], "wall_s": med("wall_s")}
        torch.cuda.synchronize()
    clk = clocks.summary()
    launches = pkg.launch_count() - launches0
    plain = None
    if not args.no_plain and prec == pkg.MIXED:
        psat = _saturated_replays(srv, sat, pkg.FP64, cfg, workloads, pinned, plain_samples)
        plain = {"value": psat["while_saturated"]["bodies_per_s"],
                 "unit": "bodies/s (saturated replay of the same trace, until its last single solve)",
                 "capacity_jobs_per_s": psat["capacity_jobs_per_s"], "saturated": psat,
                 "speedup_of_mixed": saturated["while_saturated"]["bodies_per_s"] /
                 psat["while_saturated"]["bodies_per_s"],
                 "speedup_of_mixed_whole_trace": saturated["bodies_per_s"] / psat["bodies_per_s"]}
    errs = _request_errors(pkg, datasets, workloads, sat, mixed_samples, plain_samples)
    st = srv.stats()
    srv.close()
    top = rates[f"{max(cfg['loads']):.2f}"]
    err_summary = {k: {"max": max(r[k] for r in errs if k in r), "median": float(np.median([r[k] for r in errs
                                                                                           if k in r]))}
                   for k in ("mixed_vs_direct", "plain_vs_direct", "mixed_vs_plain") if any(k in r for r in errs)}
    line = {
        "metric": "served p99 latency (Poisson arrivals at 0.8 of capacity; N log-uniform [1e3, 1e6], "
                  f"P in {{{', '.join(str(o) for o in orders)}}}, theta=0.4)",
        "value": top["p99_ms"], "unit": "ms", "n_gpus": world, "steps": cfg["replays"], "warmup": 1,
        "ms_per_step": top["mean_ms"], "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if prec == pkg.FP64 else "f32+kahan", "data": "synthetic",
        "config": {"workload": cfg["name"], "jobs_per_trace": cfg["count"], "repeat_fraction": cfg["repeat_frac"],
                   "repeat_steps": cfg["repeat_steps"], "hbm_budget_bytes": cfg["budget"],
                   "workers": args.workers, "precision": args.precision, "parallelism": f"replicas{world}",
                   "mixed_min_level": 2 if args.min_level is None else args.min_level,
                   "group_max_request_bodies": args.group_max_n, "orders": list(orders),
                   "chains": "device-resident sessions: bodies moved and tree rebuilt on the device each step",
                   "timing": "host clock: scheduled arrival (or the previous chain step's return) to results "
                             "in host memory; p50/p99 are medians over the replays, with their ranges",
                   "l2": "requests stream their bodies in and results out",
                   "host_buffers": "each request's bodies and results in pinned host memory, generated and "
                                   "allocated before the replay's clock starts"},
        "saturated": saturated, "capacity_jobs_per_s": capacity, "loads": rates,
        "served_bodies_per_s": saturated["while_saturated"]["bodies_per_s"],
        "request_rel_l2_pot": err_summary, "requests_checked": len(errs),
        "per_request": [{k: (float(f"{v:.3e}") if isinstance(v, float) else v) for k, v in r.items()} for r in errs],
        "server_stats": st,
        "e2e": {"value": top["p99_ms"], "unit": "ms", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None},
        "gpu_launches": int(launches), "clocks": clk, "roofline": None,
        "_time": top["wall_s"], "_units": top["requests"],
    }
    if plain is not None:
        line["plain_fp64"] = plain
    return line


PERIODIC = dict(name="water_1m_images3_p10", waters=333_333, P=10, theta=0.4, ncrit=64, nspawn=5000, images=3,
                cutoff=30.0, alpha_cutoff=3.8, cpu_waters=20_000)


def _run_periodic(args, pkg, datasets, prec, rank, world, local_rank):
    """Periodic water box (config 5): FMM with the lattice (images=3) and the dipole
    correction, against Ewald summation on the GPU (FP64)."""
    import torch
    cfg = PERIODIC
    x, L = datasets.water_box(cfg["waters"], seed=5 + rank)
    n = len(x)
    kw = dict(P=cfg["P"], theta=cfg["theta"], ncrit=cfg["ncrit"], nspawn=cfg["nspawn"], images=cfg["images"],
              cycle=L, device=local_rank)
    dx = torch.from_numpy(x).cuda()
    dout = torch.empty_like(dx)

    def solve(f, out):
        f.set_bodies_device(dx.data_ptr(), n)
        f.solve()
        f.dipole_correction(f.get_dipole())
        f.results_device(out.data_ptr())

    fmm = pkg.Fmm(precision=prec, **kw)
    if prec == pkg.MIXED and args.min_level is not None:
        fmm.set_mixed_policy(min_level=args.min_level)
    for _ in range(max(3, args.warmup)):
        solve(fmm, dout)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(fmm.stream())
    launches0 = pkg.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            solve(fmm, dout)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    clk = clocks.summary()
    launches = pkg.launch_count() - launches0
    phases = fmm.phase_times()
    info = fmm.info()
    mixed = dout.cpu().numpy()
    fmm.close()
    # Ewald: real part to erfc(alpha rc), wave part to exp(-K^2 / 4 alpha^2) at |k| = ksize, both ~1e-7
    alpha = cfg["alpha_cutoff"] / cfg["cutoff"]
    ksize = int(np.ceil(2 * alpha * np.sqrt(np.log(1e7)) * L / (2 * np.pi)))
    t0 = time.perf_counter()
    ew = pkg.ewald(x, ksize=ksize, alpha=alpha, sigma=0.25 / np.pi, cutoff=cfg["cutoff"], cycle=L)
    ewald_s = time.perf_counter() - t0
    q = x[:, 3]

    def vs(a, b):
        ea, eb = float(q @ a[:, 0]), float(q @ b[:, 0])
        return {"energy_rel": abs(ea - eb) / abs(eb), "grad_rel_l2": datasets.rel_l2(a[:, 1:], b[:, 1:])}

    line = {
        "metric": "periodic FMM bodies/s (water box, 1.0M charges, images=3, P=10, theta=0.4, dipole correction)",
        "value": n * args.steps / (ms / 1e3), "unit": "bodies/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if prec == pkg.FP64 else "f32+kahan", "data": "synthetic",
        "config": {"workload": cfg["name"], "charges": n, "box_edge_A": L, "P": cfg["P"], "theta": cfg["theta"],
                   "ncrit": cfg["ncrit"], "images": cfg["images"], "precision": args.precision,
                   "mixed_min_level": (2 if args.min_level is None else args.min_level) if prec == pkg.MIXED else None,
                   "parallelism": f"replicas{world}", "cells": info["ncells"], "m2l_pairs": info["n_m2l"],
                   "p2p_pairs": info["n_p2p"],
                   "ewald": {"alpha": alpha, "cutoff_A": cfg["cutoff"], "ksize": ksize, "sigma": 0.25 / np.pi,
                             "seconds": ewald_s},
                   "l2": "inputs larger than L2 (32 MB of bodies plus 0.5 GB of lists per solve)"},
        "phases_ms": phases, "vs_ewald": vs(mixed, ew), "gpu_launches": int(launches), "clocks": clk,
        "roofline": None, "_time": ms / 1e3, "_units": n * args.steps,
    }
    if not args.no_plain and prec == pkg.MIXED:
        f64 = pkg.Fmm(precision=pkg.FP64, **kw)
        plain = torch.empty_like(dx)
        solve(f64, plain)
        torch.cuda.synchronize()
        s64 = torch.cuda.ExternalStream(f64.stream())
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(s64)
        solve(f64, plain)
        p1.record(s64)
        torch.cuda.synchronize()
        pl = plain.cpu().numpy()
        line["plain_fp64"] = {"value": n / (p0.elapsed_time(p1) / 1e3), "unit": "bodies/s",
                              "ms_per_step": p0.elapsed_time(p1), "vs_ewald": vs(pl, ew),
                              "mixed_vs_plain": {"pot": datasets.rel_l2(mixed[:, 0], pl[:, 0]),
                                                 "grad": datasets.rel_l2(mixed[:, 1:], pl[:, 1:])}}
        f64.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import bindings
        if bindings.reference_available():
            xs, Ls = datasets.water_box(cfg["cpu_waters"], seed=6)
            threads = os.cpu_count() or 1
            t0 = time.perf_counter()
            bindings.Reference().solve(xs, P=cfg["P"], theta=cfg["theta"], ncrit=cfg["ncrit"], nspawn=cfg["nspawn"],
                                       images=cfg["images"], cycle=Ls, threads=threads, record_lists=False,
                                       dipole_correction=True)
            dt = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": len(xs) / dt, "unit": "bodies/s", "cores": threads, "kind": "reference",
                                    "sample": f"one periodic solve of a {len(xs)}-charge water box at the same "
                                              f"density, P, theta and images ({dt:.1f} s)"}
    return line


if __name__ == "__main__":
    main()
