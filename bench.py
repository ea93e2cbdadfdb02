"""Benchmark of the IBPM time step on B200: timesteps/s on the multi-domain
shedding-cylinder workload (400x200 cells, 5 nested domains, 157-point
cylinder, Re 200, dt 0.005, RK3, seeded 1e-3 vorticity noise in the wake).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1).  One simulation does not shard
(its multi-domain solve is global per level and levels are serially
dependent), so N GPUs run N independent replicas (weak scaling) and `value`
is the total timesteps/s of the job.  Rank 0 prints one JSON line.

* value        K steps with the state resident in HBM, CUDA events around each
               step on the solver's stream, L2 flushed (256 MB write) between
               steps outside the timed events; max over ranks.
* e2e          the same metric through the public API with host buffers: every
               step uploads omega, q, f from pinned host memory, advances one
               step and reads the boundary force f back.
* roofline     the dominant kernel (the column pass of the DST-I solve) timed
               alone with CUDA events on the solver's stream against the
               measured HBM copy bandwidth.
* cpu_baseline the reference's own CPU code (oracle/_ref/ref_driver: the
               reference sources built with -Ofast and the FFTW shim), one core,
               a bounded sample of steps of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "timesteps/s (400x200 x5-domain shedding cylinder, RK3)"
UNIT = "timesteps/s"


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _config(wl, precision):
    return {"workload": wl.name, "nx": wl.nx, "ny": wl.ny, "ngrid": wl.ngrid, "length": wl.length,
            "Re": wl.Re, "dt": wl.dt, "scheme": wl.scheme, "boundary_points": 157,
            "force_solve": "cholesky (fixed body)", "form": precision,
            "l2": "flushed between timed steps (256 MB write outside the events)",
            "initial_condition": f"seeded N(0, {wl.noise_amp:g}^2) level-0 wake vorticity (seed {wl.noise_seed})"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.p = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_rank{device}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                      stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.fh.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_baseline(wl, steps=10):
    from oracle import ref_runner
    if not ref_runner.available():
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": "unavailable: oracle/_ref/ref_driver not built"}
    r = ref_runner.run(wl, "c2", steps=steps, warmup=1)
    return {"value": r["steps_per_s"], "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"{r['timed_steps']} RK3 steps of the same workload after 1 warm-up step, Cholesky factors "
                      f"from the reference's own cache (init {r['init_s']:.1f} s excluded), "
                      f"reference sources -Ofast + project DST-I FFTW shim, 1 core of {ref_runner.host_cpu()}"}


def run_reference(args):
    ws, rank, local = _dist()
    if rank != 0:
        return 0
    from ibpm_b200 import configs
    from oracle import ref_runner
    wl = configs.c2_shedding_cylinder()
    base = {"metric": METRIC, "unit": UNIT, "n_gpus": args.gpus, "steps": None, "warmup": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": _config(wl, "reference FP64 CPU"), "impl": "reference"}
    if not ref_runner.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_driver is not built on this host"}))
        return 0
    steps = max(1, min(args.steps, 20))
    warm = max(1, min(args.warmup, 2))
    r = ref_runner.run(wl, "c2", steps=steps, warmup=warm)
    v = r["steps_per_s"]
    base.update({"steps": r["timed_steps"], "warmup": warm, "value": v, "ms_per_step": 1000.0 / v,
                 "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "reference",
                                  "sample": f"{r['timed_steps']} steps after {warm} warm-up (requested --steps "
                                            f"{args.steps}; capped at 20 to bound CPU time), Cholesky set-up "
                                            f"{r['init_s']:.1f} s excluded, single-threaded reference on "
                                            f"1 core of {ref_runner.host_cpu()}"},
                 "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    print(json.dumps(base))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32_refined"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import numpy as np
    import torch
    import torch.distributed as dist
    import ibpm_b200 as ib
    from ibpm_b200 import configs

    ws, rank, local = _dist()
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    wl = configs.c2_shedding_cylinder()
    stream = torch.cuda.Stream(device=dev)
    grid, model, s, x = ib.from_workload(wl, precision=args.precision, stream=stream.cuda_stream, device=local)
    s.init()
    s.set_state(x, with_q=False)
    W = max(3, args.warmup)
    K = max(1, args.steps)
    s.advance_resident(W)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    launches = 0
    with torch.cuda.stream(stream):
        for k in range(K):
            flush.zero_()
            ev[k][0].record(stream)
            s.advance_resident(1)
            ev[k][1].record(stream)
            launches += s.last_launch_count()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    if ws > 1:
        dist.barrier()
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = ws * K / (ms / 1000.0)
    forces = s.force_history(K)

    # ---- e2e through the public API with pinned host buffers
    Ke = min(K, 50)
    om = torch.empty(x.omega.shape, dtype=torch.float64, pin_memory=True).numpy()
    qh = torch.empty(x.q.shape, dtype=torch.float64, pin_memory=True).numpy()
    fh = torch.empty(x.f.shape, dtype=torch.float64, pin_memory=True).numpy()
    s.get_state(x)
    om[...] = x.omega
    qh[...] = x.q
    fh[...] = x.f
    xs = ib.State(grid, x.f.size // 2, omega=om, q=qh, f=fh, timestep=x.timestep, time=x.time)
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(Ke):
        s.set_state(xs)                                   # H2D omega, q, f
        s.advance_resident(1)
        ib._native.check(ib._native.lib().ibg_get_boundary_force(s.handle, ib._ptr(fh), None, None), s.handle)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if ws > 1:
        t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": ws * Ke / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": int(8 * (x.omega.size + x.q.size + x.f.size)),
           "d2h_bytes_per_step": int(8 * x.f.size)}

    # ---- roofline of the dominant kernel (DST-I column pass, finest level) timed alone
    roof = kernel_roofline(s, grid, stream)
    s.close()
    out = None
    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": W,
               "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
               "dtype": "f64" if args.precision == "fp64" else "f32+f64",
               "data": "synthetic (seeded noise initial condition, generated geometry)",
               "config": _config(wl, args.precision), "e2e": e2e, "gpu_launches": int(launches),
               "roofline": roof, "clocks": clk,
               "final_force": [float(forces[-1][0]), float(forces[-1][1])] if len(forces) else None}
        if ws == 1 and not args.no_cpu_baseline:
            try:
                out["cpu_baseline"] = cpu_baseline(wl)
            except Exception as e:  # the baseline is reported, never required
                out["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                                       "sample": f"failed: {e}"}
        print(json.dumps(out))
    if ws > 1:
        dist.destroy_process_group()
    return 0


def kernel_roofline(s, grid, stream, reps=200):
    import torch
    import ibpm_b200 as ib
    L = ib._native.lib()
    res = {}
    peak, kind = peaks()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = None
    for which, name in ((0, "dst_rows"), (1, "dst_cols"), (2, "nonlinear_node_vel")):
        L.ibg_run_kernel(s.handle, which, 5)
        torch.cuda.synchronize()
        e0.record(stream)
        nbytes = L.ibg_run_kernel(s.handle, which, reps)
        e1.record(stream)
        torch.cuda.synchronize()
        us = 1000.0 * e0.elapsed_time(e1) / reps
        res[name] = {"us_per_launch": us, "algorithmic_bytes": nbytes}
        if best is None or name == "dst_cols":
            best = name
    d = res[best]
    achieved = d["algorithmic_bytes"] / (d["us_per_launch"] * 1e-6) / 1e9
    return {"kernel": "k_dst_cols<double> (forward DST-I along i of every level of one solve)",
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_kind": f"{kind} (copy bandwidth, burst)", "traffic": None, "kernels": res}


if __name__ == "__main__":
    sys.exit(main())
