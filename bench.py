"""Benchmark of the IBPM time step on B200 (timesteps/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c2|c3|c4|c5] [--form ...]

Workloads (seeded synthetic inputs; no dataset is involved):

* c4 (default) ensemble of 64 independent ellipse runs (n in {128..512}, 1-3
  domains, seeded b, orientation, Re; dt = 0.5 dx): forms ensemble_fp32 (all
  members' steps as branches of one CUDA graph, FP32 bulk members with the
  force solve in FP64; default), ensemble_refined (the same with FP32
  transforms plus one FP64-residual refinement per solve), ensemble (FP64
  members) and serial (each member's captured FP64 step launched after the
  other on one stream: the plain path).
* c2 multi-domain shedding cylinder: 400x200 cells, 5 nested domains,
  157-point cylinder, Re 200, dt 0.005, RK3, seeded 1e-3 vorticity noise in
  the wake; forms fp32_refined (default), fp32 (FP32 bulk) and fp64 (plain).
* c3 pitching and plunging plate: 500x250 cells, 3 domains, 51 points,
  Re 300, dt 0.004, CG tolerance 1e-10; forms cholesky (flexible PCG with the
  exact inverse rebuilt every --pc-refresh steps, default), learned (flexible
  PCG with the learned preconditioner, trained first; training time
  reported, not timed) and cg (the reference's plain CG: the plain path).
* c5 two cylinders plunging in antiphase: 1024x1024 cells, 5 domains, 2 x 201
  points, Re 500, dt 0.005, CG tolerance 1e-10; forms cholesky (default),
  learned and cg (plain), as for c3.

One process per GPU (torchrun for N > 1).  One simulation does not shard
(its multi-domain solve is global per level and levels are serially
dependent), so for c2, c3 and c5 N GPUs run N independent replicas (weak
scaling) and `value` is the total timesteps/s of the job.  The c4 ensemble
shards by member (rank r advances members r, r + N, ...; strong scaling, no
exchange while they run, one all-gather of the force histories at the end)
and `value` is member-timesteps/s of all 64.  Rank 0 prints one JSON line.

* value        K steps with the state resident in HBM, CUDA events around each
               step on the stream it runs on, L2 flushed (256 MB write) between
               steps outside the timed events; max over ranks.
* plain        the plain FP64 GPU path of the same workload timed the same way in
               the same process: its timesteps/s, the speed-up of the chosen
               form over it, and the relative L2 differences of the forces over
               the same W + K steps and of the final vorticity.
* e2e          the same metric through the public API with the state on the
               host, as the reference's IBSolver::advance(State&) contract has
               it: every step uploads omega, q, f from pinned host memory,
               advances one step and reads omega, q, f back.
* roofline     the DST-I column pass (the dominant kernel), each launch timed
               alone with CUDA events on the solver's stream after an L2 flush,
               against the measured HBM copy bandwidth; traffic is null (DRAM
               bytes come from ncu runs, summarised under profiles/).
* cpu_baseline the reference's own CPU code (oracle/_ref/ref_driver: the
               reference sources built with -Ofast and the FFTW shim), one core,
               a bounded sample of steps of the same workload, with the relative
               L2 difference of its forces from the GPU run's over the same steps.
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

UNIT = "timesteps/s"
METRICS = {
    "c2": "timesteps/s (400x200 x5-domain shedding cylinder, RK3)",
    "c3": "timesteps/s (500x250 x3-domain pitching/plunging plate, RK3, CG tol 1e-10)",
    "c4": "member-timesteps/s (ensemble of 64 ellipse runs, n 128-512, 1-3 domains, RK3)",
    "c5": "timesteps/s (1024x1024 x5-domain pair of plunging cylinders, RK3, CG tol 1e-10)",
}
FORMS = {"c2": ("fp32_refined", "fp32", "fp64"), "c3": ("cholesky", "learned", "cg"),
         "c4": ("ensemble_fp32", "ensemble_refined", "ensemble", "serial"), "c5": ("cholesky", "learned", "cg")}
PLAIN = {"c2": "fp64", "c3": "cg", "c4": "serial", "c5": "cg"}
STEPS = {"c2": 200, "c3": 50, "c4": 60, "c5": 24}
WARMUP = {"c2": 10, "c3": 3, "c4": 3, "c5": 3}
PC_REFRESH = {"c3": 10, "c5": 24}  # one rebuild per timed window
L2_NOTE = "flushed between timed steps (256 MB write outside the events)"


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _workload(wlname):
    from ibpm_b200 import configs
    return {"c2": configs.c2_shedding_cylinder, "c3": configs.c3_pitching_plate,
            "c5": configs.c5_two_cylinders}[wlname]()


def workload_config(wlname, members=64):
    """What identifies the workload: the same dict for both arms."""
    from ibpm_b200 import configs
    c = {"workload": wlname, "l2": L2_NOTE}
    if wlname == "c4":
        ms = configs.ensemble_members(count=members)
        c.update({"name": f"ensemble of {members} ellipse runs", "members": members, "seed": 11,
                  "n": [w.nx for w in ms], "ngrid": [w.ngrid for w in ms],
                  "grid_points_all_levels": int(sum(w.nx * w.ny * w.ngrid for w in ms)), "scheme": "rk3",
                  "dt": "0.5 dx", "Re": "U[50, 300] seeded"})
        return c
    wl = _workload(wlname)
    c.update({"name": wl.name, "nx": wl.nx, "ny": wl.ny, "ngrid": wl.ngrid, "length": wl.length, "Re": wl.Re,
              "dt": wl.dt, "scheme": wl.scheme, "cg_tol": wl.tol})
    if wl.noise_amp:
        c["initial_condition"] = f"seeded N(0, {wl.noise_amp:g}^2) level-0 wake vorticity (seed {wl.noise_seed})"
    return c


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.p = None
        # raw samples beside the run (IBG_CLOCKS_DIR, else the temp directory); the JSON line carries the summary
        import tempfile
        self.path = os.path.join(os.environ.get("IBG_CLOCKS_DIR", tempfile.gettempdir()), f"clocks_rank{device}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.fh,
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


def rel_l2(a, b):
    import numpy as np
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own code on the host cores (bounded samples)
# ---------------------------------------------------------------------------
def _c4_sample(count):
    """(member index, workload) of the members the CPU samples: the first `count` with n <= 256
    (the larger members' CPU Cholesky set-up is minutes long)."""
    from ibpm_b200 import configs
    return [(k, w) for k, w in enumerate(configs.ensemble_members()) if w.nx <= 256][:count]


CPU_STEPS = {"c2": 10, "c3": 2, "c4": 3, "c5": 1}   # timed reference steps per sample (bounded CPU time)
CPU_WARMUP = {"c2": 3, "c3": 1, "c4": 3, "c5": 0}


def cpu_baseline(wlname, steps=None, warmup=None):
    """The reference over a bounded sample: one simulation on one host core (the reference is
    single-threaded), or for the c4 ensemble one member per usable core, side by side.  Returns
    (baseline dict, forces per sampled run (W + K steps each), member indices of the c4 sample)."""
    from oracle import ref_runner
    if not ref_runner.available():
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": "unavailable: oracle/_ref/ref_driver not built"}, None, None
    cpu = ref_runner.host_cpu()
    n = steps or CPU_STEPS[wlname]
    w = CPU_WARMUP[wlname] if warmup is None else warmup
    if wlname != "c4":
        r = ref_runner.run(_workload(wlname), wlname, steps=n, warmup=w)
        what = {"c2": "RK3 steps", "c3": "RK3 steps (plain CG force solve, tol 1e-10)",
                "c5": "RK3 steps (plain CG force solve, tol 1e-10)"}[wlname]
        return ({"value": r["steps_per_s"], "unit": UNIT, "cores": 1, "kind": "reference",
                 "sample": f"{r['timed_steps']} {what} of the same workload after {w} warm-up steps, Cholesky "
                           f"set-up (init {r['init_s']:.1f} s) excluded, reference sources -Ofast + project DST-I "
                           f"FFTW shim, 1 core of {cpu} (the reference is single-threaded)"}, [r["forces"]], None)
    # the ensemble's members are independent simulations: one per usable core, side by side
    sample = _c4_sample(len(ref_runner.usable_cpus()))
    res = ref_runner.run_parallel([(wl, f"c4_{wl.name}") for _, wl in sample], steps=n, warmup=w)
    value = sum(r["steps_per_s"] for r in res)
    sizes = sorted({(wl.nx, wl.ngrid) for _, wl in sample})
    return ({"value": value, "unit": UNIT, "cores": len(sample), "kind": "reference",
             "sample": f"{n} RK3 steps after {w} warm-up steps each of members {[k for k, _ in sample]} (the first "
                       f"{len(sample)} with n <= 256, grids (n, ngrid) {sizes}; larger members' CPU Cholesky set-up "
                       f"is too long to sample), one member per core side by side, the value the sum of their "
                       f"step rates; Cholesky set-up excluded, {len(sample)} cores of {cpu}"},
            [r["forces"] for r in res], [k for k, _ in sample])


def run_reference(args):
    ws, rank, local = _dist()
    if rank != 0:
        return 0
    from oracle import ref_runner
    wlname = args.workload
    if not ref_runner.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_driver is not built on this host"}))
        return 0
    cap = {"c2": 20, "c3": 3, "c4": 3, "c5": 1}[wlname]
    steps = max(1, min(args.steps, cap))
    warm = min(args.warmup, {"c2": 10, "c3": 1, "c4": 3, "c5": 0}[wlname])
    cb, _, _ = cpu_baseline(wlname, steps=steps, warmup=warm)
    v = cb["value"]
    out = {"metric": METRICS[wlname], "unit": UNIT, "n_gpus": args.gpus, "steps": steps, "warmup": warm,
           "value": v, "ms_per_step": 1000.0 / v, "higher_is_better": True,
           "scaling": "strong" if wlname == "c4" else "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic (seeded initial conditions and generated geometry)",
           "config": workload_config(wlname, args.members), "form": "reference FP64 CPU", "impl": "reference",
           "cpu_baseline": dict(cb, sample=cb["sample"] + f" (requested --steps {args.steps} --warmup "
                                                          f"{args.warmup}; capped at {cap} and {warm} to bound CPU "
                                                          f"time)"),
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def time_steps(K, stream, step, flush):
    """K steps, each bracketed by CUDA events on `stream`, L2 flushed before each; returns ms."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    launches = 0
    with torch.cuda.stream(stream):
        for k in range(K):
            flush.zero_()
            ev[k][0].record(stream)
            launches += step()
            ev[k][1].record(stream)
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in ev), launches


def _pinned_state(x):
    """Pinned host copies of a State's arrays plus its step counter and time."""
    import torch
    h = {}
    for k in ("omega", "q", "f"):
        a = getattr(x, k)
        h[k] = torch.empty(a.shape, dtype=torch.float64, pin_memory=True).numpy()
        h[k][...] = a
    h["ts"], h["t"] = int(x.timestep), float(x.time)
    return h


def _upload(s, h):
    import ibpm_b200 as ib
    L = ib._native.lib()
    ib._native.check(L.ibg_set_state(s.handle, ib._ptr(h["omega"]), ib._ptr(h["q"]), ib._ptr(h["f"]), h["ts"],
                                     h["t"]), s.handle)


def _download(s, h):
    import ctypes
    import ibpm_b200 as ib
    L = ib._native.lib()
    ts, t = ctypes.c_int(), ctypes.c_double()
    ib._native.check(L.ibg_get_state(s.handle, ib._ptr(h["omega"]), ib._ptr(h["q"]), ib._ptr(h["f"]),
                                     ctypes.byref(ts), ctypes.byref(t)), s.handle)
    h["ts"], h["t"] = ts.value, t.value


class Single:
    """One simulation (c2, c3, c5) in a given form."""

    def __init__(self, wlname, form, stream, device, pc_refresh=10, lpc_train=None, cg_graph=True, precision=None):
        import ibpm_b200 as ib
        self.wl = _workload(wlname)
        kw = {}
        if wlname == "c2":
            kw["precision"] = form
        else:
            kw["precond"] = {"cg": "none", "cholesky": "cholesky", "learned": "learned"}[form]
            kw["pc_refresh"] = pc_refresh
            kw["cg_graph"] = cg_graph
            if precision:
                kw["precision"] = precision
        self.grid, self.model, self.s, self.x = ib.from_workload(self.wl, stream=stream.cuda_stream, device=device,
                                                                 **kw)
        self.run = {}
        if form == "cholesky":
            self.run["pc_refresh"] = pc_refresh
        if form == "learned":
            nconf, epochs = lpc_train
            t0 = time.perf_counter()
            geom, mb = self.s.lpc_generate(nconf, 0.0, 8.0)
            t1 = time.perf_counter()
            hist = self.s.lpc_train(geom, mb, epochs=epochs, batch=4, lr=2e-3, seed=1)
            t2 = time.perf_counter()
            self.run["training"] = {"configurations": nconf, "times": [0.0, 8.0], "epochs": epochs, "batch": 4,
                                    "lr": 2e-3, "generate_s": t1 - t0, "train_s": t2 - t1,
                                    "loss_first": float(hist[0]), "loss_last": float(hist[-1])}
        self.s.init()
        self.s.set_state(self.x, with_q=False)
        self.stream = stream
        self.total = 1

    def step(self):
        self.s.advance_resident(1)
        return self.s.last_launch_count()

    def forces(self, K):
        return self.s.force_history(K)

    def omega(self):
        self.s.get_state(self.x)
        return self.x.omega.copy()

    def iterations(self):
        return self.s.cg_totals()

    def e2e(self, Ke, sync):
        """The reference's contract (src/IBSolver.cc:142-149): the State lives on
        the host; every step uploads omega, q, f, advances and reads them back."""
        import torch
        x = self.x
        self.s.get_state(x)
        host = _pinned_state(x)
        sync()
        t0 = time.perf_counter()
        for _ in range(Ke):
            _upload(self.s, host)
            self.s.advance_resident(1)
            _download(self.s, host)
        torch.cuda.synchronize()
        nb = int(8 * (x.omega.size + x.q.size + x.f.size))
        return time.perf_counter() - t0, nb, nb

    def roof_solver(self):
        return self.s, self.stream

    def close(self):
        self.s.close()


class Ens:
    """The 64-member ensemble (c4): one graph (ensemble*) or member after member (serial)."""

    def __init__(self, form, stream, device, count=64, world_size=1, rank=0, autotune=False):
        import ibpm_b200 as ib
        from ibpm_b200 import configs
        from ibpm_b200.replicas import shard
        import torch
        self.members = []
        self.total = count
        self.device = torch.device("cuda", device)
        prec = {"ensemble_fp32": "fp32", "ensemble_refined": "fp32_refined"}.get(form, "fp64")
        everyone = configs.ensemble_members(count=count)
        self.mine = shard(count, world_size, rank)
        # with several GPUs the members shard over the ranks (no exchange while they run)
        for wl in [everyone[i] for i in self.mine]:
            grid, model, s, x = ib.from_workload(wl, stream=stream.cuda_stream, device=device, precision=prec)
            s.init()
            s.set_state(x, with_q=False)
            self.members.append((wl, grid, s, x))
        self.form = form
        self.ens = None
        self.stream = stream
        self.member_stream = stream
        self.run = {"members_on_rank0": len(self.members), "member_precision": prec}
        self.pre_steps = 0  # steps every member took before the warm-up (the launch-shape trials)
        if form.startswith("ensemble"):
            self.ens = ib.Ensemble([m[2] for m in self.members])
            self.stream = torch.cuda.ExternalStream(self.ens.stream(), device=torch.device("cuda", device))
            if world_size == 1 and autotune:
                # the members' DST launch shapes per grid class, chosen by timing ensemble steps
                self.ens.advance(1)
                self.run["ensemble_shapes"] = self.ens.autotune(2)
                s0, x0 = self.members[0][2], self.members[0][3]
                s0.get_state(x0)
                self.pre_steps = int(x0.timestep)

    def step(self):
        if self.ens is not None:
            self.ens.advance(1)
            return self.ens.launches_per_step()
        n = 0
        for _, _, s, _ in self.members:
            s.advance_resident(1)
            n += s.last_launch_count()
        return n

    def forces(self, K):
        """every member's force history, in member order (one all-gather over the ranks)"""
        import numpy as np
        from ibpm_b200.replicas import gather_histories
        local = np.stack([m[2].force_history(K) for m in self.members])
        return gather_histories(local, self.total, device=self.device)

    def omega(self):
        import numpy as np
        out = []
        for _, _, s, x in self.members:
            s.get_state(x)
            out.append(x.omega.ravel().copy())
        return np.concatenate(out)

    def e2e(self, Ke, sync):
        """Every step copies every member's State in from pinned host memory and back out: in the
        ensemble forms through Ensemble.advance_host (the copies inside the ensemble's graph, each
        member's overlapping the others' steps), member by member otherwise."""
        import torch
        from types import SimpleNamespace
        hosts = []
        for wl, grid, s, x in self.members:
            s.get_state(x)
            hosts.append((s, _pinned_state(x)))
        states = [SimpleNamespace(omega=h["omega"], q=h["q"], f=h["f"]) for _, h in hosts]
        sync()
        t0 = time.perf_counter()
        for _ in range(Ke):
            if self.ens is not None:
                self.ens.advance_host(states, 1)
                continue
            for s, h in hosts:
                _upload(s, h)
            self.step()
            for s, h in hosts:
                _download(s, h)
        torch.cuda.synchronize()
        nb = sum(int(8 * (x.omega.size + x.q.size + x.f.size)) for *_, x in self.members)
        return time.perf_counter() - t0, nb, nb

    def roof_solver(self):
        # the largest member (it runs on the members' stream)
        return max(self.members, key=lambda m: m[0].nx * m[0].ny * m[0].ngrid)[2], self.member_stream

    def close(self):
        if self.ens is not None:
            self.ens.close()
        for m in self.members:
            m[2].close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=None)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c4", choices=["c2", "c3", "c4", "c5"])
    ap.add_argument("--form", default=None)
    ap.add_argument("--members", type=int, default=64, help="c4: ensemble members (the workload has 64)")
    ap.add_argument("--pc-refresh", type=int, default=None, help="c3/c5 cholesky: steps between rebuilds")
    ap.add_argument("--lpc-train", default=None, help="c3/c5 learned: CONFIGS,EPOCHS of the training run")
    ap.add_argument("--precision", default=None, choices=["fp64", "fp32_refined", "fp32"],
                    help="c3/c5: arithmetic of the bulk fields and solves (default fp64)")
    ap.add_argument("--host-cg", action="store_true",
                    help="c3/c5: the CG loop driven from the host instead of a device WHILE node in the step "
                         "graph (profilers cannot see the kernels of a graph with conditional nodes)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-path comparison run")
    ap.add_argument("--ens-autotune", action="store_true",
                    help="c4: choose the members' launch shapes per grid class by timing ensemble steps first "
                         "(the trials advance the members; the plain run takes the same steps)")
    ap.add_argument("--profile", action="store_true",
                    help="bracket the timed steps with cudaProfilerStart/Stop (for ncu --profile-from-start off) "
                         "and skip the e2e, roofline, plain and CPU legs")
    ap.add_argument("--kernel-probe", default=None, choices=["roofline", "gemm"],
                    help="for ncu --profile-from-start off: run only the c4 roofline kernel (the largest member's "
                         "FP32 column pass, members' launch shape) or four FP32 Poisson solves of a 256x256 grid "
                         "with the sine-matrix GEMM passes, bracketed by cudaProfilerStart/Stop")
    args = ap.parse_args()
    if args.kernel_probe:
        return kernel_probe(args.kernel_probe)
    wlname = args.workload
    if args.steps is None:
        args.steps = STEPS[wlname]
    if args.warmup is None:
        args.warmup = WARMUP[wlname]
    if args.impl == "reference":
        return run_reference(args)
    form = args.form or FORMS[wlname][0]
    if form not in FORMS[wlname]:
        raise SystemExit(f"--form for {wlname} must be one of {FORMS[wlname]}")
    pc_refresh = args.pc_refresh or PC_REFRESH.get(wlname, 10)
    lpc_train = tuple(int(v) for v in (args.lpc_train or ("64,1500" if wlname == "c3" else "16,300")).split(","))

    import numpy as np
    import torch
    import torch.distributed as dist

    ws, rank, local = _dist()
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2
    W = max(3, args.warmup)
    K = max(1, args.steps)

    def build(f):
        stream = torch.cuda.Stream(device=dev)
        if wlname == "c4":
            return Ens(f, stream, local, count=args.members, world_size=ws, rank=rank, autotune=args.ens_autotune)
        # the plain path is always FP64; --precision applies to the chosen form
        prec = args.precision if f != PLAIN[wlname] else None
        return Single(wlname, f, stream, local, pc_refresh=pc_refresh, lpc_train=lpc_train,
                      cg_graph=not args.host_cg, precision=prec)

    from ibpm_b200.replicas import job_throughput, max_over_ranks

    def maxrank(v):
        return max_over_ranks(v, device=dev)

    def sync():
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()

    run = build(form)
    for _ in range(W):
        run.step()
    it0 = run.iterations() if hasattr(run, "iterations") else None
    sync()
    clocks = ClockSampler(local)
    clocks.start()
    if args.profile:
        torch.cuda.cudart().cudaProfilerStart()
    ms, launches = time_steps(K, run.stream, run.step, flush)
    if args.profile:
        torch.cuda.cudart().cudaProfilerStop()
    clk = clocks.stop()
    ms = maxrank(ms)
    # units the whole job advances per step: every ensemble member (sharded over the ranks), or one
    # replica per rank
    job_units = run.total if wlname == "c4" else ws
    value = job_throughput(1, K, job_units, ms)
    pre = getattr(run, "pre_steps", 0)
    forces = run.forces(pre + W + K)
    omega = run.omega()
    cg = None
    if it0 is not None:
        it1 = run.iterations()
        solves = it1[1] - it0[1]
        cg = {"iterations_per_solve": (it1[0] - it0[0]) / max(1, solves), "solves": solves}
        if hasattr(run, "s"):
            _, mx, capped = run.s.cg_stats()
            cg["max_iterations"], cg["solves_at_the_cap"] = mx, capped  # capped solves did not converge

    if args.profile:
        run.close()
        if rank == 0:
            print(json.dumps({"metric": METRICS[wlname], "value": value, "unit": UNIT, "profile_run": True,
                              "ms_per_step": ms / K, "steps": K, "gpu_launches": int(launches)}))
        if ws > 1:
            dist.destroy_process_group()
        return 0
    Ke = min(K, 20 if wlname != "c2" else 50)
    e2e_s, bi, bo = run.e2e(Ke, sync)
    e2e_s = maxrank(e2e_s)
    e2e = {"value": job_throughput(1, Ke, job_units, 1000.0 * e2e_s), "unit": UNIT, "h2d_bytes_per_step": bi,
           "d2h_bytes_per_step": bo}
    f32 = form in ("fp32", "ensemble_fp32", "fp32_refined", "ensemble_refined") or args.precision in (
        "fp32", "fp32_refined")
    roof = kernel_roofline(*run.roof_solver(), flush, dtype="float" if f32 else "double")
    info = dict(run.run)
    import ibpm_b200 as ib
    info["autotuned_dst_shapes"] = ib.autotune_log()
    info["dst_form"] = ib.dst_form_log()
    info["sweep_form"] = ib.sweep_form_log()
    info["fp64_pass_form"] = ib.pass_form_log()
    run.close()

    plain = None
    if form != PLAIN[wlname] and not args.no_plain:
        p = build(PLAIN[wlname])
        for _ in range(pre + W):  # the same steps as the chosen form's run (its shape trials included)
            p.step()
        pit0 = p.iterations() if hasattr(p, "iterations") else None
        sync()
        pms, _ = time_steps(K, p.stream, p.step, flush)
        pms = maxrank(pms)
        pforces = p.forces(pre + W + K)
        pomega = p.omega()
        plain = {"form": PLAIN[wlname], "value": job_throughput(1, K, job_units, pms), "ms_per_step": pms / K,
                 "force_rel_l2_vs_plain": rel_l2(forces, pforces),
                 "force_max_member_rel_l2_vs_plain": (max(rel_l2(a, b) for a, b in zip(forces, pforces))
                                                      if wlname == "c4" else None),
                 "omega_rel_l2_vs_plain": rel_l2(omega, pomega) if ws == 1 else None}
        if wlname != "c4":
            # the force error of every step (largest component over the run's largest force)
            import numpy as np
            fa, fb = np.asarray(forces), np.asarray(pforces)
            n = min(len(fa), len(fb))
            scale = float(np.abs(fb[:n]).max()) or 1.0
            plain["force_err_per_step"] = [float(v) for v in np.abs(fa[:n] - fb[:n]).max(axis=1) / scale]
        if pit0 is not None:
            pit1 = p.iterations()
            plain["iterations_per_solve"] = (pit1[0] - pit0[0]) / max(1, pit1[1] - pit0[1])
        plain["speedup"] = value / plain["value"]
        p.close()

    if rank == 0:
        dtype = {"fp32": "f32+f64", "ensemble_fp32": "f32+f64", "fp32_refined": "f32+f64 refined",
                 "ensemble_refined": "f32+f64 refined"}.get(args.precision or form, "f64")
        last = forces[-1] if wlname != "c4" else forces[0][-1]
        out = {"metric": METRICS[wlname], "value": value, "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": W,
               "ms_per_step": ms / K, "higher_is_better": True,
               "scaling": "strong" if wlname == "c4" else "weak", "vs_baseline": None, "dtype": dtype,
               "data": "synthetic (seeded initial conditions and generated geometry)",
               "config": workload_config(wlname, args.members), "form": form + (
                   f" ({args.precision})" if args.precision and wlname in ("c3", "c5") else ""),
               "run": info, "e2e": e2e,
               "gpu_launches": int(launches), "roofline": roof, "clocks": clk,
               "final_force": [float(last[0]), float(last[1])] if len(forces) else None}
        if wlname != "c4":
            out["grid_point_updates_per_s"] = value * run.wl.ngrid * (run.wl.nx - 1) * (run.wl.ny - 1)
        else:
            # every member advances once per ensemble step: (member-steps/s / members) x the nodes of
            # all members' levels
            from ibpm_b200 import configs
            ms = configs.ensemble_members(count=args.members)
            nodes = sum(w.ngrid * (w.nx - 1) * (w.ny - 1) for w in ms)
            out["grid_point_updates_per_s"] = value / len(ms) * nodes
        if cg:
            out["cg"] = cg
        if plain:
            out["plain"] = plain
        if ws == 1 and not args.no_cpu_baseline:
            try:
                cb, ref_forces, sample_idx = cpu_baseline(wlname)
                if ref_forces is not None:
                    mine = [forces] if wlname != "c4" else [forces[k] for k in sample_idx]
                    errs = []
                    for a, b in zip(mine, ref_forces):
                        n = min(len(a), len(b))
                        errs.append(rel_l2(a[:n], b[:n]))
                    cb["force_rel_l2_vs_gpu_run"] = max(errs)
                    cb["force_steps_compared"] = int(min(len(a) for a in ref_forces))
                out["cpu_baseline"] = cb
            except Exception as e:  # the baseline is reported, never required
                out["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                                       "sample": f"failed: {e}"}
        print(json.dumps(out))
    if ws > 1:
        dist.destroy_process_group()
    return 0


def kernel_probe(which):
    """Launch one kernel family alone between cudaProfilerStart/Stop (for an ncu capture of just it)."""
    import ctypes
    import numpy as np
    import torch
    import ibpm_b200 as ib
    from ibpm_b200 import configs, geometry
    L = ib._native.lib()
    if which == "roofline":
        # the largest c4 member as a one-member ensemble (which applies the members' launch shape)
        wl = max(configs.ensemble_members(count=64), key=lambda w: w.nx * w.ny * w.ngrid)
        grid, model, s, x = ib.from_workload(wl, precision="fp32")
        s.init()
        s.set_state(x, with_q=False)
        ens = ib.Ensemble([s])
        ens.advance(2)
        L.ibg_run_kernel(s.handle, 1, 1)
        torch.cuda.synchronize()
        torch.cuda.cudart().cudaProfilerStart()
        nb = L.ibg_run_kernel(s.handle, 1, 3)
        torch.cuda.synchronize()
        torch.cuda.cudart().cudaProfilerStop()
        print(json.dumps({"kernel_probe": which, "member": [wl.nx, wl.ny, wl.ngrid], "algorithmic_bytes": nb}))
        ens.close()
        s.close()
        return 0
    # four FP32 Poisson solves of a 256 x 256 single-level grid with the GEMM form of the DST passes
    grid = ib.Grid(256, 256, 1, 4.0, -2.0, -2.0)
    geo = geometry.parse(configs.cylinder_geom(24, r=0.3))
    s = ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, 100.0), 0.01, "rk3", precision="fp32")
    ib._native.check(L.ibg_set_dst_gemm(s.handle, 1), s.handle)
    f = np.random.default_rng(0).standard_normal(grid.scalar().shape)
    u = np.zeros_like(f)
    fp, up = f.ctypes.data_as(ctypes.c_void_p), u.ctypes.data_as(ctypes.c_void_p)
    ib._native.check(L.ibg_solve_fp32(s.handle, -1, fp, up), s.handle)
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStart()
    for _ in range(4):
        ib._native.check(L.ibg_solve_fp32(s.handle, -1, fp, up), s.handle)
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStop()
    print(json.dumps({"kernel_probe": which, "grid": [256, 256, 1], "gemm_status": L.ibg_dst_gemm_status(s.handle)}))
    s.close()
    return 0


def kernel_roofline(s, stream, flush, reps=50, dtype="double"):
    """The dominant kernel (the DST-I column pass over every level of one solve) and two
    others, each launch timed alone with CUDA events on the solver's stream after an L2
    flush (so its operands come from HBM), against the measured copy bandwidth."""
    import torch
    import ibpm_b200 as ib
    L = ib._native.lib()
    res = {}
    peak, kind = peaks()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    for which, name in ((0, "dst_rows"), (1, "dst_cols"), (2, "nonlinear_node_vel")):
        L.ibg_run_kernel(s.handle, which, 3)
        torch.cuda.synchronize()
        nbytes = 0
        with torch.cuda.stream(stream):
            for a, b in ev:
                flush.zero_()
                a.record(stream)
                nbytes = L.ibg_run_kernel(s.handle, which, 1)
                b.record(stream)
        torch.cuda.synchronize()
        us = 1000.0 * sum(a.elapsed_time(b) for a, b in ev) / reps
        res[name] = {"us_per_launch": us, "algorithmic_bytes": nbytes,
                     "GBps": nbytes / (us * 1e-6) / 1e9 if us > 0 else None}
    d = res["dst_cols"]
    achieved = d["algorithmic_bytes"] / (d["us_per_launch"] * 1e-6) / 1e9
    return {"kernel": f"k_dst_cols<{dtype}> (forward DST-I along i of every level of one solve)",
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_kind": f"{kind} (copy bandwidth, burst)", "timing": "each launch alone after a 256 MB L2 flush",
            "traffic": None, "kernels": res}


if __name__ == "__main__":
    sys.exit(main())
