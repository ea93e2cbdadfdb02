"""Run the reference IBPM (oracle/_ref/ref_driver, the reference sources built
with -Ofast and the FFTW shim) on a named workload and report steps/s.

TEST AND BASELINE INFRASTRUCTURE ONLY: used by bench.py's CPU-baseline leg and
its `--impl reference` arm, never by the product path.  The reference is
single-threaded; one run uses one host core (pinned with taskset to a core this
process may use), and independent runs can go side by side on several cores
(`run_parallel`).  The Cholesky factors are cached with the reference's own
save/load (src/IBSolver.cc:77-108) under oracle/_ref/cache/, so repeated samples
time the steps, not the set-up; runs with keep_cache=False remove their files.
"""
from __future__ import annotations

import json
import os
import subprocess
import time

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = os.path.join(HERE, "_ref", "ref_driver")
CACHE = os.path.join(HERE, "_ref", "cache")


def available() -> bool:
    return os.path.exists(DRIVER)


def _write_inputs(wl, tag: str):
    os.makedirs(CACHE, exist_ok=True)
    gpath = os.path.join(CACHE, tag + ".geom")
    with open(gpath, "w") as fh:
        fh.write(wl.geom)
    ic = None
    w0 = wl.initial_vorticity()
    if w0 is not None:
        import numpy as np
        from oracle import ibpm_oracle as O
        from ibpm_b200 import geometry
        g = O.Grid(wl.nx, wl.ny, wl.ngrid, wl.length, wl.xoffset, wl.yoffset)
        st = O.State(g, geometry.parse(wl.geom).num_points, omega=w0)
        ic = os.path.join(CACHE, tag + "_ic.bin")
        O.save_restart(ic, st, g)
    return gpath, ic


def usable_cpus() -> list:
    """The host cores this process may run on."""
    try:
        return sorted(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return list(range(os.cpu_count() or 1))


def run(wl, tag: str, steps: int, warmup: int = 1, timeout: float = 1800.0, cpu=None,
        keep_cache: bool = True) -> dict:
    """Run W + K steps of workload `wl` on one core (`cpu`, default the first usable one); returns the
    driver's JSON plus wall time and the net force (x, y) after each of the W + K steps ("forces")."""
    import numpy as np
    gpath, ic = _write_inputs(wl, tag)
    out_prefix = os.path.join(CACHE, tag + "_run")
    args = [DRIVER, "-nx", str(wl.nx), "-ny", str(wl.ny), "-ngrid", str(wl.ngrid), "-length", repr(wl.length),
            "-xoffset", repr(wl.xoffset), "-yoffset", repr(wl.yoffset), "-geom", gpath, "-Re", repr(wl.Re),
            "-dt", repr(wl.dt), "-scheme", wl.scheme, "-nsteps", str(steps + warmup), "-warmup", str(warmup),
            "-tol", repr(wl.tol), "-cholesky_cache", os.path.join(CACHE, tag), "-out", out_prefix]
    if ic:
        args += ["-ic", ic]
    if _has_taskset():
        args = ["taskset", "-c", str(usable_cpus()[0] if cpu is None else cpu)] + args
    t0 = time.time()
    try:
        p = subprocess.run(args, capture_output=True, text=True, timeout=timeout, check=True)
        wall = time.time() - t0
        line = [l for l in p.stdout.splitlines() if l.startswith("{")][-1]
        out = json.loads(line)
        out["wall_s"] = wall
        out["forces"] = np.loadtxt(out_prefix + ".forces").reshape(-1, 6)[:, 2:4]
    finally:
        junk = [out_prefix + ".forces", out_prefix + "_final.bin"]
        if not keep_cache:
            junk += [gpath] + ([ic] if ic else [])
            junk += [os.path.join(CACHE, f) for f in os.listdir(CACHE)
                     if f.startswith(tag + "_") and f.endswith(".cholesky")]
        for f in junk:
            try:
                os.remove(f)
            except OSError:
                pass
    return out


def run_parallel(jobs, steps: int, warmup: int, timeout: float = 1800.0, keep_cache: bool = False) -> list:
    """Independent runs side by side, one per usable core (at most as many at once as there are cores):
    jobs = [(workload, tag), ...]; returns run()'s results in job order."""
    import queue
    from concurrent.futures import ThreadPoolExecutor
    cpus = usable_cpus()[:max(1, len(jobs))]
    free = queue.Queue()
    for c in cpus:
        free.put(c)

    def one(wl, tag):
        c = free.get()  # a core no other run holds
        try:
            return run(wl, tag, steps, warmup, timeout, c, keep_cache)
        finally:
            free.put(c)

    with ThreadPoolExecutor(max_workers=len(cpus)) as ex:
        futs = [ex.submit(one, wl, tag) for wl, tag in jobs]
        return [f.result() for f in futs]


def _has_taskset() -> bool:
    from shutil import which
    return which("taskset") is not None


def host_cpu() -> str:
    try:
        for l in open("/proc/cpuinfo"):
            if l.startswith("model name"):
                return l.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


if __name__ == "__main__":
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    from ibpm_b200 import configs
    name = sys.argv[1] if len(sys.argv) > 1 else "c2"
    print(run(configs.ALL[name](), name, int(sys.argv[2]) if len(sys.argv) > 2 else 0, warmup=0))
