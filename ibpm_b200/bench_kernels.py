"""Run one hot-path operation a few times on a named workload grid, for
focused profiler captures (ncu -k ...) of its kernels.

    python -m ibpm_b200.bench_kernels poisson c2 3
    python -m ibpm_b200.bench_kernels step c2 3
"""
import sys

import numpy as np


def main(argv):
    import ibpm_b200 as ib
    from ibpm_b200 import configs
    what = argv[1] if len(argv) > 1 else "poisson"
    wl = configs.ALL[argv[2] if len(argv) > 2 else "c2"]()
    reps = int(argv[3]) if len(argv) > 3 else 3
    precision = argv[4] if len(argv) > 4 else "fp64"
    grid, model, s, x = ib.from_workload(wl, precision=precision)
    if what == "poisson":
        f = np.random.default_rng(0).standard_normal(grid.scalar().shape)
        for _ in range(reps):
            u = s.poisson(f)
        print("ok", float(np.abs(u).max()))
    elif what == "step":
        s.init()
        s.set_state(x, with_q=False)
        s.advance_resident(reps)
        print("ok", s.force_history(1))
    else:
        raise SystemExit(f"unknown operation {what}")
    s.close()


if __name__ == "__main__":
    main(sys.argv)
