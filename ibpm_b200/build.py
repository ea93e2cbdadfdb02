"""Build libibpm_b200.so in-tree with nvcc for sm_100a.

    python -m ibpm_b200.build        (or __graft_entry__.build())
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libibpm_b200.so")
SOURCES = ["elliptic.cu", "ops.cu", "force.cu", "api.cu", "noalloc.cu", "lpc.cu", "lpc_tc.cu", "refine.cu", "dst_gemm.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def build(verbose: bool = False) -> str:
    objs = []
    tmp = os.path.join(HERE, "_build")
    os.makedirs(tmp, exist_ok=True)
    procs = []
    for src in SOURCES:
        obj = os.path.join(tmp, src.replace(".cu", ".o"))
        objs.append(obj)
        cmd = [nvcc(), *ARCH, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            sys.stderr.write(out.decode())
            raise RuntimeError("nvcc failed: " + " ".join(cmd))
        if verbose:
            sys.stderr.write(out.decode())
    cmd = [nvcc(), *ARCH, "-shared", "-o", OUT, *objs, "-cudart", "static"]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
