"""Builds the CUDA library of the NRG hot path in-tree (nrg_b200/libnrgb200.so) for sm_100a."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "nrg_b200", "libnrgb200.so")
SOURCES = ["capi.cu", "driver.cu", "routines.cu", "kernels.cu", "ggemm.cu", "eig.cu", "eig_large.cu",
           "noalloc.cu", "restart.cu", "tables.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "--extended-lambda", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "-Xcompiler", "-g"]


def build(force: bool = False, verbose: bool = False) -> str:
    srcs = [os.path.join(SRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".cuh", ".hpp"))]
    deps.append(os.path.join(HERE, "..", "include", "nrg_b200.h"))
    if not force and os.path.exists(OUT):
        t = os.path.getmtime(OUT)
        if all(os.path.getmtime(d) <= t for d in deps):
            return OUT
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        cmd = [NVCC, "-c", s, "-o", o] + FLAGS + ["-Xptxas", "-v"] * verbose
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT), s))
        objs.append(o)
    failed = False
    for p, s in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stderr.write(out.decode())
        if p.returncode != 0:
            failed = True
            sys.stderr.write(f"nvcc failed on {s}\n")
    if failed:
        raise RuntimeError("CUDA build failed")
    tmp = OUT + ".tmp"
    subprocess.check_call([NVCC, "-shared", "-o", tmp] + objs + ["-gencode", "arch=compute_100a,code=sm_100a",
                                                                  "-Xcompiler", "-fPIC", "-cudart", "static"])
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
