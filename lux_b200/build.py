"""Builds the CUDA library of the dense-stereo stage in-tree: lux_b200/liblux_sgm.so (sm_100a only).

    python -m lux_b200.build            # or: python lux_b200/build.py

Every kernel is compiled with --fmad=false (no multiply-add contraction) because the stage is held bit-exact against
Lux.Engine's .NET arithmetic, where every float operation rounds once.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "liblux_sgm.so")

SOURCES = ["prep.cu", "cost.cu", "sgm_emulate.cu", "sgm_uniform.cu", "sgm_split.cu", "sgm_wave.cu", "depth_cache.cu", "warp.cu", "census_sgm.cu", "lux_sgm.cu", "host_geom.cpp", "server.cpp", "dump.cpp", "color_transfer.cpp"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "--fmad=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-Xptxas", "-v",
]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, ptxas_log=None):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "lux_sgm.h"))
    objs = []
    logs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if not _stale(obj, [path] + headers):
            continue
        cmd = [nvcc()] + NVCC_FLAGS + ["-I", CSRC, "-c", path, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        logs.append(r.stdout + r.stderr)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {src}")
        if verbose:
            sys.stderr.write(r.stderr)
    if _stale(OUT, objs):
        cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", OUT] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    if ptxas_log:
        with open(ptxas_log, "w") as f:
            f.write("\n".join(logs))
    return OUT


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(OUT)
