"""Builds libbabelsim_b200.so in-tree with nvcc for sm_100a (Blackwell B200).

    python -m babelsim_b200.build [--jobs N]

Each translation unit is compiled separately (in parallel) and linked into one
shared library next to this file.  The library is the product: the Python
package only loads it.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libbabelsim_b200.so")
OBJ = os.path.join(HERE, "_build")
SOURCES = ["mesh.cpp", "mesh_io.cpp", "renumber.cpp", "geometry.cu", "fvm.cu", "krylov.cu", "gmres.cu", "amg.cu", "pcg_persistent.cu", "pcg_sell.cu", "bicgstab_sell.cu", "simple.cu", "piso.cu", "rans.cu", "results.cpp", "capi.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# The device geometry reproduces the host geometry bit for bit: no FMA contraction there.
EXTRA = {"geometry.cu": ["-fmad=false"]}


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build babelsim_b200")
    return path


def flags():
    # BSG_NVCC_FLAGS: extra nvcc flags for a tuning build (e.g. -DBSG_SELL_BATCH=8); objects are
    # rebuilt when it changes
    extra = os.environ.get("BSG_NVCC_FLAGS", "").split()
    return ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
                   "-I" + os.path.join(ROOT, "include"), "-I" + CSRC] + extra


def compile_one(src):
    obj = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    path = os.path.join(CSRC, src)
    deps = [path] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    deps.append(os.path.join(ROOT, "include", "babelsim_b200.h"))
    stamp = obj + ".flags"
    same_flags = os.path.exists(stamp) and open(stamp).read() == " ".join(flags())
    if same_flags and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
        return obj
    lang = ["-x", "cu"] if src.endswith(".cu") else []
    cmd = [nvcc()] + flags() + EXTRA.get(src, []) + lang + ["-c", path, "-o", obj]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
    with open(stamp, "w") as f:
        f.write(" ".join(flags()))
    return obj


def build(jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    if not os.path.exists(OUT) or os.path.getmtime(OUT) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    if verbose:
        print(OUT)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    a = ap.parse_args()
    try:
        build(a.jobs, verbose=True)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
