"""Build libqsmgpu.so (sm_100a) in-tree with nvcc.

Usage: python qsm.rs_b200/build.py [--force] [--jobs N]
Objects go to qsm.rs_b200/_build/, the library to qsm.rs_b200/lib/libqsmgpu.so.
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libqsmgpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=hidden", "-I", os.path.join(HERE, "..", "include")]


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers_mtime():
    m = 0.0
    for d in (CSRC, os.path.join(HERE, "..", "include")):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh")):
                m = max(m, os.path.getmtime(os.path.join(d, f)))
    return m


def compile_one(src, force, hdr_m, extra):
    obj = os.path.join(BUILD, src + ".o")
    path = os.path.join(CSRC, src)
    if not force and os.path.exists(obj):
        om = os.path.getmtime(obj)
        if om > os.path.getmtime(path) and om > hdr_m:
            return obj, None
    cmd = [NVCC] + ARCH + FLAGS + extra + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, r.stdout + r.stderr + "\n" + " ".join(cmd)
    return obj, None


def build(force=False, jobs=None, verbose_ptxas=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdr_m = headers_mtime()
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    srcs = sources()
    objs, errs = [], []
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for obj, err in ex.map(lambda s: compile_one(s, force, hdr_m, extra), srcs):
            objs.append(obj)
            if err:
                errs.append(err)
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread", "-lz"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.jobs, a.ptxas_v))
