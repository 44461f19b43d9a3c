"""Build libstgpu.so (sm_100a) in-tree with nvcc.

    python -m structure_b200.build        # incremental
    python -m structure_b200.build --force

The library is plain CUDA C++ behind the C ABI of include/stgpu.h; no torch
types cross the boundary.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libstgpu.so")
SOURCES = ["st_zpass.cu", "st_zpass_k1.cu", "st_zpass_k2.cu", "st_zpass_k3.cu",
           "st_zpass_k4.cu", "st_zpass_k5.cu", "st_zpass_k6.cu", "st_update.cu", "st_api.cu",
           "st_noalloc.cu", "st_grad.cu", "st_noadmix.cu",
           "st_popinfo.cu", "st_locprior.cu", "st_injected.cu"]
HEADERS = ["st_device.cuh", "st_types.h", "st_kernels.h", "st_zpass_fast.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=hidden", "-I" + os.path.join(ROOT, "include")]
# The data pass must round every product and sum exactly like its host
# restatement (bit-exact Z); the FP64 Metropolis/Dirichlet code may contract.
PER_FILE = {"st_update.cu": ["-fmad=true"], "st_grad.cu": ["-fmad=true"]}
DEFAULT_FMAD = ["-fmad=false"]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "stgpu.h")]
    objs, jobs = [], []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            jobs.append([NVCC] + ARCH + FLAGS + PER_FILE.get(src, DEFAULT_FMAD) + ["-c", s, "-o", o])
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4) or 1) as ex:
        for cmd, r in zip(jobs, ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), jobs)):
            if verbose:
                print(" ".join(cmd))
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise subprocess.CalledProcessError(r.returncode, cmd)
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    build_frontend(force, verbose)
    return LIB


FRONT = os.path.join(HERE, "frontend")
FRONT_LIB = os.path.join(HERE, "libstfront.so")
CLI = os.path.join(HERE, "stgpu_structure")
CXX = os.environ.get("CXX", "g++")


def build_frontend(force=False, verbose=False):
    """libstfront.so (parameters, data file, result files) and the
    stgpu_structure command line linked against libstgpu.so."""
    inc = "-I" + os.path.join(ROOT, "include")
    front = os.path.join(FRONT, "front.cpp")
    main = os.path.join(FRONT, "main.cpp")
    hdr = os.path.join(ROOT, "include", "stfront.h")
    cxx = [CXX, "-O2", "-std=c++17", "-Wall", inc]
    steps = []
    if force or _stale(FRONT_LIB, [front, hdr]):
        steps.append(cxx + ["-fPIC", "-shared", "-fvisibility=hidden", front, "-o", FRONT_LIB])
    if force or _stale(CLI, [front, main, hdr, LIB, os.path.join(ROOT, "include", "stgpu.h")]):
        steps.append(cxx + [main, front, "-L" + HERE, "-lstgpu", "-Wl,-rpath,$ORIGIN",
                            "-Wl,-rpath,/usr/local/cuda/lib64", "-o", CLI])
    for cmd in steps:
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise subprocess.CalledProcessError(r.returncode, cmd)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
