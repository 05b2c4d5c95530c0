"""Build recipe of libspmiqc_cuda.so (sm_100a) and libspmiqc_compat.so.

Compiles every csrc/*.cu with nvcc for sm_100a (one process per translation
unit, in parallel), links the shared libraries into spm-iqc_b200/lib/, and skips
objects whose sources are older than the object. Usable as a script
(`python spm-iqc_b200/build.py [-j N] [--force]`) or from Python (`build()`).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libspmiqc_cuda.so")
COMPAT_LIB = os.path.join(LIBDIR, "libspmiqc_compat.so")
BINDIR = os.path.join(HERE, "bin")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
                  "-I", os.path.join(ROOT, "include")]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(CSRC, "*.inc")) + glob.glob(os.path.join(ROOT, "include", "*.h"))


def _stale(obj: str, deps) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, obj: str, extra=()):
    cmd = [_nvcc()] + NVFLAGS + list(extra) + ["-c", src, "-o", obj]
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"nvcc failed for {os.path.basename(src)}:\n{out.stderr[-6000:]}")
    return obj


def build(jobs: int | None = None, force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    headers = _headers()
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    compat_srcs = sorted(glob.glob(os.path.join(CSRC, "compat", "*.cpp")))
    todo = []
    objs = []
    for s in srcs:
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            todo.append((s, o))
    jobs = jobs or max(1, min(len(todo), os.cpu_count() or 4))
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            futs = [ex.submit(_compile, s, o) for s, o in todo]
            for f in cf.as_completed(futs):
                o = f.result()
                if verbose:
                    print("built", os.path.basename(o), flush=True)
    if force or todo or _stale(LIB, objs):
        cmd = [_nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        out = subprocess.run(cmd, capture_output=True, text=True)
        if out.returncode != 0:
            raise RuntimeError("link failed:\n" + out.stderr[-4000:])
    if compat_srcs:
        cobjs = []
        for s in compat_srcs:
            o = os.path.join(OBJ, "compat_" + os.path.basename(s) + ".o")
            cobjs.append(o)
            if force or _stale(o, [s] + headers):
                cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-I", os.path.join(ROOT, "include"),
                       "-I", os.path.join(CUDA_HOME, "include"), "-c", s, "-o", o]
                out = subprocess.run(cmd, capture_output=True, text=True)
                if out.returncode != 0:
                    raise RuntimeError("compat compile failed:\n" + out.stderr[-4000:])
        if force or _stale(COMPAT_LIB, cobjs + [LIB]):
            # the reference's globals (N, u_R_local, ...) stay undefined here and
            # resolve against the program that links the drop-in
            cmd = ["g++", "-shared", "-o", COMPAT_LIB] + cobjs + ["-L", LIBDIR, "-lspmiqc_cuda",
                                                                   "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart",
                                                                   "-Wl,-rpath,$ORIGIN"]
            out = subprocess.run(cmd, capture_output=True, text=True)
            if out.returncode != 0:
                raise RuntimeError("compat link failed:\n" + out.stderr[-4000:])
    drivers = sorted(glob.glob(os.path.join(CSRC, "drivers", "*.cpp")))
    if drivers:
        os.makedirs(BINDIR, exist_ok=True)
        for s in drivers:
            exe = os.path.join(BINDIR, os.path.splitext(os.path.basename(s))[0])
            if force or _stale(exe, [s, LIB] + headers):
                cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                       "-I", os.path.join(CUDA_HOME, "include"), s, "-o", exe, "-L", LIBDIR, "-lspmiqc_cuda",
                       "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart", "-Wl,-rpath,$ORIGIN/../lib"]
                out = subprocess.run(cmd, capture_output=True, text=True)
                if out.returncode != 0:
                    raise RuntimeError("driver build failed:\n" + out.stderr[-4000:])
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.j, a.force, verbose=True))


if __name__ == "__main__":
    sys.exit(main())
