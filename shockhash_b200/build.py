"""Build recipe of the CUDA library ``shockhash_b200/_lib/libshg.so`` (sm_100a only).

Run as ``python -m shockhash_b200.build`` (or through ``__graft_entry__.build()``). Compiles every
``csrc/*.cu`` / ``csrc/*.cpp`` with nvcc for ``-gencode arch=compute_100a,code=sm_100a`` into one
shared library placed in-tree next to this file.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libshg.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", "--expt-relaxed-constexpr",
         "-I", INCLUDE, "-I", CSRC]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _stale(outputs, inputs):
    if not all(os.path.exists(o) for o in outputs):
        return True
    t = min(os.path.getmtime(o) for o in outputs)
    return any(os.path.getmtime(i) > t for i in inputs)


def build(verbose=False, force=False, jobs=8):
    os.makedirs(OUT_DIR, exist_ok=True)
    objdir = os.path.join(OUT_DIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "shg.h"))
    objs, procs = [], []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale([obj], [src] + headers):
            cmd = [NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj]
            if src.endswith(".cpp"):
                cmd = [NVCC] + FLAGS + ["-x", "cu", "-c", src, "-o", obj] + ARCH
            if verbose:
                print(" ".join(cmd), flush=True)
            procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
            while len([p for _, p in procs if p.poll() is None]) >= jobs:
                procs[0][1].wait()
    failed = False
    for src, p in procs:
        out, _ = p.communicate()
        if out:
            sys.stdout.write(out.decode())
        if p.returncode != 0:
            failed = True
    if failed:
        raise RuntimeError("nvcc failed")
    if force or _stale([LIB], objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
