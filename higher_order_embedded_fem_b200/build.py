"""Builds libhoefem.so (CUDA for sm_100a + host C++) in-tree with nvcc.

    python -m higher_order_embedded_fem_b200.build [--force] [--jobs N]

Objects are compiled in parallel into _build/ and linked into
higher_order_embedded_fem_b200/libhoefem.so; a source whose object is newer
than the source and the headers is not recompiled.
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libhoefem.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-O3", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def nvcc():
    for cand in [os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")]:
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(ROOT, "include", "hoefem.h"))
    return hs


def compile_one(src, force, extra):
    obj = os.path.join(BUILD, src + ".o")
    srcp = os.path.join(CSRC, src)
    newest = max([os.path.getmtime(srcp)] + [os.path.getmtime(h) for h in headers()])
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj, ""
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + extra + ["-c", srcp, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [nvcc()] + NVCC_FLAGS + extra + ["-x", "c++", "-c", srcp, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return obj, r.stderr


def build(force=False, jobs=None, verbose=False, extra=()):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(lambda s: compile_one(s, force, list(extra)), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                sys.stderr.write(log)
    if force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_verbose else []
    print(build(force=a.force or a.ptxas_verbose, jobs=a.jobs, verbose=a.ptxas_verbose, extra=extra))


if __name__ == "__main__":
    main()
