"""Build the CUDA library and the CLI in-tree.

    python -m rssieve_b200.build          # or rssieve_b200.build.build()

Outputs rssieve_b200/_lib/librssieve_b200.so (kernels for sm_100a + the C ABI
of include/rssieve_b200.h, CUDA runtime linked statically) and
rssieve_b200/_lib/rssieve (the command-line drop-in).  Object files go to
rssieve_b200/_build/.  Rebuilds only what changed.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "_lib")
OBJDIR = os.path.join(PKG, "_build")
INCLUDE = os.path.join(os.path.dirname(PKG), "include")
LIB = os.path.join(LIBDIR, "librssieve_b200.so")
CLI = os.path.join(LIBDIR, "rssieve")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["sieve.cu", "setup.cu", "bsgs.cu", "peak.cu", "engine.cu", "noalloc.cu", "batch.cu"]
CPP_SOURCES = ["host.cpp"]
HEADERS = ["mont.cuh", "rs_internal.h", "rs_host.h"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r.stdout + r.stderr


def build(verbose=False, ptxas_info=False):
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "rssieve_b200.h")]
    jobs, objs = [], []
    for src in CU_SOURCES + CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJDIR, src + ".o")
        objs.append(o)
        if not _stale(o, [s] + hdrs) and not ptxas_info:
            continue
        if src.endswith(".cu"):
            cmd = [nvcc()] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
                                     "-I", INCLUDE, "-c", s, "-o", o]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
        else:
            cmd = ["g++", "-O2", "-fPIC", "-std=c++17", "-Wall", "-I", INCLUDE, "-c", s, "-o", o]
        jobs.append(cmd)
    out = []
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for r in ex.map(_run, jobs):
            out.append(r)
    if jobs or _stale(LIB, objs):
        _run([nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xcompiler", "-fPIC"])
    cli_src = os.path.join(CSRC, "cli.cpp")
    if _stale(CLI, [cli_src, LIB] + hdrs):
        _run(["g++", "-O2", "-std=c++17", "-Wall", "-I", INCLUDE, cli_src, "-o", CLI, "-L", LIBDIR,
              "-lrssieve_b200", "-Wl,-rpath,$ORIGIN"])
    if verbose or ptxas_info:
        sys.stdout.write("".join(out))
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
