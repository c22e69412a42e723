"""Build libsplatt_b200.so (64-bit idx/val) and libsplatt_b200_w32.so (32/32)
in-tree: CUDA kernels compiled once for sm_100a with nvcc, the C host code
compiled per width with gcc, both linked against the CUDA runtime.

    python splatt-stream_b200/build.py [--force] [--jobs N]
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
           "-Xptxas", "-warn-spills"]
CFLAGS = ["-O2", "-fPIC", "-std=gnu11", "-Wall", "-Wno-unused-function"]

# per-file nvcc flags.  k_stream.cu: plain global loads cached in L2 only
# (-dlcm=cg).  The scheduled executor runs a stream's successive slices on
# whichever SMs claim them within one launch, so an SM's L1 could still hold
# rows another SM has since rewritten; L2 is coherent.
KFLAGS = {"k_stream.cu": ["-Xptxas", "-dlcm=cg"]}

KERNELS = ["k_runtime.cu", "k_sort.cu", "k_csf.cu", "k_mttkrp.cu", "k_dense.cu",
           "k_stream.cu", "k_gram_tc.cu", "k_gram_noalloc.cu", "k_ingest.cu", "k_read.cu"]
HOST = ["api.c", "io.c", "csf.c", "mttkrp.c", "cpd.c", "stream.c", "serve.c"]

LIBS = {64: os.path.join(HERE, "libsplatt_b200.so"),
        32: os.path.join(HERE, "libsplatt_b200_w32.so")}
# the `splatt cpd` command (64-bit idx/val build), linked to LIBS[64]
CLI = os.path.join(HERE, "splatt")


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r.stderr


def _headers(d):
    return [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".h", ".cuh"))]


def build(force=False, jobs=None, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    kdir = os.path.join(CSRC, "kernels")
    hdir = os.path.join(CSRC, "host")
    kh = _headers(kdir)
    hh = _headers(hdir) + [os.path.join(ROOT, "include", "splatt_b200.h")] + kh
    tasks = []
    kobjs = []
    for f in KERNELS:
        src = os.path.join(kdir, f)
        if not os.path.exists(src):
            continue
        obj = os.path.join(BUILD, f + ".o")
        kobjs.append(obj)
        if force or _stale(obj, [src] + kh):
            tasks.append([NVCC] + ARCH + NVFLAGS + KFLAGS.get(f, []) + ["-c", src, "-o", obj])
    hobjs = {64: [], 32: []}
    for w in (64, 32):
        for f in HOST:
            src = os.path.join(hdir, f)
            if not os.path.exists(src):
                continue
            obj = os.path.join(BUILD, "%s.w%d.o" % (f, w))
            hobjs[w].append(obj)
            if force or _stale(obj, [src] + hh):
                tasks.append(["gcc"] + CFLAGS + ["-DSPLATT_IDX_TYPEWIDTH=%d" % w,
                                                 "-DSPLATT_VAL_TYPEWIDTH=%d" % w,
                                                 "-c", src, "-o", obj])
    jobs = jobs or min(16, os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        for err in ex.map(_run, tasks):
            if verbose and err.strip():
                sys.stderr.write(err)
    for w in (64, 32):
        lib = LIBS[w]
        objs = kobjs + hobjs[w]
        if force or _stale(lib, objs):
            _run([NVCC] + ARCH + ["-shared", "-o", lib] + objs +
                 ["-lcudart", "-Xlinker", "-rpath," + os.path.join(CUDA, "lib64")])
    cli_src = os.path.join(CSRC, "cli", "splatt_cmd.c")
    if force or _stale(CLI, [cli_src, LIBS[64], os.path.join(ROOT, "include", "splatt_b200.h")]):
        _run(["gcc"] + CFLAGS + ["-DSPLATT_IDX_TYPEWIDTH=64", "-DSPLATT_VAL_TYPEWIDTH=64", cli_src,
                                 "-o", CLI, "-L" + HERE, "-l:libsplatt_b200.so",
                                 "-Wl,-rpath,$ORIGIN", "-lm"])
    return LIBS


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    for w, p in build(a.force, a.jobs, a.verbose).items():
        print(w, p)
