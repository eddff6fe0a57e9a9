"""Build the engine in-tree: dba_b200/libdba_b200.so and dba_b200/bin/dba_run.

nvcc cross-compiles for sm_100a (no GPU needed).  FP64 kernels are built with
-fmad=false so their arithmetic matches the CPU restatement bit for bit; FP32
kernels keep FMA contraction.  Rebuilds only what is older than its sources.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdba_b200.so")
BIN = os.path.join(HERE, "bin", "dba_run")
NVCC = os.environ.get("NVCC", "nvcc")
CXX = os.environ.get("CXX", "g++")
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = GENCODE + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
                     "-I" + os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"]

UNITS = [
    ("k_f64.cu", ["-fmad=false"]),
    ("k_f32.cu", []),
    ("api.cu", ["-fmad=false"]),
    ("noalloc.cu", ["-fmad=false"]),
    ("batch.cu", ["-fmad=false"]),
]
HEADERS = ["fpmath.h", "fpmath_coeffs.h", "k_common.cuh", "k_dendrite.cuh", "k_modelb.cuh", "k_kh.cuh",
           "k_reduce.cuh", "k_inst.cuh", "launch.h", "k_modelb_fast.cuh", "k_modelb_tile.cuh", "k_kh_tile.cuh", "k_dendrite_tile.cuh", "k_batch.cuh", "k_post.cuh", "k_pair.cuh"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build(verbose=False, jobs=4):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(BIN), exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "dba.h")]
    objs, procs = [], []
    for src, extra in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _newer(o, [s] + hdrs + [__file__]):
            cmd = [NVCC] + NVFLAGS + extra + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), flush=True)
            procs.append(subprocess.Popen(cmd))
    io_src = os.path.join(CSRC, "io.cpp")
    io_obj = os.path.join(BUILD, "io.o")
    objs.append(io_obj)
    if _newer(io_obj, [io_src] + hdrs):
        procs.append(subprocess.Popen([CXX, "-O2", "-std=c++17", "-fPIC", "-pthread", "-ffp-contract=off", "-c", io_src,
                                       "-o", io_obj]))
    bad = [p for p in procs if p.wait() != 0]
    if bad:
        raise RuntimeError("compilation failed")
    if _newer(LIB, objs):
        _run([NVCC] + GENCODE + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lcurand", "-lpthread"], verbose)
    run_src = os.path.join(CSRC, "dba_run.cpp")
    if os.path.exists(run_src) and _newer(BIN, [run_src, LIB]):
        _run([CXX, "-O2", "-std=c++17", run_src, "-o", BIN, "-L" + HERE, "-ldba_b200",
              "-Wl,-rpath,$ORIGIN/..", "-I" + os.path.join(ROOT, "include")], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
