"""Build the rh3t shared libraries in-tree (no JIT cache):

  _build/librh3t.so        FP64 kernels, compiler mul+add -> FMA contraction on
  _build/librh3t_exact.so  same sources with --fmad=false (no contraction), the
                           build whose arithmetic follows the reference operation
                           for operation

Both are compiled for sm_100a only. Host code (geometry / ghost-grid build,
context set-up) is compiled with -ffp-contract=off so the ghost discovery stays
bit-identical to the reference's.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
GXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["kernels.cu", "ghosts.cu", "flux.cu", "rhs.cu", "context.cu", "tune.cu", "adjoint.cu", "adjoint_host.cu", "noalloc.cu", "lsbuild.cu", "io.cu", "divcheck.cu"]
CPP_SOURCES = ["host/ghostgrid.cpp"]
HEADERS = ["physics.cuh", "rh3t_dev.h", "kernels.cuh", "common.cuh", "context.h", "dual.cuh", "ghost_rows.cuh", "divrn.cuh", "mbar.cuh", "host/lsbuild.h"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-1]}")
    return r.stdout + r.stderr


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    os.makedirs(OUT, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in CU_SOURCES + CPP_SOURCES + HEADERS] + \
        [os.path.join(INCLUDE, "rh3t.h"), os.path.abspath(__file__)]
    host_obj = os.path.join(OUT, "ghostgrid.o")
    if force or _stale(host_obj, deps):
        _run([GXX, "-O3", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-Wall",
              "-I", INCLUDE, "-c", os.path.join(CSRC, CPP_SOURCES[0]), "-o", host_obj])
    outputs = []
    for name, fmad in (("librh3t.so", "true"), ("librh3t_exact.so", "false")):
        target = os.path.join(OUT, name)
        outputs.append(target)
        if not (force or _stale(target, deps + [host_obj])):
            continue
        objs = []
        for src in CU_SOURCES:
            obj = os.path.join(OUT, f"{os.path.splitext(src)[0]}_{fmad}.o")
            defs = ["-DRH3T_EXACT"] if fmad == "false" else []
            log = _run([NVCC] + ARCH + defs + ["-O3", "-lineinfo", "-std=c++17", f"--fmad={fmad}", "-Xptxas", "-v",
                                        "-Xcompiler", "-fPIC,-ffp-contract=off", "-I", INCLUDE, "-c",
                                        os.path.join(CSRC, src), "-o", obj])
            if verbose:
                print(log)
            objs.append(obj)
        _run([NVCC] + ARCH + ["-shared", "-o", target] + objs + [host_obj, "-lgomp", "-lcudart"])
    return outputs


if __name__ == "__main__":
    for p in build(force="--force" in sys.argv, verbose="-v" in sys.argv):
        print(p)
