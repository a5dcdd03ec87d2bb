"""Build libb200md.so (the C-ABI engine) in-tree for sm_100a with nvcc."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libb200md.so")
SOURCES = ["api.cu", "neigh.cu", "pair_lj.cu", "pair_eam.cu", "integrate.cu", "noalloc.cu", "adjoint.cu", "replica.cu", "halo.cu"]
HEADERS = ["md_common.cuh", "md_state.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "b200md.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    if not force and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    from concurrent.futures import ThreadPoolExecutor

    objs = [os.path.join(LIBDIR, src.replace(".cu", ".o")) for src in SOURCES]
    cmds = [["nvcc", *ARCH, *FLAGS, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
            for src, obj in zip(SOURCES, objs)]
    if verbose:
        for cmd in cmds:
            print(" ".join(cmd))
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
        for r in ex.map(lambda cmd: subprocess.run(cmd), cmds):
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    cmd = ["nvcc", *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lcudart"]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
    print(LIB)
