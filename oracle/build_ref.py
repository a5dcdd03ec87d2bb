#!/usr/bin/env python
"""Build the reference LAMMPS itself (TEST INFRASTRUCTURE): oracle/_ref/.

This recipe compiles the reference's own sources where they lie (it never
copies them into the repository) with g++, into oracle/_ref/ only:

  oracle/_ref/lmp_serial  the reference's serial path: the core src/*.cpp,
                          the three EAM styles of MANYBODY (pair_eam,
                          pair_eam_alloy, pair_eam_fs), the USER-OMP files
                          whose parent style is in that set (so `-sf omp`
                          gives lj/cut/omp, eam/omp, nve/omp and the OpenMP
                          neighbor builds), and the STUBS MPI library.
  oracle/_ref/lmp_b200    the same program with this project's LAMMPS
                          package (lammps_b200/lammps: lj/cut/b200, eam/b200,
                          eam/alloy/b200, eam/fs/b200, nve/b200,
                          verlet/b200) linked against libb200md.so -- what a
                          LAMMPS user gets after `Install.sh 1` and `make`.

It does not run the reference's build system.  The only generated inputs are
the style_*.h headers: each is a list of `#include "<header>"` lines, one per
header of the selected sources that registers a style of that class (what
src/Make.sh:12-89 writes for an installed tree), written to
oracle/_ref/gen*/.

GCC >= 9 no longer treats const variables as predetermined shared, so the
reference's `#pragma omp parallel default(none)` regions fail to compile
(error "'x' not specified in enclosing 'parallel'").  OpenMP pragmas are
macro-expanded, so `-D'default(x)='` drops the `default(none)` clause without
touching a source file; the arithmetic is unchanged.

Usage: python oracle/build_ref.py [--src DIR] [--no-b200] [-j N]
The reference's src/ tree comes from --src, the LAMMPS_SRC environment
variable, or the default checkout location (DEFAULT_SRC).
"""
from __future__ import annotations

import argparse
import glob
import os
import re
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")
PKG = os.path.join(ROOT, "lammps_b200", "lammps")
LIBDIR = os.path.join(ROOT, "lammps_b200", "_lib")

MANYBODY = ["pair_eam.cpp", "pair_eam_alloy.cpp", "pair_eam_fs.cpp"]
OMP_RUNTIME = ["thr_omp.cpp", "thr_data.cpp"]
CXXFLAGS = ["-O2", "-g0", "-fopenmp", "-DLMP_USER_OMP", "-DLAMMPS_GZIP", "-D" "default(x)=",
            "-w"]

# (class macro, header prefix, style header) as src/Make.sh:60-75 lists them
STYLE_CLASSES = [("ANGLE_CLASS", "angle_", "angle"), ("ATOM_CLASS", "atom_vec_", "atom"),
                 ("BODY_CLASS", "body_", "body"), ("BOND_CLASS", "bond_", "bond"),
                 ("COMMAND_CLASS", "", "command"), ("COMPUTE_CLASS", "compute_", "compute"),
                 ("DIHEDRAL_CLASS", "dihedral_", "dihedral"), ("DUMP_CLASS", "dump_", "dump"),
                 ("FIX_CLASS", "fix_", "fix"), ("IMPROPER_CLASS", "improper_", "improper"),
                 ("INTEGRATE_CLASS", "", "integrate"), ("KSPACE_CLASS", "", "kspace"),
                 ("MINIMIZE_CLASS", "min_", "minimize"), ("PAIR_CLASS", "pair_", "pair"),
                 ("READER_CLASS", "reader_", "reader"), ("REGION_CLASS", "region_", "region")]


DEFAULT_SRC = "/root/reference/src"  # the reference checkout of the machine that builds
SOURCE_NOTE = os.path.join(OUT, "SOURCE")  # the tree the last build compiled


def ref_src(arg=None) -> str | None:
    """The reference's src/ tree: the argument, LAMMPS_SRC, or the default."""
    for src in (arg, os.environ.get("LAMMPS_SRC"), DEFAULT_SRC):
        if src and os.path.exists(os.path.join(src, "pair_lj_cut.h")):
            return src
    return None


def built_src() -> str | None:
    """The src/ tree of the last build, or LAMMPS_SRC, if it is present."""
    for src in (os.environ.get("LAMMPS_SRC"),
                open(SOURCE_NOTE).read().strip() if os.path.exists(SOURCE_NOTE) else None):
        if src and os.path.exists(os.path.join(src, "pair_lj_cut.h")):
            return src
    return None


def lmp_serial() -> str | None:
    p = os.path.join(OUT, "lmp_serial")
    return p if os.path.exists(p) else None


def lmp_b200() -> str | None:
    p = os.path.join(OUT, "lmp_b200")
    return p if os.path.exists(p) else None


def sources(src):
    """The reference sources of lmp_serial: (path, include dirs)."""
    core = sorted(glob.glob(os.path.join(src, "*.cpp")))
    many = [os.path.join(src, "MANYBODY", f) for f in MANYBODY]
    parents = {os.path.basename(p) for p in core + many}
    omp = [os.path.join(src, "USER-OMP", f) for f in OMP_RUNTIME]
    for p in sorted(glob.glob(os.path.join(src, "USER-OMP", "*_omp.cpp"))):
        b = os.path.basename(p)
        if b in OMP_RUNTIME:
            continue
        # USER-OMP/Install.sh installs a child only when its parent exists
        if b[:-len("_omp.cpp")] + ".cpp" in parents:
            omp.append(p)
    return core + many + omp


def headers_of(paths):
    return [p[:-4] + ".h" for p in paths if os.path.exists(p[:-4] + ".h")]


def write_styles(gen, hdrs):
    """style_<name>.h: one include per header that registers a style of the class."""
    os.makedirs(gen, exist_ok=True)
    for macro, prefix, name in STYLE_CLASSES:
        lines = []
        for h in sorted(hdrs, key=os.path.basename):
            b = os.path.basename(h)
            if not b.startswith(prefix):
                continue
            with open(h, errors="replace") as fh:
                if macro in fh.read():
                    lines.append(f'#include "{b}"\n')
        path = os.path.join(gen, f"style_{name}.h")
        text = "".join(lines)
        if not os.path.exists(path) or open(path).read() != text:
            with open(path, "w") as fh:
                fh.write(text)


def includes(src, gen, extra=()):
    dirs = [gen, *extra, src, os.path.join(src, "MANYBODY"), os.path.join(src, "USER-OMP"),
            os.path.join(src, "STUBS")]
    return [f"-I{d}" for d in dirs]


def obj_name(objdir, path):
    return os.path.join(objdir, os.path.basename(path)[:-4] + ".o")


def stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def compile_all(jobs, cmds):
    def run(c):
        r = subprocess.run(c, capture_output=True, text=True)
        return c, r

    failed = []
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        for c, r in ex.map(run, cmds):
            if r.returncode != 0:
                failed.append((c[-3], r.stderr[-2000:]))
    if failed:
        for f, err in failed[:5]:
            sys.stderr.write(f"--- {f}\n{err}\n")
        raise SystemExit(f"build_ref: {len(failed)} file(s) failed")


def uses_styles(path):
    with open(path, errors="replace") as fh:
        return re.search(r'#include\s+"style_', fh.read()) is not None


def build(src=None, b200=True, jobs=None, verbose=False):
    src = ref_src(src)
    if src is None:
        raise SystemExit("build_ref: reference tree not found (give --src or LAMMPS_SRC)")
    jobs = jobs or os.cpu_count() or 4
    os.makedirs(OUT, exist_ok=True)
    with open(SOURCE_NOTE, "w") as fh:
        fh.write(src + "\n")
    srcs = sources(src)
    gen = os.path.join(OUT, "gen")
    write_styles(gen, headers_of(srcs))
    objdir = os.path.join(OUT, "obj")
    os.makedirs(objdir, exist_ok=True)
    inc = includes(src, gen)
    styles = glob.glob(os.path.join(gen, "*.h"))
    cmds = []
    for p in srcs:
        o = obj_name(objdir, p)
        if stale(o, [p, *(styles if uses_styles(p) else [])]):
            cmds.append(["g++", *CXXFLAGS, *inc, "-c", p, "-o", o])
    mpi_o = os.path.join(objdir, "mpi_stubs.o")
    if stale(mpi_o, [os.path.join(src, "STUBS", "mpi.c")]):
        cmds.append(["gcc", "-O2", "-I" + os.path.join(src, "STUBS"), "-c",
                     os.path.join(src, "STUBS", "mpi.c"), "-o", mpi_o])
    if verbose:
        print(f"build_ref: {len(cmds)} of {len(srcs) + 1} objects to compile")
    compile_all(jobs, cmds)
    objs = [obj_name(objdir, p) for p in srcs] + [mpi_o]
    exe = os.path.join(OUT, "lmp_serial")
    if stale(exe, objs):
        subprocess.run(["g++", "-O2", "-fopenmp", "-o", exe + ".tmp", *objs, "-lm"], check=True)
        os.replace(exe + ".tmp", exe)
    if b200:
        build_b200(src, srcs, objs, jobs)
    return exe


def build_b200(src, srcs, objs, jobs):
    """lmp_serial plus the B200 package: the package's sources, and the
    reference files that include style headers compiled again against style
    headers that also list the package's styles."""
    lib = os.path.join(LIBDIR, "libb200md.so")
    if not os.path.exists(lib):
        raise SystemExit("build_ref: build libb200md.so first (python lammps_b200/build.py)")
    pkg_cpp = sorted(glob.glob(os.path.join(PKG, "*.cpp")))
    gen = os.path.join(OUT, "gen_b200")
    write_styles(gen, headers_of(srcs) + headers_of(pkg_cpp))
    objdir = os.path.join(OUT, "obj_b200")
    os.makedirs(objdir, exist_ok=True)
    inc = includes(src, gen, [PKG, os.path.join(ROOT, "include")])
    styles = glob.glob(os.path.join(gen, "*.h"))
    redo = [p for p in srcs if uses_styles(p)]
    cmds = []
    pkg_h = glob.glob(os.path.join(PKG, "*.h")) + [os.path.join(ROOT, "include", "b200md.h")]
    for p in redo + pkg_cpp:
        o = obj_name(objdir, p)
        if stale(o, [p, *styles, *(pkg_h if p in pkg_cpp else [])]):
            cmds.append(["g++", *CXXFLAGS, *inc, "-c", p, "-o", o])
    compile_all(jobs, cmds)
    redo_names = {os.path.basename(p)[:-4] for p in redo}
    base = [o for o in objs if os.path.basename(o)[:-2] not in redo_names]
    mine = [obj_name(objdir, p) for p in redo + pkg_cpp]
    exe = os.path.join(OUT, "lmp_b200")
    if stale(exe, base + mine + [lib]):
        subprocess.run(["g++", "-O2", "-fopenmp", "-o", exe + ".tmp", *base, *mine,
                        "-L" + LIBDIR, "-lb200md", "-Wl,-rpath,$ORIGIN/../../lammps_b200/_lib",
                        "-lm"], check=True)
        os.replace(exe + ".tmp", exe)
    return exe


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=None)
    ap.add_argument("--no-b200", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    a = ap.parse_args()
    print(build(a.src, b200=not a.no_b200, jobs=a.j, verbose=True))
