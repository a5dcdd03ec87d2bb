"""The LAMMPS package (lammps_b200/lammps/): every source compiles against
the reference's own headers (syntax check with g++, both integer widths of
src/lmptype.h), and Install.sh installs and removes the files and the
Makefile.package flags the way a LAMMPS package does."""
import glob
import os
import shutil
import subprocess

import pytest

from oracle import build_ref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "lammps_b200", "lammps")
# the reference's src/ tree: LAMMPS_SRC, or the one oracle/build_ref.py
# compiled (the tests skip when neither is present)
LAMMPS_SRC = build_ref.built_src() or ""

SOURCES = sorted(glob.glob(os.path.join(PKG, "*.cpp")))


@pytest.mark.skipif(not os.path.exists(os.path.join(LAMMPS_SRC, "pair_lj_cut.h")),
                    reason="LAMMPS source tree not available")
@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
@pytest.mark.parametrize("bigbig", [False, True])
@pytest.mark.parametrize("src", SOURCES, ids=os.path.basename)
def test_package_source_compiles_against_reference_headers(src, bigbig):
    cmd = ["g++", "-std=c++11", "-fsyntax-only", "-Wall", "-Werror",
           "-I", os.path.join(ROOT, "include"), "-I", PKG,
           "-I", LAMMPS_SRC, "-I", os.path.join(LAMMPS_SRC, "MANYBODY"),
           "-I", os.path.join(LAMMPS_SRC, "STUBS"), src]
    if bigbig:
        cmd.insert(1, "-DLAMMPS_BIGBIG")
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_every_style_header_registers_a_style():
    styles = {}
    for h in glob.glob(os.path.join(PKG, "*.h")):
        with open(h) as fh:
            for line in fh:
                for kind in ("PairStyle(", "FixStyle(", "IntegrateStyle(", "DumpStyle("):
                    if line.startswith(kind):
                        styles[line[len(kind):].split(",")[0]] = os.path.basename(h)
    assert set(styles) == {"lj/cut/b200", "eam/b200", "eam/alloy/b200", "eam/fs/b200",
                           "nve/b200", "verlet/b200", "custom/b200"}


def test_install_script_round_trip(tmp_path):
    src = tmp_path / "src"
    pkg = src / "B200"
    shutil.copytree(PKG, pkg)
    (src / "pair_eam.h").write_text("// MANYBODY present\n")
    (src / "Makefile.package").write_text("PKG_INC =   \nPKG_PATH =   \nPKG_LIB =   \n")
    subprocess.run(["sh", "Install.sh", "1"], cwd=pkg, check=True)
    for f in ("pair_lj_cut_b200.cpp", "verlet_b200.h", "b200_link.cpp"):
        assert (src / f).exists()
    mk = (src / "Makefile.package").read_text()
    assert "-I$(B200_ROOT)/include" in mk and "-lb200md" in mk
    subprocess.run(["sh", "Install.sh", "2"], cwd=pkg, check=True)
    assert (src / "Makefile.package").read_text().count("-lb200md") == 1
    subprocess.run(["sh", "Install.sh", "0"], cwd=pkg, check=True)
    assert not (src / "pair_lj_cut_b200.cpp").exists()
    assert "-lb200md" not in (src / "Makefile.package").read_text()


def test_install_requires_manybody(tmp_path):
    src = tmp_path / "src"
    pkg = src / "B200"
    shutil.copytree(PKG, pkg)
    r = subprocess.run(["sh", "Install.sh", "1"], cwd=pkg, capture_output=True, text=True)
    assert r.returncode != 0 and "MANYBODY" in r.stdout
