"""The C-ABI library loads without a GPU and exports every declared symbol."""
import os
import re

from lammps_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    with open(os.path.join(ROOT, "include", "b200md.h")) as fh:
        text = fh.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(b200_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "b200_create" in names and "b200_run" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert missing == []


def test_binding_covers_header():
    assert sorted(_abi.SIGNATURES) == declared_functions()


def test_abi_version():
    assert _abi.load().b200_abi_version() == 1
