"""ctypes binding of libb200md.so (include/b200md.h).

The library is built in-tree by ``lammps_b200/build.py``.  Loading fails
loudly when it is missing: there is no CPU fallback for the engine.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libb200md.so")

B200_OK = 0
B200_ERR_STATE = -4
STATUS_NAMES = {
    0: "B200_OK", -1: "B200_ERR_ARG", -2: "B200_ERR_CUDA", -3: "B200_ERR_NOMEM",
    -4: "B200_ERR_STATE", -5: "B200_ERR_NEIGH_OVERFLOW", -6: "B200_ERR_BOX",
    -7: "B200_ERR_LOST_ATOMS", -8: "B200_ERR_TIMEOUT",
}
PREC = {"fp64": 0, "mixed": 1}
# column groups of b200_gather (enum b200_field)
FIELDS = {"x": 1, "v": 2, "f": 4, "image": 8}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p

# name -> (restype, argtypes); every symbol declared in include/b200md.h
SIGNATURES = {
    "b200_abi_version": (C.c_int, []),
    "b200_create": (C.c_int, [C.c_int, C.c_int, C.POINTER(_vp)]),
    "b200_destroy": (C.c_int, [_vp]),
    "b200_last_error": (C.c_char_p, [_vp]),
    "b200_bytes": (C.c_longlong, [_vp]),
    "b200_set_box": (C.c_int, [_vp, _dp, _dp]),
    "b200_set_neighbor": (C.c_int, [_vp, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int]),
    "b200_set_mass": (C.c_int, [_vp, C.c_int, _dp]),
    "b200_set_lj": (C.c_int, [_vp, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp]),
    "b200_set_eam": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double, C.c_int, C.c_double, C.c_double,
                               C.c_double, C.c_int, _dp, C.c_int, _dp, C.c_int, _dp, _ip, _ip, _ip]),
    "b200_upload_atoms": (C.c_int, [_vp, C.c_int, _dp, _dp, _ip, _ip]),
    "b200_download_atoms": (C.c_int, [_vp, _dp, _dp, _dp, _ip]),
    "b200_natoms": (C.c_int, [_vp]),
    "b200_stage_atoms": (C.c_int, [_vp, C.c_int, _dp, _dp, _ip]),
    "b200_set_staged_atoms": (C.c_int, [_vp]),
    "b200_download_atoms_async": (C.c_int, [_vp, _dp, _dp, _dp, _ip]),
    "b200_wait_transfers": (C.c_int, [_vp]),
    "b200_update_positions": (C.c_int, [_vp, _dp]),
    "b200_gather": (C.c_int, [_vp, C.c_int, C.c_int, _ip, _dp]),
    "b200_set_replica_step": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int]),
    "b200_get_replica_step": (C.c_int, [_vp, _ip, _ip, _ip, _ip, _dp]),
    "b200_eam_density": (C.c_int, [_vp, C.c_int, C.c_int]),
    "b200_eam_fp_pack": (C.c_int, [_vp, C.c_int, _vp, _vp]),
    "b200_eam_fp_unpack": (C.c_int, [_vp, C.c_int, _vp, _vp]),
    "b200_eam_force": (C.c_int, [_vp, C.c_int, C.c_int, _dp, _dp, _dp, _dp]),
    "b200_neigh_build": (C.c_int, [_vp]),
    "b200_pair_compute": (C.c_int, [_vp, C.c_int, C.c_int, _dp, _dp, _dp, _dp]),
    "b200_nve_initial": (C.c_int, [_vp, C.c_double, C.c_double]),
    "b200_nve_final": (C.c_int, [_vp, C.c_double]),
    "b200_setup": (C.c_int, [_vp, _dp]),
    "b200_run": (C.c_int, [_vp, C.c_int, C.c_double, C.c_double, C.c_int, _dp, C.c_int, _ip]),
    "b200_neigh_half": (C.c_int, [_vp, _ip, _ip, _ip, C.c_longlong, C.POINTER(C.c_longlong)]),
    "b200_neigh_stats": (C.c_int, [_vp, C.POINTER(C.c_longlong), _ip, _ip, _ip, _ip]),
    "b200_get_rho_fp": (C.c_int, [_vp, _dp, _dp]),
    "b200_set_launch": (C.c_int, [_vp, C.c_int, C.c_int]),
    "b200_get_launch": (C.c_int, [_vp, _ip, _ip]),
    "b200_kernel_launches": (C.c_longlong, [_vp]),
    "b200_set_timing": (C.c_int, [_vp, C.c_int]),
    "b200_set_graphs": (C.c_int, [_vp, C.c_int]),
    "b200_get_timing": (C.c_int, [_vp, _dp, C.POINTER(C.c_longlong), C.c_int]),
    "b200_stream": (_vp, [_vp]),
    "b200_get_step_times": (C.c_int, [_vp, _dp, C.c_int, _ip, C.c_int]),
    "b200_set_ghosts": (C.c_int, [_vp, _ip]),
    "b200_neigh_check": (C.c_int, [_vp, _ip]),
    "b200_halo_pack": (C.c_int, [_vp, C.c_int, C.c_void_p, C.c_void_p]),
    "b200_halo_unpack": (C.c_int, [_vp, C.c_int, C.c_void_p, C.c_void_p]),
    "b200_set_replicas": (C.c_int, [_vp, C.c_int, _ip, _dp, _dp]),
    "b200_replica_count": (C.c_int, [_vp]),
    "b200_replica_thermo": (C.c_int, [_vp, _dp]),
    "b200_adj_set_positions": (C.c_int, [_vp, _vp]),
    "b200_adj_forces": (C.c_int, [_vp, _dp, _dp, _dp, _vp]),
    "b200_adj_backward": (C.c_int, [_vp, _dp, _dp, _dp, _vp, _vp, _dp, _dp]),
    "b200_kinetic_sum_noalloc": (C.c_int, [C.c_int, _vp, _vp, _vp, C.c_int, _vp, _vp]),
}

_lib = None


def load(build_if_missing: bool = True):
    """Load libb200md.so (building it with nvcc when absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if not build_if_missing:
            raise RuntimeError(f"libb200md.so not built: {LIB_PATH} (run lammps_b200/build.py)")
        from . import build as _build

        _build.build()
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libb200md.so missing after build: {LIB_PATH}")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def dptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


def iptr(a):
    return None if a is None else a.ctypes.data_as(_ip)


def tdptr(t):
    """double* of a contiguous float64 torch tensor (host or device)."""
    return None if t is None else C.cast(C.c_void_p(t.data_ptr()), _dp)


def tiptr(t):
    """int* of a contiguous int32 torch tensor (host or device)."""
    return None if t is None else C.cast(C.c_void_p(t.data_ptr()), _ip)


class B200Error(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code
