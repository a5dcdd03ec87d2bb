"""CPU oracle for the short-range MD step -- TEST INFRASTRUCTURE ONLY.

ctypes binding of ``oracle/md_oracle.c``, a plain-C restatement of the
reference's serial CPU path (LAMMPS 8 Aug 2014: CommBrick::borders,
Neighbor::half_bin_newton, PairLJCut::compute, PairEAM::compute, FixNVE,
Pair::virial_fdotr_compute, Thermo).  Only the tests, ``__graft_entry__.smoke``
and the CPU-baseline leg of ``bench.py`` may use it, and only to check the
engine's results or as the timed CPU baseline.  The product (``lammps_b200``) never imports it.

Parity pin: the oracle is checked against the reference's own golden thermo
logs and neighbor statistics (``tests/golden/``); see
``tests/test_oracle_golden.py``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libmdoracle.so")
_lib = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < max(
            os.path.getmtime(os.path.join(_HERE, f)) for f in ("md_oracle.c", "md_oracle.h")
        )
    ):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        sig = {
            "orc_create": (C.c_void_p, [C.c_int]),
            "orc_destroy": (None, [C.c_void_p]),
            "orc_error": (C.c_char_p, [C.c_void_p]),
            "orc_set_threads": (None, [C.c_void_p, C.c_int]),
            "orc_set_timestep": (None, [C.c_void_p, C.c_double]),
            "orc_set_box": (C.c_int, [C.c_void_p, _dp, _dp]),
            "orc_set_atoms": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp, _dp, _ip, _ip]),
            "orc_set_mass": (None, [C.c_void_p, C.c_int, C.c_double]),
            "orc_set_neighbor": (None, [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int]),
            "orc_set_thermo": (None, [C.c_void_p, C.c_int]),
            "orc_pair_lj_cut": (C.c_int, [C.c_void_p, C.c_double, C.c_int]),
            "orc_pair_lj_coeff": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double]),
            "orc_pair_eam_funcfl": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_char_p), _ip]),
            "orc_pair_eam_setfl": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int, _ip]),
            "orc_setup": (C.c_int, [C.c_void_p]),
            "orc_run": (C.c_int, [C.c_void_p, C.c_int]),
            "orc_compute": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
            "orc_thermo_rows": (C.c_int, [C.c_void_p, _dp, C.c_int]),
            "orc_nlocal": (C.c_int, [C.c_void_p]),
            "orc_nghost": (C.c_int, [C.c_void_p]),
            "orc_ncalls": (C.c_int, [C.c_void_p]),
            "orc_ndanger": (C.c_int, [C.c_void_p]),
            "orc_ntimestep": (C.c_longlong, [C.c_void_p]),
            "orc_neigh_total": (C.c_longlong, [C.c_void_p]),
            "orc_eng_vdwl": (C.c_double, [C.c_void_p]),
            "orc_virial": (None, [C.c_void_p, _dp]),
            "orc_temperature": (C.c_double, [C.c_void_p]),
            "orc_pressure": (C.c_double, [C.c_void_p]),
            "orc_kinetic": (C.c_double, [C.c_void_p]),
            "orc_get_x": (None, [C.c_void_p, _dp]),
            "orc_get_v": (None, [C.c_void_p, _dp]),
            "orc_get_f": (None, [C.c_void_p, _dp]),
            "orc_get_tag": (None, [C.c_void_p, _ip]),
            "orc_get_type": (None, [C.c_void_p, _ip]),
            "orc_get_image": (None, [C.c_void_p, _ip]),
            "orc_get_rho_fp": (None, [C.c_void_p, _dp, _dp]),
            "orc_get_eatom_vatom": (None, [C.c_void_p, _dp, _dp]),
            "orc_neigh_half": (C.c_longlong, [C.c_void_p, _ip, _ip, _ip, C.c_longlong]),
            "orc_eam_info": (C.c_int, [C.c_void_p, _ip, _dp]),
            "orc_eam_tables": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _ip, _ip, _ip]),
            "orc_lattice": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _dp]),
            "orc_lj_lattice_scale": (C.c_double, [C.c_int, C.c_double]),
            "orc_velocity_create": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


LATTICE = {"sc": 0, "bcc": 1, "fcc": 2}


def lattice(style: str, nx: int, ny: int, nz: int, scale: float) -> np.ndarray:
    """create_atoms positions in creation (tag) order."""
    nb = {"sc": 1, "bcc": 2, "fcc": 4}[style]
    x = np.zeros((nx * ny * nz * nb, 3))
    lib().orc_lattice(LATTICE[style], nx, ny, nz, scale, _d(x))
    return x


def lj_lattice_scale(style: str, rhostar: float) -> float:
    return lib().orc_lj_lattice_scale(LATTICE[style], rhostar)


class OracleSim:
    """One serial LAMMPS-like process: box, atoms, pair style, Verlet + NVE."""

    def __init__(self, units: str = "lj", threads: int = 1):
        self._L = lib()
        self._s = self._L.orc_create(1 if units == "metal" else 0)
        self._L.orc_set_threads(self._s, threads)
        self.ntypes = 1

    def close(self):
        """Free the simulation now (it is freed on garbage collection otherwise)."""
        if self._s:
            self._L.orc_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self._L.orc_error(self._s).decode())

    # ---- settings -------------------------------------------------------
    def box(self, lo, hi):
        lo = np.ascontiguousarray(lo, dtype=np.float64)
        hi = np.ascontiguousarray(hi, dtype=np.float64)
        self._check(self._L.orc_set_box(self._s, _d(lo), _d(hi)))

    def atoms(self, x, v=None, type=None, tag=None, ntypes=1):
        x = np.ascontiguousarray(x, dtype=np.float64)
        n = x.shape[0]
        v = np.zeros_like(x) if v is None else np.ascontiguousarray(v, dtype=np.float64)
        type = np.ones(n, np.int32) if type is None else np.ascontiguousarray(type, dtype=np.int32)
        tag = np.arange(1, n + 1, dtype=np.int32) if tag is None else np.ascontiguousarray(tag, dtype=np.int32)
        self.ntypes = ntypes
        self._check(self._L.orc_set_atoms(self._s, n, ntypes, _d(x), _d(v), _i(type), _i(tag)))

    def mass(self, itype, m):
        self._L.orc_set_mass(self._s, itype, m)

    def timestep(self, dt):
        self._L.orc_set_timestep(self._s, dt)

    def neighbor(self, skin, every=1, delay=10, check=True, sortfreq=1000):
        self._L.orc_set_neighbor(self._s, skin, every, delay, int(check), sortfreq)

    def thermo(self, every):
        self._L.orc_set_thermo(self._s, every)

    def lj_cut(self, cut, shift=False):
        self._check(self._L.orc_pair_lj_cut(self._s, cut, int(shift)))

    def lj_coeff(self, i, j, eps, sigma, cut=-1.0):
        self._check(self._L.orc_pair_lj_coeff(self._s, i, j, eps, sigma, cut))

    def eam_funcfl(self, files, type2file=None):
        files = [os.fsencode(f) for f in files]
        arr = (C.c_char_p * len(files))(*files)
        t2f = np.full(8, -1, np.int32)
        if type2file is None:
            type2file = [0]
        t2f[: len(type2file)] = type2file
        self._check(self._L.orc_pair_eam_funcfl(self._s, len(files), arr, _i(t2f)))

    def eam_setfl(self, path, elements_map, fs=False):
        m = np.full(8, -1, np.int32)
        m[: len(elements_map)] = elements_map
        self._check(self._L.orc_pair_eam_setfl(self._s, os.fsencode(path), int(fs), _i(m)))

    def velocity_create(self, t, seed, gaussian=False, loop_geom=True, mom=True):
        self._check(self._L.orc_velocity_create(self._s, t, seed, int(gaussian), int(loop_geom), int(mom)))

    # ---- actions --------------------------------------------------------
    def setup(self):
        self._check(self._L.orc_setup(self._s))

    def run(self, n):
        self._check(self._L.orc_run(self._s, n))

    def compute(self, eflag=1, vflag=2):
        self._check(self._L.orc_compute(self._s, eflag, vflag))

    # ---- state ----------------------------------------------------------
    @property
    def nlocal(self):
        return self._L.orc_nlocal(self._s)

    @property
    def nghost(self):
        return self._L.orc_nghost(self._s)

    @property
    def ncalls(self):
        return self._L.orc_ncalls(self._s)

    @property
    def ndanger(self):
        return self._L.orc_ndanger(self._s)

    @property
    def neigh_total(self):
        return self._L.orc_neigh_total(self._s)

    @property
    def eng_vdwl(self):
        return self._L.orc_eng_vdwl(self._s)

    @property
    def virial(self):
        v = np.zeros(6)
        self._L.orc_virial(self._s, _d(v))
        return v

    @property
    def kinetic(self):
        return self._L.orc_kinetic(self._s)

    def _vec(self, fn, cols=3, dtype=np.float64):
        a = np.zeros((self.nlocal, cols) if cols > 1 else self.nlocal, dtype)
        fn(self._s, _d(a) if dtype == np.float64 else _i(a))
        return a

    @property
    def x(self):
        return self._vec(self._L.orc_get_x)

    @property
    def v(self):
        return self._vec(self._L.orc_get_v)

    @property
    def f(self):
        return self._vec(self._L.orc_get_f)

    @property
    def tag(self):
        return self._vec(self._L.orc_get_tag, 1, np.int32)

    @property
    def type(self):
        return self._vec(self._L.orc_get_type, 1, np.int32)

    @property
    def image(self):
        return self._vec(self._L.orc_get_image, 3, np.int32)

    def rho_fp(self):
        rho = np.zeros(self.nlocal)
        fp = np.zeros(self.nlocal)
        self._L.orc_get_rho_fp(self._s, _d(rho), _d(fp))
        return rho, fp

    def eatom_vatom(self):
        e = np.zeros(self.nlocal)
        v = np.zeros((self.nlocal, 6))
        self._L.orc_get_eatom_vatom(self._s, _d(e), _d(v))
        return e, v

    def thermo_rows(self):
        n = self._L.orc_thermo_rows(self._s, None, 0)
        out = np.zeros((max(n, 1), 5))
        self._L.orc_thermo_rows(self._s, _d(out), n)
        return out[:n]

    def half_list(self):
        """(numneigh[n], jowner[m], jimage[m]) in the oracle's index order."""
        n = self.nlocal
        num = np.zeros(n, np.int32)
        m = self._L.orc_neigh_half(self._s, _i(num), None, None, 0)
        jo = np.zeros(max(m, 1), np.int32)
        ji = np.zeros(max(m, 1), np.int32)
        self._L.orc_neigh_half(self._s, _i(num), _i(jo), _i(ji), m)
        return num, jo[:m], ji[:m]

    def eam_tables(self):
        ints = np.zeros(5, np.int32)
        dbl = np.zeros(4)
        self._check(self._L.orc_eam_info(self._s, _i(ints), _d(dbl)))
        nrho, nr, nfrho, nrhor, nz2r = (int(v) for v in ints)
        fr = np.zeros((nfrho, nrho + 1, 7))
        rr = np.zeros((nrhor, nr + 1, 7))
        zr = np.zeros((nz2r, nr + 1, 7))
        nt = self.ntypes
        t2f = np.zeros(nt, np.int32)
        t2r = np.zeros((nt, nt), np.int32)
        t2z = np.zeros((nt, nt), np.int32)
        self._check(self._L.orc_eam_tables(self._s, _d(fr), _d(rr), _d(zr), _i(t2f), _i(t2r), _i(t2z)))
        return dict(nrho=nrho, nr=nr, drho=dbl[0], dr=dbl[1], rhomax=dbl[2], cutmax=dbl[3],
                    frho_spline=fr, rhor_spline=rr, z2r_spline=zr,
                    type2frho=t2f, type2rhor=t2r, type2z2r=t2z)
