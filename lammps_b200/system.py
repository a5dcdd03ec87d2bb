"""`System`: a host-side driver of one device-resident box.

It plays the role of the reference's Verlet/Thermo plumbing around the
engine: it pushes the pair tables, masses, box and atoms through the C ABI,
runs `setup` + `run N` on the device (CUDA graph per step) and turns the
device's thermo rows into the reference's thermo columns
(ComputeTemp, ComputePE, ComputePressure, Thermo; src/compute_temp.cpp:59-89,
src/compute_pressure.cpp:177-207, src/thermo.cpp:1581-1619).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .inputs import UNITS, velocity_create
from .pair import PairEAM, PairLJCut


def _torch():
    import torch
    return torch


class System:
    def __init__(self, units: str = "lj", precision: str = "fp64", device: int = 0):
        if units not in UNITS:
            raise ValueError(f"unknown units {units}")
        self._L = _abi.load()
        self.units = units
        self.u = UNITS[units]
        self.precision = precision
        self.device = f"cuda:{device}"
        h = C.c_void_p()
        rc = self._L.b200_create(device, _abi.PREC[precision], C.byref(h))
        self._h = h
        if rc != 0:
            msg = self._L.b200_last_error(h).decode() if h.value else "b200_create failed"
            raise _abi.B200Error(rc, msg)
        self.dt = self.u["dt"]
        self.thermo_every = 0
        self.n = 0
        self.ntypes = 0
        self.mass = None
        self.pair = None
        self.box_lo = self.box_hi = None
        self.ntimestep = 0
        self.thermo_rows = []
        self._staged = []   # (n, type, arrays) of staged atom sets, oldest first
        self._pending = []  # host arrays of downloads still in flight

    def __del__(self):
        try:
            if self._h:
                self._L.b200_destroy(self._h)
                self._h = None
        except Exception:
            pass

    def close(self):
        self.__del__()

    def _ck(self, rc):
        if rc != 0:
            raise _abi.B200Error(rc, self._L.b200_last_error(self._h).decode())

    # ---- settings --------------------------------------------------------
    def set_box(self, lo, hi):
        self.box_lo = np.ascontiguousarray(lo, dtype=np.float64)
        self.box_hi = np.ascontiguousarray(hi, dtype=np.float64)
        self._ck(self._L.b200_set_box(self._h, _abi.dptr(self.box_lo), _abi.dptr(self.box_hi)))

    def set_neighbor(self, skin=None, every=1, delay=10, check=True, one=0):
        skin = self.u["skin"] if skin is None else skin
        self.skin = skin
        self.every, self.delay, self.check = int(every), int(delay), bool(check)
        self._ck(self._L.b200_set_neighbor(self._h, skin, every, delay, int(check), one))

    def set_pair(self, pair):
        self.pair = pair
        self.ntypes = pair.ntypes
        t = pair.tables()
        if isinstance(pair, PairLJCut):
            self._ck(self._L.b200_set_lj(self._h, pair.ntypes, *(_abi.dptr(t[k]) for k in
                                                                ("cutsq", "lj1", "lj2", "lj3", "lj4", "offset"))))
        elif isinstance(pair, PairEAM):
            fr = np.ascontiguousarray(t["frho_spline"])
            rr = np.ascontiguousarray(t["rhor_spline"])
            zr = np.ascontiguousarray(t["z2r_spline"])
            self._keep = (fr, rr, zr)
            self._ck(self._L.b200_set_eam(
                self._h, pair.ntypes, t["nrho"], t["drho"], t["nr"], t["dr"], t["rhomax"], t["cutmax"],
                fr.shape[0], _abi.dptr(fr), rr.shape[0], _abi.dptr(rr), zr.shape[0], _abi.dptr(zr),
                _abi.iptr(np.ascontiguousarray(t["type2frho"], dtype=np.int32)),
                _abi.iptr(np.ascontiguousarray(t["type2rhor"], dtype=np.int32)),
                _abi.iptr(np.ascontiguousarray(t["type2z2r"], dtype=np.int32))))
            if self.mass is None:
                self.set_mass([m if m > 0 else 1.0 for m in pair.mass[1:]])
        else:
            raise TypeError("unsupported pair style")
        self.tables = t

    def set_mass(self, masses):
        """masses for types 1..ntypes."""
        m = np.zeros(len(masses) + 1)
        m[1:] = masses
        self.mass = m
        self._ck(self._L.b200_set_mass(self._h, len(masses), _abi.dptr(m)))

    def set_timestep(self, dt):
        self.dt = dt

    def set_thermo(self, every):
        self.thermo_every = every

    def set_launch(self, threads_per_atom=0, block=128):
        self._ck(self._L.b200_set_launch(self._h, threads_per_atom, block))

    def launch(self):
        t, b = C.c_int(), C.c_int()
        self._ck(self._L.b200_get_launch(self._h, C.byref(t), C.byref(b)))
        return t.value, b.value

    # ---- atoms -----------------------------------------------------------
    def set_atoms(self, x, type_=None, v=None):
        x = np.ascontiguousarray(x, dtype=np.float64)
        self.n = x.shape[0]
        t = np.ones(self.n, np.int32) if type_ is None else np.ascontiguousarray(type_, dtype=np.int32)
        vv = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
        self.type = t
        self._ck(self._L.b200_upload_atoms(self._h, self.n, _abi.dptr(x), _abi.dptr(vv),
                                           _abi.iptr(t), None))

    def create_velocity(self, x, t, seed, gaussian=False, loop="geom", mom=True, type_=None):
        type_ = np.ones(x.shape[0], np.int32) if type_ is None else type_
        return velocity_create(x, type_, self.mass, t, seed, self.units, gaussian, loop, mom)

    def download(self, out=None):
        """Positions, velocities, forces and image flags in the upload order.

        `out` (optional) is a dict of caller-owned arrays to fill instead of
        new ones: x, v, f as C-contiguous (n, 3) float64 and image as (n, 3)
        int32 -- e.g. page-locked host buffers, which the device copies into
        directly."""
        n = self.n
        if out is None:
            out = dict(x=np.zeros((n, 3)), v=np.zeros((n, 3)), f=np.zeros((n, 3)),
                       image=np.zeros((n, 3), np.int32))
        else:
            for k, dt in (("x", np.float64), ("v", np.float64), ("f", np.float64),
                          ("image", np.int32)):
                a = out[k]
                if a.shape != (n, 3) or a.dtype != dt or not a.flags["C_CONTIGUOUS"]:
                    raise ValueError(f"download: out[{k!r}] must be a C-contiguous ({n}, 3) {np.dtype(dt)}")
        self._ck(self._L.b200_download_atoms(self._h, _abi.dptr(out["x"]), _abi.dptr(out["v"]),
                                             _abi.dptr(out["f"]), _abi.iptr(out["image"])))
        return out

    # ---- overlapped transfers: one atom set after another -------------------
    def stage_atoms(self, x, type_=None, v=None):
        """Start copying an atom set to the device (b200_stage_atoms); it
        becomes the context's atoms at set_staged_atoms.  The arrays are held,
        and must not change, until then.  Page-locked arrays (e.g. the numpy
        view of a pinned torch tensor) let the copy run beside the steps of
        the current set."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        n = x.shape[0]
        t = np.ones(n, np.int32) if type_ is None else np.ascontiguousarray(type_, dtype=np.int32)
        vv = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
        self._ck(self._L.b200_stage_atoms(self._h, n, _abi.dptr(x), _abi.dptr(vv), _abi.iptr(t)))
        self._staged.append((n, t, (x, vv)))

    def set_staged_atoms(self):
        """The oldest staged set becomes the context's atoms (as set_atoms)."""
        if not self._staged:
            raise _abi.B200Error(_abi.B200_ERR_STATE, "no staged atom set")
        n, t, _ = self._staged.pop(0)
        self._ck(self._L.b200_set_staged_atoms(self._h))
        self.n = n
        self.type = t

    def download_async(self, out):
        """download() into the caller's arrays `out` without waiting: the
        arrays are filled while later work runs and are valid after
        wait_transfers()."""
        n = self.n
        for k, dt in (("x", np.float64), ("v", np.float64), ("f", np.float64),
                      ("image", np.int32)):
            a = out.get(k)
            if a is not None and (a.shape != (n, 3) or a.dtype != dt or
                                  not a.flags["C_CONTIGUOUS"]):
                raise ValueError(f"download_async: out[{k!r}] must be a C-contiguous ({n}, 3) "
                                 f"{np.dtype(dt)}")
        self._ck(self._L.b200_download_atoms_async(
            self._h, _abi.dptr(out.get("x")), _abi.dptr(out.get("v")), _abi.dptr(out.get("f")),
            _abi.iptr(out.get("image"))))
        self._pending.append(out)
        return out

    def wait_transfers(self):
        """Wait for every copy of stage_atoms and download_async."""
        self._ck(self._L.b200_wait_transfers(self._h))
        self._pending = []

    def gather(self, fields=("x", "v", "f", "image"), idx=None):
        """Per-atom columns straight from the device, as a dump writes them:
        {group: (m, 3) array} for the requested groups of atoms idx (caller
        indices; all atoms when None).  Image flags count box crossings since
        the upload."""
        order = [k for k in ("x", "v", "f", "image") if k in fields]
        if not order or len(order) != len(set(fields)):
            raise ValueError(f"gather: fields from x, v, f, image, not {fields}")
        bits = sum(_abi.FIELDS[k] for k in order)
        if idx is None:
            m, ip = self.n, None
        else:
            ii = np.ascontiguousarray(idx, dtype=np.int32)
            m, ip = len(ii), _abi.iptr(ii)
        out = np.zeros((m, 3 * len(order)))
        self._ck(self._L.b200_gather(self._h, bits, m, ip, _abi.dptr(out)))
        res = {k: out[:, 3 * c:3 * c + 3] for c, k in enumerate(order)}
        if "image" in res:
            res["image"] = res["image"].astype(np.int32)
        return res

    def update_positions(self, x):
        """New positions (caller order) keeping the cells and the neighbor
        list of the last build (a Pair::compute between reneighborings)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.shape != (self.n, 3):
            raise ValueError(f"update_positions: need ({self.n}, 3) positions")
        self._ck(self._L.b200_update_positions(self._h, _abi.dptr(x)))

    def cutforce(self):
        """Largest force cutoff of the pair style (Pair::cutforce)."""
        if isinstance(self.pair, PairEAM):
            return float(self.tables["cutmax"])
        return float(np.sqrt(np.max(self.tables["cutsq"])))

    # ---- spatial decomposition (lammps_b200.brick) -----------------------
    def set_ghosts(self, ghost):
        """Mark ghost atoms (caller order; None clears): not integrated, not
        distance-checked, positions set by halo_unpack.  A numpy array or an
        int32 torch tensor (host or device)."""
        if ghost is None:
            self._ck(self._L.b200_set_ghosts(self._h, None))
            return
        if hasattr(ghost, "data_ptr"):
            g = ghost.contiguous()
            if g.dtype.itemsize != 4 or tuple(g.shape) != (self.n,):
                raise ValueError(f"set_ghosts: need {self.n} int32 flags")
            if g.is_cuda:
                self._torch_ready()
            self._ck(self._L.b200_set_ghosts(self._h, _abi.tiptr(g)))
            return
        g = np.ascontiguousarray(ghost, dtype=np.int32)
        if g.shape != (self.n,):
            raise ValueError(f"set_ghosts: need {self.n} flags")
        self._ck(self._L.b200_set_ghosts(self._h, _abi.iptr(g)))

    # device-tensor forms of set_atoms / download / compute (torch tensors on
    # this context's device; no host copy)
    def _torch_ready(self):
        """Wait for the work queued on torch's current stream of this device.

        The engine runs on its own non-blocking stream, which does not wait
        for torch's stream: a tensor that torch kernels are still producing
        (an input), or a block that torch's caching allocator has just handed
        out while kernels queued earlier on torch's stream may still use it
        (an output), must be settled before the engine touches it.  Every
        engine call returns after its own stream has finished, so outputs are
        complete when the call returns."""
        _torch().cuda.current_stream(self.device).synchronize()

    def set_atoms_dev(self, x, type_, v=None):
        """x (n, 3) float64, type_ (n,) int32, v (n, 3) float64 or None."""
        x = x.contiguous()
        t = type_.contiguous()
        vv = None if v is None else v.contiguous()
        n = int(x.shape[0])
        if x.dtype != _torch().float64 or t.dtype != _torch().int32 or tuple(t.shape) != (n,):
            raise ValueError("set_atoms_dev: x float64 (n, 3), type int32 (n,)")
        self.n = n
        self.type = None
        self._torch_ready()
        self._ck(self._L.b200_upload_atoms(self._h, n, _abi.tdptr(x), _abi.tdptr(vv),
                                           _abi.tiptr(t), None))

    def download_dev(self, f=False):
        torch = _torch()
        n, dev = self.n, self.device
        out = dict(x=torch.empty((n, 3), dtype=torch.float64, device=dev),
                   v=torch.empty((n, 3), dtype=torch.float64, device=dev),
                   image=torch.empty((n, 3), dtype=torch.int32, device=dev))
        if f:
            out["f"] = torch.empty((n, 3), dtype=torch.float64, device=dev)
        self._torch_ready()
        self._ck(self._L.b200_download_atoms(self._h, _abi.tdptr(out["x"]), _abi.tdptr(out["v"]),
                                             _abi.tdptr(out.get("f")), _abi.tiptr(out["image"])))
        return out

    def compute_dev(self):
        """Forces with per-atom energy (n,) and virial (n, 6) as device tensors."""
        torch = _torch()
        ea = torch.empty(self.n, dtype=torch.float64, device=self.device)
        va = torch.empty((self.n, 6), dtype=torch.float64, device=self.device)
        self._torch_ready()
        self._ck(self._L.b200_pair_compute(self._h, 2, 4, None, None, _abi.tdptr(ea),
                                           _abi.tdptr(va)))
        return dict(eatom=ea, vatom=va)

    # split EAM compute around the forward communication of F'(rho)
    def eam_density(self, eflag=0, vflag=0):
        """Passes 1-2 of PairEAM::compute: rho, F'(rho), embedding energy."""
        self._ck(self._L.b200_eam_density(self._h, eflag, vflag))

    @staticmethod
    def _fp_args(idx, buf):
        if not (idx.is_cuda and buf.is_cuda and idx.dtype.itemsize == 4 and buf.is_contiguous()
                and idx.is_contiguous() and buf.numel() == idx.numel()):
            raise ValueError("F' halo: idx (m int32) and buf (m float64) must be contiguous CUDA tensors")
        return idx.numel(), C.c_void_p(idx.data_ptr()), C.c_void_p(buf.data_ptr())

    def eam_fp_pack(self, idx, buf):
        """buf[i] = F' of atom idx[i] (device tensors)."""
        m, pi, pb = self._fp_args(idx, buf)
        self._torch_ready()
        self._ck(self._L.b200_eam_fp_pack(self._h, m, pi, pb))

    def eam_fp_unpack(self, idx, buf):
        """F' of ghost atom idx[i] = buf[i] (device tensors)."""
        m, pi, pb = self._fp_args(idx, buf)
        self._torch_ready()
        self._ck(self._L.b200_eam_fp_unpack(self._h, m, pi, pb))

    def eam_force(self, eflag=0, vflag=0):
        """Pass 3 of PairEAM::compute after eam_density with the same flags."""
        eng = C.c_double(0.0)
        vir = np.zeros(6)
        self._ck(self._L.b200_eam_force(self._h, eflag, vflag, C.byref(eng), _abi.dptr(vir), None,
                                        None))
        return dict(eng=eng.value, virial=vir)

    def eam_force_dev(self):
        """Pass 3 with per-atom energy (n,) and virial (n, 6) as device
        tensors; the density call must have had eflag 2, vflag 4."""
        torch = _torch()
        ea = torch.empty(self.n, dtype=torch.float64, device=self.device)
        va = torch.empty((self.n, 6), dtype=torch.float64, device=self.device)
        self._torch_ready()
        self._ck(self._L.b200_eam_force(self._h, 2, 4, None, None, _abi.tdptr(ea), _abi.tdptr(va)))
        return dict(eatom=ea, vatom=va)

    def neigh_check(self):
        """The local half of Neighbor::check_distance since the last call."""
        m = C.c_int(0)
        self._ck(self._L.b200_neigh_check(self._h, C.byref(m)))
        return bool(m.value)

    def nve_initial(self):
        self._ck(self._L.b200_nve_initial(self._h, self.dt, 0.5 * self.dt * self.u["ftm2v"]))

    def nve_final(self):
        self._ck(self._L.b200_nve_final(self._h, 0.5 * self.dt * self.u["ftm2v"]))

    @staticmethod
    def _dev_args(idx, buf):
        if not (idx.is_cuda and buf.is_cuda and idx.dtype.itemsize == 4 and buf.is_contiguous()
                and idx.is_contiguous() and buf.numel() == 3 * idx.numel()):
            raise ValueError("halo: idx (m int32) and buf (3m float64) must be contiguous CUDA tensors")
        return idx.numel(), C.c_void_p(idx.data_ptr()), C.c_void_p(buf.data_ptr())

    def halo_pack(self, idx, buf):
        """buf[i] = x of atom idx[i] (device tensors)."""
        m, pi, pb = self._dev_args(idx, buf)
        self._torch_ready()
        self._ck(self._L.b200_halo_pack(self._h, m, pi, pb))

    def halo_unpack(self, idx, buf):
        """x of atom idx[i] = buf[i] (device tensors)."""
        m, pi, pb = self._dev_args(idx, buf)
        self._torch_ready()
        self._ck(self._L.b200_halo_unpack(self._h, m, pi, pb))

    # ---- actions ---------------------------------------------------------
    def neigh_build(self):
        self._ck(self._L.b200_neigh_build(self._h))

    def compute(self, eflag=1, vflag=1, per_atom=False):
        """Pair::compute on the current atoms (lists must be built)."""
        eng = C.c_double(0.0)
        vir = np.zeros(6)
        n = self.n
        ea = np.zeros(n) if per_atom else None
        va = np.zeros((n, 6)) if per_atom else None
        ef = eflag | (2 if per_atom else 0)
        vf = vflag | (4 if per_atom else 0)
        self._ck(self._L.b200_pair_compute(self._h, ef, vf, C.byref(eng), _abi.dptr(vir),
                                           _abi.dptr(ea), _abi.dptr(va)))
        out = dict(eng=eng.value, virial=vir)
        if per_atom:
            out.update(eatom=ea, vatom=va)
        return out

    def _row_to_thermo(self, row):
        return self._thermo(row, self.n, float(np.prod(self.box_hi - self.box_lo)))

    def _thermo(self, row, n, vol):
        u = self.u
        dof = 3.0 * n - 3.0
        tfactor = u["mvv2e"] / (dof * u["boltz"]) if dof > 0 else 0.0
        temp = row[1] * tfactor
        pe = row[2]
        epair = pe / n if u["normflag"] else pe
        ke = temp * 0.5 * dof * u["boltz"]
        if u["normflag"]:
            ke /= n
        press = (dof * u["boltz"] * temp + row[3] + row[4] + row[5]) / 3.0 * (1.0 / vol) * u["nktv2p"]
        return dict(Step=int(round(row[0])), Temp=temp, E_pair=epair, E_mol=0.0,
                    TotEng=epair + ke, Press=press, eng=pe, virial=np.array(row[3:9]), ke2=row[1])

    def setup(self):
        row = np.zeros(9)
        self._ck(self._L.b200_setup(self._h, _abi.dptr(row)))
        row[0] = self.ntimestep
        r = self._row_to_thermo(row)
        self.thermo_rows = [r]
        return r

    def run(self, nsteps):
        ftm2v = self.u["ftm2v"]
        nout = 1 + (nsteps // self.thermo_every if self.thermo_every > 0 else 0)
        rows = np.zeros((nout, 9))
        nr = C.c_int(0)
        self._ck(self._L.b200_run(self._h, nsteps, self.dt, ftm2v, self.thermo_every,
                                  _abi.dptr(rows), nout, C.byref(nr)))
        self.ntimestep += nsteps
        out = [self._row_to_thermo(rows[k]) for k in range(min(nr.value, nout))]
        self.thermo_rows.extend(out)
        return out

    # ---- diagnostics -----------------------------------------------------
    def neigh_stats(self):
        tot = C.c_longlong()
        nc, nd, mx, cap = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        self._ck(self._L.b200_neigh_stats(self._h, C.byref(tot), C.byref(nc), C.byref(nd),
                                          C.byref(mx), C.byref(cap)))
        return dict(full_total=tot.value, ncalls=nc.value, ndanger=nd.value, maxneigh=mx.value,
                    capacity=cap.value)

    def half_list(self):
        n = self.n
        num = np.zeros(n, np.int32)
        tot = C.c_longlong()
        self._ck(self._L.b200_neigh_half(self._h, _abi.iptr(num), None, None, 0, C.byref(tot)))
        m = tot.value
        jo = np.zeros(max(m, 1), np.int32)
        ji = np.zeros(max(m, 1), np.int32)
        self._ck(self._L.b200_neigh_half(self._h, _abi.iptr(num), _abi.iptr(jo), _abi.iptr(ji), m,
                                         C.byref(tot)))
        return num, jo[:m], ji[:m]

    def rho_fp(self):
        rho = np.zeros(self.n)
        fp = np.zeros(self.n)
        self._ck(self._L.b200_get_rho_fp(self._h, _abi.dptr(rho), _abi.dptr(fp)))
        return rho, fp

    PHASES = ("initial", "neigh", "pair1", "pair2", "final")

    def set_graphs(self, on=True):
        self._ck(self._L.b200_set_graphs(self._h, int(on)))

    def set_timing(self, on=True):
        """True (1): phase events inside every step's pieces; 2: events around
        whole pieces with the run's own step form kept."""
        self._ck(self._L.b200_set_timing(self._h, int(on)))

    def timing(self, reset=False):
        ms = np.zeros(5)
        steps = C.c_longlong()
        self._ck(self._L.b200_get_timing(self._h, _abi.dptr(ms), C.byref(steps), int(reset)))
        return dict(zip(self.PHASES, ms.tolist()), steps=steps.value)

    def step_times(self, reset=True):
        """Device milliseconds of every step timed since the last reset."""
        cnt = C.c_int()
        self._ck(self._L.b200_get_step_times(self._h, None, 0, C.byref(cnt), 0))
        ms = np.zeros(max(cnt.value, 1))
        self._ck(self._L.b200_get_step_times(self._h, _abi.dptr(ms), cnt.value, C.byref(cnt),
                                             int(reset)))
        return ms[:cnt.value]

    # ---- replicas --------------------------------------------------------
    def set_replicas(self, natoms, lo, hi):
        """Independent periodic boxes advanced together: replica r has
        natoms[r] atoms in [lo[r], hi[r]); the next set_atoms takes their
        atoms concatenated in replica order (replaces set_box)."""
        natoms = np.ascontiguousarray(natoms, dtype=np.int32)
        lo = np.ascontiguousarray(lo, dtype=np.float64).reshape(-1, 3)
        hi = np.ascontiguousarray(hi, dtype=np.float64).reshape(-1, 3)
        self._ck(self._L.b200_set_replicas(self._h, len(natoms), _abi.iptr(natoms),
                                           _abi.dptr(lo), _abi.dptr(hi)))
        self.rep_natoms = natoms
        self.rep_lo, self.rep_hi = lo, hi
        self.box_lo, self.box_hi = lo[0], hi[0]

    def set_replica_step(self, mode=0, cluster=0, block=0, tpa=0):
        """Step form of the replica batch: 0 chosen by timing on the next
        setup, 1 a graph of kernels per step, 2 one cluster launch per step
        (cluster 1/2/4, block 256/512, tpa 1/2/4; 0 = tuned)."""
        self._ck(self._L.b200_set_replica_step(self._h, mode, cluster, block, tpa))

    def replica_step(self):
        """The step form in use and the per-step times the tuning measured."""
        one, cs, bl, tp = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        ms = np.zeros(2)
        self._ck(self._L.b200_get_replica_step(self._h, C.byref(one), C.byref(cs), C.byref(bl),
                                               C.byref(tp), _abi.dptr(ms)))
        return dict(onelaunch=bool(one.value), cluster=cs.value, block=bl.value, tpa=tp.value,
                    graph_ms=float(ms[0]), onelaunch_ms=float(ms[1]))

    def replica_thermo(self):
        """Per-replica thermo (Temp, E_pair, TotEng, Press as thermo_style
        one, normalised per atom in lj units) of the current state."""
        R = len(self.rep_natoms)
        rows = np.zeros((R, 9))
        self._ck(self._L.b200_replica_thermo(self._h, _abi.dptr(rows)))
        out = []
        for r in range(R):
            row = rows[r].copy()
            n = int(round(row[0]))
            row[0] = self.ntimestep
            t = self._thermo(row, n, float(np.prod(self.rep_hi[r] - self.rep_lo[r])))
            t["natoms"] = n
            out.append(t)
        return out

    @property
    def kernel_launches(self):
        return self._L.b200_kernel_launches(self._h)

    @property
    def stream(self):
        return self._L.b200_stream(self._h)
