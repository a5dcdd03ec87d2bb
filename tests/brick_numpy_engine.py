"""A CPU stand-in for the engine's per-call entry points (lj/cut, one atom
type), for testing the decomposition driver (`lammps_b200.brick`) without a
GPU.  Test infrastructure only.

It keeps the properties the brick driver (lammps_b200.brick) relies on: atoms addressed in upload
order, lists built at rebuilds with the periodic image of each pair fixed
until the next build, each atom's forces summed over its neighbors in
ascending caller index, ghosts neither integrated nor distance-checked, and
the halo pack / unpack of positions by caller index.
"""
import numpy as np
import torch

from lammps_b200.inputs import UNITS
from lammps_b200.system import System


class NumpyLJ:
    device = "cpu"
    pair = None

    def __init__(self, lo, hi, eps=1.0, sigma=1.0, rc=2.5, mass=1.0, skin=0.3, every=1, delay=0,
                 check=True, dt=0.005, units="lj"):
        self.box_lo = np.asarray(lo, dtype=np.float64)
        self.box_hi = np.asarray(hi, dtype=np.float64)
        self.prd = self.box_hi - self.box_lo
        self.skin, self.every, self.delay, self.check = skin, every, delay, check
        self.mass = np.array([0.0, mass])
        self.dt = dt
        self.u = UNITS[units]
        self.rc = rc
        s6 = sigma ** 6
        self.lj1, self.lj2 = 48.0 * eps * s6 * s6, 24.0 * eps * s6
        self.lj3, self.lj4 = 4.0 * eps * s6 * s6, 4.0 * eps * s6
        self.moved = False

    def cutforce(self):
        return self.rc

    def _thermo(self, row, n, vol):
        return System._thermo(self, row, n, vol)

    def set_atoms(self, x, type_, v):
        self.x = np.array(x, dtype=np.float64)
        self.v = np.array(v, dtype=np.float64)
        self.type = np.array(type_)
        self.f = np.zeros_like(self.x)
        self.ghost = np.zeros(len(self.x), dtype=bool)

    def set_ghosts(self, g):
        if g is not None and hasattr(g, "numpy"):
            g = g.numpy()
        self.ghost = np.zeros(len(self.x), dtype=bool) if g is None else np.asarray(g) != 0

    def set_atoms_dev(self, x, type_, v=None):
        self.set_atoms(x.numpy(), type_.numpy(), np.zeros(tuple(x.shape)) if v is None else v.numpy())

    def download_dev(self):
        return {k: torch.from_numpy(a) for k, a in self.download().items() if k != "f"}

    def compute_dev(self):
        o = self.compute(1, 1, per_atom=True)
        return dict(eatom=torch.from_numpy(o["eatom"]), vatom=torch.from_numpy(o["vatom"]))

    def neigh_build(self):
        self.xhold = self.x.copy()
        d = self.x[:, None, :] - self.x[None, :, :]
        s = np.round(d / self.prd)
        dd = d - s * self.prd
        rsq = np.sum(dd * dd, axis=2)
        cn = (self.rc + self.skin) ** 2
        n = len(self.x)
        mask = (rsq <= cn) & ~np.eye(n, dtype=bool)
        k = max(1, int(mask.sum(axis=1).max()))
        self.J = np.zeros((n, k), np.int64)
        self.S = np.zeros((n, k, 3))
        self.ok = np.zeros((n, k), dtype=bool)
        for i in range(n):
            js = np.nonzero(mask[i])[0]
            self.J[i, :len(js)] = js
            self.S[i, :len(js)] = s[i, js]
            self.ok[i, :len(js)] = True

    def compute(self, eflag=1, vflag=1, per_atom=False):
        n = len(self.x)
        f = np.zeros((n, 3))
        e = np.zeros(n)
        w = np.zeros((n, 6))
        cutsq = self.rc * self.rc
        for k in range(self.J.shape[1]):
            j = self.J[:, k]
            dl = self.x - (self.x[j] + self.S[:, k] * self.prd)
            rsq = np.sum(dl * dl, axis=1)
            m = self.ok[:, k] & (rsq < cutsq)
            r2inv = 1.0 / np.where(m, rsq, 1.0)
            r6inv = r2inv * r2inv * r2inv
            fpair = np.where(m, r6inv * (self.lj1 * r6inv - self.lj2) * r2inv, 0.0)
            f += fpair[:, None] * dl
            e += np.where(m, 0.5 * r6inv * (self.lj3 * r6inv - self.lj4), 0.0)
            for c, (a, b) in enumerate(((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))):
                w[:, c] += 0.5 * dl[:, a] * dl[:, b] * fpair
        self.f = f
        out = dict(eng=float(e.sum()), virial=w.sum(axis=0))
        if per_atom:
            out.update(eatom=e, vatom=w)
        return out

    def nve_initial(self):
        own = ~self.ghost
        dtv, dtf = self.dt, 0.5 * self.dt * self.u["ftm2v"]
        dtfm = dtf / self.mass[self.type[own]]
        self.v[own] = self.v[own] + dtfm[:, None] * self.f[own]
        self.x[own] = self.x[own] + dtv * self.v[own]
        if self.check:
            dl = self.x[own] - self.xhold[own]
            self.moved |= bool(np.any(np.sum(dl * dl, axis=1) > 0.25 * self.skin * self.skin))

    def neigh_check(self):
        m, self.moved = self.moved, False
        return m

    def nve_final(self):
        own = ~self.ghost
        dtf = 0.5 * self.dt * self.u["ftm2v"]
        dtfm = dtf / self.mass[self.type[own]]
        self.v[own] = self.v[own] + dtfm[:, None] * self.f[own]

    def download(self):
        return dict(x=self.x.copy(), v=self.v.copy(), f=self.f.copy(),
                    image=np.zeros(self.x.shape, np.int32))

    def halo_pack(self, idx, buf):
        buf.copy_(torch.from_numpy(self.x[idx.numpy()]))

    def halo_unpack(self, idx, buf):
        self.x[idx.numpy()] = buf.numpy()


class NumpyEAM(NumpyLJ):
    """EAM stand-in with the split compute of the engine (density pass, F'
    pack/unpack by caller index, force pass): one element with analytic
    rho(r) = exp(-2 (r - r0)) s(r), F(rho) = -sqrt(rho), phi(r) = exp(-3 (r - r0)) s(r),
    s(r) = (1 - (r/rc)^2)^2 inside rc.  A ghost's own density is incomplete;
    its F' must come from its owner through eam_fp_unpack."""

    def __init__(self, lo, hi, rc=3.0, r0=1.2, mass=1.0, skin=0.3, every=1, delay=0, check=True,
                 dt=0.002, units="lj"):
        super().__init__(lo, hi, rc=rc, mass=mass, skin=skin, every=every, delay=delay,
                         check=check, dt=dt, units=units)
        from lammps_b200.pair import PairEAM
        self.pair = PairEAM(1)  # marks the engine as EAM for the brick driver
        self.r0 = r0
        self.fp = None
        self.emb = None

    def _terms(self, rsq):
        r = np.sqrt(rsq)
        q = 1.0 - rsq / (self.rc * self.rc)
        s, ds = q * q, -4.0 * q * r / (self.rc * self.rc)
        a, b = np.exp(-2.0 * (r - self.r0)), np.exp(-3.0 * (r - self.r0))
        return r, a * s, (-2.0 * a * s + a * ds), b * s, (-3.0 * b * s + b * ds)

    def _pairs(self):
        cutsq = self.rc * self.rc
        for k in range(self.J.shape[1]):
            j = self.J[:, k]
            dl = self.x - (self.x[j] + self.S[:, k] * self.prd)
            rsq = np.sum(dl * dl, axis=1)
            m = self.ok[:, k] & (rsq < cutsq)
            yield j, dl, np.where(m, rsq, 1.0), m

    def eam_density(self, eflag=0, vflag=0):
        rho = np.zeros(len(self.x))
        for j, dl, rsq, m in self._pairs():
            _, rh, _, _, _ = self._terms(rsq)
            rho += np.where(m, rh, 0.0)
        self.fp = -0.5 / np.sqrt(np.maximum(rho, 1e-300))
        self.emb = -np.sqrt(rho)

    def eam_fp_pack(self, idx, buf):
        buf.copy_(torch.from_numpy(self.fp[idx.numpy()]))

    def eam_fp_unpack(self, idx, buf):
        ii = idx.numpy()
        assert np.all(self.ghost[ii]), "F' unpack into an owned atom"
        self.fp[ii] = buf.numpy()

    def _force(self):
        n = len(self.x)
        f = np.zeros((n, 3))
        e = self.emb.copy()
        w = np.zeros((n, 6))
        for j, dl, rsq, m in self._pairs():
            r, _, drh, ph, dph = self._terms(rsq)
            fpair = np.where(m, -((self.fp + self.fp[j]) * drh + dph) / r, 0.0)
            f += fpair[:, None] * dl
            e += np.where(m, 0.5 * ph, 0.0)
            for c, (a, b) in enumerate(((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))):
                w[:, c] += 0.5 * dl[:, a] * dl[:, b] * fpair
        self.f = f
        return dict(eng=float(e.sum()), virial=w.sum(axis=0), eatom=e, vatom=w)

    def eam_force(self, eflag=0, vflag=0):
        o = self._force()
        return dict(eng=o["eng"], virial=o["virial"])

    def eam_force_dev(self):
        o = self._force()
        return dict(eatom=torch.from_numpy(o["eatom"]), vatom=torch.from_numpy(o["vatom"]))

    def compute(self, eflag=1, vflag=1, per_atom=False):
        self.eam_density()
        o = self._force()
        out = dict(eng=o["eng"], virial=o["virial"])
        if per_atom:
            out.update(eatom=o["eatom"], vatom=o["vatom"])
        return out
