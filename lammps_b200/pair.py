"""Host-side pair-style settings: the coefficient tables the device kernels use.

These classes mirror the host halves of the reference's pair styles -- the
parts a LAMMPS ``PairLJCutB200``/``PairEAMB200`` subclass inherits unchanged
(settings, coeff, init_one, read_file, file2array, array2spline) -- so that a
Python caller can drive the engine without LAMMPS.  The arithmetic follows
the reference operation for operation, so the tables are bit-identical.
"""
from __future__ import annotations

import math

import numpy as np

MAXTYPES = 8


class PairLJCut:
    """pair_style lj/cut <cut> (src/pair_lj_cut.cpp:428-602)."""

    style = "lj/cut"

    def __init__(self, cut_global: float, ntypes: int = 1, shift: bool = False, mix: str = "geometric"):
        if not (1 <= ntypes <= MAXTYPES):
            raise ValueError(f"ntypes must be 1..{MAXTYPES}")
        self.cut_global = float(cut_global)
        self.ntypes = ntypes
        self.offset_flag = bool(shift)
        self.mix = mix
        n = ntypes + 1
        self.epsilon = np.zeros((n, n))
        self.sigma = np.zeros((n, n))
        self.cut = np.zeros((n, n))
        self.setflag = np.zeros((n, n), bool)

    def coeff(self, i: int, j: int, eps: float, sigma: float, cut: float | None = None):
        """pair_coeff i j eps sigma [cut] (src/pair_lj_cut.cpp:448-476)."""
        if i > j:
            i, j = j, i
        if not (1 <= i <= self.ntypes and 1 <= j <= self.ntypes):
            raise ValueError("Incorrect args for pair coefficients")
        self.epsilon[i, j] = eps
        self.sigma[i, j] = sigma
        self.cut[i, j] = self.cut_global if cut is None else float(cut)
        self.setflag[i, j] = True

    def _mix_energy(self, e1, e2, s1, s2):
        # Pair::mix_energy (src/pair.cpp:639-650)
        if self.mix in ("geometric", "arithmetic"):
            return math.sqrt(e1 * e2)
        return 2.0 * math.sqrt(e1 * e2) * s1 ** 3 * s2 ** 3 / (s1 ** 6 + s2 ** 6)

    def _mix_distance(self, s1, s2):
        # Pair::mix_distance (src/pair.cpp:652-664)
        if self.mix == "geometric":
            return math.sqrt(s1 * s2)
        if self.mix == "arithmetic":
            return 0.5 * (s1 + s2)
        return (0.5 * (s1 ** 6 + s2 ** 6)) ** (1.0 / 6.0)

    def tables(self):
        """PairLJCut::init_one for all i<=j, mirrored (src/pair_lj_cut.cpp:545-570);
        cutsq = cut^2 as Pair::init (src/pair.cpp:214-224).  Returns flattened
        (ntypes+1)^2 arrays."""
        n = self.ntypes
        for i in range(1, n + 1):
            if not self.setflag[i, i]:
                raise ValueError("All pair coeffs are not set")
        N = n + 1
        cutsq, lj1, lj2, lj3, lj4, off = (np.zeros((N, N)) for _ in range(6))
        for i in range(1, n + 1):
            for j in range(i, n + 1):
                if not self.setflag[i, j]:
                    self.epsilon[i, j] = self._mix_energy(self.epsilon[i, i], self.epsilon[j, j],
                                                          self.sigma[i, i], self.sigma[j, j])
                    self.sigma[i, j] = self._mix_distance(self.sigma[i, i], self.sigma[j, j])
                    self.cut[i, j] = self._mix_distance(self.cut[i, i], self.cut[j, j])
                e, s, c = self.epsilon[i, j], self.sigma[i, j], self.cut[i, j]
                lj1[i, j] = 48.0 * e * math.pow(s, 12.0)
                lj2[i, j] = 24.0 * e * math.pow(s, 6.0)
                lj3[i, j] = 4.0 * e * math.pow(s, 12.0)
                lj4[i, j] = 4.0 * e * math.pow(s, 6.0)
                if self.offset_flag:
                    ratio = s / c
                    off[i, j] = 4.0 * e * (math.pow(ratio, 12.0) - math.pow(ratio, 6.0))
                for t in (lj1, lj2, lj3, lj4, off):
                    t[j, i] = t[i, j]
                cutsq[i, j] = cutsq[j, i] = c * c
        return {k: np.ascontiguousarray(v.ravel()) for k, v in
                dict(cutsq=cutsq, lj1=lj1, lj2=lj2, lj3=lj3, lj4=lj4, offset=off).items()}

    def max_cut(self):
        return float(np.sqrt(self.tables()["cutsq"].max()))


# ---------------------------------------------------------------------------
# EAM


def _grab(tokens, n):
    out = np.array([float(next(tokens)) for _ in range(n)])
    return out


def _tokens(lines):
    for line in lines:
        for tok in line.split():
            yield tok


def read_funcfl(path):
    """DYNAMO funcfl file (PairEAM::read_file, src/MANYBODY/pair_eam.cpp:433-481)."""
    with open(path) as fh:
        lines = fh.read().splitlines()
    mass = float(lines[1].split()[1])
    h = lines[2].split()
    nrho, drho, nr, dr, cut = int(h[0]), float(h[1]), int(h[2]), float(h[3]), float(h[4])
    toks = _tokens(lines[3:])
    frho = np.zeros(nrho + 1)
    zr = np.zeros(nr + 1)
    rhor = np.zeros(nr + 1)
    frho[1:] = _grab(toks, nrho)
    zr[1:] = _grab(toks, nr)
    rhor[1:] = _grab(toks, nr)
    return dict(mass=mass, nrho=nrho, drho=drho, nr=nr, dr=dr, cut=cut, frho=frho, zr=zr, rhor=rhor)


def read_setfl(path, fs=False):
    """DYNAMO setfl (eam/alloy) or Finnis-Sinclair (eam/fs) file
    (src/MANYBODY/pair_eam_alloy.cpp:115-207, src/MANYBODY/pair_eam_fs.cpp)."""
    with open(path) as fh:
        lines = fh.read().splitlines()
    words = lines[3].split()
    ne = int(words[0])
    if len(words) != ne + 1:
        raise ValueError("Incorrect element names in EAM potential file")
    elements = words[1:]
    h = lines[4].split()
    nrho, drho, nr, dr, cut = int(h[0]), float(h[1]), int(h[2]), float(h[3]), float(h[4])
    k = 5
    mass = np.zeros(ne)
    frho = np.zeros((ne, nrho + 1))
    rhor = np.zeros((ne, ne, nr + 1)) if fs else np.zeros((ne, nr + 1))
    z2r = np.zeros((ne, ne, nr + 1))
    rest = lines[k:]
    # element header lines interleave with data; walk with a line cursor
    pos = 0

    def take(n):
        nonlocal pos
        vals = []
        while len(vals) < n:
            vals.extend(float(t) for t in rest[pos].split())
            pos += 1
        return np.array(vals[:n])

    for i in range(ne):
        mass[i] = float(rest[pos].split()[1])
        pos += 1
        frho[i, 1:] = take(nrho)
        if fs:
            for j in range(ne):
                rhor[i, j, 1:] = take(nr)
        else:
            rhor[i, 1:] = take(nr)
    for i in range(ne):
        for j in range(i + 1):
            z2r[i, j, 1:] = take(nr)
    return dict(elements=elements, mass=mass, nrho=nrho, drho=drho, nr=nr, dr=dr, cut=cut,
                frho=frho, rhor=rhor, z2r=z2r, fs=fs)


def interpolate(n, delta, f):
    """PairEAM::interpolate: 7-coefficient cubic spline per knot
    (src/MANYBODY/pair_eam.cpp:723-751); knots 1..n, row 0 unused."""
    s = np.zeros((n + 1, 7))
    s[1:, 6] = f[1:n + 1]
    s6 = s[:, 6]
    s[1, 5] = s6[2] - s6[1]
    s[2, 5] = 0.5 * (s6[3] - s6[1])
    s[n - 1, 5] = 0.5 * (s6[n] - s6[n - 2])
    s[n, 5] = s6[n] - s6[n - 1]
    m = np.arange(3, n - 1)
    s[m, 5] = ((s6[m - 2] - s6[m + 2]) + 8.0 * (s6[m + 1] - s6[m - 1])) / 12.0
    m = np.arange(1, n)
    s5 = s[:, 5]
    s[m, 4] = 3.0 * (s6[m + 1] - s6[m]) - 2.0 * s5[m] - s5[m + 1]
    s[m, 3] = s5[m] + s5[m + 1] - 2.0 * (s6[m + 1] - s6[m])
    s[n, 4] = 0.0
    s[n, 3] = 0.0
    m = np.arange(1, n + 1)
    s[m, 2] = s[m, 5] / delta
    s[m, 1] = 2.0 * s[m, 4] / delta
    s[m, 0] = 3.0 * s[m, 3] / delta
    return s


def _lagrange(tab, ntab, dtab, r):
    """4-point Lagrange interpolation of a funcfl array onto the common grid
    (PairEAM::file2array, src/MANYBODY/pair_eam.cpp:536-554)."""
    sixth = 1.0 / 6.0
    p = r / dtab + 1.0
    k = p.astype(np.int64)
    k = np.minimum(k, ntab - 2)
    k = np.maximum(k, 2)
    p = p - k
    p = np.minimum(p, 2.0)
    cof1 = -sixth * p * (p - 1.0) * (p - 2.0)
    cof2 = 0.5 * (p * p - 1.0) * (p - 2.0)
    cof3 = -0.5 * p * (p + 1.0) * (p - 2.0)
    cof4 = sixth * p * (p * p - 1.0)
    return cof1 * tab[k - 1] + cof2 * tab[k] + cof3 * tab[k + 1] + cof4 * tab[k + 2]


def _z2r_index(irow, icol):
    if irow < icol:
        irow, icol = icol, irow
    return sum(m + 1 for m in range(irow)) + icol


class PairEAM:
    """pair_style eam with funcfl files (src/MANYBODY/pair_eam.cpp).

    ``coeff(i, path)`` mirrors ``pair_coeff i i file``; ``tables()`` runs
    file2array + array2spline and returns the spline arrays."""

    style = "eam"

    def __init__(self, ntypes: int = 1):
        self.ntypes = ntypes
        self.funcfl = []          # list of (path, data)
        self.map = [-1] * (ntypes + 1)
        self.mass = [0.0] * (ntypes + 1)

    def coeff(self, itype: int, path: str):
        for k, (p, _) in enumerate(self.funcfl):
            if p == path:
                break
        else:
            self.funcfl.append((path, read_funcfl(path)))
            k = len(self.funcfl) - 1
        self.map[itype] = k
        self.mass[itype] = self.funcfl[k][1]["mass"]   # atom->set_mass (:384)

    def _file2array(self):
        nt = self.ntypes
        files = [d for _, d in self.funcfl]
        dr = drho = rmax = rhomax = 0.0
        for i, f in enumerate(files):
            if i not in self.map[1:]:
                continue
            dr = max(dr, f["dr"])
            drho = max(drho, f["drho"])
            rmax = max(rmax, (f["nr"] - 1) * f["dr"])
            rhomax = max(rhomax, (f["nrho"] - 1) * f["drho"])
        nr = int(rmax / dr + 0.5)
        nrho = int(rhomax / drho + 0.5)
        nf = len(files)
        frho = np.zeros((nf + 1, nrho + 1))
        r = (np.arange(1, nrho + 1) - 1) * drho
        for i, f in enumerate(files):
            frho[i, 1:] = _lagrange(f["frho"], f["nrho"], f["drho"], r)
        t2frho = [0] + [self.map[t] if self.map[t] >= 0 else nf for t in range(1, nt + 1)]
        rr = (np.arange(1, nr + 1) - 1) * dr
        rhor = np.zeros((nf, nr + 1))
        for i, f in enumerate(files):
            rhor[i, 1:] = _lagrange(f["rhor"], f["nr"], f["dr"], rr)
        t2rhor = np.zeros((nt + 1, nt + 1), np.int32)
        for i in range(1, nt + 1):
            for j in range(1, nt + 1):
                t2rhor[i, j] = self.map[i]
        nz2r = nf * (nf + 1) // 2
        z2r = np.zeros((nz2r, nr + 1))
        n = 0
        for i in range(nf):
            for j in range(i + 1):
                zri = _lagrange(files[i]["zr"], files[i]["nr"], files[i]["dr"], rr)
                zrj = _lagrange(files[j]["zr"], files[j]["nr"], files[j]["dr"], rr)
                z2r[n, 1:] = 27.2 * 0.529 * zri * zrj
                n += 1
        cutmax = max(f["cut"] for f in files)
        return dict(nrho=nrho, drho=drho, nr=nr, dr=dr, rhomax=rhomax, cutmax=cutmax,
                    frho=frho, rhor=rhor, z2r=z2r, type2frho=np.array(t2frho, np.int32),
                    type2rhor=t2rhor)

    def _type2z2r(self):
        nt = self.ntypes
        t = np.zeros((nt + 1, nt + 1), np.int32)
        for i in range(1, nt + 1):
            for j in range(1, nt + 1):
                a, b = self.map[i], self.map[j]
                t[i, j] = 0 if (a < 0 or b < 0) else _z2r_index(a, b)
        return t

    def tables(self):
        for t in range(1, self.ntypes + 1):
            if self.map[t] < 0:
                raise ValueError("All pair coeffs are not set")
        a = self._file2array()
        # PairEAM::array2spline (src/MANYBODY/pair_eam.cpp:698-719)
        frho_s = np.stack([interpolate(a["nrho"], a["drho"], a["frho"][i]) for i in range(a["frho"].shape[0])])
        rhor_s = np.stack([interpolate(a["nr"], a["dr"], a["rhor"][i]) for i in range(a["rhor"].shape[0])])
        z2r_s = np.stack([interpolate(a["nr"], a["dr"], a["z2r"][i]) for i in range(a["z2r"].shape[0])])
        return dict(nrho=a["nrho"], drho=a["drho"], nr=a["nr"], dr=a["dr"], rhomax=a["rhomax"],
                    cutmax=a["cutmax"], frho_spline=frho_s, rhor_spline=rhor_s, z2r_spline=z2r_s,
                    type2frho=a["type2frho"], type2rhor=np.ascontiguousarray(a["type2rhor"].ravel()),
                    type2z2r=np.ascontiguousarray(self._type2z2r().ravel()))

    def max_cut(self):
        return max(d["cut"] for _, d in self.funcfl)


class PairEAMAlloy(PairEAM):
    """pair_style eam/alloy: ``coeff(path, elements)`` mirrors
    ``pair_coeff * * file E1 E2 ...`` (src/MANYBODY/pair_eam_alloy.cpp:45-109);
    an element name of None maps the type to no element (NULL)."""

    style = "eam/alloy"
    _fs = False

    def coeff(self, path, elements):
        if len(elements) != self.ntypes:
            raise ValueError("Incorrect args for pair coefficients")
        self.setfl = read_setfl(path, fs=self._fs)
        for t, name in enumerate(elements, start=1):
            if name is None:
                self.map[t] = -1
                continue
            if name not in self.setfl["elements"]:
                raise ValueError("No matching element in EAM potential file")
            self.map[t] = self.setfl["elements"].index(name)
            self.mass[t] = float(self.setfl["mass"][self.map[t]])

    def _file2array(self):
        # PairEAMAlloy::file2array (src/MANYBODY/pair_eam_alloy.cpp:213-326) and
        # PairEAMFS::file2array (src/MANYBODY/pair_eam_fs.cpp)
        s = self.setfl
        nt, ne = self.ntypes, len(s["elements"])
        nrho, nr = s["nrho"], s["nr"]
        frho = np.zeros((ne + 1, nrho + 1))
        frho[:ne] = s["frho"]
        t2frho = [0] + [self.map[t] if self.map[t] >= 0 else ne for t in range(1, nt + 1)]
        if self._fs:
            rhor = s["rhor"].reshape(ne * ne, nr + 1).copy()
        else:
            rhor = s["rhor"].copy()
        t2rhor = np.zeros((nt + 1, nt + 1), np.int32)
        for i in range(1, nt + 1):
            for j in range(1, nt + 1):
                if self._fs:
                    t2rhor[i, j] = self.map[i] * ne + self.map[j]
                else:
                    t2rhor[i, j] = self.map[i]
        z2r = np.zeros((ne * (ne + 1) // 2, nr + 1))
        n = 0
        for i in range(ne):
            for j in range(i + 1):
                z2r[n] = s["z2r"][i, j]
                n += 1
        return dict(nrho=nrho, drho=s["drho"], nr=nr, dr=s["dr"], rhomax=(nrho - 1) * s["drho"],
                    cutmax=s["cut"], frho=frho, rhor=rhor, z2r=z2r,
                    type2frho=np.array(t2frho, np.int32), type2rhor=t2rhor)

    def max_cut(self):
        return self.setfl["cut"]


class PairEAMFS(PairEAMAlloy):
    """pair_style eam/fs (Finnis-Sinclair file: one rho(r) per element pair)."""

    style = "eam/fs"
    _fs = True
