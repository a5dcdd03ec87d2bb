"""Input generation on the host: lattices, units and `velocity create`.

These reproduce the reference's input commands so that the same seeded
systems can be built without LAMMPS:
  - ``lattice fcc`` + ``create_atoms`` (src/lattice.cpp:84-94,249-256,468-485;
    src/create_atoms.cpp:726-760): positions in creation (tag) order;
  - ``velocity all create T seed [dist] [mom yes] [loop geom|all]``
    (src/velocity.cpp:136-340) with the Park-Miller generator and its
    coordinate hash (src/random_park.cpp:42-130), vectorised over atoms;
  - unit constants (src/update.cpp:118-166).
"""
from __future__ import annotations

import math

import numpy as np

UNITS = {
    "lj": dict(boltz=1.0, mvv2e=1.0, ftm2v=1.0, nktv2p=1.0, dt=0.005, skin=0.3, normflag=True),
    "metal": dict(boltz=8.617343e-5, mvv2e=1.0364269e-4, ftm2v=1.0 / 1.0364269e-4,
                  nktv2p=1.6021765e6, dt=0.001, skin=2.0, normflag=False),
}

_BASIS = {
    "sc": [(0.0, 0.0, 0.0)],
    "bcc": [(0.0, 0.0, 0.0), (0.5, 0.5, 0.5)],
    "fcc": [(0.0, 0.0, 0.0), (0.5, 0.5, 0.0), (0.5, 0.0, 0.5), (0.0, 0.5, 0.5)],
}


def lj_lattice_constant(style: str, rhostar: float) -> float:
    """scale = (nbasis / (V_primitive * rho*))^(1/3) for lj units."""
    nb = len(_BASIS[style])
    return (nb / 1.0 / rhostar) ** (1.0 / 3.0)


def lattice(style: str, nx: int, ny: int, nz: int, a: float) -> np.ndarray:
    """Atom positions of an nx*ny*nz block of unit cells, loop order k, j, i,
    basis -- the order create_atoms assigns tags 1..N."""
    basis = np.array(_BASIS[style])
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    cells = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.float64)
    pts = cells[:, None, :] + basis[None, :, :]
    return (pts.reshape(-1, 3) * a).copy()


# ---- Park-Miller RNG, vectorised over independent streams -----------------
_IA, _IM, _IQ, _IR = 16807, 2147483647, 127773, 2836
_AM = 1.0 / _IM


def _uniform(seed: np.ndarray):
    k = seed // _IQ
    seed = _IA * (seed - k * _IQ) - _IR * k
    seed = np.where(seed < 0, seed + _IM, seed)
    return seed, _AM * seed


def _geom_seeds(seed: int, x: np.ndarray) -> np.ndarray:
    """RanPark::reset(seed, coord): Jenkins one-at-a-time hash over the 4
    bytes of the seed and the 24 bytes of the coordinates, read as signed
    chars; 27-bit result; then 5 warm-up draws."""
    n = x.shape[0]
    sb = np.frombuffer(np.array([seed], dtype="<i4").tobytes(), dtype=np.int8).astype(np.int64)
    xb = np.ascontiguousarray(x, dtype="<f8").view(np.int8).reshape(n, 24).astype(np.int64)
    mask = np.uint64(0xFFFFFFFF)
    h = np.zeros(n, dtype=np.uint64)

    def mix(h, b):
        h = (h + (b.astype(np.uint64) & mask)) & mask
        h = (h + (h << np.uint64(10))) & mask
        h = h ^ (h >> np.uint64(6))
        return h

    for b in sb:
        h = mix(h, np.full(n, b, dtype=np.int64))
    for c in range(24):
        h = mix(h, xb[:, c])
    h = (h + (h << np.uint64(3))) & mask
    h = h ^ (h >> np.uint64(11))
    h = (h + (h << np.uint64(15))) & mask
    s = (h & np.uint64(0x7FFFFFF)).astype(np.int64)
    s = np.where(s == 0, 1, s)
    for _ in range(5):
        s, _u = _uniform(s)
    return s


class _Streams:
    """Independent RanPark streams with the gaussian() save/second state."""

    def __init__(self, seeds):
        self.seed = seeds.astype(np.int64)
        self.save = np.zeros(seeds.shape, bool)
        self.second = np.zeros(seeds.shape)

    def uniform(self):
        self.seed, u = _uniform(self.seed)
        return u

    def gaussian(self):
        n = self.seed.shape[0]
        first = np.empty(n)
        use = self.save.copy()
        first[use] = self.second[use]
        need = ~use
        v1 = np.zeros(n)
        v2 = np.zeros(n)
        rsq = np.zeros(n)
        todo = need.copy()
        while todo.any():
            idx = np.nonzero(todo)[0]
            s, u1 = _uniform(self.seed[idx])
            s, u2 = _uniform(s)
            self.seed[idx] = s
            a = 2.0 * u1 - 1.0
            b = 2.0 * u2 - 1.0
            r = a * a + b * b
            ok = (r < 1.0) & (r != 0.0)
            v1[idx[ok]] = a[ok]
            v2[idx[ok]] = b[ok]
            rsq[idx[ok]] = r[ok]
            todo[idx[ok]] = False
        # libm log (numpy's vectorised log may differ in the last bit)
        logs = np.array([math.log(r) for r in rsq[need].tolist()])
        fac = np.sqrt(-2.0 * logs / rsq[need])
        self.second[need] = v1[need] * fac
        first[need] = v2[need] * fac
        self.save = need
        return first


def velocity_create(x, type_, mass, t_desired, seed, units="lj", gaussian=False,
                    loop="geom", mom=True, tag=None):
    """`velocity all create t seed ...` for atoms x (creation order), per-type
    mass table mass[type]; returns v[n,3]."""
    if seed <= 0:
        raise ValueError("Illegal velocity create command")
    u = UNITS[units]
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.shape[0]
    type_ = np.asarray(type_, dtype=np.int64)
    m = np.asarray(mass, dtype=np.float64)[type_]
    if loop == "geom":
        st = _Streams(_geom_seeds(seed, x))
        draw = st.gaussian if gaussian else st.uniform
        vx, vy, vz = draw(), draw(), draw()
    elif loop == "all":
        tags = np.arange(1, n + 1) if tag is None else np.asarray(tag)
        s = seed
        save, second = False, 0.0
        vals = np.empty((n, 3))

        def unif():
            nonlocal s
            k = s // _IQ
            s = _IA * (s - k * _IQ) - _IR * k
            if s < 0:
                s += _IM
            return _AM * s

        def gauss():
            nonlocal save, second
            if not save:
                while True:
                    v1 = 2.0 * unif() - 1.0
                    v2 = 2.0 * unif() - 1.0
                    r = v1 * v1 + v2 * v2
                    if r < 1.0 and r != 0.0:
                        break
                fac = math.sqrt(-2.0 * math.log(r) / r)
                second = v1 * fac
                save = True
                return v2 * fac
            save = False
            return second

        draw = gauss if gaussian else unif
        order = np.empty(n, np.int64)
        order[np.asarray(tags) - 1] = np.arange(n)
        for t in range(n):
            vals[order[t]] = (draw(), draw(), draw())
        vx, vy, vz = vals[:, 0], vals[:, 1], vals[:, 2]
    else:
        raise ValueError("loop must be 'geom' or 'all'")
    factor = 1.0 / np.sqrt(m)
    v = np.stack([vx * factor, vy * factor, vz * factor], axis=1)
    if mom:
        # Velocity::zero_momentum via Group::mass/vcm, summed in atom order
        # (np.cumsum adds strictly left to right, like the reference loops)
        masstotal = float(np.cumsum(m)[-1])
        p = np.array([float(np.cumsum(v[:, c] * m)[-1]) for c in range(3)])
        if masstotal > 0.0:
            p = p / masstotal
        v = v - p
    t = temperature(v, m, units)
    if t == 0.0:
        raise ValueError("Attempting to rescale a 0.0 temperature")
    return v * np.sqrt(t_desired / t)


def ke_sum(v, m):
    """sum over atoms of (vx^2 + vy^2 + vz^2) * m in atom order
    (ComputeTemp::compute_scalar, src/compute_temp.cpp:59-89)."""
    terms = (v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1] + v[:, 2] * v[:, 2]) * m
    return float(np.cumsum(terms)[-1])


def temperature(v, m, units="lj"):
    u = UNITS[units]
    n = v.shape[0]
    dof = 3.0 * n - 3.0
    tfactor = u["mvv2e"] / (dof * u["boltz"]) if dof > 0 else 0.0
    return ke_sum(v, m) * tfactor
