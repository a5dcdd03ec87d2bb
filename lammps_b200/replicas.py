"""Batched replicas: many independent periodic Lennard-Jones boxes advanced
together by one engine context (b200_set_replicas).

`replica_batch` builds the seeded batch of uneven fcc boxes (atom counts
log-uniform, each box with its own reduced density and temperature);
`make_batch` loads it into a `System`, whose `setup`/`run` then advance every
replica per step with the same kernel launches, and whose `replica_thermo`
returns each replica's thermo columns.
"""
from __future__ import annotations

import numpy as np

from .inputs import lattice, lj_lattice_constant, velocity_create
from .pair import PairLJCut
from .system import System


def replica_batch(nrep: int = 256, seed: int = 20140808, nmin: int = 500, nmax: int = 8000,
                  nlo: int = 5, nhi: int = 12, rho=(0.70, 0.95), temp=(0.8, 2.0)):
    """Seeded batch of fcc LJ boxes.

    For each replica k: N_k log-uniform in [nmin, nmax], rounded to an fcc
    box of n_k^3 unit cells (4 n_k^3 atoms) with n_k = clip(round((N_k/4)^(1/3)),
    nlo, nhi); reduced density rho*_k ~ U(rho) and temperature T*_k ~ U(temp);
    velocities from `velocity all create T*_k seed_k dist gaussian mom yes
    loop geom` (src/velocity.cpp:766-787) with a per-replica seed.  Returns
    the atoms concatenated in replica order plus the per-replica tables."""
    rng = np.random.default_rng(seed)
    target = np.exp(rng.uniform(np.log(nmin), np.log(nmax), nrep))
    ncells = np.clip(np.round((target / 4.0) ** (1.0 / 3.0)), nlo, nhi).astype(int)
    rhos = rng.uniform(rho[0], rho[1], nrep)
    temps = rng.uniform(temp[0], temp[1], nrep)
    seeds = rng.integers(1, 900_000_000, nrep)
    xs, vs, lo, hi, natoms = [], [], [], [], []
    for k in range(nrep):
        a = lj_lattice_constant("fcc", rhos[k])
        n = int(ncells[k])
        x = lattice("fcc", n, n, n, a)
        v = velocity_create(x, np.ones(len(x), np.int32), np.array([0.0, 1.0]), temps[k],
                            int(seeds[k]), "lj", gaussian=True, loop="geom")
        xs.append(x)
        vs.append(v)
        lo.append(np.zeros(3))
        hi.append(np.full(3, n * a))
        natoms.append(len(x))
    return dict(x=np.concatenate(xs), v=np.concatenate(vs), natoms=np.array(natoms, np.int32),
                lo=np.array(lo), hi=np.array(hi), rho=rhos, temp=temps, ncells=ncells,
                seeds=seeds)


def shard_batch(batch: dict, rank: int, world: int) -> dict:
    """The replicas of `batch` that rank `rank` of `world` advances: a
    contiguous block of replicas, the blocks cut where the running atom count
    crosses k / world of the total, so every rank gets about the same number
    of atoms.  Replicas are independent, so the shards need no exchange.
    Returns a batch of the same form plus `replicas`, the replica indices."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of world {world}")
    nat = np.asarray(batch["natoms"], dtype=np.int64)
    cum = np.concatenate([[0], np.cumsum(nat)])
    # replica r goes to the rank whose share contains the midpoint of its atoms
    mid = (cum[:-1] + cum[1:]) / 2.0
    owner = np.minimum((mid * world / cum[-1]).astype(int), world - 1)
    idx = np.nonzero(owner == rank)[0]
    out = {"replicas": idx}
    if len(idx) == 0:
        out.update(x=np.zeros((0, 3)), v=np.zeros((0, 3)), natoms=np.zeros(0, np.int32))
        for k in ("lo", "hi"):
            out[k] = np.zeros((0, 3))
        return out
    a0, a1 = int(cum[idx[0]]), int(cum[idx[-1] + 1])
    out.update(x=batch["x"][a0:a1], v=batch["v"][a0:a1])
    for k, val in batch.items():
        if k in ("x", "v"):
            continue
        arr = np.asarray(val)
        out[k] = arr[idx] if arr.ndim >= 1 and len(arr) == len(nat) else val
    return out


def make_batch(batch: dict, precision: str = "fp64", cut: float = 2.5, skin: float = 0.3,
               every: int = 20, device: int = 0, tpa: int = 0) -> System:
    """A System advancing every replica of `batch` (lj units, eps = sigma = 1,
    rc 2.5, skin 0.3, neighbor list rebuilt every 20 steps, dt 0.005)."""
    s = System("lj", precision, device)
    s.set_replicas(batch["natoms"], batch["lo"], batch["hi"])
    p = PairLJCut(cut)
    p.coeff(1, 1, 1.0, 1.0, cut)
    s.set_pair(p)
    s.set_mass([1.0])
    s.set_neighbor(skin, every=every, delay=0, check=False)
    s.set_timestep(0.005)
    s.set_thermo(0)
    if tpa:
        s.set_launch(tpa)
    s.set_atoms(batch["x"], None, batch["v"])
    return s


def single_replica(batch: dict, k: int, precision: str = "fp64", cut: float = 2.5,
                   skin: float = 0.3, every: int = 20, device: int = 0, tpa: int = 0) -> System:
    """Replica k of `batch` as its own single-box System (same settings)."""
    a0 = int(np.sum(batch["natoms"][:k]))
    a1 = a0 + int(batch["natoms"][k])
    s = System("lj", precision, device)
    s.set_box(batch["lo"][k], batch["hi"][k])
    p = PairLJCut(cut)
    p.coeff(1, 1, 1.0, 1.0, cut)
    s.set_pair(p)
    s.set_mass([1.0])
    s.set_neighbor(skin, every=every, delay=0, check=False)
    s.set_timestep(0.005)
    s.set_thermo(0)
    if tpa:
        s.set_launch(tpa)
    s.set_atoms(batch["x"][a0:a1], None, batch["v"][a0:a1])
    return s
