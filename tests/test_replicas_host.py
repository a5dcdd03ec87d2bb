"""The seeded replica batch (no GPU)."""
import numpy as np

from lammps_b200.inputs import lj_lattice_constant
from lammps_b200.replicas import replica_batch


def test_batch_shapes_and_ranges():
    b = replica_batch(nrep=64, seed=7)
    n = b["ncells"]
    assert np.all((n >= 5) & (n <= 12))
    assert np.array_equal(b["natoms"], 4 * n ** 3)
    assert b["x"].shape == (int(b["natoms"].sum()), 3) and b["v"].shape == b["x"].shape
    assert np.all((b["rho"] >= 0.70) & (b["rho"] <= 0.95))
    assert np.all((b["temp"] >= 0.8) & (b["temp"] <= 2.0))
    for k in range(64):
        a = lj_lattice_constant("fcc", b["rho"][k])
        assert np.allclose(b["hi"][k], n[k] * a)
    # atoms of every replica inside its own box
    a0 = np.concatenate([[0], np.cumsum(b["natoms"])])
    for k in range(64):
        xk = b["x"][a0[k]:a0[k + 1]]
        assert np.all(xk >= b["lo"][k]) and np.all(xk < b["hi"][k])


def test_batch_is_seeded_and_uneven():
    a = replica_batch(nrep=32, seed=3)
    b = replica_batch(nrep=32, seed=3)
    assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["v"], b["v"])
    assert len(set(a["natoms"].tolist())) > 3


def test_velocities_have_zero_momentum_per_replica():
    b = replica_batch(nrep=8, seed=11)
    a0 = np.concatenate([[0], np.cumsum(b["natoms"])])
    for k in range(8):
        p = b["v"][a0[k]:a0[k + 1]].sum(axis=0)
        assert np.all(np.abs(p) < 1e-9)
