"""Batched replicas (b200_set_replicas) against the same replicas run one
box at a time, and the batched mixed form against the batched FP64 form."""
import numpy as np
import pytest

from lammps_b200.replicas import make_batch, replica_batch, single_replica

pytestmark = pytest.mark.gpu

NREP = 6
STEPS = 45  # crosses two rebuilds (every 20)


@pytest.fixture(scope="module")
def batch():
    return replica_batch(nrep=NREP, seed=12345)


def test_batch_matches_single_boxes(batch):
    s = make_batch(batch, "fp64", tpa=1)
    s.setup()
    t0 = s.replica_thermo()
    s.run(STEPS)
    t1 = s.replica_thermo()
    st = s.download()
    s.close()
    a0 = np.concatenate([[0], np.cumsum(batch["natoms"])])
    for k in range(NREP):
        q = single_replica(batch, k, "fp64", tpa=1)
        r0 = q.setup()
        q.run(STEPS)
        dq = q.download()  # before the extra build below wraps the positions
        q.neigh_build()
        r1 = q.compute(1, 1)
        q.close()
        for key in ("E_pair", "Press", "Temp"):
            assert abs(t0[k][key] - r0[key]) <= 1e-12 * abs(r0[key]), (k, key)
        # same cell order, lists and launch shape; the batched and single
        # kernels are separate compilations, so the last bits may differ and
        # grow slowly along the trajectory
        dx = np.max(np.abs(st["x"][a0[k]:a0[k + 1]] - dq["x"]))
        assert dx <= 1e-10, (k, dx)
        assert abs(t1[k]["eng"] - r1["eng"]) <= 1e-10 * abs(r1["eng"]), k


def test_batch_mixed_forces_within_1e5(batch):
    # off the lattice (on it the forces cancel to ~1e-14): 30 FP64 steps first
    s64 = make_batch(batch, "fp64")
    s64.setup()
    s64.run(30)
    st = s64.download()
    s64.neigh_build()
    s64.compute(1, 1)
    f64 = s64.download()["f"]
    s64.close()
    b = dict(batch, x=st["x"], v=st["v"])
    smx = make_batch(b, "mixed")
    smx.setup()
    fmx = smx.download()["f"]
    smx.close()
    a0 = np.concatenate([[0], np.cumsum(batch["natoms"])])
    for k in range(NREP):
        a, b = f64[a0[k]:a0[k + 1]], fmx[a0[k]:a0[k + 1]]
        assert np.linalg.norm(b - a) / np.linalg.norm(a) <= 1e-5, k


def test_step_times_recorded(batch):
    s = make_batch(batch, "mixed")
    s.setup()
    s.set_timing(True)
    s.run(30)
    ms = s.step_times()
    s.close()
    assert len(ms) == 30 and np.all(ms > 0)
