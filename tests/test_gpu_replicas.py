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


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_one_launch_step_equals_graph_path(batch, precision):
    """The one-launch replica step (clusters owning whole replicas) and the
    graph of kernels take the same rounded steps: identical trajectories
    through two rebuilds, for every cluster size."""
    ref = make_batch(batch, precision, tpa=1)
    ref.set_replica_step(1)
    ref.setup()
    assert not ref.replica_step()["onelaunch"]
    ref.run(STEPS)
    want = ref.download()
    ref.close()
    for cs, block in ((1, 256), (2, 512), (4, 256)):
        s = make_batch(batch, precision, tpa=1)
        s.set_replica_step(2, cs, block, 1)
        s.setup()
        st = s.replica_step()
        assert st["onelaunch"] and st["cluster"] == cs and st["block"] == block
        s.run(STEPS)
        got = s.download()
        for k in ("x", "v", "image"):
            assert np.array_equal(got[k], want[k]), (cs, block, k)
        s.close()


def test_step_form_is_tuned():
    """mode 0 times both forms on setup and reports them."""
    b = replica_batch(nrep=24, seed=99)
    s = make_batch(b, "mixed")
    s.setup()
    st = s.replica_step()
    assert st["graph_ms"] > 0 and st["onelaunch_ms"] > 0
    assert st["onelaunch"] == (st["onelaunch_ms"] < st["graph_ms"])
    s.run(25)
    s.close()
