"""The brick decomposition on the device: bricks of one box as separate
engine contexts on one GPU, stepped together in one process (`LocalComm`;
the halo exchange is a device copy and no kernel waits on another).  Each
owned atom sees the same neighbors in the same order as in the single box,
so a decomposed run must reproduce the single-box trajectory bit for bit --
for lj/cut and EAM (whose ghosts get F'(rho) from their owners between the
density and force passes), FP64 and mixed, through rebuilds (check yes) with
exchange and borders, and the per-step halo pack / unpack in between; and
the decomposed run must match the oracle's serial run."""
import os
import socket

import numpy as np
import pytest

from lammps_b200 import PairEAM, PairLJCut, System, inputs
from lammps_b200._abi import B200Error
from lammps_b200.brick import BrickRun, DistComm, LocalComm

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TPA = 4


def _lj(precision):
    a = inputs.lj_lattice_constant("fcc", 0.8442)
    x = inputs.lattice("fcc", 10, 10, 10, a)
    L = 10 * a

    def make():
        s = System("lj", precision)
        s.set_box([0.0] * 3, [L] * 3)
        p = PairLJCut(2.5)
        p.coeff(1, 1, 1.0, 1.0, 2.5)
        s.set_pair(p)
        s.set_mass([1.0])
        s.set_neighbor(0.3, every=1, delay=0, check=True)
        s.set_launch(TPA, 128)
        return s

    v = make().create_velocity(x, 1.44, 87287, gaussian=True)
    return make, x, v, 200


def _eam(precision):
    x = inputs.lattice("fcc", 10, 10, 10, 3.615)
    L = 10 * 3.615

    def make():
        s = System("metal", precision)
        s.set_box([0.0] * 3, [L] * 3)
        p = PairEAM(1)
        p.coeff(1, os.path.join(ROOT, "tests", "golden", "Cu_u3.eam"))
        s.set_pair(p)
        s.set_neighbor(1.0, every=1, delay=5, check=True)
        s.set_timestep(0.005)
        s.set_launch(TPA, 128)
        return s

    v = make().create_velocity(x, 1600.0, 376847, gaussian=True)
    return make, x, v, 100


def _brick(case, grid):
    make, x, v, steps = case
    comm = LocalComm(int(np.prod(grid)))
    b = BrickRun(comm, {r: make() for r in comm.ranks}, grid)
    b.set_atoms(x, None, v)
    b.setup()
    rows = b.run(steps, thermo_every=steps // 2)
    return b, rows, b.gather()


@pytest.mark.parametrize("style", ["lj", "eam"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_bricks_reproduce_single_box(style, precision):
    case = (_lj if style == "lj" else _eam)(precision)
    b1, rows1, ref = _brick(case, (1, 1, 1))
    assert b1.ncalls >= 2
    for grid in ((2, 1, 1), (2, 2, 1)):
        b, rows, got = _brick(case, grid)
        assert b.ncalls == b1.ncalls, grid
        for k in ("x", "v", "image"):
            assert np.array_equal(got[k], ref[k]), (grid, k, float(np.abs(got[k] - ref[k]).max()))
        assert all(s["ghost"] > 0 for s in b.stats().values())
        for r1, r2 in zip(rows1, rows):
            for k in ("Temp", "E_pair", "Press"):
                assert r2[k] == pytest.approx(r1[k], rel=1e-11, abs=1e-11), (grid, k)


@pytest.mark.parametrize("style", ["lj", "eam"])
def test_bricks_match_oracle(style):
    """Two bricks (EAM with the forward communication of F'(rho) between the
    density and force passes) against the oracle's serial run of the same
    steps: positions, velocities and image flags after the run, the thermo
    rows and the number of neighbor builds."""
    import oracle
    make, x, v, steps = (_lj if style == "lj" else _eam)("fp64")
    b, rows, got = _brick((make, x, v, steps), (2, 1, 1))
    e = make()
    o = oracle.OracleSim("lj" if style == "lj" else "metal", threads=os.cpu_count() or 4)
    o.box([0.0] * 3, e.box_hi)
    o.atoms(x, v)
    if style == "lj":
        o.mass(1, 1.0)
        o.lj_cut(2.5)
        o.lj_coeff(1, 1, 1.0, 1.0, 2.5)
        o.neighbor(0.3, 1, 0, True, 1000)
    else:
        o.eam_funcfl([os.path.join(ROOT, "tests", "golden", "Cu_u3.eam")], [0])
        o.neighbor(1.0, 1, 5, True, 1000)
    o.timestep(e.dt)
    o.thermo(steps // 2)
    o.setup()
    o.run(steps)
    order = np.argsort(o.tag)
    for k in ("x", "v"):
        ref = getattr(o, k)[order]
        err = float(np.max(np.abs(got[k] - ref)))
        assert err <= 1e-9, (k, err)
    assert np.array_equal(got["image"], o.image[order])
    assert b.ncalls == o.ncalls
    orows = o.thermo_rows()
    for r, orow in zip(rows, orows[1:]):
        assert r["Step"] == int(orow[0])
        for key, col in (("Temp", 1), ("E_pair", 2), ("Press", 4)):
            assert r[key] == pytest.approx(orow[col], rel=1e-9, abs=1e-9), (r["Step"], key)
    e.close()


@pytest.mark.parametrize("style", ["lj", "eam"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_one_brick_matches_graph_run(style, precision):
    """The per-call path of one brick and b200_run's step graphs take the same
    rounded steps: same trajectory, same thermo.  For lj/cut b200_run steps
    through the one-launch step kernel (forces and both half-steps, with the
    position buffers alternating), the per-call path through separate
    pair and half-step kernels."""
    make, x, v, steps = (_lj if style == "lj" else _eam)(precision)
    b1, rows1, ref = _brick((make, x, v, steps), (1, 1, 1))
    s = make()
    s.set_atoms(x, None, v)
    s.set_thermo(steps // 2)
    s.setup()
    rows = s.run(steps)
    d = s.download()
    assert np.array_equal(d["x"], ref["x"])
    assert np.array_equal(d["v"], ref["v"])
    assert np.array_equal(d["image"], ref["image"])
    assert s.neigh_stats()["ncalls"] == b1.ncalls
    by_step = {r["Step"]: r for r in rows}
    assert steps in by_step
    for r1 in rows1:
        r2 = by_step[r1["Step"]]
        for k in ("Temp", "E_pair", "Press"):
            assert r2[k] == pytest.approx(r1[k], rel=1e-11, abs=1e-11), k


def test_halo_index_errors_are_reported():
    make, x, v, _ = _lj("fp64")
    s = make()
    s.set_atoms(x, None, v)
    s.neigh_build()
    idx = torch.tensor([0, len(x)], dtype=torch.int32, device="cuda")
    buf = torch.zeros((2, 3), dtype=torch.float64, device="cuda")
    with pytest.raises(B200Error, match="outside"):
        s.halo_pack(idx, buf)
    # the context stays usable
    s.halo_pack(idx[:1], buf[:1])
    assert buf[0].cpu().numpy().tolist() == list(x[0])
    # with ghosts marked, unpack writes ghosts only: an owned atom's index is
    # refused and its position is left as it was
    g = np.zeros(len(x), np.int32)
    g[len(x) // 2:] = 1
    s.set_ghosts(g)
    idx = torch.tensor([len(x) - 1, 3], dtype=torch.int32, device="cuda")
    buf = torch.full((2, 3), 0.5, dtype=torch.float64, device="cuda")
    with pytest.raises(B200Error, match="owned"):
        s.halo_unpack(idx, buf)
    after = s.download()["x"]
    assert after[3].tolist() == list(x[3])
    s.halo_unpack(idx[:1], buf[:1])
    assert s.download()["x"][len(x) - 1].tolist() == [0.5, 0.5, 0.5]
    # b200_run decides rebuilds alone: it refuses a context with ghosts
    s.set_ghosts(np.ones(len(x)))
    s.setup()
    with pytest.raises(B200Error, match="ghost"):
        s.run(1)


def _nccl_worker(port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        make, x, v, steps = _lj("fp64")
        b = BrickRun(DistComm(), {0: make()}, (1, 1, 1))
        b.set_atoms(x, None, v)
        b.setup()
        rows = b.run(steps // 4, thermo_every=steps // 8)
        g = b.gather()
        np.savez(out, x=g["x"], v=g["v"], ncalls=b.ncalls, temp=[r["Temp"] for r in rows])
    finally:
        dist.destroy_process_group()


def test_nccl_transport_one_rank(tmp_path):
    """DistComm over NCCL (one rank: the all-to-alls of the exchange and
    borders, the MAX and SUM all-reduces) gives the in-process result."""
    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    out = str(tmp_path / "nccl.npz")
    p = mp.get_context("spawn").Process(target=_nccl_worker, args=(port, out))
    p.start()
    p.join(timeout=300)
    assert p.exitcode == 0, p.exitcode
    make, x, v, steps = _lj("fp64")
    b = BrickRun(LocalComm(1), {0: make()}, (1, 1, 1))
    b.set_atoms(x, None, v)
    b.setup()
    rows = b.run(steps // 4, thermo_every=steps // 8)
    ref = b.gather()
    res = np.load(out)
    assert int(res["ncalls"]) == b.ncalls
    assert np.array_equal(res["x"], ref["x"])
    assert np.array_equal(res["v"], ref["v"])
    assert np.allclose(res["temp"], [r["Temp"] for r in rows], rtol=1e-13)
