"""The brick decomposition's host logic on CPU (`lammps_b200.brick`): brick
geometry, Domain::pbc, and whole decomposed runs with a CPU stand-in engine
-- in one process (`LocalComm`) and as two `gloo` ranks (`DistComm`, world
size 2, spawned processes, 127.0.0.1).  Every decomposition must give the
single-box trajectory bit for bit: each owned atom sees the same neighbors in
the same order.  No GPU is touched."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from lammps_b200 import inputs  # noqa: E402
from lammps_b200.brick import BrickGrid, BrickRun, DistComm, LocalComm, pbc  # noqa: E402

from brick_numpy_engine import NumpyEAM, NumpyLJ  # noqa: E402

NCELL = 5
STEPS = 60


def _system():
    a = inputs.lj_lattice_constant("fcc", 0.8442)
    x = inputs.lattice("fcc", NCELL, NCELL, NCELL, a)
    rng = np.random.default_rng(5)
    v = rng.normal(scale=1.3, size=x.shape)
    v -= v.mean(axis=0)
    # a few atoms start just outside the box: the first wrap moves them
    x[:7, 0] -= NCELL * a
    return x, v, NCELL * a


def _run(comm, grid, ranks=None):
    x, v, L = _system()
    ranks = comm.ranks if ranks is None else ranks
    eng = {r: NumpyLJ([0.0] * 3, [L] * 3, every=1, delay=0, check=True) for r in ranks}
    b = BrickRun(comm, eng, grid)
    b.set_atoms(x, None, v)
    b.setup()
    rows = b.run(STEPS, thermo_every=20)
    return b, rows, b.gather()


def test_brick_grid_bounds_owner_near():
    lo, hi = np.zeros(3), np.array([10.0, 7.0, 5.0])
    g = BrickGrid(lo, hi, (3, 2, 1))
    assert g.nranks == 6
    rng = np.random.default_rng(1)
    x = rng.uniform(0, 1, size=(4000, 3)) * hi
    own = g.owner(x)
    for r in range(6):
        blo, bhi = g.bounds(r)
        inside = np.all((x >= blo) & (x < bhi), axis=1)
        assert np.array_equal(inside, own == r)
        # reference brick bounds: boxlo + prd * (i * 1.0 / p), last = boxhi
        cx, cy, cz = g.coords(r)
        assert blo[0] == lo[0] + 10.0 * (cx * 1.0 / 3)
        # near() contains every atom within depth (Euclidean, periodic) of an
        # atom inside the brick
        depth = 1.3
        near = g.near(x, r, depth)
        ins = np.nonzero(own == r)[0]
        d = x[:, None, :] - x[None, ins, :]
        d -= np.round(d / hi) * hi
        close = np.any(np.sum(d * d, axis=2) <= depth * depth, axis=1)
        assert not np.any(close & ~near)


def test_pbc_rule():
    lo, hi = np.zeros(3), np.full(3, 4.0)
    # -1e-17 + 4.0 rounds to 4.0 = hi: the second test takes it back to lo
    x = np.array([[-0.5, 4.0, 2.0], [3.9, -1e-17, 5.0]])
    xw, im = pbc(x, np.zeros((2, 3), np.int64), lo, hi)
    assert np.all((xw >= lo) & (xw < hi))
    assert im.tolist() == [[-1, 1, 0], [0, 0, 1]]
    assert xw[0, 0] == -0.5 + 4.0 and xw[0, 1] == 0.0 and xw[1, 1] == 0.0


def test_local_decompositions_match_single_box_bit_for_bit():
    b1, rows1, ref = _run(LocalComm(1), (1, 1, 1))
    assert b1.ncalls >= 2  # rebuilds happened (check yes)
    for grid in ((2, 1, 1), (1, 2, 2), (3, 1, 1)):
        comm = LocalComm(int(np.prod(grid)))
        b, rows, got = _run(comm, grid)
        assert b.ncalls == b1.ncalls, grid
        for k in ("x", "v", "image"):
            assert np.array_equal(got[k], ref[k]), (grid, k)
        st = b.stats()
        assert sum(s["owned"] for s in st.values()) == len(ref["x"])
        assert all(s["ghost"] > 0 for s in st.values())
        for r1, r2 in zip(rows1, rows):
            for k in ("Temp", "E_pair", "Press"):
                assert r2[k] == pytest.approx(r1[k], rel=1e-12, abs=1e-12), (grid, k)
    # the trajectory left the starting box: image flags record it
    assert np.any(ref["image"] != 0)


def _worker(rank, port, result_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=2)
    try:
        b, rows, got = _run(DistComm(), (2, 1, 1))
        np.savez(os.path.join(result_dir, f"brick{rank}.npz"), x=got["x"], v=got["v"],
                 image=got["image"], ncalls=b.ncalls, temp=[r["Temp"] for r in rows],
                 epair=[r["E_pair"] for r in rows])
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_match_single_box(tmp_path):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0, p.exitcode
    b1, rows1, ref = _run(LocalComm(1), (1, 1, 1))
    for r in range(2):
        res = np.load(tmp_path / f"brick{r}.npz")
        assert int(res["ncalls"]) == b1.ncalls
        for k in ("x", "v", "image"):
            assert np.array_equal(res[k], ref[k]), k
        assert np.allclose(res["temp"], [q["Temp"] for q in rows1], rtol=1e-12)
        assert np.allclose(res["epair"], [q["E_pair"] for q in rows1], rtol=1e-12)


def test_merge_by_gid():
    from lammps_b200.brick import _merge_by_gid, _W, _GID
    rng = np.random.default_rng(9)
    gid = rng.permutation(1000)
    for na, nb in ((600, 400), (0, 1000), (1000, 0), (999, 1)):
        a = np.zeros((na, _W)); a[:, _GID] = np.sort(gid[:na]); a[:, 5] = rng.normal(size=na)
        b = np.zeros((nb, _W)); b[:, _GID] = gid[na:na + nb]; b[:, 5] = rng.normal(size=nb)
        out, pa, pb = _merge_by_gid(torch.from_numpy(a), torch.from_numpy(b))
        out = out.numpy()
        assert np.array_equal(out[:, _GID], np.arange(na + nb) if na + nb == 1000 else np.sort(gid[:na + nb]))
        assert np.array_equal(out[pa.numpy()], a)
        assert np.array_equal(out[pb.numpy()], b)


def _run_eam(comm, grid, ranks=None, steps=30):
    """EAM over bricks: the density pass, the forward communication of F'
    to the ghosts, the force pass (PairEAM::compute's passes and
    forward_comm_pair, src/MANYBODY/pair_eam.cpp:160-303)."""
    # 8 x 4 x 4 cells at a = 1.6: along x a brick of a 2 x 1 x 1 grid (6.4)
    # plus its ghost depth (rc + skin = 2.3 each side) does not span the box,
    # so the outermost ghosts lack part of their neighborhood and their own
    # densities are wrong: only the forwarded F' gives the right forces
    a = 1.6
    x = inputs.lattice("fcc", 8, 4, 4, a)
    rng = np.random.default_rng(11)
    x = x + rng.normal(scale=0.03, size=x.shape)
    v = rng.normal(scale=0.3, size=x.shape)
    v -= v.mean(axis=0)
    hi = [8 * a, 4 * a, 4 * a]
    ranks = comm.ranks if ranks is None else ranks
    eng = {r: NumpyEAM([0.0] * 3, hi, rc=2.0, every=1, delay=0, check=True) for r in ranks}
    b = BrickRun(comm, eng, grid)
    assert b.fp_halo == (comm.world > 1)
    b.set_atoms(x, None, v)
    b.setup()
    rows = b.run(steps, thermo_every=20)
    return b, rows, b.gather()


def test_eam_bricks_reproduce_single_box():
    """Ghosts carry their owners' F': every decomposition gives the
    single-box trajectory bit for bit (with the ghosts' own, incomplete
    densities the forces would differ)."""
    b1, rows1, ref = _run_eam(LocalComm(1), (1, 1, 1))
    for grid in ((2, 1, 1), (1, 2, 2)):
        b, rows, got = _run_eam(LocalComm(int(np.prod(grid))), grid)
        assert b.ncalls == b1.ncalls, grid
        for k in ("x", "v", "image"):
            assert np.array_equal(got[k], ref[k]), (grid, k)
        for r1, r2 in zip(rows1, rows):
            for k in ("Temp", "E_pair", "Press"):
                assert r2[k] == pytest.approx(r1[k], rel=1e-12, abs=1e-12), (grid, k)


def _eam_worker(rank, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=2)
    try:
        b, rows, g = _run_eam(DistComm(), (2, 1, 1), ranks=[rank])
        if rank == 0:
            np.savez(out, x=g["x"], v=g["v"], ncalls=b.ncalls, temp=[r["Temp"] for r in rows])
    finally:
        dist.destroy_process_group()


def test_eam_two_gloo_ranks_reproduce_single_box(tmp_path):
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    out = str(tmp_path / "eam.npz")
    mp.start_processes(_eam_worker, args=(port, out), nprocs=2, start_method="spawn", join=True)
    b1, rows1, ref = _run_eam(LocalComm(1), (1, 1, 1))
    res = np.load(out)
    assert int(res["ncalls"]) == b1.ncalls
    assert np.array_equal(res["x"], ref["x"])
    assert np.array_equal(res["v"], ref["v"])
