"""Host transfers through the C ABI: b200_upload_atoms / b200_download_atoms
stage through one device buffer that the context keeps and grows between
calls.  Round trips must be exact for growing and shrinking atom counts, and
a download into caller-owned (page-locked) arrays must equal one into new
arrays."""
import numpy as np
import pytest

from lammps_b200 import PairLJCut, System, inputs
from lammps_b200._abi import B200Error

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _system(edge=20.0, tpa=None):
    """An FP64 LJ context; `tpa` fixes the pair kernels' launch shape (without
    it the first setup picks one by timing, and contexts with different
    shapes agree to rounding, not bit for bit)."""
    s = System("lj", "fp64")
    s.set_box([0.0, 0.0, 0.0], [edge] * 3)
    p = PairLJCut(2.5)
    p.coeff(1, 1, 1.0, 1.0, 2.5)
    s.set_pair(p)
    s.set_mass([1.0])
    s.set_neighbor(0.3, 20, 0, False)
    if tpa:
        s.set_launch(tpa, 128)
    return s


def test_round_trip_growing_and_shrinking():
    s = _system()
    rng = np.random.default_rng(7)
    for n in (100, 5000, 37, 5000, 20001, 1):
        x = rng.uniform(0.0, 20.0, size=(n, 3))
        v = rng.normal(size=(n, 3))
        s.set_atoms(x, None, v)
        out = s.download()
        assert np.array_equal(out["x"], x), n
        assert np.array_equal(out["v"], v), n
        assert not out["image"].any(), n
    s.close()


def test_download_into_page_locked_buffers():
    a = inputs.lj_lattice_constant("fcc", 0.8442)
    x = inputs.lattice("fcc", 9, 9, 9, a)
    n = len(x)
    s = _system(9 * a)
    rng = np.random.default_rng(11)
    s.set_atoms(x, None, rng.normal(size=(n, 3)))
    s.setup()
    s.run(5)
    ref = s.download()
    keep = []

    def pinned(shape, dt):
        t = torch.zeros(shape, dtype=dt, pin_memory=True)
        keep.append(t)
        return t.numpy()

    out = {k: pinned((n, 3), torch.float64) for k in ("x", "v", "f")}
    out["image"] = pinned((n, 3), torch.int32)
    got = s.download(out)
    assert got is out
    for k in ("x", "v", "f", "image"):
        assert np.array_equal(out[k], ref[k]), k
    with pytest.raises(ValueError):
        s.download({"x": np.zeros((n, 2)), "v": out["v"], "f": out["f"], "image": out["image"]})
    s.close()


def test_device_pointer_upload_download():
    """Upload from and download into device memory (unified addressing): same
    atoms as the host path; an out-of-range type in a device array is found by
    the upload kernel and reported with its index."""
    s = _system()
    rng = np.random.default_rng(3)
    n = 3000
    x = rng.uniform(0.0, 20.0, size=(n, 3))
    v = rng.normal(size=(n, 3))
    xt = torch.from_numpy(x).cuda()
    vt = torch.from_numpy(v).cuda()
    tt = torch.ones(n, dtype=torch.int32, device="cuda")
    s.set_atoms_dev(xt, tt, vt)
    d = s.download_dev()
    assert torch.equal(d["x"], xt) and torch.equal(d["v"], vt)
    assert not d["image"].any()
    h = s.download()
    assert np.array_equal(h["x"], x) and np.array_equal(h["v"], v)
    tt[1234] = 7
    with pytest.raises(B200Error, match="atom 1234"):
        s.set_atoms_dev(xt, tt, vt)
    s.close()


def _sets():
    """Three atom sets: two LJ lattices of one size with different
    velocities, and a smaller lattice."""
    a = inputs.lj_lattice_constant("fcc", 0.8442)
    out = []
    for cells, seed in ((8, 1), (8, 2), (6, 3)):
        x = inputs.lattice("fcc", cells, cells, cells, a)
        v = np.random.default_rng(seed).normal(size=(len(x), 3))
        out.append((x, v, cells * a))
    return out


def test_overlapped_transfers_match_blocking():
    """Stage the next set while the current one runs, download without
    waiting: every set's results equal those of the blocking calls."""
    keep = []

    def pinned(a):
        t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        keep.append(t)
        return t.numpy()

    sets = _sets()
    ref = []
    for x, v, edge in sets:
        s = _system(edge, tpa=4)
        s.set_atoms(x, None, v)
        s.setup()
        s.run(10)
        ref.append(s.download())
        s.close()
    got = []
    s = None
    for k, (x, v, edge) in enumerate(sets):
        if s is None or s.box_hi[0] != edge:
            if s is not None:
                s.wait_transfers()
                s.close()
            s = _system(edge, tpa=4)
            s.stage_atoms(pinned(x), pinned(np.ones(len(x), np.int32)), pinned(v))
        s.set_staged_atoms()
        if k + 1 < len(sets) and sets[k + 1][2] == edge:
            nx, nv, _ = sets[k + 1]
            s.stage_atoms(pinned(nx), pinned(np.ones(len(nx), np.int32)), pinned(nv))
        s.setup()
        s.run(10)
        n = len(x)
        out = {"x": pinned(np.zeros((n, 3))), "v": pinned(np.zeros((n, 3))),
               "f": pinned(np.zeros((n, 3))), "image": pinned(np.zeros((n, 3), np.int32))}
        got.append(s.download_async(out))
    s.wait_transfers()
    s.close()
    for k, (r, g) in enumerate(zip(ref, got)):
        for key in ("x", "v", "f", "image"):
            assert np.array_equal(g[key], r[key]), (k, key)


def test_staging_errors_leave_the_context_usable():
    x, v, edge = _sets()[0]
    n = len(x)
    s = _system(edge)
    with pytest.raises(B200Error, match="STATE"):
        s.set_staged_atoms()
    bad = np.ones(n, np.int32)
    bad[17] = 3
    s.stage_atoms(x, bad, v)
    s.stage_atoms(x, None, v)
    with pytest.raises(B200Error, match="two atom sets"):
        s.stage_atoms(x, None, v)
    with pytest.raises(B200Error, match="atom 17"):
        s.set_staged_atoms()
    s.set_staged_atoms()
    s.setup()
    s.run(5)
    out = {k: np.zeros((n, 3)) for k in ("x", "v", "f")}
    s.download_async(out)
    s.wait_transfers()
    assert np.array_equal(out["x"], s.download()["x"])
    s.close()
