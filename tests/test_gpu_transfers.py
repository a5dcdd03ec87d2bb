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


def _system(edge=20.0):
    s = System("lj", "fp64")
    s.set_box([0.0, 0.0, 0.0], [edge] * 3)
    p = PairLJCut(2.5)
    p.coeff(1, 1, 1.0, 1.0, 2.5)
    s.set_pair(p)
    s.set_mass([1.0])
    s.set_neighbor(0.3, 20, 0, False)
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
