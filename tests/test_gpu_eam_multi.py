"""Two-element EAM on the device against the oracle: eam/alloy and eam/fs
setfl tables (PairEAMAlloy / PairEAMFS, src/MANYBODY/pair_eam_alloy.cpp and
pair_eam_fs.cpp), where every pair looks its spline rows up through the
type2rhor / type2z2r maps -- the path the one-element specialization of the
kernels does not take.  Bars as in the other parity tests: FP64 forces,
energy and virial within 1e-12, the half list bit-exact, mixed forces within
1e-5."""
import numpy as np
import pytest

import oracle
from gpu_cases import force_errors, half_sets, virial_errors
from lammps_b200 import PairEAMAlloy, PairEAMFS, System, inputs

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 1e-5
RC = 5.0
NR = NRHO = 800


def _block(vals):
    return [" ".join(f"{v:.16e}" for v in vals[k:k + 5]) for k in range(0, len(vals), 5)]


def _switch(r):
    """C1 cubic switch from 1 at r = 4.4 to 0 at RC, so the tables end smoothly."""
    t = np.clip((r - 4.4) / (RC - 4.4), 0.0, 1.0)
    return 1.0 - t * t * (3.0 - 2.0 * t)


def write_two_element(path, fs):
    """A two-element setfl file (element A: mass 60, element B: mass 40).
    eam/alloy: one density function per element; eam/fs: one per element pair."""
    r = np.arange(NR) * (RC / (NR - 1))
    rho = np.arange(NRHO) * (40.0 / (NRHO - 1))
    lines = ["two-element test tables", "generated by tests/test_gpu_eam_multi.py", "third comment line",
             "2 A B", f"{NRHO} {40.0 / (NRHO - 1):.16e} {NR} {RC / (NR - 1):.16e} {RC:.16e}"]
    for i in range(2):
        lines.append(f"{i + 1} {60.0 - 20.0 * i} 3.6 fcc")
        lines += _block(-(1.0 + 0.3 * i) * np.sqrt(rho))
        dens = [np.exp(-(2.0 + 0.25 * i + 0.15 * j) * (r - 2.55)) * _switch(r)
                for j in range(2 if fs else 1)]
        for d in dens:
            lines += _block(d)
    for i in range(2):
        for j in range(i + 1):
            a = 1.4 + 0.1 * (i + j)
            phi = 0.5 * (np.exp(-2 * a * (r - 2.55)) - 2 * np.exp(-a * (r - 2.55))) * _switch(r)
            lines += _block(r * phi)
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    return path


def _atoms():
    """fcc 6^3 (864 atoms) at a = 3.6 A with seeded 0.08 A jitter and a
    seeded 50/50 split of the two types."""
    x = inputs.lattice("fcc", 6, 6, 6, 3.6)
    rng = np.random.default_rng(4242)
    x = x + rng.normal(scale=0.08, size=x.shape)
    t = np.ones(len(x), np.int32)
    t[rng.permutation(len(x))[: len(x) // 2]] = 2
    return x, t, np.array([6 * 3.6] * 3)


@pytest.fixture(scope="module", params=["alloy", "fs"])
def case(request, tmp_path_factory):
    fs = request.param == "fs"
    path = write_two_element(str(tmp_path_factory.mktemp("eam2") / f"ab.eam.{request.param}"), fs)
    x, t, hi = _atoms()
    o = oracle.OracleSim("metal")
    o.box([0, 0, 0], hi)
    o.atoms(x, None, t, ntypes=2)
    o.eam_setfl(path, [0, 1], fs=fs)
    o.neighbor(1.0, 1, 0, True, 0)
    o.setup()
    o.compute(eflag=1, vflag=1)
    snap = dict(f=o.f, eng=o.eng_vdwl, virial=o.virial, half=o.half_list(), x=o.x, type=o.type)
    return dict(fs=fs, path=path, hi=hi, snap=snap)


def _device(case, precision):
    s = System("metal", precision)
    s.set_box([0.0, 0.0, 0.0], case["hi"])
    p = PairEAMFS(2) if case["fs"] else PairEAMAlloy(2)
    p.coeff(case["path"], ["A", "B"])
    s.set_pair(p)
    s.set_neighbor(1.0, 1, 0, True)
    snap = case["snap"]
    s.set_atoms(snap["x"], snap["type"], np.zeros_like(snap["x"]))
    s.neigh_build()
    return s


def test_two_element_fp64_forces_energy_virial(case):
    s = _device(case, "fp64")
    r = s.compute(eflag=1, vflag=1)
    f = s.download()["f"]
    snap = case["snap"]
    rel, mx = force_errors(f, snap["f"])
    assert rel <= FP64_TOL and mx <= 1e-11, (rel, mx)
    assert abs(r["eng"] - snap["eng"]) <= FP64_TOL * abs(snap["eng"])
    d, o = virial_errors(r["virial"], snap["virial"])
    assert d <= FP64_TOL and o <= FP64_TOL, (d, o)
    s.close()


def test_two_element_half_list_bit_exact(case):
    s = _device(case, "fp64")
    num, jo, ji = s.half_list()
    onum, ojo, oji = case["snap"]["half"]
    assert np.array_equal(num, onum)
    for a, b in zip(half_sets(num, jo, ji), half_sets(onum, ojo, oji)):
        assert np.array_equal(a, b)
    s.close()


def test_two_element_mixed_within_1e5(case):
    s = _device(case, "mixed")
    s.compute(eflag=1, vflag=1)
    f = s.download()["f"]
    rel, _ = force_errors(f, case["snap"]["f"])
    assert rel <= MIXED_TOL, rel
    s.close()
