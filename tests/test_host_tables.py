"""Host-side mirrors of the reference's input commands and pair tables are
bit-identical to the oracle (which is pinned to the reference's logs)."""
import os

import numpy as np
import pytest

import oracle
from lammps_b200 import PairEAM, PairEAMAlloy, PairEAMFS, PairLJCut, inputs
from lammps_b200.eam_synth import write_setfl

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_lattice_and_lj_scale_match():
    a = inputs.lj_lattice_constant("fcc", 0.8442)
    assert a == oracle.lj_lattice_scale("fcc", 0.8442)
    x = inputs.lattice("fcc", 5, 4, 3, a)
    assert np.array_equal(x, oracle.lattice("fcc", 5, 4, 3, a))


@pytest.mark.parametrize("gaussian", [False, True])
@pytest.mark.parametrize("loop", ["geom", "all"])
def test_velocity_create_bit_identical(gaussian, loop):
    a = inputs.lj_lattice_constant("fcc", 0.8442)
    x = inputs.lattice("fcc", 6, 6, 6, a)
    mass = np.array([0.0, 1.0])
    v = inputs.velocity_create(x, np.ones(len(x), np.int32), mass, 1.44, 87287, "lj",
                               gaussian=gaussian, loop=loop)
    s = oracle.OracleSim("lj")
    s.box([0, 0, 0], [6 * a] * 3)
    s.atoms(x)
    s.mass(1, 1.0)
    s.velocity_create(1.44, 87287, gaussian=gaussian, loop_geom=(loop == "geom"))
    assert np.array_equal(v, s.v)


def test_velocity_metal_units():
    x = inputs.lattice("fcc", 5, 5, 5, 3.615)
    mass = np.array([0.0, 63.55])
    v = inputs.velocity_create(x, np.ones(len(x), np.int32), mass, 1600.0, 376847, "metal",
                               gaussian=True)
    s = oracle.OracleSim("metal")
    s.box([0, 0, 0], [5 * 3.615] * 3)
    s.atoms(x)
    s.mass(1, 63.55)
    s.velocity_create(1600.0, 376847, gaussian=True)
    assert np.array_equal(v, s.v)


def _oracle_lj_tables(p):
    s = oracle.OracleSim("lj")
    s.box([0, 0, 0], [10, 10, 10])
    s.atoms(np.zeros((1, 3)), type=np.ones(1, np.int32), ntypes=p.ntypes)
    return s


def test_lj_tables_two_types_with_mixing():
    p = PairLJCut(2.5, ntypes=2, shift=True)
    p.coeff(1, 1, 1.0, 1.0)
    p.coeff(2, 2, 0.7, 1.1, 2.75)
    t = p.tables()
    # mixed 1-2 entry: geometric epsilon and sigma, cutoff sqrt(2.5*2.75)
    assert t["cutsq"][1 * 3 + 2] == np.sqrt(2.5 * 2.75) ** 2
    assert t["lj1"][1 * 3 + 2] == 48.0 * np.sqrt(0.7) * np.sqrt(1.1) ** 12
    assert t["offset"][1 * 3 + 1] != 0.0


def test_eam_funcfl_tables_bit_identical():
    path = os.path.join(GOLDEN, "Cu_u3.eam")
    p = PairEAM(1)
    p.coeff(1, path)
    t = p.tables()
    s = oracle.OracleSim("metal")
    s.box([0, 0, 0], [20, 20, 20])
    s.atoms(np.array([[1.0, 1.0, 1.0]]))
    s.eam_funcfl([path], [0])
    s.compute()
    o = s.eam_tables()
    for k in ("nrho", "nr", "drho", "dr", "rhomax", "cutmax"):
        assert t[k] == o[k], k
    for k in ("frho_spline", "rhor_spline", "z2r_spline"):
        assert np.array_equal(t[k], o[k]), k
    assert p.mass[1] == 63.55


def test_eam_setfl_tables_bit_identical(tmp_path):
    path = write_setfl(str(tmp_path / "synth.eam.alloy"), nr=600, nrho=600)
    p = PairEAMAlloy(1)
    p.coeff(path, ["Cu"])
    t = p.tables()
    s = oracle.OracleSim("metal")
    s.box([0, 0, 0], [20, 20, 20])
    s.atoms(np.array([[1.0, 1.0, 1.0]]))
    s.eam_setfl(path, [0])
    s.compute()
    o = s.eam_tables()
    for k in ("frho_spline", "rhor_spline", "z2r_spline"):
        assert np.array_equal(t[k], o[k]), k
    assert np.array_equal(t["type2z2r"].reshape(2, 2)[1:, 1:], o["type2z2r"])


def _write_fs(path, ne=2, nr=300, nrho=300):
    """Small two-element Finnis-Sinclair file for table checks."""
    r = np.arange(nr) * (5.0 / (nr - 1))
    rho = np.arange(nrho) * (30.0 / (nrho - 1))
    def block(vals):
        return [" ".join(f"{v:.16e}" for v in vals[k:k + 5]) for k in range(0, len(vals), 5)]

    lines = ["fs test", "two elements", "generated for tests", f"{ne} A B",
             f"{nrho} {30.0 / (nrho - 1):.16e} {nr} {5.0 / (nr - 1):.16e} 5.0"]
    for i in range(ne):
        lines.append(f"{i + 1} {50.0 + i} 3.6 fcc")
        lines += block(-(1 + 0.1 * i) * np.sqrt(rho))
        for j in range(ne):
            lines += block(np.exp(-(1.5 + 0.2 * i + 0.1 * j) * (r - 2.5)))
    for i in range(ne):
        for j in range(i + 1):
            lines += block(r * 0.3 * np.exp(-(1.0 + 0.1 * (i + j)) * (r - 2.5)))
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    return path


def test_eam_fs_two_element_tables(tmp_path):
    path = _write_fs(str(tmp_path / "ab.eam.fs"))
    p = PairEAMFS(2)
    p.coeff(path, ["A", "B"])
    t = p.tables()
    s = oracle.OracleSim("metal")
    s.box([0, 0, 0], [20, 20, 20])
    s.atoms(np.array([[1.0, 1.0, 1.0], [3.0, 1.0, 1.0]]), type=np.array([1, 2], np.int32), ntypes=2)
    s.eam_setfl(path, [0, 1], fs=True)
    s.compute()
    o = s.eam_tables()
    for k in ("frho_spline", "rhor_spline", "z2r_spline"):
        assert np.array_equal(t[k], o[k]), k
    assert np.array_equal(t["type2rhor"].reshape(3, 3)[1:, 1:], o["type2rhor"])
    assert np.array_equal(t["type2z2r"].reshape(3, 3)[1:, 1:], o["type2z2r"])
