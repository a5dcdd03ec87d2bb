"""Failure paths of the C ABI: status codes, never a device fault.

Each failure is made on the host side (a bad input or a too-small limit);
the device turns it into a status word that the host maps to an error code,
as the reference maps the GPU package's negative codes to error->all
(src/GPU/gpu_extra.h:26-64).
"""
import json
import os

import numpy as np
import pytest

from gpu_cases import device_case
from lammps_b200 import PairLJCut, System, inputs
from lammps_b200._abi import B200Error

pytestmark = pytest.mark.gpu

with open(os.path.join(os.path.dirname(__file__), "golden", "reference_logs.json")) as fh:
    LOGS = json.load(fh)


def _small_lj(n_cells=6, one=0):
    a = inputs.lj_lattice_constant("fcc", 0.8442)
    x = inputs.lattice("fcc", n_cells, n_cells, n_cells, a)
    s = System("lj", "fp64")
    s.set_box([0, 0, 0], [n_cells * a] * 3)
    p = PairLJCut(2.5)
    p.coeff(1, 1, 1.0, 1.0, 2.5)
    s.set_pair(p)
    s.set_mass([1.0])
    s.set_neighbor(0.3, 20, 0, False, one)
    return s, x


def test_hard_neighbor_limit_reports_overflow():
    s, x = _small_lj(one=40)
    s.set_atoms(x)
    with pytest.raises(B200Error) as e:
        s.setup()
    assert e.value.code == -5
    assert "boost neigh_modify one" in str(e.value)


def test_soft_capacity_grows_and_run_matches_reference_log():
    case = LOGS["melt"]
    dev = device_case(case, "fp64")
    dev.set_neighbor(case["neighbor"]["skin"], case["neighbor"]["every"],
                     case["neighbor"]["delay"], case["neighbor"]["check"], -24)
    rows = [dev.setup()] + dev.run(case["run"])
    for got, want in zip(rows, case["thermo_rows"]):
        for col in ("Temp", "E_pair", "TotEng", "Press"):
            assert "%.8g" % got[col] == want[col], (want["Step"], col)
    assert dev.neigh_stats()["capacity"] > 24


def test_non_finite_coordinate_is_lost_atom():
    s, x = _small_lj()
    x = x.copy()
    x[5, 1] = np.nan
    s.set_atoms(x)
    with pytest.raises(B200Error) as e:
        s.setup()
    assert e.value.code == -7


def test_mixed_box_not_longer_than_twice_the_list_cutoff():
    # 3 x 3 x 3 fcc cells: edge 5.04 sigma, longer than the list cutoff (2.8)
    # but not twice it.  The mixed form forms separations at the minimum
    # image of 32-bit fixed-point coordinates, which needs the longer box.
    a = inputs.lj_lattice_constant("fcc", 0.8442)
    x = inputs.lattice("fcc", 3, 3, 3, a)
    s = System("lj", "mixed")
    s.set_box([0, 0, 0], [3 * a] * 3)
    p = PairLJCut(2.5)
    p.coeff(1, 1, 1.0, 1.0, 2.5)
    s.set_pair(p)
    s.set_mass([1.0])
    s.set_atoms(x)
    with pytest.raises(B200Error) as e:
        s.setup()
    assert e.value.code == -6
    assert "twice the list cutoff" in str(e.value)


def test_box_smaller_than_ghost_cutoff():
    a = inputs.lj_lattice_constant("fcc", 0.8442)
    x = inputs.lattice("fcc", 1, 1, 1, a)
    s = System("lj", "fp64")
    s.set_box([0, 0, 0], [a] * 3)
    p = PairLJCut(2.5)
    p.coeff(1, 1, 1.0, 1.0, 2.5)
    s.set_pair(p)
    s.set_mass([1.0])
    s.set_atoms(x)
    with pytest.raises(B200Error) as e:
        s.setup()
    assert e.value.code == -6


def test_calls_out_of_order():
    s, x = _small_lj()
    with pytest.raises(B200Error) as e:
        s.compute()
    assert e.value.code == -4
    s.set_atoms(x)
    with pytest.raises(B200Error) as e:
        s.run(5)
    assert e.value.code == -4


def test_bad_arguments():
    s, x = _small_lj()
    with pytest.raises(B200Error):
        s.set_launch(3)
    with pytest.raises(B200Error):
        s.set_atoms(x, type_=np.full(len(x), 2, np.int32))
