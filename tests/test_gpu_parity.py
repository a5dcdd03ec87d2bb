"""Parity of the CUDA engine (through the C ABI) with the pinned CPU oracle.

Bars: neighbor lists bit-exact as sorted per-atom sets of (owner, image);
FP64 forces within 1e-12 norm-wise relative, energy and virial diagonal
within 1e-12 relative, virial off-diagonals within 1e-12 of |trace|;
mixed precision within 1e-5 (force).
"""
import json
import os

import numpy as np
import pytest

import oracle
from lammps_b200 import PairLJCut, System, inputs

from gpu_cases import (device_case, device_from_snapshot, force_errors, half_sets,
                       oracle_snapshot, virial_errors)

pytestmark = pytest.mark.gpu

with open(os.path.join(os.path.dirname(__file__), "golden", "reference_logs.json")) as fh:
    LOGS = json.load(fh)

FP64_TOL = 1e-12
MIXED_TOL = 1e-5


@pytest.fixture(scope="module")
def lj_snap():
    return oracle_snapshot(LOGS["bench_lj"], steps=10)


@pytest.fixture(scope="module")
def eam_snap():
    return oracle_snapshot(LOGS["bench_eam"], steps=10)


def _check_fp64(case, snap, tpa=0):
    dev = device_from_snapshot(case, snap, "fp64", tpa)
    dev.neigh_build()
    r = dev.compute(eflag=1, vflag=1)
    f = dev.download()["f"]
    rel, mx = force_errors(f, snap["f"])
    assert rel <= FP64_TOL, rel
    assert mx <= 1e-11, mx
    assert abs(r["eng"] - snap["eng"]) <= FP64_TOL * abs(snap["eng"])
    d, o = virial_errors(r["virial"], snap["virial"])
    assert d <= FP64_TOL and o <= FP64_TOL, (d, o)
    return dev


def test_lj_fp64_forces_energy_virial(lj_snap):
    _check_fp64(LOGS["bench_lj"], lj_snap)


@pytest.mark.parametrize("tpa", [1, 2, 4, 8])
def test_lj_fp64_every_launch_shape(lj_snap, tpa):
    _check_fp64(LOGS["bench_lj"], lj_snap, tpa)


def test_lj_half_list_bit_exact(lj_snap):
    dev = device_from_snapshot(LOGS["bench_lj"], lj_snap)
    dev.neigh_build()
    num, jo, ji = dev.half_list()
    onum, ojo, oji = lj_snap["half"]
    assert int(num.sum()) == lj_snap["neigh_total"]
    assert np.array_equal(num, onum)
    for a, b in zip(half_sets(num, jo, ji), half_sets(onum, ojo, oji)):
        assert np.array_equal(a, b)
    st = dev.neigh_stats()
    assert st["full_total"] == 2 * lj_snap["neigh_total"]


def test_eam_fp64_forces_density_embedding(eam_snap):
    dev = _check_fp64(LOGS["bench_eam"], eam_snap)
    rho, fp = dev.rho_fp()
    assert np.max(np.abs(rho - eam_snap["rho"]) / np.abs(eam_snap["rho"])) <= FP64_TOL
    assert np.max(np.abs(fp - eam_snap["fp"]) / np.abs(eam_snap["fp"])) <= FP64_TOL


def test_eam_half_list_bit_exact(eam_snap):
    dev = device_from_snapshot(LOGS["bench_eam"], eam_snap)
    dev.neigh_build()
    num, jo, ji = dev.half_list()
    onum, ojo, oji = eam_snap["half"]
    assert np.array_equal(num, onum)
    for a, b in zip(half_sets(num, jo, ji), half_sets(onum, ojo, oji)):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("name", ["bench_lj", "bench_eam"])
def test_mixed_precision_within_1e5(name, lj_snap, eam_snap):
    snap = lj_snap if name == "bench_lj" else eam_snap
    dev = device_from_snapshot(LOGS[name], snap, "mixed")
    dev.neigh_build()
    r = dev.compute(eflag=1, vflag=1)
    f = dev.download()["f"]
    rel, mx = force_errors(f, snap["f"])
    assert rel <= MIXED_TOL, rel
    assert abs(r["eng"] - snap["eng"]) <= MIXED_TOL * abs(snap["eng"])
    d, o = virial_errors(r["virial"], snap["virial"])
    assert d <= MIXED_TOL and o <= MIXED_TOL, (d, o)


def _fmt(v):
    return "%.8g" % v


@pytest.mark.parametrize("name", ["bench_lj", "bench_eam", "potentials_lj", "melt"])
def test_device_run_reproduces_reference_log(name):
    """The device Verlet loop prints the reference's thermo digits and
    neighbor statistics (regress/benchmark.py compares these columns)."""
    case = LOGS[name]
    dev = device_case(case, "fp64")
    rows = [dev.setup()] + dev.run(case["run"])
    ref = case["thermo_rows"]
    assert len(rows) == len(ref)
    for got, want in zip(rows, ref):
        assert got["Step"] == int(want["Step"])
        for col in ("Temp", "E_pair", "TotEng", "Press"):
            assert _fmt(got[col]) == want[col], (name, want["Step"], col, got[col], want[col])
    st = dev.neigh_stats()
    assert st["ncalls"] == case["stats"]["builds"]
    assert st["ndanger"] == case["stats"]["dangerous"]
    assert st["full_total"] == 2 * case["stats"]["neighbors"]


def test_eager_launches_match_graph_replay():
    """The graph path (device-conditional rebuild) and the kernel-by-kernel
    path run the same kernels in the same order: identical thermo.  Both
    contexts get the same launch shape (the search picks one by timing, so
    two searched contexts may sum in different orders)."""
    case = LOGS["potentials_lj"]
    a = device_case(case, "fp64", tpa=2)
    b = device_case(case, "fp64", tpa=2)
    b.set_graphs(False)
    ra = [a.setup()] + a.run(case["run"])
    rb = [b.setup()] + b.run(case["run"])
    for x, y in zip(ra, rb):
        for col in ("Temp", "E_pair", "Press"):
            assert x[col] == y[col]
    assert a.neigh_stats()["ncalls"] == b.neigh_stats()["ncalls"]


def test_piece_timing_keeps_the_step_form():
    """Timing mode 2 brackets whole pieces with stream events and keeps the
    run's own step form (the one-launch lj/cut step): the thermo equals an
    untimed run's, every step is timed, and the force pieces carry the time.
    Both contexts get the same launch shape, as above."""
    case = LOGS["potentials_lj"]
    a = device_case(case, "fp64", tpa=2)
    b = device_case(case, "fp64", tpa=2)
    b.set_timing(2)
    ra = [a.setup()] + a.run(case["run"])
    rb = [b.setup()] + b.run(case["run"])
    for x, y in zip(ra, rb):
        for col in ("Temp", "E_pair", "Press"):
            assert x[col] == y[col]
    ph = b.timing()
    assert ph["steps"] == case["run"]
    assert ph["pair1"] > 0 and ph["neigh"] > 0 and ph["initial"] > 0
    assert ph["pair2"] == 0 and ph["final"] == 0
    ms = b.step_times()
    assert len(ms) == case["run"]
    assert abs(sum(ms) - (ph["initial"] + ph["neigh"] + ph["pair1"])) <= 1e-6 * sum(ms)


def _noncubic_oracle(steps, thermo):
    """fcc 6 x 7 x 8 cells at rho* 0.8442: three different box edges (10.1,
    11.8 and 13.4 sigma), Gaussian velocities at T* 1.44; the oracle run for
    `steps` steps with thermo rows every `thermo`."""
    a = inputs.lj_lattice_constant("fcc", 0.8442)
    x = inputs.lattice("fcc", 6, 7, 8, a)
    hi = np.array([6 * a, 7 * a, 8 * a])
    v = inputs.velocity_create(x, np.ones(len(x), np.int32), np.array([0.0, 1.0]), 1.44, 4928,
                               "lj", gaussian=True, loop="geom")
    o = oracle.OracleSim("lj", threads=4)
    o.box([0.0, 0.0, 0.0], hi)
    o.atoms(x, v)
    o.mass(1, 1.0)
    o.lj_cut(2.5)
    o.lj_coeff(1, 1, 1.0, 1.0, 2.5)
    o.neighbor(0.3, 10, 0, False, 0)
    o.thermo(thermo)
    o.setup()
    o.run(steps)
    return o, x, v, hi


def _noncubic_device(prec, hi):
    s = System("lj", prec)
    s.set_box([0.0, 0.0, 0.0], hi)
    p = PairLJCut(2.5)
    p.coeff(1, 1, 1.0, 1.0, 2.5)
    s.set_pair(p)
    s.set_mass([1.0])
    s.set_neighbor(0.3, 10, 0, False)
    return s


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
def test_noncubic_box_forces_and_run(prec, tol):
    """Unequal box edges: the mixed form scales each fixed-point component by
    its own unit (no common unit, the two-kernel step), the FP64 form takes
    the one-launch step.  Forces after 10 oracle steps within the form's bar,
    and a 30-step device run's thermo rows against the oracle's."""
    o, x, v, hi = _noncubic_oracle(10, 0)
    o.compute(1, 1)
    dev = _noncubic_device(prec, hi)
    dev.set_atoms(o.x, None, o.v)
    dev.neigh_build()
    dev.compute(1, 1)
    rel, _ = force_errors(dev.download()["f"], o.f)
    assert rel <= tol, rel
    o2, _, _, _ = _noncubic_oracle(30, 10)
    want = o2.thermo_rows()
    dev = _noncubic_device(prec, hi)
    dev.set_thermo(10)
    dev.set_atoms(x, None, v)
    rows = [dev.setup()] + dev.run(30)
    assert len(rows) == len(want)
    rtol = 1e-9 if prec == "fp64" else 1e-5
    for got, ref in zip(rows, want):
        assert got["Step"] == int(ref[0])
        for key, col in (("Temp", 1), ("E_pair", 2), ("Press", 4)):
            assert got[key] == pytest.approx(ref[col], rel=rtol, abs=rtol), (got["Step"], key)
