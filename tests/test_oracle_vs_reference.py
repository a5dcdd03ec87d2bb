"""The oracle against the reference itself, atom by atom.

oracle/build_ref.py compiles the reference's own serial LAMMPS
(oracle/_ref/lmp_serial).  Here it runs the benchmark configurations --
plain LJ with uniform and with Gaussian velocities (bench/in.lj and the
32,000-atom LJ configuration), EAM with the Cu_u3 funcfl table
(bench/in.eam), and EAM with the synthetic 5000-point setfl table through
eam/alloy (the 32,000-atom EAM configuration) -- and dumps, at steps 0 and
10, every atom's position, force, energy (compute pe/atom) and virial
(compute stress/atom NULL virial, which is -nktv2p times the per-atom virial
that Pair::ev_tally accumulates, src/pair.cpp:795,838 and
src/MANYBODY/pair_eam.cpp:226, folded into the owners by reverse
communication).  The oracle runs the same steps from the same inputs.

Bars: positions and forces equal to 1e-13 (norm-wise relative; at step 0,
where the lattice forces cancel to about 1e-13, the largest force difference
within 1e-13 of the RMS force at step 10), per-atom energy and virial to
1e-12 (at step 0 the virial's largest difference against its RMS at step
10, for the same reason).  These pin the oracle on the per-atom outputs the golden logs do not
print.
"""
import os

import numpy as np
import pytest

import oracle
from lammps_runs import input_script, read_dump, run_lammps
from oracle import build_ref
from oracle_cases import build_oracle_case

LMP = build_ref.lmp_serial()
pytestmark = pytest.mark.skipif(LMP is None, reason="reference binary not built "
                                                    "(python oracle/build_ref.py)")

LJ = {"units": "lj", "lattice": 0.8442, "cells": [20, 20, 20], "mass": 1.0,
      "velocity": {"t": 1.44, "seed": 87287, "loop": "geom", "dist": "uniform"},
      "pair": {"style": "lj/cut", "cut": 2.5, "eps": 1.0, "sigma": 1.0},
      "neighbor": {"skin": 0.3, "every": 20, "delay": 0, "check": False},
      "dt": 0.005, "thermo": 5, "run": 10}
EAM = {"units": "metal", "lattice": 3.615, "cells": [20, 20, 20],
       "velocity": {"t": 1600.0, "seed": 376847, "loop": "geom", "dist": "uniform"},
       "pair": {"style": "eam", "file": "Cu_u3.eam"},
       "neighbor": {"skin": 1.0, "every": 1, "delay": 5, "check": True},
       "dt": 0.005, "thermo": 5, "run": 10}
NKTV2P = {"lj": 1.0, "metal": 1.6021765e6}  # src/update.cpp:118-166


def _gauss(case):
    c = dict(case)
    c["velocity"] = dict(case["velocity"], dist="gaussian")
    return c


CASES = {
    "lj_uniform": (LJ, None),
    "lj_gaussian": (_gauss(LJ), None),      # the 32,000-atom LJ configuration
    "eam_funcfl": (EAM, None),
    "eam_synth_setfl": (_gauss(EAM), "synth"),  # the 32,000-atom EAM configuration
}


def _reference(name, case, kind, tmp):
    work = str(tmp / name)
    os.makedirs(work, exist_ok=True)
    coeff = None
    pair_style = None
    if kind == "synth":
        from lammps_b200.eam_synth import write_setfl
        write_setfl(os.path.join(work, "Cu_synth.eam.alloy"))
        pair_style, coeff = "eam/alloy", "pair_coeff * * Cu_synth.eam.alloy Cu"
    extra = ["compute pe all pe/atom", "compute st all stress/atom NULL virial",
             "dump d all custom 10 dump.txt id x y z fx fy fz c_pe " +
             " ".join(f"c_st[{k}]" for k in range(1, 7)),
             "dump_modify d sort id format \"%d" + " %.17g" * 13 + "\""]
    script = input_script(case, pair_style=pair_style, pair_coeff=coeff, extra=extra)
    run_lammps(LMP, script, work)
    return read_dump(os.path.join(work, "dump.txt")), work


def _oracle(case, kind, work, steps):
    if kind == "synth":
        from oracle_cases import case_lattice
        x, hi = case_lattice(case)
        s = oracle.OracleSim("metal", threads=4)
        s.box([0.0, 0.0, 0.0], hi)
        s.atoms(x)
        s.eam_setfl(os.path.join(work, "Cu_synth.eam.alloy"), [0])
        v = case["velocity"]
        s.velocity_create(v["t"], v["seed"], gaussian=True, loop_geom=True)
        nb = case["neighbor"]
        s.neighbor(nb["skin"], nb["every"], nb["delay"], nb["check"], 1000)
        s.timestep(case["dt"])
        s.thermo(case["thermo"])
    else:
        s = build_oracle_case(case, threads=4)
    s.setup()
    if steps:
        s.run(steps)
    x, f, tag = s.x, s.f, s.tag
    s.compute(eflag=3, vflag=5)
    e, va = s.eatom_vatom()
    order = np.argsort(tag)
    return x[order], f[order], e[order], va[order], s.thermo_rows()


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_matches_reference_per_atom(name, tmp_path):
    case, kind = CASES[name]
    frames, work = _reference(name, case, kind, tmp_path)
    nktv2p = NKTV2P[case["units"]]
    frms = float(np.sqrt(np.mean(np.sum(frames[10][:, 4:7] ** 2, axis=1))))
    vrms = float(np.sqrt(np.mean(frames[10][:, 8:14] ** 2))) / nktv2p
    for step in (0, 10):
        ref = frames[step]
        assert ref.shape[0] == 32000
        x, f, e, va, _ = _oracle(case, kind, work, step)
        assert np.array_equal(ref[:, 0].astype(int), np.arange(1, 32001))
        assert _rel(x, ref[:, 1:4]) <= 1e-13, (step, "x")
        vref = -ref[:, 8:14] / nktv2p
        if step == 0:
            assert float(np.abs(f - ref[:, 4:7]).max()) <= 1e-13 * frms, (step, "f")
            assert float(np.abs(va - vref).max()) <= 1e-12 * vrms, (step, "vatom")
        else:
            assert _rel(f, ref[:, 4:7]) <= 1e-13, (step, "f")
            assert _rel(va, vref) <= 1e-12, (step, "vatom")
        assert _rel(e, ref[:, 7]) <= 1e-12, (step, "eatom")


@pytest.mark.parametrize("name", ["bench_lj", "bench_eam", "melt"])
def test_reference_binary_reproduces_golden_log(name, tmp_path):
    """The input scripts written from the golden cases' parameters, run by
    the reference's own binary, print the thermo digits and neighbor
    statistics of the reference's logs -- so the same scripts can drive
    lmp_b200 (tests/test_gpu_lammps_package.py)."""
    import json

    from lammps_runs import GOLDEN, parse_log
    with open(os.path.join(GOLDEN, "reference_logs.json")) as fh:
        case = json.load(fh)[name]
    out = parse_log(run_lammps(LMP, input_script(case), str(tmp_path)))
    assert [r["Step"] for r in out["rows"]] == [r["Step"] for r in case["thermo_rows"]]
    for got, want in zip(out["rows"], case["thermo_rows"]):
        for col in ("Temp", "E_pair", "TotEng", "Press"):
            assert got[col] == want[col], (name, want["Step"], col)
    assert out["builds"] == case["stats"]["builds"]
    assert out["dangerous"] == case["stats"]["dangerous"]
    assert out["neighbors"] == case["stats"]["neighbors"]
