"""Build oracle simulations from the run parameters in tests/golden (test helper)."""
import os

import numpy as np

import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def case_lattice(case):
    """(positions in creation order, box hi) for a case's fcc block."""
    nx, ny, nz = case["cells"]
    if case["units"] == "lj":
        a = oracle.lj_lattice_scale("fcc", case["lattice"])
    else:
        a = case["lattice"]
    x = oracle.lattice("fcc", nx, ny, nz, a)
    return x, np.array([nx * a, ny * a, nz * a])


def build_oracle_case(case, threads=1, sortfreq=1000):
    x, hi = case_lattice(case)
    s = oracle.OracleSim(case["units"], threads=threads)
    s.box([0.0, 0.0, 0.0], hi)
    s.atoms(x)
    p = case["pair"]
    if p["style"] == "lj/cut":
        s.mass(1, case["mass"])
        s.lj_cut(p["cut"])
        s.lj_coeff(1, 1, p["eps"], p["sigma"], p["cut"])
    else:
        s.eam_funcfl([os.path.join(GOLDEN, p["file"])], [0])
    v = case["velocity"]
    s.velocity_create(v["t"], v["seed"], gaussian=v["dist"] == "gaussian",
                      loop_geom=v["loop"] == "geom")
    nb = case["neighbor"]
    s.neighbor(nb["skin"], nb["every"], nb["delay"], nb["check"], sortfreq)
    s.timestep(case["dt"])
    s.thermo(case["thermo"])
    return s
