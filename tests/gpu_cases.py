"""Helpers that build matched oracle / device systems for the GPU parity tests."""
import os

import numpy as np

import oracle
from lammps_b200 import PairEAM, PairEAMAlloy, PairLJCut, System, inputs
from oracle_cases import GOLDEN, build_oracle_case, case_lattice


def device_case(case, precision="fp64", tpa=0):
    """System configured like a golden-log case, with the reference's
    lattice and `velocity create` generated on the host."""
    x, hi = case_lattice(case)
    sysm = System(case["units"], precision)
    sysm.set_box([0.0, 0.0, 0.0], hi)
    p = case["pair"]
    if p["style"] == "lj/cut":
        pair = PairLJCut(p["cut"])
        pair.coeff(1, 1, p["eps"], p["sigma"], p["cut"])
        sysm.set_pair(pair)
        sysm.set_mass([case["mass"]])
    else:
        pair = PairEAM(1)
        pair.coeff(1, os.path.join(GOLDEN, p["file"]))
        sysm.set_pair(pair)
    vel = case["velocity"]
    v = inputs.velocity_create(x, np.ones(len(x), np.int32), sysm.mass, vel["t"], vel["seed"],
                               case["units"], gaussian=vel["dist"] == "gaussian", loop=vel["loop"])
    nb = case["neighbor"]
    sysm.set_neighbor(nb["skin"], nb["every"], nb["delay"], nb["check"])
    sysm.set_timestep(case["dt"])
    sysm.set_thermo(case["thermo"])
    if tpa:
        sysm.set_launch(tpa)
    sysm.set_atoms(x, None, v)
    return sysm


def oracle_snapshot(case, steps=10, threads=4):
    """Run the oracle `steps` steps, then rebuild lists and evaluate forces
    with energy and pairwise virial on the resulting positions."""
    s = build_oracle_case(case, threads=threads)
    s.setup()
    if steps:
        s.run(steps)
    s.compute(eflag=1, vflag=1)
    out = dict(x=s.x, v=s.v, f=s.f, type=s.type, eng=s.eng_vdwl, virial=s.virial,
               nghost=s.nghost, half=s.half_list(), neigh_total=s.neigh_total)
    if case["pair"]["style"] != "lj/cut":
        out["rho"], out["fp"] = s.rho_fp()
    return out


def device_from_snapshot(case, snap, precision="fp64", tpa=0):
    sysm = device_case(case, precision, tpa)
    sysm.set_atoms(snap["x"], snap["type"], snap["v"])
    return sysm


def force_errors(f, fref):
    """Norm-wise relative error and max |dF_i| / RMS(F_ref)."""
    d = f - fref
    rel = np.linalg.norm(d) / np.linalg.norm(fref)
    rms = np.sqrt(np.mean(np.sum(fref * fref, axis=1)))
    mx = np.max(np.linalg.norm(d, axis=1)) / rms
    return rel, mx


def virial_errors(v, vref):
    trace = abs(vref[0] + vref[1] + vref[2])
    diag = np.max(np.abs(v[:3] - vref[:3]) / np.abs(vref[:3]))
    off = np.max(np.abs(v[3:] - vref[3:])) / trace
    return diag, off


def half_sets(num, jowner, jimage):
    """Per-atom sorted arrays of (owner*27 + image) codes."""
    codes = jowner.astype(np.int64) * 27 + jimage
    out = []
    o = 0
    for k in num:
        out.append(np.sort(codes[o:o + k]))
        o += k
    return out
