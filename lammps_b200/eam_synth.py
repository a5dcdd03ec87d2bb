"""Synthetic single-element setfl (eam/alloy) table for the EAM benchmark.

Functions (r in Angstrom, energies in eV), each multiplied by a C1 cubic
switch S(r) = 1 - 3t^2 + 2t^3, t = (r - 4.5)/0.45, that takes rho and phi
smoothly to zero over [4.5, 4.95]:
    rho(r) = exp(-2.0 (r - 2.556)) S(r)
    F(rho) = -sqrt(rho)
    phi(r) = 0.5 (exp(-2*1.4 (r - 2.556)) - 2 exp(-1.4 (r - 2.556))) S(r)
A funcfl file cannot hold this phi (funcfl stores an effective charge Z(r)
with phi = 27.2*0.529 Z^2 / r >= 0, src/MANYBODY/pair_eam.cpp:661), so the
table is written in the setfl layout, which stores r*phi(r) directly
(src/MANYBODY/pair_eam_alloy.cpp:198-202).  5000 points for rho in
[0, 40] and for r in [0, 4.95].
"""
from __future__ import annotations

import os

import numpy as np

R0 = 2.556
RC = 4.95
RS = 4.5
NR = NRHO = 5000
RHOMAX = 40.0
MASS = 63.55
A0 = 3.615


def switch(r):
    t = np.clip((r - RS) / (RC - RS), 0.0, 1.0)
    return 1.0 - 3.0 * t * t + 2.0 * t * t * t


def rho_r(r):
    return np.exp(-2.0 * (r - R0)) * switch(r)


def phi_r(r):
    return 0.5 * (np.exp(-2.0 * 1.4 * (r - R0)) - 2.0 * np.exp(-1.4 * (r - R0))) * switch(r)


def f_rho(rho):
    return -np.sqrt(rho)


def write_setfl(path: str, nr: int = NR, nrho: int = NRHO) -> str:
    dr = RC / (nr - 1)
    drho = RHOMAX / (nrho - 1)
    r = np.arange(nr) * dr
    rho = np.arange(nrho) * drho
    lines = [
        "synthetic Cu-like EAM: rho=exp(-2(r-2.556)), F=-sqrt(rho), Morse-like phi",
        "C1 cubic switch to zero over [4.5, 4.95] A",
        "generated by lammps_b200/eam_synth.py",
        "1 Cu",
        f"{nrho} {drho:.16e} {nr} {dr:.16e} {RC:.16e}",
        f"29 {MASS} {A0} fcc",
    ]

    def block(vals):
        out = []
        for k in range(0, len(vals), 5):
            out.append(" ".join(f"{v:.16e}" for v in vals[k:k + 5]))
        return out

    lines += block(f_rho(rho))
    lines += block(rho_r(r))
    lines += block(r * phi_r(r))
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    return path
