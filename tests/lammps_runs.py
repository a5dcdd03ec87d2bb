"""Run a LAMMPS binary (the reference's own lmp_serial, or lmp_b200 with this
project's package linked in) on input scripts written from the run
parameters of tests/golden/reference_logs.json, and read back its thermo
rows, neighbor statistics and dumps (test helper).

The scripts are written here from each case's parameters (lattice, box,
velocity, pair, neighbor, timestep, thermo, run length), in LAMMPS's input
syntax, so that nothing at run time reads the reference checkout.
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def input_script(case, *, pair_style=None, pair_coeff=None, fix="nve", run_style=None,
                 velocity_dist=None, extra=(), run=None, thermo=None, pre=()):
    """LAMMPS commands for a golden case; keyword arguments override parts."""
    nx, ny, nz = case["cells"]
    p = case["pair"]
    v = case["velocity"]
    nb = case["neighbor"]
    dist = velocity_dist or v.get("dist", "uniform")
    lines = [f"units {case['units']}", "atom_style atomic", *pre,
             f"lattice fcc {case['lattice']}",
             f"region box block 0 {nx} 0 {ny} 0 {nz}", "create_box 1 box", "create_atoms 1 box"]
    if "mass" in case:
        lines.append(f"mass 1 {case['mass']}")
    # the pair style first: an EAM file sets the mass that velocity needs
    if p["style"] == "lj/cut":
        lines.append(f"pair_style {pair_style or 'lj/cut'} {p['cut']}")
        lines.append(pair_coeff or f"pair_coeff 1 1 {p['eps']} {p['sigma']} {p['cut']}")
    else:
        lines.append(f"pair_style {pair_style or 'eam'}")
        lines.append(pair_coeff or f"pair_coeff 1 1 {p['file']}")
    lines.append(f"velocity all create {v['t']} {v['seed']} dist {dist} loop {v['loop']}")
    lines.append(f"neighbor {nb['skin']} bin")
    lines.append(f"neigh_modify delay {nb['delay']} every {nb['every']} "
                 f"check {'yes' if nb['check'] else 'no'}")
    lines.append(f"fix 1 all {fix}")
    if run_style:
        lines.append(f"run_style {run_style}")
    lines.append(f"timestep {case['dt']}")
    th = case["thermo"] if thermo is None else thermo
    if th:
        lines.append(f"thermo {th}")
    lines += list(extra)
    lines.append(f"run {case['run'] if run is None else run}")
    return "\n".join(lines) + "\n"


def run_lammps(exe, script, workdir, args=(), env=None, timeout=600, files=("Cu_u3.eam",)):
    """Run `exe -in in.test` in workdir (with the golden potential files
    beside it); returns the screen output.  A non-zero exit raises with the
    output's tail."""
    os.makedirs(workdir, exist_ok=True)
    for f in files:
        src = os.path.join(GOLDEN, f)
        if os.path.exists(src) and not os.path.exists(os.path.join(workdir, f)):
            shutil.copy(src, workdir)
    with open(os.path.join(workdir, "in.test"), "w") as fh:
        fh.write(script)
    e = dict(os.environ)
    e.setdefault("OMP_NUM_THREADS", "1")
    if env:
        e.update(env)
    r = subprocess.run([exe, "-in", "in.test", "-log", "log.test", *args], cwd=workdir,
                       capture_output=True, text=True, env=e, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"{os.path.basename(exe)} exited {r.returncode}:\n"
                           f"{(r.stdout + r.stderr)[-3000:]}")
    return r.stdout


def parse_log(text):
    """Thermo rows (column -> printed string), neighbor statistics and the
    loop time of the last run in a LAMMPS screen output."""
    lines = text.splitlines()
    rows, cols = [], None
    for ln in lines:
        t = ln.split()
        if t and t[0] == "Step":
            cols, rows = t, []
            continue
        if cols and t and len(t) == len(cols) and re.fullmatch(r"-?\d+", t[0]):
            rows.append(dict(zip(cols, t)))
            continue
        if ln.startswith("Loop time"):
            cols = None
    out = {"rows": rows}
    for key, pat in (("neighbors", r"Total # of neighbors = (\S+)"),
                     ("builds", r"Neighbor list builds = (\d+)"),
                     ("dangerous", r"Dangerous builds = (\d+)"),
                     ("loop_time", r"Loop time of (\S+) on")):
        m = re.findall(pat, text)
        if m:
            out[key] = float(m[-1]) if key in ("loop_time", "neighbors") else int(m[-1])
    return out


def read_dump(path):
    """{step: array (natoms, ncols)} of a `dump custom` text file sorted by id."""
    frames, step = {}, None
    with open(path) as fh:
        lines = fh.read().splitlines()
    k = 0
    while k < len(lines):
        if lines[k].startswith("ITEM: TIMESTEP"):
            step = int(lines[k + 1])
            k += 2
        elif lines[k].startswith("ITEM: NUMBER OF ATOMS"):
            n = int(lines[k + 1])
            k += 2
        elif lines[k].startswith("ITEM: ATOMS"):
            frames[step] = np.loadtxt(lines[k + 1:k + 1 + n], ndmin=2)
            k += 1 + n
        else:
            k += 1
    return frames
