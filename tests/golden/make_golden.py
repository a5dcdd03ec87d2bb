"""Extract the reference's golden thermo lines and neighbor statistics.

Reads the log files that ship with the reference (LAMMPS 8 Aug 2014) next to
their input scripts and writes ``reference_logs.json``: per case, the run
parameters (transcribed from the matching ``in.*`` script) and the printed
thermo rows, ghost count, neighbor total and build counts.  Also copies the
``Cu_u3.eam`` funcfl table the EAM benchmark reads.

Run from the repository root, naming the reference checkout (the directory
that holds bench/, examples/ and src/) as the argument or in LAMMPS_ROOT:

    python tests/golden/make_golden.py REFERENCE
"""
import json
import os
import re
import shutil
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LAMMPS_ROOT")
if not REF:
    sys.exit("usage: make_golden.py REFERENCE  (or set LAMMPS_ROOT)")
HERE = os.path.dirname(os.path.abspath(__file__))

# Run parameters of each input script.  lattice "fcc" with rho* (lj units) or
# the lattice constant (metal units); box = block 0 n 0 n 0 n in lattice units.
CASES = {
    "bench_lj": {
        "log": "bench/log.1Feb14.lj.fixed.linux.1", "input": "bench/in.lj",
        "units": "lj", "lattice": 0.8442, "cells": [20, 20, 20], "mass": 1.0,
        "velocity": {"t": 1.44, "seed": 87287, "loop": "geom", "dist": "uniform"},
        "pair": {"style": "lj/cut", "cut": 2.5, "eps": 1.0, "sigma": 1.0},
        "neighbor": {"skin": 0.3, "every": 20, "delay": 0, "check": False},
        "dt": 0.005, "thermo": 0, "run": 100,
    },
    "bench_lj_np4": {
        "log": "bench/log.1Feb14.lj.fixed.linux.4", "input": "bench/in.lj", "same_as": "bench_lj",
    },
    "bench_eam": {
        "log": "bench/log.1Feb14.eam.fixed.linux.1", "input": "bench/in.eam",
        "units": "metal", "lattice": 3.615, "cells": [20, 20, 20],
        "velocity": {"t": 1600.0, "seed": 376847, "loop": "geom", "dist": "uniform"},
        "pair": {"style": "eam", "file": "Cu_u3.eam"},
        "neighbor": {"skin": 1.0, "every": 1, "delay": 5, "check": True},
        "dt": 0.005, "thermo": 50, "run": 100,
    },
    "potentials_lj": {
        "log": "bench/POTENTIALS/log.26Jun12.lj.1", "input": "bench/POTENTIALS/in.lj",
        "units": "lj", "lattice": 0.8442, "cells": [20, 20, 20], "mass": 1.0,
        "velocity": {"t": 1.44, "seed": 87287, "loop": "geom", "dist": "uniform"},
        "pair": {"style": "lj/cut", "cut": 2.5, "eps": 1.0, "sigma": 1.0},
        "neighbor": {"skin": 0.3, "every": 1, "delay": 5, "check": True},
        "dt": 0.005, "thermo": 0, "run": 100,
    },
    "potentials_eam": {
        "log": "bench/POTENTIALS/log.26Jun12.eam.1", "input": "bench/POTENTIALS/in.eam",
        "units": "metal", "lattice": 3.615, "cells": [20, 20, 20],
        "velocity": {"t": 1600.0, "seed": 376847, "loop": "geom", "dist": "uniform"},
        "pair": {"style": "eam", "file": "Cu_u3.eam"},
        "neighbor": {"skin": 1.0, "every": 1, "delay": 5, "check": True},
        "dt": 0.005, "thermo": 0, "run": 100,
    },
    "melt": {
        "log": "examples/melt/log.melt.1Feb14.linux.1", "input": "examples/melt/in.melt",
        "units": "lj", "lattice": 0.8442, "cells": [10, 10, 10], "mass": 1.0,
        "velocity": {"t": 3.0, "seed": 87287, "loop": "all", "dist": "uniform"},
        "pair": {"style": "lj/cut", "cut": 2.5, "eps": 1.0, "sigma": 1.0},
        "neighbor": {"skin": 0.3, "every": 20, "delay": 0, "check": False},
        "dt": 0.005, "thermo": 50, "run": 250,
    },
}


def parse_log(path):
    rows, stats = [], {}
    with open(path) as fh:
        lines = fh.read().splitlines()
    for k, line in enumerate(lines):
        if line.startswith("Step "):
            cols = line.split()
            for nxt in lines[k + 1:]:
                if not re.match(r"^\s*\d", nxt):
                    break
                vals = nxt.split()
                rows.append({c: v for c, v in zip(cols, vals)})
        m = re.match(r"^Nghost:\s+(\S+) ave", line)
        if m:
            stats["nghost_ave"] = m.group(1)
        m = re.match(r"^Total # of neighbors = (\d+)", line)
        if m:
            stats["neighbors"] = int(m.group(1))
        m = re.match(r"^Neighbor list builds = (\d+)", line)
        if m:
            stats["builds"] = int(m.group(1))
        m = re.match(r"^Dangerous builds = (\d+)", line)
        if m:
            stats["dangerous"] = int(m.group(1))
    return rows, stats


def main():
    out = {}
    for name, case in CASES.items():
        rows, stats = parse_log(os.path.join(REF, case["log"]))
        entry = dict(case)
        entry["thermo_rows"] = rows
        entry["stats"] = stats
        out[name] = entry
    with open(os.path.join(HERE, "reference_logs.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
    shutil.copyfile(os.path.join(REF, "bench", "Cu_u3.eam"), os.path.join(HERE, "Cu_u3.eam"))
    print("wrote", len(out), "cases")


if __name__ == "__main__":
    main()
