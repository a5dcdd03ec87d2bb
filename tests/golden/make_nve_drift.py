"""NVE energy drift of the plain FP64 LJ configuration over 10^4 steps, from
the CPU oracle (the reference's serial algorithm), as a fixture for the GPU
drift test.

Configuration: 32,000 atoms, fcc 20^3 at rho* 0.8442, eps = sigma = m = 1,
rc 2.5, skin 0.3, `neigh_modify every 20 delay 0 check no`, `velocity all
create 1.44 87287 dist gaussian mom yes loop geom`, dt 0.005, thermo every
100 steps.  Writes nve_drift_lj32k.json: the TotEng series (per atom, lj
units) and its least-squares slope per step.

    python tests/golden/make_nve_drift.py [threads]
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

STEPS = 10000
EVERY = 100


def main():
    threads = int(sys.argv[1]) if len(sys.argv) > 1 else (os.cpu_count() or 1)
    a = oracle.lj_lattice_scale("fcc", 0.8442)
    x = oracle.lattice("fcc", 20, 20, 20, a)
    hi = [20 * a] * 3
    s = oracle.OracleSim("lj", threads=threads)
    s.box([0.0, 0.0, 0.0], hi)
    s.atoms(x)
    s.mass(1, 1.0)
    s.lj_cut(2.5)
    s.lj_coeff(1, 1, 1.0, 1.0, 2.5)
    s.velocity_create(1.44, 87287, gaussian=True, loop_geom=True)
    s.neighbor(0.3, 20, 0, False, 1000)
    s.timestep(0.005)
    s.thermo(EVERY)
    t0 = time.time()
    s.setup()
    s.run(STEPS)
    rows = s.thermo_rows()
    # columns: Step, Temp, E_pair, TotEng, Press
    steps = [int(r[0]) for r in rows]
    etot = [float(r[3]) for r in rows]
    slope = float(np.polyfit(steps, etot, 1)[0])
    out = {"config": __doc__.split("\n\n")[1], "steps": steps, "toteng": etot,
           "slope_per_step": slope, "threads": threads, "seconds": time.time() - t0}
    with open(os.path.join(HERE, "nve_drift_lj32k.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print(f"slope {slope:.3e} per step over {STEPS} steps, {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
