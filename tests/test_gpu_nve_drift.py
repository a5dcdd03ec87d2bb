"""NVE energy drift over 10^4 steps of the plain LJ configuration (32,000
atoms, rho* 0.8442, T* 1.44 Gaussian, every 20), FP64 and mixed, against the
oracle's drift (tests/golden/nve_drift_lj32k.json, made by
make_nve_drift.py).

Trajectories of a chaotic system separate after a few hundred steps, so the
comparison is statistical: the least-squares slope of TotEng(step) per atom
and the RMS fluctuation around that line.  FP64 must drift like the oracle
(both slopes are rounding-level); the mixed form, whose forces carry ~1e-6
relative error, must keep the drift below a bound that still makes it a
usable NVE integrator."""
import json
import os

import numpy as np
import pytest

from lammps_b200 import PairLJCut, System, inputs

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

HERE = os.path.dirname(os.path.abspath(__file__))
STEPS = 10000
EVERY = 100


@pytest.fixture(scope="module")
def ref():
    with open(os.path.join(HERE, "golden", "nve_drift_lj32k.json")) as fh:
        return json.load(fh)


def _run(precision):
    a = inputs.lj_lattice_constant("fcc", 0.8442)
    x = inputs.lattice("fcc", 20, 20, 20, a)
    v = inputs.velocity_create(x, np.ones(len(x), np.int32), np.array([0.0, 1.0]), 1.44, 87287,
                               "lj", gaussian=True, loop="geom")
    s = System("lj", precision)
    s.set_box([0.0] * 3, [20 * a] * 3)
    p = PairLJCut(2.5)
    p.coeff(1, 1, 1.0, 1.0, 2.5)
    s.set_pair(p)
    s.set_mass([1.0])
    s.set_neighbor(0.3, every=20, delay=0, check=False)
    s.set_timestep(0.005)
    s.set_thermo(EVERY)
    s.set_atoms(x, None, v)
    s.setup()
    s.run(STEPS)
    rows = s.thermo_rows
    s.close()
    steps = np.array([r["Step"] for r in rows], float)
    etot = np.array([r["TotEng"] for r in rows])
    return steps, etot


def _fit(steps, etot, start=1000):
    """Slope per step and RMS residual of TotEng after the first `start`
    steps (the lattice start relaxes during the first few hundred)."""
    m = steps >= start
    k, b = np.polyfit(steps[m], etot[m], 1)
    resid = etot[m] - (k * steps[m] + b)
    return k, float(np.sqrt(np.mean(resid ** 2)))


def _ref_fit(ref):
    return _fit(np.array(ref["steps"], float), np.array(ref["toteng"]))


def test_fp64_drift_matches_oracle(ref):
    steps, etot = _run("fp64")
    assert steps[0] == 0 and steps[-1] == STEPS
    # the same trajectory as the oracle's at first: sums in another order
    assert abs(etot[0] - ref["toteng"][0]) <= 1e-11 * abs(ref["toteng"][0])
    assert abs(etot[1] - ref["toteng"][1]) <= 1e-11 * abs(ref["toteng"][1])
    k, rms = _fit(steps, etot)
    k_ref, rms_ref = _ref_fit(ref)
    # later the trajectories separate; the drift rate (about -1.3e-7 per step
    # per atom for dt 0.005 with the unshifted cutoff) and the fluctuation
    # around it are properties of the integrator and must agree
    assert abs(k - k_ref) <= 0.1 * abs(k_ref), (k, k_ref)
    assert rms <= 1.5 * rms_ref, (rms, rms_ref)


def test_mixed_drift_bounded(ref):
    steps, etot = _run("mixed")
    k, rms = _fit(steps, etot)
    k_ref, rms_ref = _ref_fit(ref)
    assert abs(k - k_ref) <= 0.2 * abs(k_ref), (k, k_ref)
    assert rms <= 2.0 * rms_ref, (rms, rms_ref)
