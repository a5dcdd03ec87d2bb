"""The reference arm's sampling scheme against fresh runs of the reference.

bench.py times the reference's own program (oracle/_ref/lmp_serial) on
samples that each start from the seeded initial state.  It builds that state
once with the workload's own commands, saves it with write_restart, and runs
every sample in one process as `clear` + `read_restart` + the workload's pair,
neighbor, fix and timestep commands + `run`.  A sample must then be the same
run as a fresh process of the whole script: the same thermo rows to every
printed digit, for every sample of the loop.  Checked with the plain styles
(one thread) on the 32,000-atom LJ and EAM configurations.
"""
import os
import re
import subprocess

import pytest

import bench
from oracle import build_ref

LMP = build_ref.lmp_serial()
pytestmark = pytest.mark.skipif(LMP is None, reason="reference binary not built "
                                                    "(python oracle/build_ref.py)")

STEPS = 20
THERMO_ROW = re.compile(r"^\s+\d+\s+-?\d")


def _run(workdir, name, text):
    with open(os.path.join(workdir, name), "w") as fh:
        fh.write(text)
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run([LMP, "-in", name, "-log", "none", "-echo", "none"], cwd=workdir,
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.stdout + r.stderr)[-800:]
    return r.stdout


def _rows(out):
    return [line.split() for line in out.splitlines() if THERMO_ROW.match(line)]


@pytest.mark.parametrize("workload", ["lj32k", "eam32k"])
def test_restart_samples_equal_fresh_runs(workload, tmp_path):
    work = str(tmp_path)
    if workload == "eam32k":
        from lammps_b200.eam_synth import write_setfl
        write_setfl(os.path.join(work, "Cu_synth.eam.alloy"))
    script = bench.WORKLOADS[workload]["script"]
    fresh = _rows(_run(work, "in.fresh",
                       "\n".join(script + [f"thermo {STEPS // 2}", f"run {STEPS}"]) + "\n"))
    assert len(fresh) == 3
    prep, loop = bench.reference_scripts(workload, 2, STEPS)
    # the loop's thermo prints every STEPS steps: rows 0 and STEPS of each sample
    _run(work, "in.prep", prep)
    out = _run(work, "in.bench", loop)
    assert len(re.findall(r"Loop time of", out)) == 2
    assert _rows(out) == [fresh[0], fresh[2]] * 2


def test_replica_scripts_are_the_replica_batch(tmp_path):
    """The reference inputs of the batched-replica CPU rows build the same
    boxes as the batch the engine runs: for the three smallest replicas, the
    reference's thermo rows over 20 steps equal the oracle's run from the
    batch's own positions and velocities (to the printed digits)."""
    import numpy as np

    import oracle
    from lammps_b200.replicas import replica_batch

    b = replica_batch()
    start = np.concatenate([[0], np.cumsum(b["natoms"])])
    reps = bench.replica_scripts(20)
    for k in np.argsort(b["natoms"], kind="stable")[:3]:
        script = [("thermo 10" if line == "thermo 20" else line) for line in reps[k][1]]
        out = _run(str(tmp_path), f"in.rep{k}", "\n".join(script) + "\n")
        ref = [[float(v) for v in row] for row in _rows(out)]
        assert [r[0] for r in ref] == [0, 10, 20]
        o = oracle.OracleSim("lj", threads=1)
        o.box([0.0] * 3, b["hi"][k])
        o.atoms(b["x"][start[k]:start[k + 1]], b["v"][start[k]:start[k + 1]])
        o.mass(1, 1.0)
        o.lj_cut(2.5)
        o.lj_coeff(1, 1, 1.0, 1.0, 2.5)
        o.neighbor(0.3, 20, 0, False, 1000)
        o.timestep(0.005)
        o.thermo(10)
        o.setup()
        o.run(20)
        rows = o.thermo_rows()
        o.close()
        assert len(rows) == 3, k
        for r, orow in zip(ref, rows):
            # printed: Step Temp E_pair E_mol TotEng Press; oracle: step temp epair etotal press
            for col, ocol in ((1, 1), (2, 2), (4, 3), (5, 4)):
                assert r[col] == pytest.approx(orow[ocol], rel=2e-7, abs=1e-7), (k, r[0], col)
