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
