"""Pin the CPU oracle against the reference's own golden logs.

The reference ships no unit tests; its regression harness compares printed
thermo columns of ``bench/in.*`` and ``examples/melt`` runs with stored logs
(regress/benchmark.py:22-80).  The oracle must reproduce those printed values
digit for digit (thermo format %.8g, src/thermo.cpp), together with the
ghost-atom count, neighbor-pair total and neighbor-build counts printed at the
end of each run.
"""
import json
import os

import pytest

import oracle
from oracle_cases import build_oracle_case

with open(os.path.join(os.path.dirname(__file__), "golden", "reference_logs.json")) as fh:
    LOGS = json.load(fh)


def _fmt(v):
    return "%.8g" % v


@pytest.mark.parametrize("name", ["bench_lj", "bench_eam", "potentials_lj", "potentials_eam", "melt"])
def test_oracle_reproduces_reference_log(name):
    case = LOGS[name]
    sim = build_oracle_case(case, threads=1)
    sim.setup()
    sim.run(case["run"])
    rows = sim.thermo_rows()
    ref = case["thermo_rows"]
    assert len(rows) == len(ref)
    for got, want in zip(rows, ref):
        assert int(got[0]) == int(want["Step"])
        assert _fmt(got[1]) == want["Temp"], (name, want["Step"], "Temp")
        assert _fmt(got[2]) == want["E_pair"], (name, want["Step"], "E_pair")
        assert _fmt(got[3]) == want["TotEng"], (name, want["Step"], "TotEng")
        assert _fmt(got[4]) == want["Press"], (name, want["Step"], "Press")
    st = case["stats"]
    assert sim.neigh_total == st["neighbors"]
    assert sim.ncalls == st["builds"]
    assert sim.ndanger == st["dangerous"]
    assert str(sim.nghost) == st["nghost_ave"]


def test_four_process_log_matches_serial():
    """The 4-process log prints the same thermo as the serial one; so does the oracle."""
    a, b = LOGS["bench_lj"], LOGS["bench_lj_np4"]
    assert a["thermo_rows"] == b["thermo_rows"]
    assert a["stats"]["neighbors"] == b["stats"]["neighbors"]


def test_threaded_oracle_agrees_with_serial():
    case = LOGS["melt"]
    s1 = build_oracle_case(case, threads=1)
    s4 = build_oracle_case(case, threads=4)
    for s in (s1, s4):
        s.setup()
        s.run(40)
    r1, r4 = s1.thermo_rows(), s4.thermo_rows()
    assert abs(r1[-1][2] - r4[-1][2]) < 1e-10 * abs(r1[-1][2])
    assert s1.neigh_total == s4.neigh_total
