"""The LAMMPS package on the GPU: the reference's own program with the B200
styles linked in (oracle/_ref/lmp_b200, made by oracle/build_ref.py from the
reference's sources and lammps_b200/lammps/) runs the benchmark inputs.

Each run must
  - instantiate the /b200 class, shown by the banner line the style prints
    at init (the -sf fallback of src/force.cpp:154-175 is silent, so a run
    that fell back to the plain style would otherwise pass unnoticed);
  - print the thermo digits of the reference's own logs
    (bench/log.1Feb14.{lj,eam}.fixed.linux.1, bench/POTENTIALS/log.26Jun12.lj.1),
    with the reference's neighbor-build and dangerous-build counts;
in both ways the package runs: per call (Pair::compute inside the
reference's Verlet::run, following its reneighbor schedule) and resident
(run_style verlet/b200 with fix nve/b200: the run advances on the device).
"""
import json
import os

import numpy as np
import pytest

from lammps_runs import GOLDEN, input_script, parse_log, run_lammps
from oracle import build_ref

pytestmark = pytest.mark.gpu

LMP = build_ref.lmp_b200()
needs_binary = pytest.mark.skipif(LMP is None, reason="lmp_b200 not built (python oracle/build_ref.py)")

with open(os.path.join(GOLDEN, "reference_logs.json")) as fh:
    LOGS = json.load(fh)

ENV = {"LD_LIBRARY_PATH": os.environ.get("LD_LIBRARY_PATH", "") + ":/usr/local/cuda/lib64",
       "B200_DEVICE": "0"}


def _styles(case, mode, precision="fp64"):
    """pair_style, fix and run_style of a mode."""
    pair = "lj/cut/b200" if case["pair"]["style"] == "lj/cut" else "eam/b200"
    if precision != "fp64":
        pair += " precision " + precision
    if mode == "per_call":
        return dict(pair_style=pair, fix="nve", run_style=None)
    return dict(pair_style=pair, fix="nve/b200", run_style="verlet/b200")


def _run(case, tmp, mode, precision="fp64", args=()):
    st = _styles(case, mode, precision)
    if case["pair"]["style"] == "lj/cut":
        # lj/cut/b200 takes the cutoff before the precision keyword
        name, _, rest = st["pair_style"].partition(" ")
        script = input_script(case, fix=st["fix"], run_style=st["run_style"])
        script = script.replace(f"pair_style lj/cut {case['pair']['cut']}",
                                f"pair_style {name} {case['pair']['cut']} {rest}".rstrip())
    else:
        script = input_script(case, pair_style=st["pair_style"], fix=st["fix"],
                              run_style=st["run_style"])
    text = run_lammps(LMP, script, str(tmp), args=args, env=ENV)
    return text, parse_log(text)


def _golden(case, out, exact=True, rel=0.0):
    """exact: every printed digit; else step 0 within `rel` in every column
    and the conserved TotEng within `rel` on every row."""
    ref = case["thermo_rows"]
    assert [r["Step"] for r in out["rows"]] == [r["Step"] for r in ref]
    for got, want in zip(out["rows"], ref):
        for col in ("Temp", "E_pair", "TotEng", "Press"):
            if exact:
                assert got[col] == want[col], (want["Step"], col, got[col], want[col])
            elif want["Step"] == "0" or col == "TotEng":
                g, w = float(got[col]), float(want[col])
                assert abs(g - w) <= rel * abs(w), (want["Step"], col, g, w)
    assert out["builds"] == case["stats"]["builds"]
    assert out["dangerous"] == case["stats"]["dangerous"]


@needs_binary
@pytest.mark.parametrize("name", ["bench_lj", "bench_eam", "potentials_lj"])
@pytest.mark.parametrize("mode", ["per_call", "resident"])
def test_lmp_b200_reproduces_reference_log(name, mode, tmp_path):
    case = LOGS[name]
    text, out = _run(case, tmp_path, mode)
    cls = "PairLJCutB200" if case["pair"]["style"] == "lj/cut" else "PairEAMB200"
    assert f"({cls})" in text
    assert ("resident mode" in text) == (mode == "resident")
    _golden(case, out)


@needs_binary
@pytest.mark.parametrize("name", ["bench_lj", "bench_eam"])
def test_suffix_b200_selects_the_device_styles(name, tmp_path):
    """`-sf b200` on the reference's unmodified input: lj/cut -> lj/cut/b200
    (eam -> eam/b200), nve -> nve/b200, verlet -> verlet/b200 (resident)."""
    case = LOGS[name]
    text = run_lammps(LMP, input_script(case), str(tmp_path), args=("-sf", "b200"), env=ENV)
    cls = "PairLJCutB200" if case["pair"]["style"] == "lj/cut" else "PairEAMB200"
    assert f"({cls})" in text and "resident mode" in text
    _golden(case, parse_log(text))


@needs_binary
@pytest.mark.parametrize("name", ["bench_lj", "bench_eam"])
def test_mixed_precision_keyword(name, tmp_path):
    """`precision mixed`: the step-0 thermo columns and the total energy of
    every row within 1e-5 of the reference's digits, and the same builds."""
    case = LOGS[name]
    text, out = _run(case, tmp_path, "resident", "mixed")
    assert "mixed precision" in text
    _golden(case, out, exact=False, rel=1e-5)


@needs_binary
@pytest.mark.parametrize("name", ["bench_lj", "bench_eam"])
def test_dump_custom_b200_matches_reference_dump(name, tmp_path):
    """`dump custom/b200` in a resident run (its columns gathered on the
    device at the output steps between the run's ends) against `dump custom`
    of the reference's own binary on the same input: positions, velocities
    and forces at steps 0, 50 and 100, and the image flags, which count the
    box crossings of the whole run."""
    from lammps_runs import read_dump
    ref_exe = build_ref.lmp_serial()
    if ref_exe is None:
        pytest.skip("reference binary not built")
    case = LOGS[name]
    cols = "id x y z vx vy vz fx fy fz ix iy iz"
    fmt = "\"%d" + " %.17g" * 9 + " %d %d %d\""

    def script(style):
        st = _styles(case, "resident")
        extra = [f"dump d all {style} 50 dump.txt {cols}", f"dump_modify d sort id format {fmt}"]
        if style == "custom":
            return input_script(case, extra=extra)
        if case["pair"]["style"] == "lj/cut":
            sc = input_script(case, fix=st["fix"], run_style=st["run_style"], extra=extra)
            return sc.replace("pair_style lj/cut ", "pair_style lj/cut/b200 ")
        return input_script(case, pair_style=st["pair_style"], fix=st["fix"],
                            run_style=st["run_style"], extra=extra)

    run_lammps(ref_exe, script("custom"), str(tmp_path / "ref"))
    text = run_lammps(LMP, script("custom/b200"), str(tmp_path / "b200"), env=ENV)
    assert "resident mode" in text
    ref = read_dump(str(tmp_path / "ref" / "dump.txt"))
    got = read_dump(str(tmp_path / "b200" / "dump.txt"))
    assert sorted(ref) == sorted(got) == [0, 50, 100]
    # on the step-0 lattice the forces cancel to ~1e-13: their differences
    # are measured against the RMS force of step 50
    frms = float(np.sqrt(np.mean(np.sum(ref[50][:, 7:10] ** 2, axis=1))))
    for step in (0, 50, 100):
        r, g = ref[step], got[step]
        assert np.array_equal(r[:, 0], g[:, 0])
        assert np.array_equal(r[:, 10:13], g[:, 10:13]), step  # image flags
        for c0, what in ((1, "x"), (4, "v"), (7, "f")):
            a, b = g[:, c0:c0 + 3], r[:, c0:c0 + 3]
            if step == 0 and what == "f":
                err = float(np.abs(a - b).max()) / frms
            else:
                err = np.linalg.norm(a - b) / np.linalg.norm(b)
            assert err <= 1e-9, (step, what, err)
    # some atoms crossed the box during the run
    assert np.abs(ref[100][:, 10:13]).sum() > 0
