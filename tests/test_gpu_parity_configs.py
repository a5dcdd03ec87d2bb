"""Parity with the oracle on the benchmark configurations themselves.

The oracle (pinned atom by atom against the reference's own binary in
tests/test_oracle_vs_reference.py) runs each configuration from its seeded
initial state; the CUDA engine, through the C ABI, gets the oracle's
positions and must reproduce its neighbor lists and forces:

  - 32,000-atom LJ with Gaussian velocities (fcc 20^3, rho* 0.8442, T* 1.44,
    rc 2.5, skin 0.3);
  - 32,000-atom EAM with the synthetic 5000-point setfl tables through
    eam/alloy (fcc 20^3, a = 3.615 A, 1600 K Gaussian, skin 1.0);
  - per-atom energy and virial (eflag_atom / vflag_atom: Pair::ev_tally's
    eatom[i] += epairhalf and vatom[i][k] += 0.5 v[k], src/pair.cpp:795,838,
    and the embedding energy eatom[i] += phi of src/MANYBODY/pair_eam.cpp:226),
    LJ and EAM;
  - batched replicas, each replica against its own oracle run;
  - 4,000,000-atom LJ (fcc 100^3) at step 0 and after 10 steps.

Bars: half lists bit-exact as sorted per-atom sets of (owner, image); FP64
forces, energy, virial, density and embedding derivative within 1e-12
(norm-wise relative for per-atom arrays, off-diagonal virial relative to
|trace|); mixed precision within 1e-5 of the oracle.
"""
import os

import numpy as np
import pytest

import oracle
from gpu_cases import force_errors, virial_errors
from lammps_b200 import PairEAMAlloy, PairLJCut, System, inputs

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 1e-5
THREADS = os.cpu_count() or 4


# ---------------------------------------------------------------------------
# cases

def lj_case(cells):
    a = inputs.lj_lattice_constant("fcc", 0.8442)
    x = inputs.lattice("fcc", cells, cells, cells, a)
    return dict(kind="lj", x=x, hi=np.array([cells * a] * 3), t=1.44, seed=87287, skin=0.3,
                every=20, delay=0, check=False, units="lj")


def eam_case(setfl):
    x = inputs.lattice("fcc", 20, 20, 20, 3.615)
    return dict(kind="eam", x=x, hi=np.array([20 * 3.615] * 3), t=1600.0, seed=376847, skin=1.0,
                every=1, delay=5, check=True, units="metal", setfl=setfl)


def oracle_sim(case):
    s = oracle.OracleSim(case["units"], threads=THREADS)
    s.box([0.0, 0.0, 0.0], case["hi"])
    s.atoms(case["x"])
    if case["kind"] == "lj":
        s.mass(1, 1.0)
        s.lj_cut(2.5)
        s.lj_coeff(1, 1, 1.0, 1.0, 2.5)
    else:
        s.eam_setfl(case["setfl"], [0])
    s.velocity_create(case["t"], case["seed"], gaussian=True, loop_geom=True)
    s.neighbor(case["skin"], case["every"], case["delay"], case["check"], 1000)
    s.timestep(0.005)
    return s


def snapshot(s, per_atom=False, half=True):
    """State of the oracle: forces from its own step, then a compute on the
    same positions with energy, virial (and per-atom tallies)."""
    s.compute(eflag=3 if per_atom else 1, vflag=5 if per_atom else 1)
    out = dict(x=s.x, type=s.type, f=s.f, eng=s.eng_vdwl, virial=s.virial)
    if half:
        out["half"] = s.half_list()
    if per_atom:
        out["eatom"], out["vatom"] = s.eatom_vatom()
    return out


def device(case, precision, snap):
    d = System(case["units"], precision)
    d.set_box([0.0, 0.0, 0.0], case["hi"])
    if case["kind"] == "lj":
        p = PairLJCut(2.5)
        p.coeff(1, 1, 1.0, 1.0, 2.5)
        d.set_pair(p)
        d.set_mass([1.0])
    else:
        p = PairEAMAlloy(1)
        p.coeff(case["setfl"], ["Cu"])
        d.set_pair(p)
    d.set_neighbor(case["skin"], case["every"], case["delay"], case["check"])
    d.set_atoms(snap["x"], snap["type"], None)
    d.neigh_build()
    return d


def exact_totals(snap):
    """Energy and virial of the oracle's state as exactly rounded sums of its
    per-atom tallies.  The oracle's own totals are sequential sums, like the
    reference's: on the 4M-atom lattice, where every pair term is nearly the
    same, their rounding drifts one way and the total is off by ~1e-10
    relative, more than the bar; the per-atom tallies (sums of ~40 terms)
    are exact to ~1e-15."""
    import math
    eng = math.fsum(snap["eatom"])
    vir = np.array([math.fsum(snap["vatom"][:, k]) for k in range(6)])
    return eng, vir


def check_forces(d, snap, tol, fscale=None):
    r = d.compute(eflag=1, vflag=1)
    f = d.download()["f"]
    if fscale is None:
        rel, mx = force_errors(f, snap["f"])
        assert rel <= tol, rel
    else:  # on the lattice the forces cancel: compare against a force scale
        assert float(np.abs(f - snap["f"]).max()) <= tol * fscale
    eng, vir = exact_totals(snap) if "eatom" in snap else (snap["eng"], snap["virial"])
    assert abs(r["eng"] - eng) <= tol * abs(eng), (r["eng"], eng)
    dg, off = virial_errors(r["virial"], vir)
    assert dg <= tol and off <= tol, (dg, off)


def canonical_half(num, jo, ji):
    """Every (atom, owner, image) entry as one sorted int64 key: equal keys
    mean equal per-atom sets."""
    n = len(num)
    atom = np.repeat(np.arange(n, dtype=np.int64), num)
    key = atom * (27 * np.int64(n)) + jo.astype(np.int64) * 27 + ji.astype(np.int64)
    key.sort()
    return key


def check_half(d, snap):
    num, jo, ji = d.half_list()
    onum, ojo, oji = snap["half"]
    assert np.array_equal(num, onum)
    assert np.array_equal(canonical_half(num, jo, ji), canonical_half(onum, ojo, oji))


# ---------------------------------------------------------------------------
# 32,000-atom LJ, Gaussian velocities

@pytest.fixture(scope="module")
def lj32k():
    case = lj_case(20)
    s = oracle_sim(case)
    s.setup()
    s.run(10)
    return case, snapshot(s, per_atom=True)


def test_lj32k_gaussian_fp64(lj32k):
    case, snap = lj32k
    d = device(case, "fp64", snap)
    check_half(d, snap)
    check_forces(d, snap, FP64_TOL)


def test_lj32k_gaussian_mixed(lj32k):
    case, snap = lj32k
    check_forces(device(case, "mixed", snap), snap, MIXED_TOL)


@pytest.mark.parametrize("tpa", [1, 2, 4, 8, 16, 32])
def test_lj32k_mixed_every_launch_shape(lj32k, tpa):
    """The mixed pair kernel in each launch shape: one thread per atom walks
    its slabs; several lanes per atom take consecutive list entries."""
    case, snap = lj32k
    d = device(case, "mixed", snap)
    d.set_launch(tpa)
    check_forces(d, snap, MIXED_TOL)


def _run_from_oracle_state(case, precision, tpa, steps):
    """Largest position difference (minimum image) between the engine and
    the oracle after `steps` steps from the oracle's state after 10 steps,
    both with the same list schedule (a rebuild at the start, then the
    case's every / delay / check rule)."""
    s10 = oracle_sim(case)
    s10.setup()
    s10.run(10)
    o10 = np.argsort(s10.tag)
    x10, t10, v10 = s10.x[o10], s10.type[o10], s10.v[o10]
    s10.close()
    o = oracle.OracleSim(case["units"], threads=THREADS)
    o.box([0.0, 0.0, 0.0], case["hi"])
    o.atoms(x10, v=v10)
    if case["kind"] == "lj":
        o.mass(1, 1.0)
        o.lj_cut(2.5)
        o.lj_coeff(1, 1, 1.0, 1.0, 2.5)
    else:
        o.eam_setfl(case["setfl"], [0])
    o.neighbor(case["skin"], case["every"], case["delay"], case["check"], 1000)
    o.timestep(0.005)
    o.setup()
    o.run(steps)
    ox = o.x[np.argsort(o.tag)]
    o.close()
    d = System(case["units"], precision)
    d.set_box([0.0, 0.0, 0.0], case["hi"])
    if case["kind"] == "lj":
        p = PairLJCut(2.5)
        p.coeff(1, 1, 1.0, 1.0, 2.5)
        d.set_pair(p)
        d.set_mass([1.0])
    else:
        p = PairEAMAlloy(1)
        p.coeff(case["setfl"], ["Cu"])
        d.set_pair(p)
    d.set_neighbor(case["skin"], case["every"], case["delay"], case["check"])
    if tpa:
        d.set_launch(tpa)
    d.set_atoms(x10, t10, v10)
    d.set_timestep(0.005)
    d.setup()
    d.run(steps)
    st = d.download()
    d.close()
    # the two runs wrap atoms into the box at different steps
    d_x = st["x"] - ox
    d_x -= case["hi"] * np.round(d_x / case["hi"])
    return float(np.max(np.abs(d_x)))


@pytest.mark.parametrize("tpa", [1, 2, 4, 8])
@pytest.mark.parametrize("precision,bar", [("fp64", 1e-9), ("mixed", 1e-4)])
def test_lj32k_step_every_launch_shape(lj32k, precision, bar, tpa):
    """The one-launch MD step (forces and both half-steps) in each launch
    shape, 20 steps against the oracle's.  Two runs whose lists are rebuilt at
    different steps legitimately drift apart by ~1e-4 in 20 steps here: with
    rebuilds every 20 steps and no displacement check, pairs come within the
    cutoff between rebuilds.  With the same schedule, positions must agree
    within 1e-9 (FP64).  For mixed precision, a pair within FP32 rounding of
    the cutoff may be counted on one side and not the other for a step,
    which moves positions by up to ~1e-5, so the bar is 1e-4.  A wiring
    mistake in the step (a force lost or doubled) moves them by ~1e-2."""
    case, _ = lj32k
    dx = _run_from_oracle_state(case, precision, tpa, 20)
    print(precision, "tpa", tpa, "max |dx|", dx)
    assert dx <= bar, dx


@pytest.mark.parametrize("precision,bar", [("fp64", 1e-9), ("mixed", 1e-3)])
def test_lj32k_run_repeats_the_launch_shape_search(lj32k, precision, bar):
    """With the launch shape left to the search, the first run repeats the
    search 50 steps in, between two steps, and may switch shapes there; the
    state is left as it was, so 100 steps stay on the oracle's own 100.  The
    mixed bar is wider than over 20 steps: more cutoff-rounding events, each
    grown over more steps; a lost or doubled force would move atoms ~0.1."""
    case, _ = lj32k
    dx = _run_from_oracle_state(case, precision, 0, 100)
    print(precision, "searched", "max |dx|", dx)
    assert dx <= bar, dx


# ---------------------------------------------------------------------------
# 32,000-atom EAM, synthetic 5000-point setfl tables

@pytest.fixture(scope="module")
def eam32k(tmp_path_factory):
    from lammps_b200.eam_synth import write_setfl
    setfl = write_setfl(str(tmp_path_factory.mktemp("synth") / "Cu_synth.eam.alloy"))
    case = eam_case(setfl)
    s = oracle_sim(case)
    s.setup()
    s.run(10)
    snap = snapshot(s, per_atom=True)
    snap["rho"], snap["fp"] = s.rho_fp()
    return case, snap


def test_eam32k_synthetic_fp64(eam32k):
    case, snap = eam32k
    d = device(case, "fp64", snap)
    check_half(d, snap)
    check_forces(d, snap, FP64_TOL)
    rho, fp = d.rho_fp()
    assert np.max(np.abs(rho - snap["rho"]) / np.abs(snap["rho"])) <= FP64_TOL
    assert np.max(np.abs(fp - snap["fp"]) / np.abs(snap["fp"])) <= FP64_TOL


def test_eam32k_synthetic_mixed(eam32k):
    case, snap = eam32k
    check_forces(device(case, "mixed", snap), snap, MIXED_TOL)


@pytest.mark.parametrize("tpa", [1, 2, 4, 8])
@pytest.mark.parametrize("precision,bar", [("fp64", 1e-9), ("mixed", 1e-4)])
def test_eam32k_step_every_launch_shape(eam32k, precision, bar, tpa):
    """The one-launch EAM step (density pass, then forces and both
    half-steps) in each launch shape, 20 steps against the oracle's from the
    same state.  The lists are rebuilt on a displacement check with a 1.0 A
    skin, so they hold every pair within the cutoff whenever they are
    rebuilt.  A mixed decision that differs from the oracle's therefore
    changes no force.  Bars as for the LJ step."""
    case, _ = eam32k
    dx = _run_from_oracle_state(case, precision, tpa, 20)
    print("eam", precision, "tpa", tpa, "max |dx|", dx)
    assert dx <= bar, dx


# ---------------------------------------------------------------------------
# per-atom energy and virial

@pytest.mark.parametrize("style", ["lj", "eam"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_per_atom_energy_and_virial(style, precision, lj32k, eam32k):
    case, snap = lj32k if style == "lj" else eam32k
    tol = FP64_TOL if precision == "fp64" else MIXED_TOL
    d = device(case, precision, snap)
    r = d.compute(eflag=1, vflag=1, per_atom=True)
    ea, va = r["eatom"], r["vatom"]
    assert np.linalg.norm(ea - snap["eatom"]) <= tol * np.linalg.norm(snap["eatom"])
    assert np.linalg.norm(va - snap["vatom"]) <= tol * np.linalg.norm(snap["vatom"])
    # the tallies sum to the global energy and virial
    assert abs(ea.sum() - r["eng"]) <= 1e-12 * abs(r["eng"])
    assert np.allclose(va.sum(axis=0), r["virial"], rtol=1e-11, atol=1e-11 * abs(r["virial"][:3].sum()))


# ---------------------------------------------------------------------------
# batched replicas, each against its own oracle run

def test_replicas_each_match_their_oracle_run():
    from lammps_b200.replicas import make_batch, replica_batch
    batch = replica_batch(nrep=3, seed=777)
    steps = 45  # crosses two rebuilds (every 20)
    s = make_batch(batch, "fp64")
    s.setup()
    s.run(steps)
    rows = s.replica_thermo()
    st = s.download()
    s.close()
    a0 = np.concatenate([[0], np.cumsum(batch["natoms"])])
    for k in range(3):
        x = batch["x"][a0[k]:a0[k + 1]]
        v = batch["v"][a0[k]:a0[k + 1]]
        o = oracle.OracleSim("lj", threads=THREADS)
        o.box(batch["lo"][k], batch["hi"][k])
        o.atoms(x, v)
        o.mass(1, 1.0)
        o.lj_cut(2.5)
        o.lj_coeff(1, 1, 1.0, 1.0, 2.5)
        o.neighbor(0.3, 20, 0, False, 1000)
        o.timestep(0.005)
        o.thermo(steps)
        o.setup()
        o.run(steps)
        orow = o.thermo_rows()[-1]  # step, temp, epair, etotal, press
        order = np.argsort(o.tag)
        dx = np.max(np.abs(st["x"][a0[k]:a0[k + 1]] - o.x[order]))
        assert dx <= 1e-10, (k, dx)
        for key, col in (("Temp", 1), ("E_pair", 2), ("TotEng", 3), ("Press", 4)):
            assert abs(rows[k][key] - orow[col]) <= 1e-10 * abs(orow[col]), (k, key)


# ---------------------------------------------------------------------------
# 4,000,000-atom LJ

@pytest.fixture(scope="module")
def lj4m():
    case = lj_case(100)
    s = oracle_sim(case)
    s.setup()
    s0 = snapshot(s, per_atom=True)
    s.run(10)
    s10 = snapshot(s, per_atom=True)
    s.close()
    return case, s0, s10


def test_lj4m_step0_fp64(lj4m):
    case, s0, s10 = lj4m
    d = device(case, "fp64", s0)
    check_half(d, s0)
    fscale = float(np.sqrt(np.mean(np.sum(s10["f"] ** 2, axis=1))))
    check_forces(d, s0, FP64_TOL, fscale=fscale)


def test_lj4m_step10_fp64(lj4m):
    case, _, s10 = lj4m
    d = device(case, "fp64", s10)
    check_half(d, s10)
    check_forces(d, s10, FP64_TOL)


def test_lj4m_step10_mixed(lj4m):
    case, _, s10 = lj4m
    check_forces(device(case, "mixed", s10), s10, MIXED_TOL)


# ---------------------------------------------------------------------------
# per-atom columns gathered on the device (what a dump writes)

def test_gather_columns_match_oracle_state(lj32k):
    """b200_gather of x, v, f and image flags after 50 FP64 steps against
    the oracle after the same 50 steps, and against a full download."""
    case = lj_case(20)
    steps = 50
    o = oracle_sim(case)
    o.setup()
    o.run(steps)
    order = np.argsort(o.tag)
    d = System("lj", "fp64")
    d.set_box([0.0, 0.0, 0.0], case["hi"])
    p = PairLJCut(2.5)
    p.coeff(1, 1, 1.0, 1.0, 2.5)
    d.set_pair(p)
    d.set_mass([1.0])
    d.set_neighbor(0.3, 20, 0, False)
    # the oracle's initial velocities in tag order (its own order is sorted
    # by cell at setup)
    o2 = oracle_sim(case)
    o2.setup()
    d.set_atoms(case["x"], None, o2.v[np.argsort(o2.tag)])
    o2.close()
    d.setup()
    d.run(steps)
    g = d.gather(("x", "v", "f", "image"))
    full = d.download()
    for k in ("x", "v", "f", "image"):
        assert np.array_equal(g[k], full[k]), k
    for k in ("x", "v", "f"):
        ref = getattr(o, k)[order]
        err = np.linalg.norm(g[k] - ref) / np.linalg.norm(ref)
        assert err <= 1e-10, (k, err)
    # the oracle's image flags against the device's crossings since upload
    assert np.array_equal(g["image"], o.image[order])
    idx = np.array([5, 31999, 0, 17], np.int32)
    sub = d.gather(("v", "image"), idx)
    assert np.array_equal(sub["v"], full["v"][idx])
    assert np.array_equal(sub["image"], full["image"][idx])
    with pytest.raises(Exception, match="outside"):
        d.gather(("x",), np.array([32000], np.int32))
    o.close()
