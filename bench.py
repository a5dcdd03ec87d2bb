#!/usr/bin/env python
"""Throughput of the short-range MD step on B200, in Matom-steps/s.

Headline workload (one bench step = the first 100 NVE timesteps from the
seeded initial state; restore and Verlet setup are untimed): the
4,000,000-atom LJ configuration -- fcc 100^3 at rho* 0.8442, Gaussian
velocities at T* 1.44 (seed 87287, loop geom), lj/cut rc 2.5, skin 0.3,
rebuild every 20 steps, dt 0.005 -- in FP32-mixed precision, with the FP64
form, their ratio and both forms' errors against the oracle beside it.  The
32,000-atom EAM configuration (synthetic 5000-point setfl tables) is a block
of its own (eam_32k) with the same figures.  Inputs are seeded synthetic data
of the reference's benchmark shapes.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Timing: W untimed bench steps, then K bench steps bracketed by a barrier and
torch.cuda.synchronize(); each bench step is timed with CUDA events on the
engine's stream, after an L2 flush (a 256 MB write) that is outside the
events.  `value` is the aggregate over ranks (max time over ranks).  `e2e` is
the same metric through the public API with page-locked host buffers: upload
of x, v, type, setup, 100 steps, download of x, v, f, image per bench step,
each step's copies overlapping its neighbours' device work (staged upload,
asynchronous download), wall clock from the first upload to the last
download; `e2e.blocking_value` is the same with blocking calls.  Under
torchrun each rank runs its own replica (weak
scaling, no data-path collective).  `--impl reference` times the reference's
own CPU build (oracle/_ref/lmp_serial, -sf omp on all host cores) on the same
workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Matom-steps/s LJ+EAM: FP32-mixed vs FP64 on 1 B200 at ≤1e-5 rel force error"
MD_STEPS = 100          # NVE timesteps per bench step
DEVICE = 0              # CUDA device of this rank
FLUSH_BYTES = 256 << 20  # > 126 MB L2


# ---------------------------------------------------------------------------
# workloads

def eam32k_inputs():
    from lammps_b200 import inputs
    x = inputs.lattice("fcc", 20, 20, 20, 3.615)
    v = inputs.velocity_create(x, np.ones(len(x), np.int32), np.array([0.0, 63.55]), 1600.0,
                               376847, "metal", gaussian=True, loop="geom")
    return x, v, np.array([20 * 3.615] * 3)


def eam4m_inputs():
    """The EAM workload at 4,000,000 atoms: fcc 100^3 at a = 3.615 A, the same
    Gaussian 1600 K velocities (seed 376847, loop geom)."""
    from lammps_b200 import inputs
    x = inputs.lattice("fcc", 100, 100, 100, 3.615)
    v = inputs.velocity_create(x, np.ones(len(x), np.int32), np.array([0.0, 63.55]), 1600.0,
                               376847, "metal", gaussian=True, loop="geom")
    return x, v, np.array([100 * 3.615] * 3)


def make_eam32k(precision, setfl, x, v, hi):
    from lammps_b200 import PairEAMAlloy, System
    s = System("metal", precision, device=DEVICE)
    s.set_box([0.0, 0.0, 0.0], hi)
    p = PairEAMAlloy(1)
    p.coeff(setfl, ["Cu"])
    s.set_pair(p)
    s.set_neighbor(1.0, every=1, delay=5, check=True)
    s.set_timestep(0.005)
    s.set_thermo(0)
    s.set_atoms(x, None, v)
    return s


def make_eam_cu(precision):
    """The reference's own EAM benchmark (bench/in.eam): Cu_u3 funcfl table,
    fcc 20^3 at a = 3.615, uniform velocities at 1600 K (seed 376847, loop
    geom), skin 1.0, every 1 delay 5 check yes, dt 5 fs."""
    from lammps_b200 import PairEAM, System, inputs
    x = inputs.lattice("fcc", 20, 20, 20, 3.615)
    s = System("metal", precision, device=DEVICE)
    s.set_box([0.0, 0.0, 0.0], [20 * 3.615] * 3)
    p = PairEAM(1)
    p.coeff(1, os.path.join(ROOT, "tests", "golden", "Cu_u3.eam"))
    s.set_pair(p)
    v = inputs.velocity_create(x, np.ones(len(x), np.int32), s.mass, 1600.0, 376847, "metal")
    s.set_neighbor(1.0, every=1, delay=5, check=True)
    s.set_timestep(0.005)
    s.set_thermo(0)
    s.set_atoms(x, None, v)
    return s, (x, v)


def lj4m_inputs():
    from lammps_b200 import inputs
    a = inputs.lj_lattice_constant("fcc", 0.8442)
    x = inputs.lattice("fcc", 100, 100, 100, a)
    v = inputs.velocity_create(x, np.ones(len(x), np.int32), np.array([0.0, 1.0]), 1.44, 87287,
                               "lj", gaussian=True, loop="geom")
    return x, v, np.array([100 * a] * 3)


def make_lj(precision, x, v, hi, atoms=True):
    from lammps_b200 import PairLJCut, System
    s = System("lj", precision, device=DEVICE)
    s.set_box([0.0, 0.0, 0.0], hi)
    p = PairLJCut(2.5)
    p.coeff(1, 1, 1.0, 1.0, 2.5)
    s.set_pair(p)
    s.set_mass([1.0])
    s.set_neighbor(0.3, every=20, delay=0, check=False)
    s.set_timestep(0.005)
    s.set_thermo(0)
    if atoms:
        s.set_atoms(x, None, v)
    return s


# ---------------------------------------------------------------------------
# clocks during the timed region

class NvmlClockSampler:
    """SM clock and clock-event reasons sampled in-process through NVML every
    `period` seconds while the timed region runs (the bench's timed region is
    tens of milliseconds, too short for nvidia-smi's 200 ms loop).  Reads
    only; changes no GPU setting."""

    def __init__(self, device, period=0.005):
        import pynvml
        import torch
        self.nv = pynvml
        pynvml.nvmlInit()
        pr = torch.cuda.get_device_properties(device)
        bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
        try:
            self.h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device)
        self.period = period
        self.samples = []
        self.stop_ev = threading.Event()
        self.t = None

    def _run(self):
        nv = self.nv
        while not self.stop_ev.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.samples.append((sm, rs))
            except Exception:
                pass
            self.stop_ev.wait(self.period)

    def start(self):
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def stop(self):
        self.stop_ev.set()
        if self.t:
            self.t.join(timeout=2)
        nv = self.nv
        try:
            mx = float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM))
        except Exception:
            mx = None
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        reasons = sorted({k for _, r in self.samples for k, b in bits.items() if r & b})
        sm = [float(c) for c, _ in self.samples]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": reasons, "samples": len(sm), "source": "nvml"}


def clock_sampler(device):
    """NVML sampler when NVML loads, else the nvidia-smi loop."""
    try:
        return NvmlClockSampler(device)
    except Exception:
        return ClockSampler(device)


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------

def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic():
    """dram bytes per launch of the profiled kernels, from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
            return json.load(fh)
    except Exception:
        return {}


STEP_BYTES_PER_ATOM = 96.0  # one-launch LJ step: x and v read and written (FP64)
EAM_BYTES_PER_ATOM_STEP = 200.0   # x, v, f, rho, fp traffic of one EAM step (FP64 state)
EAM_HALF_PAIRS = 21.0             # half pairs inside 4.95 A per atom on the fcc lattice
EAM_FLOP_PER_ATOM_STEP = 80.0 * EAM_HALF_PAIRS + 15.0


LJ_BYTES_PER_ATOM_STEP = 168.0   # x read for forces, f write, fused NVE x, v, f read, x, v write
LJ_HALF_PAIRS = 27.6             # half pairs inside rc = 2.5 per atom in the fluid at rho* 0.8442
LJ_FLOP_PER_ATOM_STEP = 27.0 * LJ_HALF_PAIRS


def step_roofline(n, step_ms, hbm_peak, clk, bytes_per_atom=EAM_BYTES_PER_ATOM_STEP,
                  flop_per_atom=EAM_FLOP_PER_ATOM_STEP):
    """Whole-step fractions: algorithmic bytes against the measured copy
    bandwidth and algorithmic FLOPs against the nominal FP32 FMA peak
    (148 SMs x 128 lanes x 2 FLOP x the sampled maximum SM clock)."""
    rate = n / (step_ms * 1e-3)  # atom-steps per second
    mhz = (clk or {}).get("sm_max_mhz") or 1965.0
    fp32_peak = 148 * 128 * 2 * mhz * 1e6 / 1e12
    gbs = bytes_per_atom * rate / 1e9
    tflops = flop_per_atom * rate / 1e12
    return {"alg_bytes_per_atom_step": bytes_per_atom, "achieved_gbs": gbs,
            "hbm_frac": gbs / hbm_peak, "alg_flop_per_atom_step": flop_per_atom,
            "achieved_tflops": tflops, "fp32_peak_tflops_nominal": fp32_peak,
            "fp32_frac": tflops / fp32_peak}


def device_time_run(sysm, torch, ext, flush, nsteps, start=None):
    """One bench step: (untimed) restore of the initial state and Verlet
    setup, L2 flush, then `nsteps` NVE steps timed with CUDA events on the
    engine's stream.  Restarting from the same state keeps every bench step
    the same workload: the synthetic EAM box is far from equilibrium and
    densifies as it runs, so a continuing trajectory would drift."""
    if start is not None:
        sysm.set_atoms(start[0], None, start[1])
        sysm.setup()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(ext):
        flush.zero_()
    e0.record(ext)
    sysm.run(nsteps)
    e1.record(ext)
    e1.synchronize()
    return e0.elapsed_time(e1)


def time_form(sysm, torch, flush, K, W, start, timing=False):
    """Warm up, then K timed bench steps; returns (total ms, per-step ms list)."""
    ext = torch.cuda.ExternalStream(sysm.stream)
    sysm.setup()
    sysm.set_timing(timing)
    for _ in range(W):
        device_time_run(sysm, torch, ext, flush, MD_STEPS, start)
    sysm.timing(reset=True)
    ms = [device_time_run(sysm, torch, ext, flush, MD_STEPS, start) for _ in range(K)]
    return sum(ms), ms


_PINNED = []  # torch tensors that own the page-locked memory of the e2e buffers


def pinned(torch, a):
    """A page-locked host copy of array `a` (a numpy view of a pinned torch tensor)."""
    t = torch.empty(a.shape, dtype=getattr(torch, str(a.dtype)), pin_memory=True)
    _PINNED.append(t)
    out = t.numpy()
    out[...] = a
    return out


def e2e_run(sysm, x_pin, v_pin, t_pin, out_pin, K):
    """Public-API end to end: page-locked host buffers in, host results out,
    per bench step (upload, setup, the MD steps, download)."""
    n = x_pin.shape[0]
    t0 = time.perf_counter()
    for _ in range(K):
        sysm.set_atoms(x_pin, t_pin, v_pin)
        sysm.setup()
        sysm.run(MD_STEPS)
        out = sysm.download(out_pin)
    t1 = time.perf_counter()
    h2d = x_pin.nbytes + v_pin.nbytes + t_pin.nbytes
    d2h = out["x"].nbytes + out["v"].nbytes + out["f"].nbytes + out["image"].nbytes
    return (t1 - t0) * 1e3, h2d, d2h


def e2e_run_overlapped(sysm, x_pin, v_pin, t_pin, outs, K):
    """e2e_run with each bench step's copies overlapping its neighbours'
    device work (b200_stage_atoms / b200_download_atoms_async): the next
    step's inputs are copied on the upload stream while this step runs, and
    this step's results are copied to the host on the download stream while
    the next one runs.  Every step's copies are inside the timed region: the
    clock starts before the first upload and stops after the last download
    has arrived."""
    n = x_pin.shape[0]
    t0 = time.perf_counter()
    sysm.stage_atoms(x_pin, t_pin, v_pin)
    for k in range(K):
        sysm.set_staged_atoms()
        if k + 1 < K:
            sysm.stage_atoms(x_pin, t_pin, v_pin)
        sysm.setup()
        sysm.run(MD_STEPS)
        sysm.download_async(outs[k % 2])
    sysm.wait_transfers()
    t1 = time.perf_counter()
    h2d = x_pin.nbytes + v_pin.nbytes + t_pin.nbytes
    d2h = sum(outs[0][k].nbytes for k in ("x", "v", "f", "image"))
    assert outs[0]["x"].shape == (n, 3)
    return (t1 - t0) * 1e3, h2d, d2h


def host_cpu():
    """The host's CPU model and the cores this process may use."""
    model = None
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count() or 1
    return {"model": model, "cores": cores}


# The reference's own CPU path: oracle/_ref/lmp_serial, the reference's
# LAMMPS built from its sources (oracle/build_ref.py), on the workload of the
# GPU arm -- the same lattice, velocities, potential, neighbor settings and
# timestep, from the seeded initial state, one process per sample.  One core:
# the plain styles; all cores: `-sf omp` (lj/cut/omp, eam/alloy/omp, nve/omp,
# OpenMP neighbor builds) with OMP_NUM_THREADS threads.
WORKLOADS = {
    "eam32k": {"atoms": 32000, "script": [
        "units metal", "atom_style atomic", "lattice fcc 3.615",
        "region box block 0 20 0 20 0 20", "create_box 1 box", "create_atoms 1 box",
        "pair_style eam/alloy", "pair_coeff * * Cu_synth.eam.alloy Cu",
        "velocity all create 1600.0 376847 dist gaussian loop geom",
        "neighbor 1.0 bin", "neigh_modify every 1 delay 5 check yes", "fix 1 all nve",
        "timestep 0.005"]},
    "lj32k": {"atoms": 32000, "script": [
        "units lj", "atom_style atomic", "lattice fcc 0.8442",
        "region box block 0 20 0 20 0 20", "create_box 1 box", "create_atoms 1 box",
        "mass 1 1.0", "velocity all create 1.44 87287 dist gaussian loop geom",
        "pair_style lj/cut 2.5", "pair_coeff 1 1 1.0 1.0 2.5", "neighbor 0.3 bin",
        "neigh_modify delay 0 every 20 check no", "fix 1 all nve", "timestep 0.005"]},
    "lj4m": {"atoms": 4000000, "script": [
        "units lj", "atom_style atomic", "lattice fcc 0.8442",
        "region box block 0 100 0 100 0 100", "create_box 1 box", "create_atoms 1 box",
        "mass 1 1.0", "velocity all create 1.44 87287 dist gaussian loop geom",
        "pair_style lj/cut 2.5", "pair_coeff 1 1 1.0 1.0 2.5", "neighbor 0.3 bin",
        "neigh_modify delay 0 every 20 check no", "fix 1 all nve", "timestep 0.005"]},
}


def reference_binary():
    p = os.path.join(ROOT, "oracle", "_ref", "lmp_serial")
    return p if os.access(p, os.X_OK) else None


# Commands of a workload that build its initial state (written once to a
# binary restart file, which holds positions, velocities, image flags, types
# and masses exactly) and commands each sample gives again after reading it.
SETUP_COMMANDS = ("units", "atom_style", "lattice", "region", "create_box", "create_atoms",
                  "velocity")


def reference_scripts(workload, samples, steps):
    """(preparation script, sampling script) of the reference's own program:
    the first builds the seeded initial state and writes it as a restart
    file; the second runs `samples` fresh runs of the first `steps` steps in
    one process, each from `clear` + `read_restart` of that state with the
    workload's pair, neighbor, fix and timestep commands."""
    w = WORKLOADS[workload]["script"]
    last = max(i for i, c in enumerate(w) if c.split()[0] == "velocity")
    prep = w[:last + 1] + ["write_restart start.restart"]
    again = [c for c in w if c.split()[0] not in SETUP_COMMANDS]
    loop = ([f"variable sample loop {samples}", "label next_sample", "clear",
             "read_restart start.restart"] + again +
            [f"thermo {steps}", f"run {steps}", "next sample", "jump SELF next_sample"])
    return "\n".join(prep) + "\n", "\n".join(loop) + "\n"


def reference_cpu(workload, threads, samples, steps=MD_STEPS, setfl=None, timeout=900):
    """Matom-steps/s of the reference's own binary: `samples` fresh runs of
    the first `steps` steps from the seeded state; the median of the `Loop
    time` rates (setup excluded, as the GPU arm's events exclude it).  The
    seeded state is built once (untimed) and each sample reads it back, so a
    sample costs its setup and its loop, not the lattice construction."""
    import re
    import shutil
    exe = reference_binary()
    w = WORKLOADS[workload]
    tmp = tempfile.mkdtemp(prefix="b200ref_")
    if setfl:
        shutil.copy(setfl, os.path.join(tmp, "Cu_synth.eam.alloy"))
    prep, loop = reference_scripts(workload, samples, steps)
    for name, text in (("in.prep", prep), ("in.bench", loop)):
        with open(os.path.join(tmp, name), "w") as fh:
            fh.write(text)
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    base = [exe, "-log", "none", "-echo", "none"] + (["-sf", "omp"] if threads > 1 else [])
    try:
        out = ""
        for name, limit in (("in.prep", timeout), ("in.bench", timeout * max(1, samples))):
            r = subprocess.run(base + ["-in", name], cwd=tmp, env=env, capture_output=True,
                               text=True, timeout=limit)
            if r.returncode != 0:
                raise RuntimeError(f"lmp_serial {name} failed ({r.returncode}): "
                                   f"{(r.stdout + r.stderr)[-500:]}")
            out = r.stdout
        secs = [float(s) for s in re.findall(r"Loop time of (\S+) on", out)]
        if len(secs) != samples:
            raise RuntimeError(f"lmp_serial ran {len(secs)} of {samples} samples: {out[-500:]}")
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    rates = [w["atoms"] * steps / s / 1e6 for s in secs]
    style = "-sf omp, " if threads > 1 else "plain styles, "
    return dict(value=statistics.median(rates), unit="Matom-steps/s", cores=threads,
                kind="reference", samples=rates,
                sample=f"{workload}: {samples} fresh runs of the first {steps} NVE steps from the "
                       f"seeded state (built once, written with write_restart, read back by each "
                       f"run), reference lmp_serial ({style}{threads} thread(s)) in one process, "
                       f"median of the Loop-time rates ({sum(secs):.1f} s of loop time)")


def port_cpu(setfl, x, v, hi, threads, samples):
    """Fallback when the reference binary is absent: the oracle port of the
    reference's algorithm on the same first-100-steps workload."""
    import oracle
    rates, secs = [], []
    for _ in range(samples):
        s = oracle.OracleSim("metal", threads=threads)
        s.box([0.0, 0.0, 0.0], hi)
        s.atoms(x, v)
        s.eam_setfl(setfl, [0])
        s.neighbor(1.0, 1, 5, True, 1000)
        s.timestep(0.005)
        s.setup()
        t0 = time.perf_counter()
        s.run(MD_STEPS)
        secs.append(time.perf_counter() - t0)
        rates.append(len(x) * MD_STEPS / secs[-1] / 1e6)
        s.close()
    return dict(value=statistics.median(rates), unit="Matom-steps/s", cores=threads, kind="port",
                samples=rates,
                sample=f"eam32k: {samples} runs of the first {MD_STEPS} NVE steps from the seeded "
                       f"state, oracle port (OpenMP {threads} threads), median ({sum(secs):.1f} s)")


def port_cpu_lj4m(threads, samples, steps):
    """Fallback when the reference binary is absent: the oracle port on the
    LJ-4M workload's first `steps` steps."""
    import oracle
    from lammps_b200 import inputs
    a = inputs.lj_lattice_constant("fcc", 0.8442)
    rates, secs = [], []
    for _ in range(samples):
        o = oracle.OracleSim("lj", threads=threads)
        o.box([0.0, 0.0, 0.0], [100 * a] * 3)
        o.atoms(oracle.lattice("fcc", 100, 100, 100, a))
        o.mass(1, 1.0)
        o.lj_cut(2.5)
        o.lj_coeff(1, 1, 1.0, 1.0, 2.5)
        o.velocity_create(1.44, 87287, gaussian=True, loop_geom=True)
        o.neighbor(0.3, 20, 0, False, 1000)
        o.timestep(0.005)
        o.setup()
        t0 = time.perf_counter()
        o.run(steps)
        secs.append(time.perf_counter() - t0)
        rates.append(4000000 * steps / secs[-1] / 1e6)
        o.close()
    return dict(value=statistics.median(rates), unit="Matom-steps/s", cores=threads, kind="port",
                samples=rates,
                sample=f"lj4m: {samples} runs of the first {steps} NVE steps from the seeded "
                       f"state, oracle port (OpenMP {threads} threads), median ({sum(secs):.1f} s)")


def cpu_baseline_eam32k(setfl, x, v, hi, samples=3):
    """All host cores (the baseline) plus a one-core row."""
    host = host_cpu()
    if reference_binary():
        out = reference_cpu("eam32k", host["cores"], samples, setfl=setfl)
        out["one_core"] = reference_cpu("eam32k", 1, 2, setfl=setfl)
    else:
        out = port_cpu(setfl, x, v, hi, host["cores"], samples)
        out["one_core"] = port_cpu(setfl, x, v, hi, 1, 1)
    out["cpu_model"] = host["model"]
    out["nproc"] = host["cores"]
    return out


def errors_vs(f, eng, vir, ref):
    """Force, energy and virial errors against a reference state: norm-wise
    relative force error and the largest |dF_i| over the RMS force; relative
    energy and virial diagonal; off-diagonal virial over |trace|."""
    d = f - ref["f"]
    rms = float(np.sqrt(np.mean(np.sum(ref["f"] ** 2, axis=1))))
    tr = abs(float(np.sum(ref["virial"][:3])))
    return {"force": float(np.linalg.norm(d) / np.linalg.norm(ref["f"])),
            "force_max_over_rms": float(np.max(np.linalg.norm(d, axis=1)) / rms),
            "energy": abs(eng - ref["eng"]) / abs(ref["eng"]),
            "virial_diag": float(np.max(np.abs(vir[:3] - ref["virial"][:3]) / np.abs(ref["virial"][:3]))),
            "virial_offdiag_over_trace": float(np.max(np.abs(vir[3:] - ref["virial"][3:])) / tr)}


def lj4m_oracle_state(hi, steps=10):
    """The oracle (all host threads) after `steps` steps of the LJ-4M
    configuration, with forces, energy and pairwise virial of that state."""
    import oracle
    from lammps_b200 import inputs
    a = inputs.lj_lattice_constant("fcc", 0.8442)
    o = oracle.OracleSim("lj", threads=host_cpu()["cores"])
    o.box([0.0, 0.0, 0.0], hi)
    o.atoms(oracle.lattice("fcc", 100, 100, 100, a))
    o.mass(1, 1.0)
    o.lj_cut(2.5)
    o.lj_coeff(1, 1, 1.0, 1.0, 2.5)
    o.velocity_create(1.44, 87287, gaussian=True, loop_geom=True)
    o.neighbor(0.3, 20, 0, False, 1000)
    o.timestep(0.005)
    o.setup()
    o.run(steps)
    o.compute(eflag=1, vflag=1)
    out = dict(x=o.x, f=o.f, eng=o.eng_vdwl, virial=o.virial)
    o.close()
    return out


def eam32k_oracle_state(setfl, x, hi, steps=10):
    """The oracle after `steps` steps of the EAM-32k configuration, with the
    forces, energy and pairwise virial of that state."""
    import oracle
    o = oracle.OracleSim("metal", threads=host_cpu()["cores"])
    o.box([0.0, 0.0, 0.0], hi)
    o.atoms(x)
    o.eam_setfl(setfl, [0])
    o.velocity_create(1600.0, 376847, gaussian=True, loop_geom=True)
    o.neighbor(1.0, 1, 5, True, 1000)
    o.timestep(0.005)
    o.setup()
    o.run(steps)
    o.compute(eflag=1, vflag=1)
    out = dict(x=o.x, f=o.f, eng=o.eng_vdwl, virial=o.virial)
    o.close()
    return out


def replica_bench(prec, batch, torch, steps=1000, lat_steps=200):
    """Batched replicas: replica-steps/s over `steps` NVE steps of every
    replica (graph replay, events on the engine stream), then the device time
    of each of `lat_steps` steps with phase events on (p50 / p99)."""
    from lammps_b200.replicas import make_batch
    s = make_batch(batch, prec, device=DEVICE)
    s.setup()
    s.run(40)
    ext = torch.cuda.ExternalStream(s.stream)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(ext)
    s.run(steps)
    e1.record(ext)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    s.set_timing(True)
    s.run(20)
    s.step_times(reset=True)
    s.run(lat_steps)
    st = s.step_times(reset=True)
    s.set_timing(False)
    nrep = len(batch["natoms"])
    form = s.replica_step()
    out = {"replica_steps_per_s": nrep * steps / (ms * 1e-3),
           "step_form": ("one launch per step: clusters of %d CTAs x %d threads, %d thread(s) "
                         "per atom" % (form["cluster"], form["block"], form["tpa"])
                         if form["onelaunch"] else "graph of kernels per step"),
           "tuned_ms_per_step": {"graph": form["graph_ms"], "one_launch": form["onelaunch_ms"]},
           "matom_steps_per_s": float(batch["natoms"].sum()) * steps / (ms * 1e3),
           "ms_per_step": ms / steps, "launch": s.launch(),
           "step_ms_p50": float(np.percentile(st, 50)), "step_ms_p99": float(np.percentile(st, 99))}
    s.close()
    return out


def brick_bench(torch, x, v, hi, steps=40, warm=40):
    """One box split into bricks (lammps_b200.brick) on this one GPU: the
    per-call step of one brick, and of 2 bricks (2 x 1 x 1) as separate
    contexts whose halo exchange is a device copy.  The bricks of a step run
    one after the other here; on N GPUs they run side by side.  Wall time
    around host-synchronous steps (each entry point returns after its
    stream)."""
    from lammps_b200.brick import BrickRun, LocalComm
    out = {"atoms": len(x), "steps": steps,
           "note": "LJ fcc 4M, rc 2.5, skin 0.3, every 20 check no; per-call steps with "
                   "rebuild (exchange + borders) every 20 steps and a halo exchange on the others"}
    for prec in ("fp64", "mixed"):
        for grid in ((1, 1, 1), (2, 1, 1)):
            comm = LocalComm(int(np.prod(grid)))
            b = BrickRun(comm, {r: make_lj(prec, x, v, hi, atoms=False) for r in comm.ranks}, grid)
            b.set_atoms(x, None, v)
            b.setup()
            b.run(warm)
            torch.cuda.synchronize()
            b.timers = {k: 0.0 for k in b.timers}
            t0 = time.perf_counter()
            b.run(steps)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            key = f"{prec}_{'x'.join(map(str, grid))}"
            st = b.stats()
            out[key] = {"ms_per_step": dt / steps * 1e3,
                        "matom_steps_per_s": len(x) * steps / dt / 1e6,
                        "ghost_atoms": sum(q["ghost"] for q in st.values()),
                        "rebuilds": b.ncalls,
                        "ms_per_step_by_phase": {k: t / steps * 1e3 for k, t in b.timers.items()}}
            for e in b.st.values():
                e.engine.close()
    return out


def dist_setup():
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def _reduce(val, ws, torch, op):
    if ws == 1:
        return val
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([val], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def allmax(val, ws, torch):
    """The maximum of `val` over the ranks (device times: the slowest rank)."""
    import torch.distributed as dist
    return _reduce(val, ws, torch, dist.ReduceOp.MAX if ws > 1 else None)


def allsum(val, ws, torch):
    """The sum of `val` over the ranks (work done by all ranks)."""
    import torch.distributed as dist
    return _reduce(val, ws, torch, dist.ReduceOp.SUM if ws > 1 else None)


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def profile_case(args):
    """One form of one workload, W warm-up + K bench steps, for ncu captures."""
    import torch
    torch.cuda.set_device(0)
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    work, prec = args.case.split("-")
    if work == "eam32k":
        tmp = tempfile.mkdtemp(prefix="b200prof_")
        from lammps_b200.eam_synth import write_setfl
        setfl = write_setfl(os.path.join(tmp, "Cu_synth.eam.alloy"))
        x, v, hi = eam32k_inputs()
        s = make_eam32k(prec, setfl, x, v, hi)
    elif work == "lj4m":
        x, v, hi = lj4m_inputs()
        s = make_lj(prec, x, v, hi)
    elif work == "lj32k":
        from lammps_b200 import inputs
        a = inputs.lj_lattice_constant("fcc", 0.8442)
        x = inputs.lattice("fcc", 20, 20, 20, a)
        v = inputs.velocity_create(x, np.ones(len(x), np.int32), np.array([0.0, 1.0]), 1.44,
                                   87287, "lj", gaussian=True, loop="geom")
        s = make_lj(prec, x, v, np.array([20 * a] * 3))
    elif work == "eam4m":
        tmp = tempfile.mkdtemp(prefix="b200prof_")
        from lammps_b200.eam_synth import write_setfl
        setfl = write_setfl(os.path.join(tmp, "Cu_synth.eam.alloy"))
        x, v, hi = eam4m_inputs()
        s = make_eam32k(prec, setfl, x, v, hi)
    elif work == "c3":
        from lammps_b200.replicas import make_batch, replica_batch
        batch = replica_batch(nrep=256)
        x, v = batch["x"], batch["v"]
        s = make_batch(batch, prec)
    else:
        raise SystemExit(f"unknown case {args.case}")
    if args.eager:
        s.set_graphs(False)
    if args.tpa:
        s.set_launch(args.tpa)
    total, per = time_form(s, torch, flush, args.steps, max(args.warmup, 1), (x, v))
    s.set_timing(True)
    ext = torch.cuda.ExternalStream(s.stream)
    device_time_run(s, torch, ext, flush, MD_STEPS, (x, v))
    ph = s.timing(reset=True)
    pieces = piece_times(s, torch, flush, (x, v), runs=1)
    print(json.dumps({"case": args.case, "atoms": s.n, "steps": args.steps,
                      "matom_steps_per_s": s.n * MD_STEPS * args.steps / (total * 1e3),
                      "launch": s.launch(), "neigh": s.neigh_stats(),
                      "phases_ms_per_md_step": {k: ph[k] / max(ph["steps"], 1) for k in s.PHASES},
                      "pieces_ms_per_md_step": pieces}))
    s.close()


def headline_timed(s, torch, flush, K, W, start, ws, dev):
    """W untimed and K timed bench steps of one form, bracketed by a barrier
    and a synchronize on both sides, with the SM clocks sampled during the
    timed region: (value over all ranks, max-over-ranks total ms, launches,
    clocks)."""
    ext = torch.cuda.ExternalStream(s.stream)
    s.setup()
    for _ in range(W):
        device_time_run(s, torch, ext, flush, MD_STEPS, start)
    barrier(ws)
    torch.cuda.synchronize()
    clocks = clock_sampler(dev)
    clocks.start()
    l0 = s.kernel_launches
    per = [device_time_run(s, torch, ext, flush, MD_STEPS, start) for _ in range(K)]
    torch.cuda.synchronize()
    launches = s.kernel_launches - l0
    barrier(ws)
    clk = clocks.stop()
    total_ms = allmax(sum(per), ws, torch)
    atoms_all = allsum(s.n, ws, torch)  # every rank advances its own box
    return atoms_all * MD_STEPS * K / (total_ms * 1e3), total_ms, launches, clk


def phase_times(s, torch, flush, start, runs=2):
    """Per-MD-step device time of each phase, from the CUDA events recorded
    inside the step graphs (a separate pass: the events cost time)."""
    ext = torch.cuda.ExternalStream(s.stream)
    s.set_timing(True)
    device_time_run(s, torch, ext, flush, MD_STEPS, start)
    s.timing(reset=True)
    for _ in range(runs):
        device_time_run(s, torch, ext, flush, MD_STEPS, start)
    ph = s.timing(reset=True)
    s.set_timing(False)
    return {k: ph[k] / max(ph["steps"], 1) for k in s.PHASES}


def piece_times(s, torch, flush, start, runs=2):
    """Per-MD-step device time of whole step pieces with the run's own step
    form (timing mode 2: two stream events around each piece): "initial"
    (chunk starts), "neigh" (rebuilds) and "pair1" (forces with both
    half-steps: the one-launch step kernel for lj/cut)."""
    ext = torch.cuda.ExternalStream(s.stream)
    s.set_timing(2)
    device_time_run(s, torch, ext, flush, MD_STEPS, start)
    s.timing(reset=True)
    for _ in range(runs):
        device_time_run(s, torch, ext, flush, MD_STEPS, start)
    ph = s.timing(reset=True)
    s.set_timing(False)
    return {k: ph[k] / max(ph["steps"], 1) for k in ("initial", "neigh", "pair1")}


def e2e_block(torch, s, x, v, K, ws=1):
    """The form's metric through the public API with page-locked host
    buffers: upload x, v, type; setup; 100 steps; download x, v, f, image."""
    n = len(x)
    x_pin = pinned(torch, np.ascontiguousarray(x, dtype=np.float64))
    v_pin = pinned(torch, np.ascontiguousarray(v, dtype=np.float64))
    t_pin = pinned(torch, np.ones(n, np.int32))
    o_pin = {k: pinned(torch, np.zeros((n, 3), dt)) for k, dt in
             (("x", np.float64), ("v", np.float64), ("f", np.float64), ("image", np.int32))}
    o_pin2 = {k: pinned(torch, np.zeros((n, 3), dt)) for k, dt in
              (("x", np.float64), ("v", np.float64), ("f", np.float64), ("image", np.int32))}
    e2e_run(s, x_pin, v_pin, t_pin, o_pin, 1)
    s_ms, h2d, d2h = e2e_run(s, x_pin, v_pin, t_pin, o_pin, K)
    e2e_run_overlapped(s, x_pin, v_pin, t_pin, (o_pin, o_pin2), 2)
    e_ms, h2d2, d2h2 = e2e_run_overlapped(s, x_pin, v_pin, t_pin, (o_pin, o_pin2), K)
    assert (h2d2, d2h2) == (h2d, d2h)
    _PINNED.clear()
    e_ms = allmax(e_ms, ws, torch)
    s_ms = allmax(s_ms, ws, torch)
    atoms_all = allsum(n, ws, torch)
    return {"value": atoms_all * MD_STEPS * K / (e_ms * 1e3), "unit": "Matom-steps/s",
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "form": "overlapped transfers: each bench step uploads x, v, type from page-locked "
                    "host buffers (staged while the previous step runs), sets them, runs setup "
                    "and the MD steps, and downloads x, v, f, image (copied while the next step "
                    "runs); wall clock from the first upload to the last download",
            "blocking_value": atoms_all * MD_STEPS * K / (s_ms * 1e3)}


def oracle_errors(make, ref):
    """Both forms' force, energy and virial errors on the oracle's state."""
    errs = {}
    for prec in ("fp64", "mixed"):
        s = make(prec)
        s.set_atoms(ref["x"], None, None)
        s.neigh_build()
        r = s.compute(1, 1)
        errs[prec] = errors_vs(s.download()["f"], r["eng"], r["virial"], ref)
        s.close()
    return errs


def eam32k_block(torch, flush, K, W, setfl, clk, no_cpu, oracle=True):
    """The 32,000-atom EAM configuration (synthetic 5000-point setfl) as a
    line of its own: mixed and FP64, the dominant kernel's roofline, end to
    end through the API, errors against the oracle, the reference's CPU
    path on the same workload (all cores and one core)."""
    x, v, hi = eam32k_inputs()
    n = len(x)
    out = {"workload": "eam-32k: fcc 20^3 a=3.615 A, synthetic 5000-point setfl (eam/alloy), "
                       "1600 K Gaussian (seed 376847, loop geom), skin 1.0, every 1 delay 5 check "
                       "yes, dt 5 fs; one bench step = the first 100 NVE steps from the seeded state",
           "atoms": n, "unit": "Matom-steps/s",
           "l2": "flushed (256 MB write) before every timed bench step"}
    for prec in ("mixed", "fp64"):
        s = make_eam32k(prec, setfl, x, v, hi)
        t, _ = time_form(s, torch, flush, K, W, (x, v))
        out[prec] = n * MD_STEPS * K / (t * 1e3)
        out[prec + "_ms_per_md_step"] = t / (K * MD_STEPS)
        ph = phase_times(s, torch, flush, (x, v))
        out[prec + "_phases_ms_per_md_step"] = ph
        if prec == "mixed":
            out["e2e"] = e2e_block(torch, s, x, v, K)
            peak, peak_kind = load_peaks()
            dom = max(("pair1", "pair2"), key=lambda k: ph[k])
            # force pass: x (24 B) and F' (8 B) read, f (24 B) written; density
            # pass: x (24 B) read, rho and F' (16 B) written
            bpa = 56.0 if dom == "pair2" else 40.0
            ach = bpa * n / (ph[dom] * 1e-3) / 1e9
            out["roofline"] = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                               "frac": ach / peak, "traffic": load_traffic().get(f"eam32k_mixed_{dom}"),
                               "kernel": "k_eam_force (mixed)" if dom == "pair2" else "k_eam_rho (mixed)",
                               "kernel_ms": ph[dom], "peak_source": f"{peak_kind} hbm_gbs",
                               "step": step_roofline(n, out["mixed_ms_per_md_step"], peak, clk)}
        s.close()
    out["value"] = out["mixed"]
    out["mixed_over_fp64"] = out["mixed"] / out["fp64"]
    if oracle:
        ref = eam32k_oracle_state(setfl, x, hi)
        out["error_vs_oracle"] = oracle_errors(lambda p: make_eam32k(p, setfl, x, None, hi), ref)
        out["error_vs_oracle"]["state"] = "oracle after 10 steps from the seeded state"
    if not no_cpu:
        out["cpu_baseline"] = cpu_baseline_eam32k(setfl, x, v, hi)
    return out


def replica_scripts(steps, every=1):
    """(atoms, reference input) of every `every`-th replica of the 256-replica
    batch: the box as the batch builds it (fcc at the replica's density, its
    Gaussian velocities from its seed with loop geom), lj/cut rc 2.5, skin 0.3,
    every 20 delay 0 check no, dt 0.005, the first `steps` NVE steps."""
    from lammps_b200.replicas import replica_batch
    b = replica_batch()
    out = []
    for k in range(0, len(b["natoms"]), every):
        n = int(b["ncells"][k])
        out.append((int(b["natoms"][k]), [
            "units lj", "atom_style atomic", f"lattice fcc {b['rho'][k]:.17g}",
            f"region box block 0 {n} 0 {n} 0 {n}", "create_box 1 box", "create_atoms 1 box",
            "mass 1 1.0",
            f"velocity all create {b['temp'][k]:.17g} {int(b['seeds'][k])} dist gaussian loop geom",
            "pair_style lj/cut 2.5", "pair_coeff 1 1 1.0 1.0 2.5", "neighbor 0.3 bin",
            "neigh_modify delay 0 every 20 check no", "fix 1 all nve", "timestep 0.005",
            f"thermo {steps}", f"run {steps}", "clear"]))
    return out


def reference_cpu_replicas(procs, steps, every=1, timeout=900):
    """Matom-steps/s of the reference's own binary on the 256-replica batch
    (or every `every`-th replica): `procs` concurrent single-threaded
    processes (plain styles), each running its share of the replicas one
    after another; the rate is the atom-steps of all replicas over the
    largest per-process sum of Loop times (setup excluded, as elsewhere)."""
    import re
    import shutil
    exe = reference_binary()
    reps = replica_scripts(steps, every)
    # largest replicas first, each to the process with the least work so far
    order = sorted(range(len(reps)), key=lambda k: -reps[k][0])
    share = [[] for _ in range(procs)]
    load = [0] * procs
    for k in order:
        p = load.index(min(load))
        share[p].append(k)
        load[p] += reps[k][0]
    tmp = tempfile.mkdtemp(prefix="b200rep_")
    env = dict(os.environ, OMP_NUM_THREADS="1")
    try:
        runs = []
        for p, ks in enumerate(share):
            if not ks:
                continue
            name = f"in.share{p}"
            with open(os.path.join(tmp, name), "w") as fh:
                fh.write("\n".join(line for k in ks for line in reps[k][1]) + "\n")
            runs.append((ks, subprocess.Popen([exe, "-in", name, "-log", "none", "-echo", "none"],
                                              cwd=tmp, env=env, stdout=subprocess.PIPE,
                                              stderr=subprocess.STDOUT, text=True)))
        secs = []
        for ks, pr in runs:
            out, _ = pr.communicate(timeout=timeout)
            t = [float(x) for x in re.findall(r"Loop time of (\S+) on", out)]
            if pr.returncode != 0 or len(t) != len(ks):
                raise RuntimeError(f"lmp_serial replica share failed ({pr.returncode}): {out[-500:]}")
            secs.append(sum(t))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    atoms = sum(r[0] for r in reps)
    return {"value": atoms * steps / max(secs) / 1e6, "unit": "Matom-steps/s", "processes": procs,
            "replicas": len(reps), "atoms": atoms, "steps": steps,
            "replica_steps_per_s": len(reps) * steps / max(secs)}


def cpu_rows(setfl):
    """The reference's own CPU path on each configuration that runs on a
    CPU in seconds: one core (plain styles) and all cores (-sf omp)."""
    host = host_cpu()
    rows = {"cpu_model": host["model"], "nproc": host["cores"]}
    rows["lj_32k"] = {"one_core": reference_cpu("lj32k", 1, 1)["value"],
                      "all_cores": reference_cpu("lj32k", host["cores"], 3)["value"]}
    rows["eam_32k"] = {"one_core": reference_cpu("eam32k", 1, 1, setfl=setfl)["value"],
                       "all_cores": reference_cpu("eam32k", host["cores"], 3, setfl=setfl)["value"]}
    rows["replicas_256"] = {
        "one_core": reference_cpu_replicas(1, MD_STEPS, every=4),
        "all_cores": reference_cpu_replicas(host["cores"], MD_STEPS),
        "note": "the first 100 steps of each replica; one core: every 4th replica in one "
                "process; all cores: all 256 replicas over one single-threaded process per core"}
    rows["note"] = ("Matom-steps/s of fresh runs of the first 100 steps from the seeded state "
                    "(median of the all-core runs); lj_4M is in cpu_baseline")
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-extras", action="store_true", help="only the headline line")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline samples")
    ap.add_argument("--eager", action="store_true",
                    help="with --case: launch kernels one by one (for profilers)")
    ap.add_argument("--tpa", type=int, default=0,
                    help="with --case: threads per atom of the pair kernels (0 = autotuned)")
    ap.add_argument("--case", default=None,
                    help="profile one form only: eam32k-mixed, eam32k-fp64, lj4m-mixed, lj4m-fp64, lj32k-mixed, lj32k-fp64, "
                         "eam4m-mixed, eam4m-fp64, c3-mixed, c3-fp64 (256 replicas)")
    args = ap.parse_args()
    if args.case:
        return profile_case(args)
    K, W = args.steps, max(args.warmup, 3)
    ws, rank, local = dist_setup()
    config = {"workload": "lj-4M: fcc 100^3 (4,000,000 atoms), rho* 0.8442, T* 1.44 Gaussian "
                          "(seed 87287, loop geom), lj/cut rc 2.5, skin 0.3, every 20 delay 0 "
                          "check no, dt 0.005, mixed precision; one bench step = the first 100 "
                          "NVE steps from the seeded initial state",
              "atoms": 4000000, "md_steps_per_step": MD_STEPS, "precision": "mixed",
              "l2": "inputs larger than L2 (4M atoms), and flushed (256 MB write) before every "
                    "timed bench step",
              "parallelism": f"replicas x{ws}"}
    n4 = WORKLOADS["lj4m"]["atoms"]
    RS = 20  # MD steps of one reference sample of LJ-4M (one neighbor rebuild)

    if args.impl == "reference":
        # the reference's own CPU path on all host cores; each bench step is a
        # fresh run of the first RS steps of the workload (W discarded)
        if rank == 0:
            host = host_cpu()
            if reference_binary():
                cpu = reference_cpu("lj4m", host["cores"], W + K, steps=RS)
                timed = cpu["samples"][W:]
                secs = [n4 * RS / (r * 1e6) for r in timed]
                value = n4 * RS * K / sum(secs) / 1e6
                cpu["sample"] += f"; first {W} runs discarded as warm-up"
            else:
                cpu = port_cpu_lj4m(host["cores"], W + K, RS)
                timed = cpu["samples"][W:]
                secs = [n4 * RS / (r * 1e6) for r in timed]
                value = n4 * RS * K / sum(secs) / 1e6
                cpu["sample"] = "reference binary absent: " + cpu["sample"]
            cpu.update(value=value, cpu_model=host["model"], nproc=host["cores"])
            line = {"metric": METRIC, "value": value, "unit": "Matom-steps/s", "n_gpus": ws,
                    "steps": K, "warmup": W, "ms_per_step": sum(secs) * 1e3 / K,
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                    "dtype": "f64", "data": "synthetic (seeded fcc lattice + Gaussian velocities)",
                    "config": config, "impl": "reference", "cpu_baseline": cpu,
                    "e2e": {"value": value, "unit": "Matom-steps/s", "h2d_bytes_per_step": 0,
                            "d2h_bytes_per_step": 0}}
            print(json.dumps(line))
        return

    import torch
    global DEVICE
    dev = local if torch.cuda.device_count() > 1 else 0
    DEVICE = dev
    torch.cuda.set_device(dev)
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    tmp = tempfile.mkdtemp(prefix="b200bench_")
    from lammps_b200.eam_synth import write_setfl
    setfl = write_setfl(os.path.join(tmp, "Cu_synth.eam.alloy"))
    x4, v4, hi4 = lj4m_inputs()
    assert len(x4) == n4
    start = (x4, v4)

    # ---- headline: LJ-4M, mixed precision, device-timed -------------------
    sysm = make_lj("mixed", x4, v4, hi4)
    value, total_ms, launches, clk = headline_timed(sysm, torch, flush, K, W, start, ws, dev)
    phases = phase_times(sysm, torch, flush, start)
    pieces = piece_times(sysm, torch, flush, start)
    peak, peak_kind = load_peaks()
    # the dominant kernel is the one-launch step k_lj_step (forces, this
    # step's final and the next initial half-step); its algorithmic bytes per
    # atom, FP64 state: x read and written (48 B), v read and written (48 B);
    # the forces stay in registers.  Its time is the step piece's (with the
    # one-thread k_decide after it), from events around the piece.
    achieved = STEP_BYTES_PER_ATOM * n4 / (pieces["pair1"] * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": load_traffic().get("lj4m_mixed_step"),
                "kernel": "k_lj_step", "kernel_ms": pieces["pair1"],
                "alg_bytes_per_atom": STEP_BYTES_PER_ATOM,
                # what bounds the kernel: the L1 data pipe of its neighbour
                # gathers (ncu capture in profiles/k_lj_step_lj4m.md)
                "l1tex_pct_of_peak": load_traffic().get("lj4m_mixed_step_l1tex_pct"),
                "pair_kernel": {"kernel": "k_lj_mixed (phase-timed steps)",
                                "ms": phases["pair1"],
                                "achieved_gbs": 48.0 * n4 / (phases["pair1"] * 1e-3) / 1e9},
                "peak_source": f"{peak_kind} hbm_gbs",
                # whole-step figures from the headline runs (timing events off),
                # so that they follow from `value`
                "step": step_roofline(n4, total_ms / (K * MD_STEPS), peak, clk,
                                      LJ_BYTES_PER_ATOM_STEP, LJ_FLOP_PER_ATOM_STEP)}
    e2e = e2e_block(torch, sysm, x4, v4, K, ws)
    sysm.close()

    # ---- the FP64 form of the same workload -------------------------------
    s64 = make_lj("fp64", x4, v4, hi4)
    v64, t64, _, _ = headline_timed(s64, torch, flush, K, W, start, ws, dev)
    ph64 = phase_times(s64, torch, flush, start)
    pc64 = piece_times(s64, torch, flush, start)
    s64.close()

    extras = {"fp64": v64, "mixed_over_fp64": value / v64,
              "ms_per_md_step": {"mixed": total_ms / (K * MD_STEPS), "fp64": t64 / (K * MD_STEPS)},
              "phases_ms_per_md_step": {"mixed": phases, "fp64": ph64},
              "pieces_ms_per_md_step": {"mixed": pieces, "fp64": pc64}}
    if not args.no_extras:
        if rank == 0:  # the oracle uses every host core: one rank at a time
            ref = lj4m_oracle_state(hi4)
            extras["error_vs_oracle"] = oracle_errors(
                lambda p: make_lj(p, x4, v4, hi4, atoms=False), ref)
            extras["error_vs_oracle"]["state"] = ("oracle after 10 steps from the seeded state "
                                                  "(all host threads)")
        # NVE energy conservation over 1000 steps (thermo every 100), both
        # forms from the same state
        nve, etot = {}, {}
        for prec in ("mixed", "fp64"):
            s = make_lj(prec, x4, v4, hi4)
            s.set_thermo(100)
            rows = [s.setup()] + s.run(1000)
            st = np.array([r["Step"] for r in rows], dtype=float)
            e = np.array([r["TotEng"] for r in rows])
            etot[prec] = e
            nve[prec] = {"etot_first": float(e[0]), "etot_last": float(e[-1]),
                         "slope_per_step": float(np.polyfit(st, e, 1)[0])}
            s.close()
        nve["max_abs_etot_diff"] = float(np.max(np.abs(etot["mixed"] - etot["fp64"])))
        extras["nve_1000"] = nve

        extras["eam_32k"] = eam32k_block(torch, flush, K, W, setfl, clk,
                                         args.no_cpu or rank != 0 or ws != 1, oracle=rank == 0)
        cu = {}
        for prec in ("mixed", "fp64"):
            scu, st = make_eam_cu(prec)
            t, _ = time_form(scu, torch, flush, K, W, st)
            cu[prec] = scu.n * MD_STEPS * K / (t * 1e3)
            scu.close()
        cu["mixed_over_fp64"] = cu["mixed"] / cu["fp64"]
        extras["eam_cu_u3_32k"] = cu
        # the plain LJ configuration of 32,000 atoms (fcc 20^3, Gaussian
        # velocities, every 20 check no), the workload of the lj_32k CPU rows
        from lammps_b200 import inputs as _inputs
        a32 = _inputs.lj_lattice_constant("fcc", 0.8442)
        x32 = _inputs.lattice("fcc", 20, 20, 20, a32)
        v32 = _inputs.velocity_create(x32, np.ones(len(x32), np.int32), np.array([0.0, 1.0]),
                                      1.44, 87287, "lj", gaussian=True, loop="geom")
        lj32 = {"atoms": len(x32), "note": "fcc 20^3 rho* 0.8442, T* 1.44 Gaussian (seed 87287, "
                "loop geom), rc 2.5, skin 0.3, every 20 check no; one bench step = the first 100 "
                "NVE steps from the seeded state"}
        for prec in ("mixed", "fp64"):
            s32 = make_lj(prec, x32, v32, np.array([20 * a32] * 3))
            t, _ = time_form(s32, torch, flush, K, W, (x32, v32))
            lj32[prec] = s32.n * MD_STEPS * K / (t * 1e3)
            s32.close()
        lj32["mixed_over_fp64"] = lj32["mixed"] / lj32["fp64"]
        extras["lj_32k"] = lj32
        # the EAM workload at 4M atoms: the density and force kernels at a
        # size where they are not launch- and latency-bound
        xe, ve, hie = eam4m_inputs()
        em = {"atoms": len(xe), "note": "fcc 100^3 a=3.615, synthetic setfl, 1600 K, skin 1.0, "
                                       "every 1 delay 5 check yes, 100 steps per bench step"}
        for prec in ("mixed", "fp64"):
            s = make_eam32k(prec, setfl, xe, ve, hie)
            k4 = max(2, K // 3)
            t, _ = time_form(s, torch, flush, k4, 2, (xe, ve))
            ph = phase_times(s, torch, flush, (xe, ve), runs=1)
            em[prec] = len(xe) * MD_STEPS * k4 / (t * 1e3)
            em[prec + "_phases_ms_per_step"] = ph
            # algorithmic bytes: density pass 40 B/atom, force pass 56 B/atom
            em[prec + "_rho_kernel_gbs"] = 40.0 * len(xe) / (ph["pair1"] * 1e-3) / 1e9
            em[prec + "_force_kernel_gbs"] = 56.0 * len(xe) / (ph["pair2"] * 1e-3) / 1e9
            s.close()
        em["mixed_over_fp64"] = em["mixed"] / em["fp64"]
        extras["eam_4M"] = em
        extras["bricks_lj_4M"] = brick_bench(torch, x4, v4, hi4)

        from lammps_b200.replicas import replica_batch, shard_batch
        full = replica_batch(nrep=256)
        # under torchrun the 256 replicas are sharded across the ranks (no
        # exchange); throughput is all replicas over the slowest rank's time
        batch = shard_batch(full, rank, ws) if ws > 1 else full
        rep = {"replicas": 256, "atoms": int(full["natoms"].sum()),
               "natoms_min": int(full["natoms"].min()), "natoms_max": int(full["natoms"].max()),
               "ranks": ws, "steps": 1000,
               "note": "256 fcc LJ boxes, 4n^3 atoms with n = 5..12 from log-uniform "
                       "500-8000, rho* U(0.70,0.95), T* U(0.8,2.0), rc 2.5 skin 0.3 "
                       "every 20; one set of launches per step for all replicas; "
                       "p50/p99 with phase events recorded in the step graphs"}
        for prec in ("mixed", "fp64"):
            r = replica_bench(prec, batch, torch)
            if ws > 1:
                ms = allmax(r["ms_per_step"], ws, torch)
                r["ms_per_step"] = ms
                r["replica_steps_per_s"] = 256 / (ms * 1e-3)
                r["matom_steps_per_s"] = float(full["natoms"].sum()) / (ms * 1e3)
                r["step_ms_p50"] = allmax(r["step_ms_p50"], ws, torch)
                r["step_ms_p99"] = allmax(r["step_ms_p99"], ws, torch)
            rep[prec] = r
        rep["mixed_over_fp64"] = rep["mixed"]["replica_steps_per_s"] / rep["fp64"]["replica_steps_per_s"]
        extras["replicas_256"] = rep
        from lammps_b200.forcematch import force_matching_case, gradient_check
        fm = force_matching_case()
        rng = np.random.default_rng(99)
        eps0 = fm["eps"] * (1 + 0.08 * rng.standard_normal(3))
        sig0 = fm["sigma"] * (1 + 0.02 * rng.standard_normal(3))
        extras["force_matching_8k"] = gradient_check(fm, eps0, sig0, device=DEVICE)
        extras["force_matching_8k"]["note"] = (
            "2-type lj/cut, 8000 atoms, 10x10x20 fcc rho*=0.85 + 0.05 jitter; errors of "
            "dL/d(eps,sigma) vs FP64 central differences (h=1e-5, cutoffs held) relative to "
            "the largest component, and of dL/dx along 8 unit directions relative to |dL/dx|")

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        host = host_cpu()
        if reference_binary():
            cpu = reference_cpu("lj4m", host["cores"], 3, steps=RS)
            cpu["one_core"] = reference_cpu("lj4m", 1, 1, steps=5)
            cpu["one_core"]["sample"] += (" (no rebuild inside the 5 steps: the set-up build is "
                                          "untimed)")
            if not args.no_extras:
                cpu["rows"] = cpu_rows(setfl)
        else:
            cpu = port_cpu_lj4m(host["cores"], 1, RS)
        cpu.update(cpu_model=host["model"], nproc=host["cores"])

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "Matom-steps/s", "n_gpus": ws, "steps": K,
                "warmup": W, "ms_per_step": total_ms / K, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32-mixed (f64 positions/sums)",
                "data": "synthetic (seeded fcc lattice + Gaussian velocities; synthetic setfl EAM)",
                "config": config, "clocks": clk, "e2e": e2e, "gpu_launches": int(launches),
                "roofline": roofline, "cpu_baseline": cpu}
        line.update(extras)
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
