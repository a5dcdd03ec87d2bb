"""b200_kinetic_sum_noalloc: the allocation-free kinetic-energy sum agrees
with the sum the engine's own setup row carries (sum m v^2 of
ComputeTemp::compute_scalar, src/compute_temp.cpp:59-89), on two calls in a
row, and rejects sizes beyond its limits.  Collected last on purpose: it must
pass both alone in a fresh process and after every other GPU test."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from lammps_b200 import _abi

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

REL = 1e-12  # FP64 tolerance of the parity tests; only the summation order differs


def _noalloc(n, v, t, m, ntypes, out, stream=None):
    lib = _abi.load()
    s = torch.cuda.current_stream().cuda_stream if stream is None else stream
    return lib.b200_kinetic_sum_noalloc(n, C.c_void_p(v.data_ptr()), C.c_void_p(t.data_ptr()),
                                        C.c_void_p(m.data_ptr()), ntypes,
                                        C.c_void_p(out.data_ptr()), C.c_void_p(s))


def _device(v, t, m):
    dev = torch.device("cuda:0")
    return (torch.from_numpy(np.ascontiguousarray(v, np.float64)).to(dev),
            torch.from_numpy(np.ascontiguousarray(t, np.int32)).to(dev),
            torch.from_numpy(np.ascontiguousarray(m, np.float64)).to(dev))


def test_matches_setup_row_twice():
    from gpu_cases import device_case
    from oracle_cases import GOLDEN

    with open(os.path.join(GOLDEN, "reference_logs.json")) as fh:
        case = json.load(fh)["bench_lj"]
    sysm = device_case(case)
    row = sysm.setup()
    v = sysm.download()["v"]
    n = v.shape[0]
    t = np.ones(n, np.int32)
    m = np.asarray(sysm.mass, np.float64)
    dv, dt, dm = _device(v, t, m)
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda:0")
    assert _noalloc(n, dv, dt, dm, len(m) - 1, out[0:1]) == 0
    assert _noalloc(n, dv, dt, dm, len(m) - 1, out[1:2]) == 0
    torch.cuda.synchronize()
    a, b = out.cpu().numpy()
    ref = row["ke2"]
    assert abs(a - ref) <= REL * abs(ref)
    assert abs(b - ref) <= REL * abs(ref)
    assert a == b  # fixed summation order: repeat calls agree bit for bit
    sysm.close()


def test_large_grid_two_types():
    """More atoms than the fixed 1184 x 256 threads (grid-stride path) and
    two atom types, against an extended-precision host sum."""
    rng = np.random.default_rng(7)
    n = 1_500_000
    v = rng.normal(size=(n, 3))
    t = rng.integers(1, 3, size=n).astype(np.int32)
    m = np.array([0.0, 1.0, 2.5])
    terms = (v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1] + v[:, 2] * v[:, 2]) * m[t]
    ref = float(np.sum(terms.astype(np.longdouble)))
    dv, dt, dm = _device(v, t, m)
    out = torch.zeros(2, dtype=torch.float64, device="cuda:0")
    for k in range(2):
        assert _noalloc(n, dv, dt, dm, 2, out[k:k + 1]) == 0
    torch.cuda.synchronize()
    a, b = out.cpu().numpy()
    assert abs(a - ref) <= REL * abs(ref)
    assert a == b


def test_rejects_sizes_beyond_limits():
    dv, dt, dm = _device(np.zeros((4, 3)), np.ones(4), np.ones(2))
    out = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    assert _noalloc(1 << 26, dv, dt, dm, 1, out) == -1  # B200_ERR_ARG
    assert _noalloc(0, dv, dt, dm, 1, out) == -1  # B200_ERR_ARG
    assert _noalloc(4, dv, dt, dm, 9, out) == -1  # B200_ERR_ARG


def test_type_outside_range_gives_nan():
    """A type outside 1..ntypes is never used as an index into mass[]: the
    sum comes back NaN, and a following call with valid types is exact."""
    n = 1000
    rng = np.random.default_rng(3)
    v = rng.normal(size=(n, 3))
    t = np.ones(n, np.int32)
    t[417] = 3  # ntypes = 2
    m = np.array([0.0, 1.0, 2.0])
    dv, dt, dm = _device(v, t, m)
    out = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    assert _noalloc(n, dv, dt, dm, 2, out) == 0
    torch.cuda.synchronize()
    assert np.isnan(out.cpu().numpy()[0])
    dt[417] = 2
    assert _noalloc(n, dv, dt, dm, 2, out) == 0
    torch.cuda.synchronize()
    tt = t.copy()
    tt[417] = 2
    ref = float(np.sum(((v * v).sum(axis=1) * m[tt]).astype(np.longdouble)))
    assert abs(out.cpu().numpy()[0] - ref) <= REL * abs(ref)
