"""Force matching with the engine's adjoint kernel (2-type lj/cut, 8,000
atoms on a jittered 10x10x20 fcc lattice at rho* 0.85).

Checks:
  - FP64 forward forces == the oracle's PairLJCut forces (1e-12);
  - mixed forward within 1e-5 of FP64;
  - dL/d(eps_ij, sigma_ij) against FP64 central finite differences, h = 1e-5
    (cutoffs held at their values, so no pair crosses a cutoff);
  - dL/dx against directional central differences along 8 random unit
    directions (atoms in pairs within 10 h of a cutoff are held still, since
    the force jumps there), and the mixed Hessian-vector product against the
    FP64 one over all atoms.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from lammps_b200.forcematch import LJForceField, force_matching_case, pair_matrix  # noqa: E402

pytestmark = pytest.mark.gpu

H = 1e-5
CUT = 2.5


@pytest.fixture(scope="module")
def case():
    c = force_matching_case()
    rng = np.random.default_rng(99)
    # parameters at which the gradient is taken: the hidden ones, perturbed
    c["eps0"] = c["eps"] * (1 + 0.08 * rng.standard_normal(3))
    c["sigma0"] = c["sigma"] * (1 + 0.02 * rng.standard_normal(3))
    c["max_cut"] = CUT * 1.1 * 1.05
    return c


def _field(case, precision):
    return LJForceField(case["lo"], case["hi"], case["x"], case["types"], 2, case["max_cut"],
                        precision=precision)


@pytest.fixture(scope="module")
def fields(case):
    f64 = _field(case, "fp64")
    fmx = _field(case, "mixed")
    yield f64, fmx
    f64.close()
    fmx.close()


def _mats(eps, sigma):
    e = pair_matrix(torch.as_tensor(eps, dtype=torch.float64), 2)
    s = pair_matrix(torch.as_tensor(sigma, dtype=torch.float64), 2)
    return e, s


def test_fp64_forward_matches_oracle(case, fields):
    import oracle

    f64, _ = fields
    x = torch.tensor(case["x"], dtype=torch.float64, device="cuda")
    e, s = _mats(case["eps"], case["sigma"])
    with torch.no_grad():
        fd = f64.forces(x, e, s).cpu().numpy()
    o = oracle.OracleSim("lj", threads=4)
    o.box(case["lo"], case["hi"])
    o.atoms(case["x"], type=case["types"], ntypes=2)
    o.mass(1, 1.0)
    o.mass(2, 1.0)
    o.lj_cut(CUT)
    k = 0
    for i in (1, 2):
        for j in range(i, 3):
            o.lj_coeff(i, j, case["eps"][k], case["sigma"][k], CUT * case["sigma"][k])
            k += 1
    o.neighbor(0.3, 1, 0, False, 0)
    o.setup()
    fo = np.zeros_like(fd)
    fo[o.tag - 1] = o.f
    err = np.linalg.norm(fd - fo) / np.linalg.norm(fo)
    assert err <= 1e-12, err


def test_mixed_forward_within_1e5(case, fields):
    f64, fmx = fields
    x = torch.tensor(case["x"], dtype=torch.float64, device="cuda")
    e, s = _mats(case["eps0"], case["sigma0"])
    with torch.no_grad():
        a = f64.forces(x, e, s)
        b = fmx.forces(x, e, s)
    err = float(torch.linalg.norm(b - a) / torch.linalg.norm(a))
    assert err <= 1e-5, err


@pytest.fixture(scope="module")
def report(case):
    from lammps_b200.forcematch import gradient_check

    return gradient_check(case, case["eps0"], case["sigma0"], h=H, ndirs=8, cut_factor=CUT)


def test_parameter_gradient_vs_central_differences(report):
    assert report["theta_grad_err_fp64"] <= 1e-6, report
    # the mixed (FP32 pair math) adjoint meets the same 1e-6 bar
    assert report["theta_grad_err_mixed"] <= 1e-6, report


def test_position_gradient_directional_and_full(report):
    assert report["x_dir_err_fp64"] <= 1e-6, report
    assert report["x_dir_err_mixed"] <= 1e-6, report
    assert report["x_hvp_mixed_vs_fp64"] <= 1e-5, report
