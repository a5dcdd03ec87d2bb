"""Differentiable force matching for pair_style lj/cut on the B200 engine.

`LJForceField` holds one box of typed atoms in an engine context; its
`forces(x, eps, sigma)` returns per-atom forces as a torch tensor that is
differentiable with respect to the positions and to the per-type-pair
epsilon and sigma.  Forward and backward both run on the GPU: the forward
pass is PairLJCut's pair force (src/pair_lj_cut.cpp:100-113) with
lj1 = 48 eps sigma^12 and lj2 = 24 eps sigma^6 (PairLJCut::init_one,
src/pair_lj_cut.cpp:560-563), and the backward pass is the engine's adjoint
kernel (dL/dx as the Hessian-vector product of the forces with dL/dF, and
dL/dlj1, dL/dlj2 per type pair); torch carries the chain rule from lj1, lj2
to epsilon and sigma.

The cutoff of a type pair is `cut_factor * sigma` (2.5 sigma by default) and
is not differentiated: a pair that crosses the cutoff under a parameter
change contributes a jump that finite differences see and a gradient cannot.

With precision "mixed" the pair arithmetic is FP32 on separations formed from
32-bit fixed-point coordinates and every sum is FP64; "fp64" is the FP64
reference form.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .system import System

MAX_TYPES = 4  # MD_ADJ_MAXTYPES of the engine


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def lj_tables(eps, sigma, cut_factor: float = 2.5):
    """(ntypes+1)^2 tables from symmetric per-type-pair eps and sigma.

    eps, sigma: torch tensors of shape (ntypes+1, ntypes+1) (row and column 0
    unused).  Returns (lj1, lj2) as differentiable flattened tensors and
    cutsq as a detached numpy array."""
    lj1 = 48.0 * eps * sigma ** 12
    lj2 = 24.0 * eps * sigma ** 6
    cut = cut_factor * sigma.detach().cpu().numpy()
    cutsq = np.ascontiguousarray((cut * cut).ravel(), dtype=np.float64)
    return lj1.reshape(-1), lj2.reshape(-1), cutsq


def pair_matrix(values, ntypes: int):
    """Symmetric (ntypes+1)^2 tensor from the upper-triangle values
    (1,1), (1,2), ..., (1,n), (2,2), ... (torch, differentiable)."""
    import torch

    m = torch.zeros((ntypes + 1, ntypes + 1), dtype=values.dtype, device=values.device)
    k = 0
    rows, cols = [], []
    for i in range(1, ntypes + 1):
        for j in range(i, ntypes + 1):
            rows.append(i)
            cols.append(j)
            k += 1
    if values.numel() != k:
        raise ValueError(f"expected {k} pair values for {ntypes} types, got {values.numel()}")
    r = torch.tensor(rows)
    c = torch.tensor(cols)
    m = m.index_put((r, c), values)
    m = m.index_put((c, r), values)
    return m


class LJForceField:
    """A box of typed atoms whose LJ forces can be differentiated.

    box_lo, box_hi: orthogonal periodic box; types: 1-based ints (n);
    x0: initial positions (n, 3) used to size the context; skin: list skin
    added to the largest cutoff the force field will be asked for
    (max_cut)."""

    def __init__(self, box_lo, box_hi, x0, types, ntypes: int, max_cut: float,
                 precision: str = "mixed", skin: float = 0.3, device: int = 0):
        if not (1 <= ntypes <= MAX_TYPES):
            raise ValueError(f"force matching supports 1..{MAX_TYPES} types")
        self.ntypes = ntypes
        self.precision = precision
        self.sys = System("lj", precision, device)
        self._L = self.sys._L
        self.sys.set_box(box_lo, box_hi)
        self.sys.set_neighbor(skin, every=1, delay=0, check=False)
        w = ntypes + 1
        # the list is built once for the largest cutoff; any cutsq up to it
        # can then be evaluated without a rebuild
        big = np.zeros(w * w)
        for a in range(1, w):
            for b in range(1, w):
                big[a * w + b] = max_cut * max_cut
        z = np.zeros(w * w)
        self.sys._ck(self._L.b200_set_lj(self.sys._h, ntypes, _dp(big), _dp(z), _dp(z), _dp(z),
                                         _dp(z), _dp(z)))
        self.sys.ntypes = ntypes
        self.sys.set_mass([1.0] * ntypes)
        self.max_cutsq = max_cut * max_cut
        self.sys.set_atoms(np.asarray(x0, dtype=np.float64),
                           np.asarray(types, dtype=np.int32), None)
        self.sys.neigh_build()
        self.n = len(types)
        self._x_ptr = None

    def close(self):
        self.sys.close()

    def set_positions(self, x):
        """Device positions (torch, float64, (n, 3), contiguous) -> context
        and a fresh neighbor list."""
        if x.dtype.is_floating_point is False or x.shape != (self.n, 3):
            raise ValueError("positions must be a float tensor of shape (n, 3)")
        import torch

        xc = x.detach().to(dtype=torch.float64).contiguous()
        # the engine reads xc on its own stream: finish torch's work on it first
        torch.cuda.synchronize(xc.device)
        self.sys._ck(self._L.b200_adj_set_positions(self.sys._h, C.c_void_p(xc.data_ptr())))
        self._x_ptr = xc

    def _check_cutsq(self, cutsq):
        if np.any(cutsq > self.max_cutsq * (1 + 1e-12)):
            raise ValueError("a cutoff exceeds the max_cut the force field was built for")

    def forces_raw(self, lj1: np.ndarray, lj2: np.ndarray, cutsq: np.ndarray, out):
        """F for the current positions into the device tensor `out` (n, 3)."""
        self._check_cutsq(cutsq)
        self.sys._ck(self._L.b200_adj_forces(self.sys._h, _dp(lj1), _dp(lj2), _dp(cutsq),
                                             C.c_void_p(out.data_ptr())))
        return out

    def backward_raw(self, lj1, lj2, cutsq, g, gx):
        """dL/dx into `gx` and (dL/dlj1, dL/dlj2) as numpy tables, given g = dL/dF."""
        w = self.ntypes + 1
        glj1 = np.zeros(w * w)
        glj2 = np.zeros(w * w)
        self.sys._ck(self._L.b200_adj_backward(self.sys._h, _dp(lj1), _dp(lj2), _dp(cutsq),
                                               C.c_void_p(g.data_ptr()),
                                               C.c_void_p(gx.data_ptr()), _dp(glj1), _dp(glj2)))
        return glj1, glj2

    def forces(self, x, eps, sigma, cut_factor: float = 2.5):
        """Differentiable forces: x (n, 3) float64 CUDA tensor; eps, sigma
        (ntypes+1, ntypes+1) symmetric tensors (CPU or CUDA)."""
        lj1, lj2, cutsq = lj_tables(eps, sigma, cut_factor)
        return _LJForces.apply(x, lj1, lj2, self, cutsq)


def _make_function():
    import torch

    class LJForces(torch.autograd.Function):
        @staticmethod
        def forward(ctx, x, lj1, lj2, ff, cutsq):
            ff.set_positions(x)
            l1 = np.ascontiguousarray(lj1.detach().cpu().numpy(), dtype=np.float64)
            l2 = np.ascontiguousarray(lj2.detach().cpu().numpy(), dtype=np.float64)
            f = torch.empty((ff.n, 3), dtype=torch.float64, device=x.device)
            torch.cuda.synchronize(x.device)
            ff.forces_raw(l1, l2, cutsq, f)
            ctx.save_for_backward(x, lj1, lj2)
            ctx.ff, ctx.cutsq, ctx.l1, ctx.l2 = ff, cutsq, l1, l2
            return f

        @staticmethod
        def backward(ctx, gf):
            x, lj1, lj2 = ctx.saved_tensors
            ff = ctx.ff
            ff.set_positions(x)
            g = gf.detach().to(torch.float64).contiguous()
            gx = torch.empty((ff.n, 3), dtype=torch.float64, device=x.device)
            torch.cuda.synchronize(x.device)
            glj1, glj2 = ff.backward_raw(ctx.l1, ctx.l2, ctx.cutsq, g, gx)
            t1 = torch.from_numpy(glj1).to(dtype=lj1.dtype, device=lj1.device)
            t2 = torch.from_numpy(glj2).to(dtype=lj2.dtype, device=lj2.device)
            return gx, t1, t2, None, None

    return LJForces


class _Lazy:
    fn = None

    def apply(self, *args):
        if _Lazy.fn is None:
            _Lazy.fn = _make_function()
        return _Lazy.fn.apply(*args)


_LJForces = _Lazy()


def force_matching_case(nx: int = 10, ny: int = 10, nz: int = 20, rho: float = 0.85,
                        jitter: float = 0.05, seed: int = 4242):
    """The 2-type force-matching configuration: fcc nx x ny x nz cells at
    reduced density rho, Gaussian jitter (sigma units), types split 50/50 by a
    seeded shuffle; hidden eps_ij ~ U(0.5, 1.5) and sigma_ij ~ U(0.9, 1.1)
    for (1,1), (1,2), (2,2).  Returns a dict of numpy inputs."""
    from .inputs import lattice, lj_lattice_constant

    rng = np.random.default_rng(seed)
    a = lj_lattice_constant("fcc", rho)
    x = lattice("fcc", nx, ny, nz, a)
    x = x + rng.normal(scale=jitter, size=x.shape)
    n = len(x)
    types = np.ones(n, np.int32)
    types[rng.permutation(n)[: n // 2]] = 2
    eps = rng.uniform(0.5, 1.5, size=3)
    sigma = rng.uniform(0.9, 1.1, size=3)
    hi = np.array([nx * a, ny * a, nz * a])
    x = np.mod(x, hi)
    return dict(x=x, types=types, lo=np.zeros(3), hi=hi, eps=eps, sigma=sigma, ntypes=2)


def gradient_check(case: dict, eps0, sigma0, h: float = 1e-5, ndirs: int = 8,
                   cut_factor: float = 2.5, seed: int = 5, device: int = 0):
    """Gradients of the force-matching loss L = mean_i |F_i(theta) - F_target_i|^2
    at (eps0, sigma0) from the FP64 and mixed adjoints, against FP64 central
    differences with step h: the 6 parameters (cutoffs held at their values)
    and `ndirs` random unit directions in position space (atoms of pairs
    within 10 h of a cutoff held still).  Targets are the FP64 forces at the
    case's hidden parameters.  Returns the errors (relative to the largest
    finite difference, or to |dL/dx|) and the wall time of one mixed
    forward + backward."""
    import time

    import torch
    from scipy.spatial import cKDTree

    nt = case["ntypes"]
    max_cut = cut_factor * max(np.max(case["sigma"]), np.max(sigma0)) * 1.05
    f64 = LJForceField(case["lo"], case["hi"], case["x"], case["types"], nt, max_cut, "fp64",
                       device=device)
    fmx = LJForceField(case["lo"], case["hi"], case["x"], case["types"], nt, max_cut, "mixed",
                       device=device)
    dev = torch.device("cuda", device)

    def mats(e, s):
        return (pair_matrix(torch.as_tensor(np.asarray(e), dtype=torch.float64), nt),
                pair_matrix(torch.as_tensor(np.asarray(s), dtype=torch.float64), nt))

    x0 = torch.tensor(case["x"], dtype=torch.float64, device=dev)
    with torch.no_grad():
        ft = f64.forces(x0, *mats(case["eps"], case["sigma"]), cut_factor=cut_factor)

    def grads(field):
        x = x0.clone().requires_grad_(True)
        ev = torch.tensor(np.asarray(eps0), dtype=torch.float64, requires_grad=True)
        sv = torch.tensor(np.asarray(sigma0), dtype=torch.float64, requires_grad=True)
        f = field.forces(x, pair_matrix(ev, nt), pair_matrix(sv, nt), cut_factor=cut_factor)
        loss = ((f - ft) ** 2).sum(dim=1).mean()
        gx, ge, gs = torch.autograd.grad(loss, (x, ev, sv))
        return loss.detach().item(), gx.detach(), np.concatenate([ge.numpy(), gs.numpy()])

    sig = pair_matrix(torch.as_tensor(np.asarray(sigma0), dtype=torch.float64), nt).numpy()
    cutsq = np.ascontiguousarray(((cut_factor * sig) ** 2).ravel())

    def loss_fixed(x, e, s):
        em, sm = mats(e, s)
        lj1 = np.ascontiguousarray((48.0 * em * sm ** 12).reshape(-1).numpy())
        lj2 = np.ascontiguousarray((24.0 * em * sm ** 6).reshape(-1).numpy())
        f64.set_positions(x)
        f = torch.empty_like(x)
        f64.forces_raw(lj1, lj2, cutsq, f)
        return float(((f - ft) ** 2).sum(dim=1).mean())

    L64, gx64, gt64 = grads(f64)
    Lmx, gxmx, gtmx = grads(fmx)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(5):
        grads(fmx)
    torch.cuda.synchronize(dev)
    t_fb = (time.perf_counter() - t0) / 5

    th = np.concatenate([np.asarray(eps0, float), np.asarray(sigma0, float)])
    k = len(th) // 2
    fd = np.zeros(len(th))
    for p in range(len(th)):
        tp, tm = th.copy(), th.copy()
        tp[p] += h
        tm[p] -= h
        fd[p] = (loss_fixed(x0, tp[:k], tp[k:]) - loss_fixed(x0, tm[:k], tm[k:])) / (2 * h)
    scale = np.max(np.abs(fd))

    xs = case["x"]
    t = case["types"]
    hi = case["hi"]
    tree = cKDTree(xs, boxsize=hi)
    pairs = tree.query_pairs(max_cut, output_type="ndarray")
    d = xs[pairs[:, 0]] - xs[pairs[:, 1]]
    d -= hi * np.round(d / hi)
    r = np.linalg.norm(d, axis=1)
    near = np.abs(r - cut_factor * sig[t[pairs[:, 0]], t[pairs[:, 1]]]) < 10 * h
    still = np.zeros(len(xs), bool)
    still[pairs[near, 0]] = True
    still[pairs[near, 1]] = True
    rng = np.random.default_rng(seed)
    gnorm = float(torch.linalg.norm(gx64))
    dir64 = dirmx = 0.0
    for _ in range(ndirs):
        u = rng.standard_normal(xs.shape)
        u[still] = 0.0
        u /= np.linalg.norm(u)
        ut = torch.tensor(u, dtype=torch.float64, device=dev)
        fdu = (loss_fixed(x0 + h * ut, th[:k], th[k:]) - loss_fixed(x0 - h * ut, th[:k], th[k:])) / (2 * h)
        dir64 = max(dir64, abs(float((gx64 * ut).sum()) - fdu) / gnorm)
        dirmx = max(dirmx, abs(float((gxmx * ut).sum()) - fdu) / gnorm)
    out = {
        "atoms": len(xs), "loss_fp64": L64, "loss_mixed": Lmx,
        "theta_grad_err_fp64": float(np.max(np.abs(gt64 - fd)) / scale),
        "theta_grad_err_mixed": float(np.max(np.abs(gtmx - fd)) / scale),
        "x_dir_err_fp64": dir64, "x_dir_err_mixed": dirmx,
        "x_hvp_mixed_vs_fp64": float(torch.linalg.norm(gxmx - gx64) / torch.linalg.norm(gx64)),
        "atoms_held_still": int(still.sum()), "h": h, "directions": ndirs,
        "mixed_forward_backward_ms": 1e3 * t_fb,
    }
    f64.close()
    fmx.close()
    return out
