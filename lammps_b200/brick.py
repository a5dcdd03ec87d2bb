"""Spatial decomposition of one periodic box over ranks: the CommBrick path
(src/comm_brick.cpp) on top of the engine's per-call entry points.

Rank r owns the atoms inside brick r of a px x py x pz grid, with the
reference's brick bounds: sublo = boxlo + prd * (i * 1.0 / p), the last
brick ending at boxhi, an atom owned where sublo <= x < subhi
(Domain::set_local_box src/domain.cpp:292-316, Comm::set_proc_grid
src/comm.cpp:543-547).  A rank's context holds the WHOLE periodic box with
its owned atoms and, as ghosts, every atom of another rank whose periodic
distance to the brick, per dimension, is at most the ghost depth -- at the
atom's own coordinates: the builder forms periodic images as it does for a
single box.

How it differs from the reference, and why:

- Full neighbor lists with owner-only force writes, so no reverse
  communication of forces (CommBrick::reverse_comm, src/comm_brick.cpp:513).
- For EAM the ghost depth is twice the list cutoff: every ghost within the
  list cutoff of the brick then has its whole neighborhood on the rank and
  gets its own density, so the forward communication of F'(rho) in
  PairEAM::compute (src/MANYBODY/pair_eam.cpp:232) is not needed.
- A rank orders its atoms (owned and ghost) by global id.  The builder orders
  each cell by caller index, so every owned atom's neighbor list holds the
  same entries in the same order as in the single box: forces, and with them
  whole trajectories, are bit-identical to the single-box run.
- The exchange and borders steps (src/comm_brick.cpp:573-864) run at each
  rebuild through host memory; the per-step forward communication of ghost
  positions (src/comm_brick.cpp:444-511) stays on the device
  (b200_halo_pack / b200_halo_unpack and one all-to-all).

The ranks may all live in one process (`LocalComm`: one engine per rank, the
exchange a copy) or one per process (`DistComm`: torch.distributed, NCCL for
CUDA tensors, gloo for CPU tensors).  Every collective is taken by every rank
in the same order.
"""
from __future__ import annotations

import numpy as np
import torch

from .pair import PairEAM

# record columns of an atom sent between ranks
_GID, _TYPE, _IMG, _X, _V, _W = 0, 1, 2, 5, 8, 11


def pbc(x, image, lo, hi):
    """Domain::pbc for an orthogonal box (src/domain.cpp:478-560): x < lo ->
    x + prd, image - 1; x >= hi -> x - prd, max(x, lo), image + 1.  Same
    rounded operations as the device's wrap."""
    x = np.array(x, dtype=np.float64, copy=True)
    image = np.array(image, dtype=np.int64, copy=True)
    prd = hi - lo
    for d in range(3):
        xd = x[:, d]
        m = xd < lo[d]
        xd[m] = xd[m] + prd[d]
        image[m, d] -= 1
        m = xd >= hi[d]
        xd[m] = np.maximum(xd[m] - prd[d], lo[d])
        image[m, d] += 1
    return x, image


class BrickGrid:
    """px x py x pz bricks of the box [lo, hi); rank = cx + px*(cy + py*cz)."""

    def __init__(self, lo, hi, grid):
        self.lo = np.asarray(lo, dtype=np.float64)
        self.hi = np.asarray(hi, dtype=np.float64)
        self.prd = self.hi - self.lo
        self.grid = tuple(int(g) for g in grid)
        if len(self.grid) != 3 or min(self.grid) < 1:
            raise ValueError("brick grid must be three positive counts")
        self.nranks = self.grid[0] * self.grid[1] * self.grid[2]
        # split planes: boxlo + prd * (i * 1.0 / p); the last one is boxhi
        self.splits = []
        for d in range(3):
            p = self.grid[d]
            s = np.array([self.lo[d] + self.prd[d] * (i * 1.0 / p) for i in range(p)] + [self.hi[d]])
            self.splits.append(s)

    def coords(self, rank):
        px, py, _ = self.grid
        return rank % px, (rank // px) % py, rank // (px * py)

    def bounds(self, rank):
        c = self.coords(rank)
        blo = np.array([self.splits[d][c[d]] for d in range(3)])
        bhi = np.array([self.splits[d][c[d] + 1] for d in range(3)])
        return blo, bhi

    def owner(self, x):
        """Rank owning each (wrapped) position."""
        c = [np.searchsorted(self.splits[d][1:-1], x[:, d], side="right") for d in range(3)]
        px, py, _ = self.grid
        return (c[0] + px * (c[1] + py * c[2])).astype(np.int64)

    def near(self, x, rank, depth):
        """Atoms whose periodic distance to brick `rank` is at most `depth` in
        every dimension (a superset of those within `depth` in space)."""
        blo, bhi = self.bounds(rank)
        ok = np.ones(len(x), dtype=bool)
        tol = depth * (1.0 + 1e-12) + 1e-12 * float(np.max(self.prd))
        for d in range(3):
            if self.grid[d] == 1:
                continue
            xd = x[:, d]
            inside = (xd >= blo[d]) & (xd < bhi[d])
            L = self.prd[d]
            dist = np.minimum(np.mod(blo[d] - xd, L), np.mod(xd - bhi[d], L))
            ok &= inside | (dist <= tol)
        return ok


# ---- communicators ------------------------------------------------------------

class LocalComm:
    """Every rank of the decomposition in this process; an exchange is a copy."""

    def __init__(self, world):
        self.world = int(world)
        self.ranks = list(range(self.world))

    def alltoall_rows(self, send, send_counts, recv_counts=None):
        parts = {p: torch.split(send[p], list(send_counts[p])) for p in self.ranks}
        out = {}
        for q in self.ranks:
            rc = [int(send_counts[p][q]) for p in self.ranks]
            out[q] = (torch.cat([parts[p][q] for p in self.ranks]), rc)
        return out

    def allreduce(self, vals, op="sum"):
        a = np.array([np.asarray(vals[r], dtype=np.float64) for r in self.ranks])
        return a.max(axis=0) if op == "max" else a.sum(axis=0)


class DistComm:
    """One rank per process over torch.distributed (NCCL for CUDA tensors,
    gloo for CPU tensors); `alltoall_rows` is one all_to_all_single with the
    per-rank row counts as split sizes."""

    def __init__(self, device=None):
        import torch.distributed as dist
        self.dist = dist
        self.world = dist.get_world_size()
        self.rank = dist.get_rank()
        self.ranks = [self.rank]
        backend = dist.get_backend()
        if device is None:
            device = (f"cuda:{torch.cuda.current_device()}" if backend == "nccl" else "cpu")
        self.dev = torch.device(device)

    def alltoall_rows(self, send, send_counts, recv_counts=None):
        r = self.rank
        sc = [int(c) for c in send_counts[r]]
        if recv_counts is None:
            t = torch.tensor(sc, dtype=torch.int64, device=self.dev)
            o = torch.empty_like(t)
            self.dist.all_to_all_single(o, t)
            rc = [int(c) for c in o.tolist()]
        else:
            rc = [int(c) for c in recv_counts[r]]
        x = send[r]
        src_dev = x.device
        x = x.to(self.dev).contiguous()
        out = torch.empty((sum(rc),) + tuple(x.shape[1:]), dtype=x.dtype, device=self.dev)
        self.dist.all_to_all_single(out, x, output_split_sizes=rc, input_split_sizes=sc)
        return {r: (out.to(src_dev), rc)}

    def allreduce(self, vals, op="sum"):
        t = torch.tensor(np.asarray(vals[self.rank], dtype=np.float64), device=self.dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX if op == "max" else self.dist.ReduceOp.SUM)
        return t.cpu().numpy()


# ---- the decomposed run ---------------------------------------------------------

class _Rank:
    def __init__(self, rank, engine):
        self.rank = rank
        self.engine = engine
        self.dev = torch.device(engine.device)


def _records(gid, typ, img, x, v):
    r = np.zeros((len(gid), _W))
    r[:, _GID] = gid
    r[:, _TYPE] = typ
    r[:, _IMG:_IMG + 3] = img
    r[:, _X:_X + 3] = x
    r[:, _V:_V + 3] = v
    return r


class BrickRun:
    """Verlet with fix nve over a brick-decomposed box (Verlet::setup and
    Verlet::run, src/verlet.cpp:88-142, 207-309, with CommBrick's exchange,
    borders and forward_comm and Neighbor::decide, src/neighbor.cpp:1294-1372).

    `engines` maps each rank of `comm.ranks` to a configured engine
    (`System`: box, pair style, masses, neighbor settings and timestep set;
    no atoms).  All engines must share those settings."""

    def __init__(self, comm, engines, grid):
        self.comm = comm
        self.grid = BrickGrid(*self._box(engines), grid)
        if self.grid.nranks != comm.world:
            raise ValueError(f"brick grid {grid} has {self.grid.nranks} bricks for {comm.world} ranks")
        if sorted(engines) != sorted(comm.ranks):
            raise ValueError("one engine per rank of this process")
        self.st = {r: _Rank(r, engines[r]) for r in comm.ranks}
        e0 = engines[comm.ranks[0]]
        self.every, self.delay, self.check = e0.every, e0.delay, e0.check
        self.cutneigh = e0.cutforce() + e0.skin
        self.depth = self.cutneigh * (2.0 if isinstance(e0.pair, PairEAM) else 1.0)
        self.mass = np.asarray(e0.mass, dtype=np.float64)
        self.e0 = e0
        self.natoms = 0
        self.ntimestep = 0
        self.ago = 0
        self.ncalls = 0
        self.ndanger = 0
        self.thermo_every = 0
        self.thermo_rows = []

    @staticmethod
    def _box(engines):
        e = next(iter(engines.values()))
        return np.asarray(e.box_lo, dtype=np.float64), np.asarray(e.box_hi, dtype=np.float64)

    # ---- atoms in, atoms out ------------------------------------------------
    def set_atoms(self, x, type_=None, v=None):
        """Distribute a whole system: every process passes the same arrays (as
        every rank reads a data file); global ids are the row numbers."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        n = len(x)
        typ = np.ones(n, np.int64) if type_ is None else np.asarray(type_, dtype=np.int64)
        v = np.zeros((n, 3)) if v is None else np.asarray(v, dtype=np.float64)
        xw, img = pbc(x, np.zeros((n, 3), np.int64), self.grid.lo, self.grid.hi)
        own = self.grid.owner(xw)
        gid = np.arange(n, dtype=np.int64)
        owned = {}
        for r in self.comm.ranks:
            m = own == r
            owned[r] = _records(gid[m], typ[m], img[m], xw[m], v[m])
        self.natoms = n
        self._borders(owned)

    def gather(self):
        """Positions, velocities and image flags of all atoms by global id, on
        every rank (for checks and output)."""
        send, cnt = {}, {}
        for r, s in self.st.items():
            own = self._owned_records(s, wrap=False)
            send[r] = torch.from_numpy(np.tile(own, (self.comm.world, 1)))
            cnt[r] = [len(own)] * self.comm.world
        got = self.comm.alltoall_rows(send, cnt)
        rows = got[self.comm.ranks[0]][0].cpu().numpy()
        order = np.argsort(rows[:, _GID], kind="stable")
        rows = rows[order]
        return dict(x=rows[:, _X:_X + 3].copy(), v=rows[:, _V:_V + 3].copy(),
                    image=rows[:, _IMG:_IMG + 3].astype(np.int64), type=rows[:, _TYPE].astype(np.int64))

    def _owned_records(self, s, wrap):
        d = s.engine.download()
        own = ~s.ghost
        x = d["x"][own]
        img = s.image[own] + d["image"][own]
        if wrap:
            x, img = pbc(x, img, self.grid.lo, self.grid.hi)
        return _records(s.gid[own], s.type[own], img, x, d["v"][own])

    # ---- CommBrick::exchange + borders ---------------------------------------
    def _exchange(self, owned):
        """Send every owned atom to the rank whose brick holds it."""
        send, cnt = {}, {}
        for r, rec in owned.items():
            dest = self.grid.owner(rec[:, _X:_X + 3])
            order = np.argsort(dest, kind="stable")
            send[r] = torch.from_numpy(np.ascontiguousarray(rec[order]))
            cnt[r] = np.bincount(dest, minlength=self.comm.world).tolist()
        got = self.comm.alltoall_rows(send, cnt)
        out = {}
        for r, (rows, _) in got.items():
            rows = rows.cpu().numpy()
            out[r] = rows[np.argsort(rows[:, _GID], kind="stable")]
        return out

    def _borders(self, owned):
        """Ghosts: each rank sends to every other rank its owned atoms within
        the ghost depth of that rank's brick; then each rank orders its atoms
        by global id, uploads them and builds its lists."""
        send, cnt, sel = {}, {}, {}
        for r, rec in owned.items():
            x = rec[:, _X:_X + 3]
            parts, c, ss = [], [], []
            for q in range(self.comm.world):
                k = (np.zeros(0, np.int64) if q == r
                     else np.nonzero(self.grid.near(x, q, self.depth))[0])
                g = rec[k].copy()
                g[:, _IMG:_IMG + 3] = 0
                g[:, _V:_V + 3] = 0
                parts.append(g)
                c.append(len(k))
                ss.append(k)
            send[r] = torch.from_numpy(np.concatenate(parts) if parts else np.zeros((0, _W)))
            cnt[r] = c
            sel[r] = ss
        got = self.comm.alltoall_rows(send, cnt)
        for r, (grec, rc) in got.items():
            s = self.st[r]
            own = owned[r]
            grec = grec.cpu().numpy()
            allr = np.concatenate([own, grec])
            order = np.argsort(allr[:, _GID], kind="stable")
            pos = np.empty(len(allr), np.int64)
            pos[order] = np.arange(len(allr))
            rows = allr[order]
            s.gid = rows[:, _GID].astype(np.int64)
            s.type = rows[:, _TYPE].astype(np.int64)
            s.image = rows[:, _IMG:_IMG + 3].astype(np.int64)
            s.ghost = np.zeros(len(rows), dtype=bool)
            s.ghost[pos[len(own):]] = True
            s.send_counts = list(cnt[r])
            s.recv_counts = list(rc)
            s.send_idx = torch.from_numpy(
                np.concatenate([pos[k] for k in sel[r]]).astype(np.int32)).to(s.dev)
            s.recv_idx = torch.from_numpy(pos[len(own):].astype(np.int32)).to(s.dev)
            e = s.engine
            e.set_atoms(rows[:, _X:_X + 3], s.type.astype(np.int32), rows[:, _V:_V + 3])
            e.set_ghosts(s.ghost.astype(np.int32) if s.ghost.any() else None)
            e.neigh_build()

    def _rebuild(self):
        owned = {r: self._owned_records(s, wrap=True) for r, s in self.st.items()}
        self._borders(self._exchange(owned))
        self.ago = 0
        self.ncalls += 1

    # ---- CommBrick::forward_comm ---------------------------------------------
    def _forward(self):
        send, cnt, rcnt = {}, {}, {}
        for r, s in self.st.items():
            buf = torch.empty((len(s.send_idx), 3), dtype=torch.float64, device=s.dev)
            s.engine.halo_pack(s.send_idx, buf)
            send[r], cnt[r], rcnt[r] = buf, s.send_counts, s.recv_counts
        got = self.comm.alltoall_rows(send, cnt, rcnt)
        for r, (buf, _) in got.items():
            s = self.st[r]
            if s.dev.type == "cuda":
                torch.cuda.current_stream(s.dev).synchronize()
            s.engine.halo_unpack(s.recv_idx, buf.contiguous())

    # ---- Neighbor::decide ------------------------------------------------------
    def _decide(self, moved):
        self.ago += 1
        if self.ago >= self.delay and self.ago % self.every == 0:
            if not self.check:
                return True
            flag = bool(self.comm.allreduce({r: [float(m)] for r, m in moved.items()}, "max")[0])
            if flag and self.ago == max(self.every, self.delay):
                self.ndanger += 1
            return flag
        return False

    # ---- thermo ----------------------------------------------------------------
    def _force(self, thermo):
        rows = {}
        for r, s in self.st.items():
            if thermo:
                o = s.engine.compute(1, 1, per_atom=True)
                own = ~s.ghost
                rows[r] = np.concatenate([[0.0, o["eatom"][own].sum()], o["vatom"][own].sum(axis=0)])
            else:
                s.engine.compute(0, 0)
        return rows

    def _thermo_row(self, rows):
        for r, s in self.st.items():
            d = s.engine.download()
            own = ~s.ghost
            v = d["v"][own]
            rows[r][0] = float(np.sum(self.mass[s.type[own]] * np.sum(v * v, axis=1)))
        tot = self.comm.allreduce(rows, "sum")
        row = np.concatenate([[float(self.ntimestep)], tot])
        vol = float(np.prod(self.grid.prd))
        return self.e0._thermo(row, self.natoms, vol)

    # ---- Verlet ------------------------------------------------------------------
    def setup(self):
        rows = self._force(True)
        r = self._thermo_row(rows)
        self.thermo_rows = [r]
        self.ago = 0
        self.ncalls = 0
        return r

    def run(self, nsteps, thermo_every=0):
        out = []
        for k in range(1, nsteps + 1):
            self.ntimestep += 1
            thermo = (thermo_every > 0 and k % thermo_every == 0) or k == nsteps
            for s in self.st.values():
                s.engine.nve_initial()
            moved = {r: (s.engine.neigh_check() if self.check else False) for r, s in self.st.items()}
            if self._decide(moved):
                self._rebuild()
            else:
                self._forward()
            rows = self._force(thermo)
            for s in self.st.values():
                s.engine.nve_final()
            if thermo:
                out.append(self._thermo_row(rows))
        self.thermo_rows.extend(out)
        return out

    def stats(self):
        """Atoms held per rank: owned and ghost."""
        return {r: dict(owned=int((~s.ghost).sum()), ghost=int(s.ghost.sum()))
                for r, s in self.st.items()}
