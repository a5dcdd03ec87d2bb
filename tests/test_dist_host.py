"""The multi-rank host path on CPU: two `gloo` ranks (world size 2, spawned
processes, rendezvous on 127.0.0.1).  Each rank takes its shard of a replica
batch (`replicas.shard_batch`: contiguous, atom-balanced, no exchange), and
the bench's rank reductions give the slowest rank's time and the summed
work.  No GPU is touched."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

WORLD = 2


def _batch():
    from lammps_b200.replicas import replica_batch
    return replica_batch(nrep=9, seed=7, nmin=32, nmax=600, nlo=2, nhi=5)


def _worker(rank, port, result_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD)
    try:
        import bench
        from lammps_b200.replicas import shard_batch
        full = _batch()
        sh = shard_batch(full, rank, WORLD)
        got = [None] * WORLD
        dist.all_gather_object(got, sh["replicas"].tolist())
        t_max = bench.allmax(1.0 + rank, WORLD, torch)
        n_sum = bench.allsum(float(len(sh["x"])), WORLD, torch)
        np.savez(os.path.join(result_dir, f"rank{rank}.npz"), replicas=np.array(sh["replicas"]),
                 natoms=sh["natoms"], x=sh["x"], gathered=np.array(sum(got, [])),
                 t_max=t_max, n_sum=n_sum)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_shard_replicas_and_reduce(tmp_path):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, port, str(tmp_path))) for r in range(WORLD)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0, p.exitcode
    full = _batch()
    res = [np.load(tmp_path / f"rank{r}.npz") for r in range(WORLD)]
    # the shards partition the batch, in order, with each rank's atoms
    allrep = np.concatenate([r["replicas"] for r in res])
    assert np.array_equal(allrep, np.arange(len(full["natoms"])))
    assert np.array_equal(res[0]["gathered"], allrep)
    assert np.array_equal(np.concatenate([r["x"] for r in res]), full["x"])
    # atom-balanced: no shard holds more than half the atoms plus one replica
    tot = int(full["natoms"].sum())
    for r in res:
        assert int(r["natoms"].sum()) <= tot / WORLD + int(full["natoms"].max())
    # the bench's reductions: slowest rank's time, summed work
    assert all(float(r["t_max"]) == 2.0 for r in res)
    assert all(float(r["n_sum"]) == float(tot) for r in res)


def test_shard_batch_single_rank_is_identity():
    from lammps_b200.replicas import shard_batch
    full = _batch()
    sh = shard_batch(full, 0, 1)
    assert np.array_equal(sh["x"], full["x"])
    assert np.array_equal(sh["natoms"], full["natoms"])
    with pytest.raises(ValueError):
        shard_batch(full, 2, 2)
