"""The multi-GPU path's exchange logic on CPU: two gloo ranks.

KPM probes are sharded across ranks; each rank's raw dot products are
all-gathered and the moments accumulated in the global probe order.  The
result must equal, bit for bit, the accumulation of all dots in one process.
Slice results are gathered in slice order.  The per-rank dots come from the
CPU oracle here (on GPUs they come from the library)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from evsl_b200 import parallel as P

MDEG, NVEC, INTV = 25, 7, [0.9, 2.4, 0.0, 12.0]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import torch.distributed as dist

    from oracle import evsl_oracle as O

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ia, ja, a = O.lap_csr(6, 5, 4)
        n = len(ia) - 1
        probes = O.seeded_rademacher(NVEC, n, 21)
        s0, s1 = P.shard(NVEC, rank, world)
        local = O.kpm_raw_dots(MDEG, probes[s0:s1], INTV, ia, ja, a)
        mu, ec = P.combine_kpm_dots(local, NVEC, MDEG, 1, n, INTV)
        ev = O.exeiglap3(6, 5, 4, -1, 100)
        sli = np.linspace(0.5, 6.0, 6)
        res = P.solve_slices_sharded(lambda s: int(np.count_nonzero((ev >= sli[s]) & (ev < sli[s + 1]))), 5)
        q.put((rank, mu, ec, res))
    finally:
        dist.destroy_process_group()


def test_shard_partitions():
    for count in (0, 1, 5, 7, 64):
        for world in (1, 2, 3, 8):
            parts = [P.shard(count, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == count
            assert all(parts[i][1] == parts[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in parts]
            assert max(sizes) - min(sizes) <= 1


def test_two_rank_kpm_and_slices_match_single_process():
    from oracle import evsl_oracle as O
    import evsl_b200

    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ia, ja, a = O.lap_csr(6, 5, 4)
    n = len(ia) - 1
    probes = O.seeded_rademacher(NVEC, n, 21)
    dots = O.kpm_raw_dots(MDEG, probes, INTV, ia, ja, a)
    mu1, ec1 = evsl_b200.kpm_accumulate(MDEG, 1, n, INTV, dots)
    mu_ref, ec_ref = O.kpmdos(MDEG, 1, probes, INTV, ia, ja, a)
    ev = O.exeiglap3(6, 5, 4, -1, 100)
    sli = np.linspace(0.5, 6.0, 6)
    counts = [int(np.count_nonzero((ev >= sli[s]) & (ev < sli[s + 1]))) for s in range(5)]
    for rank, mu, ec, res in out:
        assert np.array_equal(mu, mu1) and ec == ec1, rank
        assert res == counts
    assert np.max(np.abs(mu1 - mu_ref)) <= 1e-13 * np.max(np.abs(mu_ref))
