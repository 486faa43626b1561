"""Multi-GPU distribution of the spectrum-slicing path (one process per GPU).

EVSL has no distributed layer; its units of work are independent:

* slices (and slice requests) -- each rank solves its own share with no
  exchange at all (weak scaling);
* KPM probe vectors -- each rank runs the moment recurrence for its share of
  the probes, and the only exchange is one all-gather of the raw dot products
  (Mdeg x nvec doubles, a few hundred KB), after which every rank accumulates
  the moments in the global probe order.  Because each probe's dot products
  do not depend on which probes share its block (fixed reduction order), the
  sharded result is bit for bit the single-GPU kpmdos result.

The exchange uses torch.distributed (NCCL on GPUs, gloo on CPUs); the numerics
are the library's (`evsl_b200.Library`, `evsl_b200.kpm_accumulate`).
"""
from __future__ import annotations

import numpy as np


def shard(count: int, rank: int, world: int):
    """Contiguous block [start, stop) of `count` units for `rank` of `world`
    (the first count % world ranks get one more)."""
    base, extra = divmod(count, world)
    start = rank * base + min(rank, extra)
    stop = start + base + (1 if rank < extra else 0)
    return start, stop


def gather_columns(local: np.ndarray, count: int, group=None, device=None) -> np.ndarray:
    """All-gather the column blocks (rows x cols_r) of every rank, in rank
    order, into one rows x count array on every rank.  Ranks own contiguous
    blocks given by `shard`."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rows = local.shape[0]
    widths = [shard(count, r, world) for r in range(world)]
    maxw = max(b - a for a, b in widths)
    dev = device if device is not None else "cpu"
    buf = torch.zeros((rows, maxw), dtype=torch.float64, device=dev)
    buf[:, : local.shape[1]] = torch.from_numpy(np.ascontiguousarray(local)).to(dev)
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = np.empty((rows, count))
    for r, (a, b) in enumerate(widths):
        out[:, a:b] = parts[r][:, : b - a].cpu().numpy()
    return out


def combine_kpm_dots(local_dots: np.ndarray, nvec: int, Mdeg: int, damping: int, n: int, intv, group=None,
                     device=None):
    """Exchange the per-rank KPM dot products and accumulate the moments
    (identical on every rank)."""
    from . import kpm_accumulate

    dots = gather_columns(local_dots, nvec, group=group, device=device)
    return kpm_accumulate(Mdeg, damping, n, intv, dots)


def kpmdos_sharded(lib, Mdeg: int, damping: int, nvec: int, intv, group=None, device=None):
    """kpmdos over all ranks: rank r draws the generator's draws of its probe
    shard (the draws the single-GPU kpmdos would use), computes their dot
    products on its GPU, and the moments are combined.  Returns (mu, ecnt)
    equal bit for bit to `lib.kpmdos(Mdeg, damping, nvec, intv)` after the
    same `set_seed`."""
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    a, b = shard(nvec, rank, world)
    n = lib.n
    if b > a:
        probes = lib.draw_probes(n, a, b - a)
        local = lib.kpm_dots(Mdeg, intv, probes, b - a)
        probes.free()
    else:
        local = np.zeros((Mdeg, 0))
    return combine_kpm_dots(local, nvec, Mdeg, damping, n, intv, group=group, device=device)


def solve_slices_sharded(solve_one, nslices: int, group=None):
    """Run `solve_one(s)` for this rank's slices and gather every slice's
    result (a small picklable object) on every rank, in slice order."""
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    a, b = shard(nslices, rank, world)
    mine = [(s, solve_one(s)) for s in range(a, b)]
    everyone = [None] * world
    dist.all_gather_object(everyone, mine, group=group)
    out = [None] * nslices
    for part in everyone:
        for s, res in part:
            out[s] = res
    return out
