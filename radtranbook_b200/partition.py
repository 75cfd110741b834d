"""Particle-partitioned steps over several processes (one GPU each).

The reference's process-parallel IMC (IMC/IMC1DMPI.py, IMC/IMC2DMPI.py) gives every rank a
share of the particles (`_local_count`, IMC/IMC1DMPI.py:38-42 and :156-159), sums the
per-cell deposition and intensity over the ranks before the material update
(IMC/IMC1DMPI.py:282-285, IMC/IMC2DMPI.py:321-324), combs each rank's census locally to its
share of Nmax, and sums the ledger terms.  The same partition here, with two differences:

  - the ranks' shares add up to the totals exactly (N // world, plus one on the first
    N % world ranks; the reference gives every rank max(1, N // world));
  - every rank issues 1/world of the step's source energy (emission, fixed source, boundary
    faces and the initial census) with its share of the particles, so the union of the
    ranks' sources carries that energy once.  The reference's wrappers call the serial
    samplers with the local count, which issue the full energy on every rank
    (IMC/IMC2DMPI.py:205-299), so its radiation energy grows with the rank count.

Random numbers: a rank draws its sources and tracking with Philox particle ids offset by
rank * (2^32 // world), so the ranks' histories use disjoint counters of the one key (a bank
split into id ranges tracks exactly as the unsplit bank); its comb and initial census use a
per-rank key.  The only data exchange is one SUM all-reduce of the per-cell tallies per step
(plus the comb discrepancy when it is booked into the material) and one of a few ledger
scalars.
"""
from __future__ import annotations

import numpy as np
import torch

GOLDEN64 = 0x9E3779B97F4A7C15
MASK64 = (1 << 64) - 1


def local_count(n: int, rank: int, world: int) -> int:
    """This rank's share of n particles: the shares of all ranks add up to n."""
    n = int(n)
    if n <= 0:
        return 0
    return n // world + (1 if rank < n % world else 0)


def id_base(rank: int, world: int) -> int:
    """First Philox particle id of this rank's sources and bank entries."""
    return (rank * ((1 << 32) // world)) & 0xFFFFFFFF


def rank_key(seed: int, rank: int) -> int:
    """Philox key of this rank's comb and initial census (the seed itself on rank 0)."""
    return (int(seed) + rank * GOLDEN64) & MASK64


def world_of(dist) -> tuple[int, int]:
    """(rank, world) of a torch.distributed module, or (0, 1) for None."""
    if dist is None:
        return 0, 1
    return dist.get_rank(), dist.get_world_size()


def sum_tensors(dist, tensors: list) -> None:
    """Sum every tensor over the ranks in place, with one all-reduce of their concatenation."""
    if dist is None or dist.get_world_size() == 1:
        return
    sizes = [t.numel() for t in tensors]
    buf = torch.cat([t.reshape(-1).to(torch.float64) for t in tensors])
    dist.all_reduce(buf)
    o = 0
    for t, n in zip(tensors, sizes):
        t.copy_(buf[o:o + n].view_as(t))
        o += n


def sum_scalars(dist, values: list, device) -> list:
    """Sum a few FP64 scalars over the ranks (one all-reduce); returns Python floats."""
    if dist is None or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t)
    return [float(x) for x in t.cpu()]


def summary_totals(dist, sm, n_particles: int, device) -> dict:
    """The ledger terms and counts of a step summary (imc_step_summary) summed over the ranks
    with one all-reduce: radiation energy after the comb ('rad') and before ('comb_before'),
    boundary emission and escape by side, fixed-source and emission energy, tracked weight,
    census entries after the comb ('n_particles'), tracked entries ('n_bank') and the event
    statistics.  e_side_total / escaped_total: the sums over the sides."""
    if dist is None or dist.get_world_size() == 1:
        # one rank: the summary's own fields (this runs in the host time between two steps)
        return {"rad": sm.comb_after, "comb_before": sm.comb_before, "e_side": np.array(sm.e_side),
                "escaped": np.array(sm.escaped), "e_side_total": sum(sm.e_side), "escaped_total": sum(sm.escaped),
                "source_emission": sm.source_emission, "emission_total": sm.emission_total,
                "weight_sum": sm.weight_sum, "n_particles": int(n_particles), "n_bank": int(sm.n_bank),
                "stats": np.array(sm.stats, dtype=np.int64)}
    vals = ([float(sm.comb_after), float(sm.comb_before)] + [float(x) for x in sm.e_side]
            + [float(x) for x in sm.escaped]
            + [float(sm.source_emission), float(sm.emission_total), float(sm.weight_sum), float(n_particles),
               float(sm.n_bank)] + [float(x) for x in sm.stats])
    v = sum_scalars(dist, vals, device)
    return {"rad": v[0], "comb_before": v[1], "e_side": np.array(v[2:6]), "escaped": np.array(v[6:10]),
            "e_side_total": sum(v[2:6]), "escaped_total": sum(v[6:10]),
            "source_emission": v[10], "emission_total": v[11], "weight_sum": v[12], "n_particles": int(v[13]),
            "n_bank": int(v[14]), "stats": np.array(v[15:], dtype=np.int64)}
