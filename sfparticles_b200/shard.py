"""Running one job on several GPUs, one process per GPU.

Particles never interact and the fields are analytic, so a job splits across
GPUs with no data exchange during the run:
- one collision's beam is split by particle (``split_counts``);
- a batch of independent collisions is split by expected work
  (``assign_instances``).

Each rank then runs its share as an ordinary ``Simulation`` or ``Ensemble``
with its own Philox key (``rank_seed``).  Nothing is exchanged per step.
The collectives are reductions of kilobytes:
- ``reduce_diagnostics``: every species' buffered and alive counts, the
  particle-steps and the photon energy spectrum, summed over the ranks in
  one all-reduce; ``JobDiagnostics`` runs it as a Simulation ``monitor`` at
  every ``print_every`` boundary and at the end of ``start``;
- ``reduce_job``: the maximum of the ranks' device times and the sum of
  their work (``sum_over_ranks`` for other totals, such as bytes copied).
They work with any ``torch.distributed`` backend: NCCL on GPUs (the vector
on the rank's device), gloo on CPUs.

This is an extension of the reference, which runs on one device.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np


def rank_seed(base: int, rank: int) -> int:
    """Philox key of `rank`'s share of a job keyed `base` (64-bit)."""
    return (int(base) + 0x9E3779B97F4A7C15 * (int(rank) + 1)) & (2 ** 64 - 1)


def split_counts(total: int, world: int) -> List[Tuple[int, int]]:
    """(start, count) of each rank's slice of `total` particles; the first
    `total % world` ranks take one more."""
    if world <= 0:
        raise ValueError("world size must be positive")
    base, extra = divmod(int(total), int(world))
    out, start = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((start, n))
        start += n
    return out


def assign_instances(costs: Sequence[float], world: int) -> List[List[int]]:
    """Instances (by index) for each rank. Longest expected work first, each
    to the rank with the least work so far; every rank's list stays in
    instance order."""
    if world <= 0:
        raise ValueError("world size must be positive")
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += float(costs[i])
    for lst in out:
        lst.sort()
    return out


def sum_over_ranks(values: Sequence[float], device=None) -> List[float]:
    """Each of `values` summed over the ranks (one all-reduce); the values
    themselves when torch.distributed is not initialised.  Every rank must
    call it at the same point with the same number of values."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [float(v) for v in t.tolist()]


def reduce_job(ms: float, particle_steps: float, device=None) -> Tuple[float, float]:
    """(max over ranks of `ms`, sum over ranks of `particle_steps`); the
    values themselves when torch.distributed is not initialised.  Every
    rank must call it at the same point."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(ms), float(particle_steps)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    w = torch.tensor([float(particle_steps)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    return float(t.item()), float(w.item())


def _dist_on():
    import torch.distributed as dist
    return dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1


def local_diagnostics(species, particle_steps: float, bins: int = 64, lo: float = 2.0, hi: float = 2500.0):
    """This rank's diagnostics as one float64 vector: per species its
    buffered and its alive count, then the particle-steps, then the photon
    spectrum (alive photons of every massless species, `bins` log10 bins of
    energy / m_e c^2 over [lo, hi])."""
    from .diagnostics import photon_histogram
    v = []
    for p in species:
        v += [float(p.N_buffered), float(p.Npart)]
    v.append(float(particle_steps))
    h = np.zeros(bins)
    for p in species:
        if p.m == 0:
            h = h + photon_histogram(p, bins, lo, hi)
    return np.concatenate([np.asarray(v, dtype=np.float64), h])


def reduce_diagnostics(species, particle_steps: float, bins: int = 64, lo: float = 2.0, hi: float = 2500.0,
                       device=None) -> dict:
    """Job-wide diagnostics: `local_diagnostics` of every rank summed by one
    all-reduce (the local values when torch.distributed is not initialised).
    Every rank must call it at the same point, with species in the same
    order.  Returns {"buffered": {name: n}, "alive": {name: n},
    "particle_steps": n, "spectrum": counts[bins], "spectrum_range": (lo, hi)}."""
    v = local_diagnostics(species, particle_steps, bins, lo, hi)
    if _dist_on():
        import torch
        import torch.distributed as dist
        t = torch.as_tensor(v, dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        v = t.cpu().numpy()
    n = len(species)
    names = [p.name for p in species]
    return {"buffered": {nm: float(v[2 * i]) for i, nm in enumerate(names)},
            "alive": {nm: float(v[2 * i + 1]) for i, nm in enumerate(names)},
            "particle_steps": float(v[2 * n]), "spectrum": np.asarray(v[2 * n + 1:]), "spectrum_range": (lo, hi)}


class JobDiagnostics:
    """A Simulation ``monitor``: at every ``print_every`` boundary and at the
    end of ``start`` it reduces the counters and the photon spectrum over
    the ranks (``reduce_diagnostics``) and keeps (step, result) in
    ``history`` on every rank.  Every rank's Simulation must run the same
    steps with the same ``print_every``, so that the ranks reduce together."""

    def __init__(self, bins: int = 64, lo: float = 2.0, hi: float = 2500.0, device=None):
        self.bins, self.lo, self.hi, self.device = bins, lo, hi, device
        self.history = []

    def __call__(self, sim):
        r = reduce_diagnostics(sim.all_particles, sim.particle_steps, self.bins, self.lo, self.hi, self.device)
        self.history.append((sim.step, r))
        return r
