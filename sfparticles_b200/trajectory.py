"""Device-side trajectories of selected particles.

The reference serves trajectory recording through ``Simulation.start``'s
``call_back(istep)`` (simulation.py:140-141, as used by
example/trajectory.py:62-70), which a device-resident step can only honour by
stopping after every step.  A ``Trajectory`` instead names the buffer slots
and the attributes to record and a period ``every``: the step loop ends its
device chunks on multiples of ``every`` and, after each such chunk, gathers
the slots' values into small device arrays (one host synchronisation per
record, none per step).  ``numpy()`` copies the records to the host once.

Slots are buffer indices.  Electrons and positrons are never pruned, so
their slots are stable for the whole simulation; photon slots are compacted
when ``start()`` returns (``_prune``), so a photon trajectory is valid within
one ``start()``.  A slot not yet filled when a record is taken (at or past
``N_buffered``) records NaN.  This is an extension of the reference.
"""
from __future__ import annotations

from typing import Dict, Iterable, List, Optional, Sequence

import numpy as np

_DEFAULT = ("x", "y", "z", "ux", "uy", "uz")
_SPIN = ("sx", "sy", "sz")
_STATE = _DEFAULT + _SPIN + ("tau",)  # what the fused step keeps per particle


class Trajectory(object):
    def __init__(self, species, index: Sequence[int], every: int = 1, attrs: Optional[Iterable[str]] = None):
        every = int(every)
        if every < 1:
            raise ValueError("every must be a positive number of steps")
        idx = np.asarray(index, dtype=np.int64).reshape(-1)
        if idx.size and idx.min() < 0:
            raise ValueError("slot indices must be non-negative")
        if attrs is None:
            attrs = _DEFAULT + tuple(a for a in _SPIN if a in species.attrs)
        attrs = tuple(attrs)
        for a in attrs:
            if a not in species.attrs or a not in _STATE:
                raise ValueError(f"{species.name} has no recordable attribute {a!r} (one of {_STATE})")
        self.species = species
        self.index = idx
        self.every = every
        self.attrs = attrs
        self.steps: List[int] = []  # steps completed when each record was taken
        self._rows: Dict[str, list] = {a: [] for a in attrs}
        self._idx = None  # the index as a tensor on the species' device

    def due(self, step: int) -> bool:
        """Whether a record belongs after `step` completed steps (each step
        once, whatever the chunking)."""
        return step % self.every == 0 and (not self.steps or self.steps[-1] != step)

    def steps_to_next(self, step: int) -> int:
        """Steps from `step` to the next record: a device chunk ends there."""
        return self.every - step % self.every

    def capture(self, step: int) -> None:
        """Record the slots' current values (device arrays of the species)."""
        import torch
        p = self.species
        n = int(p.N_buffered)
        first = p._d(self.attrs[0])
        dev = first.device
        if self._idx is None or self._idx.device != dev:
            self._idx = torch.as_tensor(self.index, dtype=torch.int64, device=dev)
        idx = self._idx
        valid = idx < n
        safe = torch.where(valid, idx, torch.zeros_like(idx))
        nan = torch.full((idx.numel(),), float("nan"), dtype=torch.float64, device=dev)
        for a in self.attrs:
            if n == 0 or idx.numel() == 0:
                self._rows[a].append(nan.clone())
                continue
            v = p._d(a).index_select(0, safe)
            self._rows[a].append(torch.where(valid, v, nan))
        if dev.type == "cuda":
            # the fused run steps on its own stream: its next launch must not
            # overwrite the arrays while these gathers still read them
            torch.cuda.current_stream(dev).synchronize()
        self.steps.append(int(step))

    def numpy(self) -> Dict[str, np.ndarray]:
        """{attribute: array [records, slots]} on the host, plus 'step'."""
        import torch
        out = {"step": np.asarray(self.steps, dtype=np.int64)}
        for a in self.attrs:
            rows = self._rows[a]
            out[a] = (torch.stack(rows).cpu().numpy() if rows
                      else np.zeros((0, self.index.size), dtype=np.float64))
        return out
