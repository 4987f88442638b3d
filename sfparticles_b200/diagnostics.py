"""Diagnostics used to judge arithmetic forms against each other.

Photon energy spectrum dN/dlog10(eps) in log bins over [threshold, max] and
its relative L1 distance; pair yield and its relative difference.  Inputs
are host arrays of pruned species (after ``Simulation.start``)."""
from __future__ import annotations

import numpy as np


def photon_energies(photons) -> np.ndarray:
    """Photon energies in units of m_e c^2 (|u| of each photon)."""
    ux, uy, uz = photons.ux, photons.uy, photons.uz
    return np.sqrt(ux * ux + uy * uy + uz * uz)


def photon_spectrum(photons, bins: int = 64, lo: float = 2.0, hi: float = None, energies=None):
    """Counts in `bins` log10 bins over [lo, hi] (hi defaults to the largest energy)."""
    e = photon_energies(photons) if energies is None else np.asarray(energies)
    if e.size == 0:
        return np.zeros(bins), (lo, lo * 10)
    hi = float(e.max()) if hi is None else hi
    h, _ = np.histogram(np.log10(e), bins=bins, range=(np.log10(lo), np.log10(max(hi, lo * 1.0001))))
    return h.astype(float), (lo, hi)


def photon_spectrum_device(photons, bins: int = 64, lo: float = 2.0, hi: float = 2500.0) -> np.ndarray:
    """Counts in `bins` log10 bins over [lo, hi] of the alive photons of a
    species whose state is on the device (a run in progress), computed there;
    energies outside the range are not counted."""
    import torch
    n = photons.N_buffered
    if n == 0:
        return np.zeros(bins)
    alive = photons._d("_to_be_pruned")[:n] == 0
    ux, uy, uz = (photons._d(k)[:n] for k in ("ux", "uy", "uz"))
    le = 0.5 * torch.log10(ux * ux + uy * uy + uz * uz)
    le = le[alive & (le >= np.log10(lo)) & (le <= np.log10(hi))]
    h = torch.histc(le, bins=bins, min=float(np.log10(lo)), max=float(np.log10(hi)))
    return h.double().cpu().numpy()


def photon_histogram(photons, bins: int = 64, lo: float = 2.0, hi: float = 2500.0) -> np.ndarray:
    """Counts in `bins` log10 bins over [lo, hi] of the alive photons of a
    species, wherever its state is (device: computed there; host: numpy)."""
    if photons._gpu:
        return photon_spectrum_device(photons, bins, lo, hi)
    n = photons.N_buffered
    if n == 0:
        return np.zeros(bins)
    alive = ~np.asarray(photons._arr["_to_be_pruned"][:n], dtype=bool)
    ux, uy, uz = (np.asarray(photons._arr[k][:n])[alive] for k in ("ux", "uy", "uz"))
    le = 0.5 * np.log10(ux * ux + uy * uy + uz * uz)
    h, _ = np.histogram(le, bins=bins, range=(np.log10(lo), np.log10(hi)))
    return h.astype(float)


def spectrum_rel_l1(a: np.ndarray, b: np.ndarray) -> float:
    """sum |a - b| / sum b."""
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    return float(np.abs(a - b).sum() / max(b.sum(), 1e-300))


def rel_diff(a: float, b: float) -> float:
    return float(abs(a - b) / max(abs(b), 1e-300))
