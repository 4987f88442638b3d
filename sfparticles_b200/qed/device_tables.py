"""QED tables resident on the CUDA device, with their C-ABI descriptors."""
from __future__ import annotations

import numpy as np

from .. import _lib
from . import tables

_dev = {}


def _tensor(a, device):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=device).contiguous()


def rs_table(device):
    """(RSTable, keep-alive tensors) for the rejection-sampling method."""
    key = ("rs", str(device))
    if key not in _dev:
        iA, dA, zN, zmax = tables.rs_tables()
        ti, td = _tensor(iA, device), _tensor(dA, device)
        t = _lib.RSTable(ti.data_ptr(), td.data_ptr(), zN, 0, zmax)
        _dev[key] = (t, (ti, td))
    return _dev[key][0]


def od_tables(device):
    """(photon ODTable, pair ODTable) for the optical-depth method."""
    key = ("od", str(device))
    if key not in _dev:
        d = tables.od_tables()
        keep = []
        out = []
        for kind in ("photon", "pair"):
            rt = _tensor(d[f"{kind}_rate_total"], device)
            cu = _tensor(d[f"{kind}_cumulative"], device)
            keep += [rt, cu]
            n = int(rt.numel())
            lcm = float(d["log_chi_min"])
            lcd = float(d["log_chi_delta"])
            out.append(_lib.ODTable(rt.data_ptr(), cu.data_ptr(), n, int(cu.shape[1]), lcm, lcd, lcm + (n - 1) * lcd,
                                    float(d["log_delta_min"]), float(d["log_delta_delta"])))
        _dev[key] = (tuple(out), keep)
    return _dev[key][0]
