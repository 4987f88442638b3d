"""Particle species: the reference's ``Particles`` / ``SpinParticles`` API
(sfparticles/particles.py) over device-resident SoA buffers.

Same constructor arguments, assertions, attribute names (``x, y, z, ux, uy,
uz, inv_gamma, chi, Ex..Bz, _to_be_pruned``, plus ``event``, ``photon_delta``
/ ``pair_delta``, ``tau`` and ``sx, sy, sz``), ``N_buffered`` /
``buffer_size`` bookkeeping with the reference growth rule, and the private
step methods the reference's tests call directly (``_eval_field``,
``_calculate_chi``, ``_photon_event``, ``_pair_event``, ``_pick_hard_photon``,
``_create_photon``, ``_create_pair``, ``_push_position``, ``_push_momentum``,
``_extend``, ``_prune``, ``_to_gpu``, ``_to_host``).

Storage: every attribute array lives either on the host (numpy) or on the
CUDA device (torch tensors used as raw device memory).  Reading an attribute
always returns a numpy array -- the host array itself while the species is on
the host, a (cached) copy while it is on the device, as the reference's
GPU mode returns host data after ``start``.  The compute methods move the
species to the device and run libsfp.so kernels; nothing computes on the host.

Arrays the reference keeps as per-step scratch (``chi``, ``Ex..Bz``,
``event``, ``photon_delta`` / ``pair_delta``) are created on first use; the
fused ``Simulation`` step keeps only positions, momenta, spin, optical depth
and the prune flags in HBM and does not refresh the scratch arrays.
"""
from __future__ import annotations

import ctypes
import os
from enum import Enum, auto
from typing import Tuple
from weakref import ref

import numpy as np

from . import _lib, qed
from .constants import C as c, E_CHARGE as e, EPSILON_0 as epsilon_0, HBAR as hbar, M_E as m_e, PI as pi  # noqa
from .fields import Fields


class RadiationReactionType(Enum):
    """Radiation reaction type (particles.py:27-40).

    NONE: no radiation reaction; PHOTON: through photon emission (recoil);
    LL: Landau-Lifshitz force for gamma >> 1; CLL: quantum-corrected LL."""
    NONE = auto()
    PHOTON = auto()
    LL = auto()
    CLL = auto()


_RR_CODE = {RadiationReactionType.NONE: 1, RadiationReactionType.PHOTON: 2, RadiationReactionType.LL: 3,
            RadiationReactionType.CLL: 4}
_FLOAT_ATTRS_LAZY = ("chi", "Ex", "Ey", "Ez", "Bx", "By", "Bz", "photon_delta", "pair_delta")
_BOOL_ATTRS_LAZY = ("event",)
_BOOL_ATTRS = ("_to_be_pruned", "event")
# attributes a device-resident run may hold as of its position epoch (photons)
_POSITIONS = ("x", "y", "z")
_SPECIES_COUNTER = [0]


def _stream_ptr():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _device():
    import torch
    if not torch.cuda.is_available():
        raise _lib.SFPError("sfparticles_b200 needs a CUDA device; none is available")
    return torch.device("cuda", torch.cuda.current_device())


def _host_empty(shape, dtype):
    """Host tensor for device-to-host copies: page-locked memory from torch's
    caching host allocator (DMA in both directions, blocks reused from call
    to call), or pageable memory where page-locking fails."""
    import torch
    try:
        return torch.empty(shape, dtype=dtype, pin_memory=True)
    except RuntimeError:
        return torch.empty(shape, dtype=dtype)


def _random_seed() -> int:
    return int.from_bytes(os.urandom(8), "little")


class Particles(object):
    def __init__(self, name: str, q: int, m: float, N: int = 0, props: Tuple = None,
                 RR: RadiationReactionType = RadiationReactionType.PHOTON, push=True) -> None:
        """Initialise a species (particles.py:44-146).

        q: charge in units of e; m: mass in units of m_e (0 for photons);
        N: number of particles; props: (x, y, z, ux, uy, uz) arrays of
        length N (lists, arrays, or scalars when N == 1); RR: radiation
        reaction type; push: whether the species is moved.
        """
        d = self.__dict__
        d["_arr"] = {}
        d["_gpu"] = False
        d["_host_cache"] = {}
        d["_version"] = 0
        self.name = name
        self.q = q * e
        self.m = m * m_e
        self.RR = RR
        self.push = push
        self.bw = False
        self.radiating = False
        self.seed = _random_seed()
        self.rng_stream = _SPECIES_COUNTER[0] & 0xFFFFFFFF
        _SPECIES_COUNTER[0] += 1
        self._rng_step = 0
        N = int(N)

        assert m >= 0, 'negative mass'
        if m == 0:
            assert q == 0, 'photons cannot have mass'
        assert isinstance(RR, RadiationReactionType), 'RR must be RadiationReactionType'

        arr = self._arr
        if props is None:
            if m == 0:
                assert N == 0, "cannot initialize photons with only N without props."
            for k in ("x", "y", "z", "ux", "uy", "uz"):
                arr[k] = np.zeros(N)
        if props:
            assert len(props) == 6, 'given properties must has length of 6'
            props_ = prepare_props(props, N)
            for k, v in zip(("x", "y", "z", "ux", "uy", "uz"), props_):
                arr[k] = np.ascontiguousarray(v, dtype=np.float64)
        self.attrs = ['x', 'y', 'z', 'ux', 'uy', 'uz']
        ux, uy, uz = arr["ux"], arr["uy"], arr["uz"]
        if m > 0:
            arr["inv_gamma"] = 1. / np.sqrt(1 + ux ** 2 + uy ** 2 + uz ** 2)
        else:
            assert (ux ** 2 + uy ** 2 + uz ** 2 > 0).all(), "photon momentum cannot be 0"
            arr["inv_gamma"] = 1. / np.sqrt(ux ** 2 + uy ** 2 + uz ** 2)
        self.attrs += ['inv_gamma', 'chi', 'Ex', 'Ey', 'Ez', 'Bx', 'By', 'Bz']
        self.N_buffered = N
        self.buffer_size = N
        arr["_to_be_pruned"] = np.full(N, False)
        self.attrs += ['_to_be_pruned']

    # ------------------------------------------------------------------
    # attribute storage
    # ------------------------------------------------------------------
    def __getattr__(self, name):
        d = self.__dict__
        arr = d.get("_arr")
        attrs = d.get("attrs", ())
        if arr is None or name not in attrs:
            raise AttributeError(f"{type(self).__name__!s} has no attribute {name!r}")
        if name not in arr:
            self._materialize(name)
        if d["_gpu"] and name in _POSITIONS:
            self._sync_positions()
        a = arr[name]
        if not d["_gpu"]:
            return a
        hit = d["_host_cache"].get(name)
        if hit is not None and hit[0] == d["_version"]:
            return hit[1]
        h = a.cpu().numpy()
        if name in _BOOL_ATTRS:
            h = h.astype(bool)
        d["_host_cache"][name] = (d["_version"], h)
        return h

    def __setattr__(self, name, value):
        d = self.__dict__
        if name in d.get("attrs", ()) and "_arr" in d:
            if d["_gpu"]:
                import torch
                v = np.asarray(value)
                dt = torch.uint8 if name in _BOOL_ATTRS else torch.float64
                d["_arr"][name] = torch.as_tensor(v.astype(np.uint8) if name in _BOOL_ATTRS else v.astype(np.float64),
                                                  device=_device()).to(dt).contiguous()
                self._touch()
            else:
                v = np.asarray(value)
                d["_arr"][name] = v.astype(bool) if name in _BOOL_ATTRS else np.ascontiguousarray(v, dtype=np.float64)
            return
        object.__setattr__(self, name, value)

    def _touch(self):
        self.__dict__["_version"] += 1

    def _sync_positions(self):
        """A device-resident run that holds this photon species stores its
        positions as of the run's position epoch (photons fly straight, and
        the step kernels advance them in registers): have the run write them
        out before they are read."""
        f = self.__dict__.get("_pos_sync")
        if f is not None:
            f()

    def _materialize(self, name):
        n = self.buffer_size
        if name == "inv_gamma":  # derived from u (particles.py:118-123)
            self._arr[name] = self._inv_gamma_from_u()
            return
        if self._gpu:
            import torch
            dt = torch.uint8 if name in _BOOL_ATTRS else torch.float64
            self._arr[name] = torch.zeros(n, dtype=dt, device=_device())
        else:
            self._arr[name] = np.zeros(n, dtype=bool) if name in _BOOL_ATTRS else np.zeros(n)

    def _inv_gamma_from_u(self):
        if self._gpu:
            import torch
            ig = torch.empty(self.buffer_size, dtype=torch.float64, device=_device())
            if self.buffer_size:
                _lib.call("sfp_inv_gamma", ctypes.c_void_p(self._arr["ux"].data_ptr()),
                          ctypes.c_void_p(self._arr["uy"].data_ptr()), ctypes.c_void_p(self._arr["uz"].data_ptr()),
                          ctypes.c_void_p(ig.data_ptr()), self.buffer_size, 1 if self.m == 0 else 0, _stream_ptr())
            return ig
        ux, uy, uz = self._arr["ux"], self._arr["uy"], self._arr["uz"]
        with np.errstate(divide="ignore"):
            if self.m > 0:
                return 1. / np.sqrt(1 + ux ** 2 + uy ** 2 + uz ** 2)
            return 1. / np.sqrt(ux ** 2 + uy ** 2 + uz ** 2)

    _SCRATCH = ("inv_gamma", "chi", "Ex", "Ey", "Ez", "Bx", "By", "Bz", "event", "photon_delta", "pair_delta")

    def _drop_scratch(self):
        """Free the per-step scratch arrays and the stored 1/gamma; the fused
        step keeps neither (1/gamma is recomputed from u on access)."""
        for k in self._SCRATCH:
            self._arr.pop(k, None)
        self._touch()

    def _d(self, name, sync=True):
        """Device tensor of an attribute (species must be on the device).
        sync=False: photon positions as stored (for handing the arrays to a
        run, not for reading them)."""
        if not self._gpu:
            self._to_gpu()
        if name not in self._arr:
            self._materialize(name)
        if sync and name in _POSITIONS:
            self._sync_positions()
        return self._arr[name]

    def _p(self, name):
        return ctypes.c_void_p(self._d(name).data_ptr())

    def _to_gpu(self) -> None:
        """Move every materialised attribute to the CUDA device (particles.py:148-155)."""
        if self._gpu:
            return
        import torch
        dev = _device()
        _lib.load()
        # host arrays that _to_host left in page-locked memory go by DMA,
        # asynchronously; the sources stay referenced until the copies end
        src = []
        for k, v in list(self._arr.items()):
            a = np.ascontiguousarray(v, dtype=np.uint8 if k in _BOOL_ATTRS else np.float64)
            src.append(a)
            self._arr[k] = torch.from_numpy(a).to(dev, non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
        del src
        self.__dict__["_gpu"] = True
        self.__dict__["_host_cache"] = {}

    def _to_host(self) -> None:
        """Move every attribute back to host numpy arrays (particles.py:157-164)."""
        if not self._gpu:
            return
        import torch
        self._sync_positions()
        outs = []
        for k, v in list(self._arr.items()):
            h = _host_empty(v.shape, v.dtype)
            h.copy_(v, non_blocking=True)
            outs.append((k, h))
        torch.cuda.current_stream(_device()).synchronize()
        for k, h in outs:
            a = h.numpy()
            self._arr[k] = a.astype(bool) if k in _BOOL_ATTRS else a
        self.__dict__["_gpu"] = False
        self.__dict__["_host_cache"] = {}

    # ------------------------------------------------------------------
    @property
    def Npart(self) -> int:
        """Number of particles not marked for pruning (particles.py:166-174)."""
        if self.N_buffered == 0:
            return 0
        if not self._gpu:
            return int(self.N_buffered - np.count_nonzero(self._arr["_to_be_pruned"][: self.N_buffered]))
        return self.N_buffered - self._bool_sum("_to_be_pruned")

    @property
    def gamma(self):
        """Lorentz factor (energy / m_e c^2 for photons): 1 / inv_gamma."""
        return 1.0 / self.inv_gamma

    def _bool_sum(self, name) -> int:
        import torch
        out = torch.zeros(1, dtype=torch.int64, device=_device())
        _lib.call("sfp_bool_sum", self._p(name), self.N_buffered, ctypes.c_void_p(out.data_ptr()), _stream_ptr())
        return int(out.item())

    def set_photon(self, photon: 'Particles') -> None:
        """Emit photons into `photon` (particles.py:187-212)."""
        assert self.m > 0, 'photon cannot radiate photon'
        assert self.RR != RadiationReactionType.LL and self.RR != RadiationReactionType.CLL, \
            'LL equation does not radiate photon'
        assert isinstance(photon, Particles), 'photon must be Particle class'
        assert photon.m == 0 and photon.q == 0, 'photon must be m=0 and q=0'
        self.radiating = True
        self.photon_ref = ref(photon)
        self.attrs += ["event", "photon_delta"]
        if qed.use_optical_depth():
            self.attrs += ['tau']
            self._materialize('tau')
        self.__dict__["_od"] = qed.use_optical_depth()

    def set_pair(self, electron: 'Particles', positron: 'Particles') -> None:
        """Create Breit-Wheeler pairs into (electron, positron) (particles.py:215-242)."""
        assert self.m == 0, 'massive particle cannot create BW pair'
        assert isinstance(electron, Particles) and isinstance(positron, Particles), \
            'pair must be tuple or list of Particle class'
        assert electron.m == m_e and electron.q == -e, 'first of the pair must be electron'
        assert positron.m == m_e and positron.q == e, 'second of the pair must be positron'
        self.bw = True
        self.bw_electron_ref = ref(electron)
        self.bw_positron_ref = ref(positron)
        self.attrs += ["event", "pair_delta"]
        if qed.use_optical_depth():
            self.attrs += ['tau']
            self._materialize('tau')
        self.__dict__["_od"] = qed.use_optical_depth()

    @property
    def uses_optical_depth(self) -> bool:
        return bool(self.__dict__.get("_od", False))

    # ------------------------------------------------------------------
    # per-op kernels (the reference's kernel boundary, particles.py:244-473)
    # ------------------------------------------------------------------
    def _push_momentum(self, dt: float) -> None:
        """Boris push, then LL / CLL (particles.py:244-281)."""
        if self.m == 0:
            return
        _lib.call("sfp_boris", self._p("ux"), self._p("uy"), self._p("uz"), self._p("inv_gamma"),
                  *[self._p(k) for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz")], self.q, self.N_buffered,
                  self._p("_to_be_pruned"), dt, _stream_ptr())
        self._touch()
        if self.RR in (RadiationReactionType.LL, RadiationReactionType.CLL):
            self._calculate_chi()
            fn = "sfp_LL_push" if self.RR == RadiationReactionType.LL else "sfp_CLL_push"
            _lib.call(fn, self._p("ux"), self._p("uy"), self._p("uz"), self._p("inv_gamma"), self._p("chi"),
                      self.N_buffered, self._p("_to_be_pruned"), dt, _stream_ptr())

    def _push_position(self, dt: float) -> None:
        """x += c dt u / gamma (particles.py:284-296)."""
        _lib.call("sfp_push_position", self._p("x"), self._p("y"), self._p("z"), self._p("ux"), self._p("uy"),
                  self._p("uz"), self._p("inv_gamma"), self.N_buffered, self._p("_to_be_pruned"), dt, _stream_ptr())
        self._touch()

    def _eval_field(self, fields: Fields, t: float) -> None:
        """Fields at particle positions (particles.py:299-323)."""
        from . import program
        mod = program.get_module(fields, form=None, qed=None)
        prm = fields.params_device(_device())
        _lib.call("sfp_field_eval", mod.handle, ctypes.c_void_p(prm.data_ptr()), self._p("x"), self._p("y"),
                  self._p("z"), float(t), self.N_buffered, self._p("_to_be_pruned"),
                  *[self._p(k) for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz")], _stream_ptr())
        self._touch()

    def _calculate_chi(self) -> None:
        """Quantum parameter chi (particles.py:326-339)."""
        _lib.call("sfp_update_chi", *[self._p(k) for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "ux", "uy", "uz",
                                                              "inv_gamma", "chi")],
                  self.N_buffered, self._p("_to_be_pruned"), _stream_ptr())
        self._touch()

    def _next_rng_step(self) -> int:
        s = self._rng_step
        self._rng_step = (s + 1) & 0xFFFFFFFF
        return s

    def _events(self, delta_name: str, pair: bool, dt: float):
        from .qed import device_tables
        dev = _device()
        step = self._next_rng_step()
        if self.uses_optical_depth:
            t_ph, t_pa = device_tables.od_tables(dev)
            tab = t_pa if pair else t_ph
            _lib.call("sfp_update_tau", self._p("tau"), self._p("inv_gamma"), self._p("chi"), dt, self.N_buffered,
                      self._p("_to_be_pruned"), self._p("event"), self._p(delta_name), ctypes.byref(tab),
                      self.seed & (2 ** 64 - 1), self.rng_stream, step, _stream_ptr())
        else:
            tab = device_tables.rs_table(dev)
            fn = "sfp_pair_from_rejection_sampling" if pair else "sfp_photon_from_rejection_sampling"
            _lib.call(fn, self._p("inv_gamma"), self._p("chi"), dt, self.N_buffered, self._p("_to_be_pruned"),
                      self._p("event"), self._p(delta_name), ctypes.byref(tab), self.seed & (2 ** 64 - 1),
                      self.rng_stream, step, _stream_ptr())
        self._touch()

    def _photon_event(self, dt: float):
        """Photon emission events and energy fractions (particles.py:342-361)."""
        self._events("photon_delta", False, dt)
        return self.event, self.photon_delta

    def _pair_event(self, dt: float):
        """Pair creation events and energy fractions (particles.py:364-383)."""
        self._events("pair_delta", True, dt)
        return self.event, self.pair_delta

    def _pick_hard_photon(self, threshold: float = 2.0) -> None:
        """Drop emission events below `threshold` m_e c^2 (particles.py:386-396)."""
        _lib.call("sfp_pick_hard_photon", self._p("event"), self._p("photon_delta"), self._p("inv_gamma"),
                  float(threshold), self.N_buffered, _stream_ptr())
        self._touch()

    def _event_index(self, n_event: int):
        import torch
        ws_bytes = int(_lib.load().sfp_find_event_index_workspace(self.N_buffered))
        ws = torch.empty(max(1, ws_bytes // 8), dtype=torch.int64, device=_device())
        idx = torch.empty(n_event, dtype=torch.int64, device=_device())
        _lib.call("sfp_find_event_index", self._p("event"), n_event, self.N_buffered,
                  ctypes.c_void_p(idx.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ws.numel() * 8, _stream_ptr())
        return idx

    def _create_photon(self, pho: 'Particles') -> None:
        """Append photons for the events, then recoil (particles.py:399-431)."""
        n = self._bool_sum("event")
        if n == 0:
            return
        if hasattr(self, 'photon_ref'):
            idx = self._event_index(n)
            pho._extend(n)
            pho._to_gpu()
            _lib.call("sfp_create_photon", *[self._p(k) for k in ("x", "y", "z", "ux", "uy", "uz")],
                      *[pho._p(k) for k in ("x", "y", "z", "ux", "uy", "uz", "inv_gamma", "_to_be_pruned")],
                      ctypes.c_void_p(idx.data_ptr()), self._p("photon_delta"), pho.N_buffered, n, _stream_ptr())
            pho.N_buffered += n
            pho._touch()
        if self.RR == RadiationReactionType.PHOTON:
            _lib.call("sfp_photon_recoil", self._p("ux"), self._p("uy"), self._p("uz"), self._p("inv_gamma"),
                      self._p("event"), self._p("photon_delta"), self.N_buffered, self._p("_to_be_pruned"),
                      _stream_ptr())
            self._touch()

    def _create_pair(self, ele: 'Particles', pos: 'Particles') -> None:
        """Append e-/e+ for the events, prune the photons (particles.py:433-473)."""
        n = self._bool_sum("event")
        if n == 0:
            return
        if hasattr(self, 'bw_electron_ref'):
            idx = self._event_index(n)
            ele._extend(n)
            pos._extend(n)
            for dst, inv in ((ele, 0), (pos, 1)):
                dst._to_gpu()
                _lib.call("sfp_create_pair", *[self._p(k) for k in ("x", "y", "z", "ux", "uy", "uz")],
                          self._p("_to_be_pruned"),
                          *[dst._p(k) for k in ("x", "y", "z", "ux", "uy", "uz", "inv_gamma", "_to_be_pruned")],
                          ctypes.c_void_p(idx.data_ptr()), self._p("pair_delta"), dst.N_buffered, n, inv,
                          _stream_ptr())
            ele.N_buffered += n
            pos.N_buffered += n
            ele._touch()
            pos._touch()
            self._touch()

    # ------------------------------------------------------------------
    def _extend(self, N_new: int) -> None:
        """Grow buffers: buffer_size += N_buffered//4 + N_new when the free
        space is below N_new (particles.py:476-500).  New slots are pruned,
        event-free, and zero (spin and optical depth of appended particles
        start at zero)."""
        if (self.buffer_size - self.N_buffered) < N_new:
            new = self.buffer_size + int(self.N_buffered / 4) + N_new
            self._resize(new)

    def _resize(self, new: int):
        """Reallocate every array at `new` slots.  On the device the outgrown
        blocks go back to the caching allocator, which reuses them or frees
        them on a later allocation that would not fit; the simulation empties
        the cache only once a run has ended, since emptying it synchronises
        the device."""
        old = self.buffer_size
        for k, v in list(self._arr.items()):
            if self._gpu:
                import torch
                t = torch.empty(new, dtype=v.dtype, device=v.device)
                m = min(old, new)
                t[:m] = v[:m]
                if new > old:
                    t[old:] = 1 if k == "_to_be_pruned" else 0
                self._arr[k] = t
                del v
            else:
                a = np.zeros(new, dtype=v.dtype)
                a[: min(old, new)] = v[: min(old, new)]
                if k == "_to_be_pruned" and new > old:
                    a[old:] = True
                self._arr[k] = a
        self.buffer_size = new
        self._touch()

    def _prune(self) -> None:
        """Remove pruned particles and compact every array (particles.py:503-516)."""
        if self._gpu:
            import torch
            self._sync_positions()
            # the kept slots once, then one gather per array
            idx = torch.nonzero(self._arr["_to_be_pruned"] == 0).flatten()
            for k, v in list(self._arr.items()):
                self._arr[k] = torch.index_select(v, 0, idx)
            N = int(idx.numel())
        else:
            keep = ~self._arr["_to_be_pruned"].astype(bool)
            for k, v in list(self._arr.items()):
                self._arr[k] = np.ascontiguousarray(v[keep])
            N = int(keep.sum())
        self.buffer_size = N
        self.N_buffered = N
        self._touch()


class SpinParticles(Particles):
    """Particles with spin, pushed with Boris + Thomas-BMT (particles.py:518-604)."""

    def __init__(self, name: str, q: int, m: float, N: int = 0, props: Tuple = None,
                 RR: RadiationReactionType = RadiationReactionType.PHOTON, ae: float = 1.14e-3,
                 push: bool = True) -> None:
        """props: (x, y, z, ux, uy, uz, sx, sy, sz); ae: anomalous moment (g-2)/2."""
        if props is None:
            if m == 0:
                assert N == 0, "cannot initialize photons with only N without props."
            super().__init__(name, q, m, N, props, RR, push)
            for k in ("sx", "sy", "sz"):
                self._arr[k] = np.zeros(int(N))
        if props:
            assert len(props) == 9, 'given properties must has length of 9'
            super().__init__(name, q, m, N, props[:6], RR, push)
            for k, v in zip(("sx", "sy", "sz"), prepare_props(props[6:], int(N))):
                self._arr[k] = np.ascontiguousarray(v, dtype=np.float64)
        self.ae = ae
        self.attrs += ['sx', 'sy', 'sz']

    def _push_momentum(self, dt: float) -> None:
        """Boris-TBMT, then LL (particles.py:575-604; no CLL branch there)."""
        if self.m == 0:
            return
        _lib.call("sfp_boris_tbmt", self._p("ux"), self._p("uy"), self._p("uz"), self._p("inv_gamma"),
                  self._p("sx"), self._p("sy"), self._p("sz"),
                  *[self._p(k) for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz")], self.q, self.ae, self.N_buffered,
                  self._p("_to_be_pruned"), dt, _stream_ptr())
        self._touch()
        if self.RR == RadiationReactionType.LL:
            self._calculate_chi()
            _lib.call("sfp_LL_push", self._p("ux"), self._p("uy"), self._p("uz"), self._p("inv_gamma"),
                      self._p("chi"), self.N_buffered, self._p("_to_be_pruned"), dt, _stream_ptr())


def prepare_props(props: Tuple, N: int) -> list:
    """Convert arrays / lists / scalars into float64 vectors of length N
    (particles.py:606-635)."""
    props_ = []
    for prop in props:
        if isinstance(prop, np.ndarray):
            assert len(prop.shape) == 1, 'given property is not vector'
            assert prop.shape[0] == N, 'given N does not match given property length'
            props_.append(prop)
        if isinstance(prop, (int, float)):
            assert N == 1, 'given N does not match given property length'
            props_.append(np.asarray([prop], dtype=np.float64))
        if isinstance(prop, (list, tuple)):
            assert len(prop) == N, 'given N does not match given property length'
            props_.append(np.asarray(prop, dtype=np.float64))
    return props_
