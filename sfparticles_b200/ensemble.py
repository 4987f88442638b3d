"""Ensemble: many independent collisions advanced by one set of launches.

Each member is an ordinary ``Simulation`` with its own species, field
parameters and Philox seed.  One ensemble step is one set of persistent
launches over every member's species.  The massive and photon kernels take
tiles of all members by ticket, so members of very different sizes share the
GPU with no launch per member, and the step loop is replayed from CUDA graphs.

Members must share dt, photon_threshold, the arithmetic form, the QED method
and the field *structure*: the field program is one NVRTC module, and its
numeric parameters (a0, waist, duration, ...) are per member.

A member's results are the ones it gets when run alone.  Its particles draw
from its own Philox key, with streams numbered by species within the member,
and its children are appended in its own order (the append scan restarts at
each member's first tile, per destination).

This is an extension with no reference counterpart: the reference runs one
collision per ``Simulation``.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

from . import _lib, program
from .particles import _device, _stream_ptr
from .simulation import (MIN_ROOM, Simulation, _release_cached_blocks, attach_position_sync, detach_position_sync,
                         observe_rates, plan_chunk, resolve_pending, sync_positions)


class Ensemble(object):
    def __init__(self, sims: Sequence[Simulation], graph_chunk: int = 64, m_stages: int = 0, min_blocks: int = 0,
                 p_stages: int = 0, p_min_blocks: int = 0) -> None:
        sims = list(sims)
        if not sims:
            raise ValueError("an ensemble needs at least one simulation")
        first = sims[0]
        for s in sims:
            if s.engine != "fused":
                raise ValueError("ensemble members use the fused engine")
            if (s.dt, s.photon_threshold, s.form, s.qed_method, s.sampler) != (
                    first.dt, first.photon_threshold, first.form, first.qed_method, first.sampler):
                raise ValueError("ensemble members must share dt, photon_threshold, form, QED method and sampler")
            if s.fields.structure() != first.fields.structure():
                raise ValueError("ensemble members must share the field structure (parameters may differ)")
            if (s.step, s.t) != (first.step, first.t):
                raise ValueError("ensemble members must start at the same step and time")
        ids = [id(p) for s in sims for p in s.all_particles]
        if len(set(ids)) != len(ids):
            raise ValueError("a species belongs to more than one ensemble member")
        self.sims = sims
        self.form, self.qed_method, self.dt = first.form, first.qed_method, first.dt
        self.step, self.t = first.step, first.t
        self.graph_chunk = int(graph_chunk)
        self.m_stages = int(m_stages) or first.m_stages
        self.min_blocks = int(min_blocks) or first.min_blocks
        self.p_stages = int(p_stages) or first.p_stages
        self.p_min_blocks = int(p_min_blocks) or first.p_min_blocks
        self.particle_steps = 0   # sum over executed steps of all members' N_buffered
        self.kernel_launches = 0  # libsfp kernels launched by start()/run_on_device()
        self._run = None

    @property
    def species(self):
        return [p for s in self.sims for p in s.all_particles]

    def _segments(self):
        """Members' segment tables back to back; destinations offset to the
        member's first segment, instance = member index."""
        allp = self.species
        segs = (_lib.Segment * len(allp))()
        base = 0
        for k, sim in enumerate(self.sims):
            one = sim._segments()
            for i in range(len(sim.all_particles)):
                s = segs[base + i]
                ctypes.memmove(ctypes.byref(s), ctypes.byref(one[i]), ctypes.sizeof(_lib.Segment))
                for f in ("photon_dest", "ele_dest", "pos_dest"):
                    if getattr(s, f) >= 0:
                        setattr(s, f, getattr(s, f) + base)
                s.instance = k
            base += len(sim.all_particles)
        return segs

    def _launches_per_step(self):
        ps = self.species
        return (1 + any(p.m != 0 for p in ps) + any(p.m == 0 for p in ps)
                + 2 * any(p.bw or p.radiating for p in ps))

    def _begin(self):
        for p in self.species:
            p._to_gpu()
            p._drop_scratch()
        first = self.sims[0]
        mod = program.get_module(first.fields, form=self.form, qed=self.qed_method)
        dev = _device()
        params = [s.fields.params_device(dev) for s in self.sims]
        inst = (_lib.Instance * len(self.sims))()
        base = 0
        for k, s in enumerate(self.sims):
            inst[k].seed = s.seed
            inst[k].field_params = params[k].data_ptr()
            inst[k].first_seg = base
            inst[k].n_seg = len(s.all_particles)
            base += len(s.all_particles)
        segs = self._segments()
        allp = self.species
        nbuf = (ctypes.c_int64 * len(allp))(*[p.N_buffered for p in allp])
        cfg = first._run_config()
        cfg.t0, cfg.step0 = self.t, self.step
        cfg.m_stages, cfg.min_blocks = self.m_stages, self.min_blocks
        cfg.p_stages, cfg.p_min_blocks = self.p_stages, self.p_min_blocks
        run = ctypes.c_void_p()
        _lib.call("sfp_run_create", mod.handle, ctypes.byref(cfg), len(self.sims), inst, len(allp), segs, nbuf,
                  ctypes.byref(run))
        self._run = run
        self._keep = (mod, params)
        self._ps_base = self.particle_steps
        attach_position_sync(self, allp)

    def _sync_positions(self):
        sync_positions(self, self.species)

    def _end(self):
        if self._run is not None:
            self._sync_positions()
            detach_position_sync(self.species)
            _lib.load().sfp_run_destroy(self._run)
        self._run = None
        self._keep = None

    def _update_run(self, counts=True):
        allp = self.species
        nbuf = (ctypes.c_int64 * len(allp))(*[p.N_buffered for p in allp]) if counts else None
        _lib.call("sfp_run_update", self._run, len(allp), self._segments(), nbuf)

    def _sync_state(self, st, nbuf) -> int:
        """Read the run's state into every member; returns the steps
        completed since the last read."""
        _lib.check(_lib.load().sfp_run_read_state(self._run, ctypes.byref(st), nbuf, _stream_ptr()),
                   "sfp_run_read_state")
        if st.error:
            raise _lib.SFPError(f"device error in the step kernel: {_lib.DEV_ERRORS.get(st.error, st.error)}")
        done = int(st.step) - self.step
        for i, p in enumerate(self.species):
            p.N_buffered = int(nbuf[i])
            if done > 0:
                p._touch()
        self.particle_steps = self._ps_base + int(st.particle_steps)
        self.step, self.t = int(st.step), float(st.t)
        for s in self.sims:
            s.step, s.t = self.step, self.t
        return done

    def _loop(self, nstep: int):
        L = _lib.load()
        allp = self.species
        nbuf = (ctypes.c_int64 * len(allp))()
        st = _lib.RunState()
        remaining = int(nstep)
        max_chunk = 4 * self.graph_chunk if self.graph_chunk > 0 else 256
        rates = self.__dict__.setdefault("_rates", {})
        while remaining > 0:
            target = min(remaining, max_chunk if rates else (self.graph_chunk or 64))
            # many members: a smaller minimum room each, so the total stays near one simulation's
            grew, fit = plan_chunk(allp, rates, target, min_room=max(1 << 12, MIN_ROOM // max(1, len(self.sims))))
            chunk = min(target, fit)
            if grew:
                self._update_run()
            before = [p.N_buffered for p in allp]
            _lib.check(L.sfp_run_steps(self._run, chunk, self.graph_chunk if chunk >= self.graph_chunk else 0,
                                       _stream_ptr()), "sfp_run_steps")
            self._pos_dirty = True
            self.kernel_launches += self._launches_per_step() * chunk + 1
            done = self._sync_state(st, nbuf)
            halted = bool(st.halted)
            if halted:
                if st.appends_pending:
                    # finishing the stopped step completes it: count it
                    resolve_pending(self._run, allp, lambda: self._update_run(counts=False))
                    done += self._sync_state(st, nbuf)
                else:
                    _lib.check(L.sfp_run_clear_halt(self._run, _stream_ptr()), "sfp_run_clear_halt")
            remaining -= done
            observe_rates(allp, before, done, rates)
            if done == 0 and not halted:
                raise _lib.SFPError("the step made no progress")

    def time_step_kernel(self, nstep: int):
        """Advance `nstep` steps with eager launches and return, per step, the
        CUDA-event durations [ms] of its (massive, photon, scan + appends)
        kernels, with the buffered counts before and after."""
        if self._run is None:
            self._begin()
        L = _lib.load()
        allp = self.species
        before = [p.N_buffered for p in allp]
        st = _lib.RunState()
        nbuf = (ctypes.c_int64 * len(allp))()
        out = []
        for _ in range(int(nstep)):
            ms = (ctypes.c_float * 3)()
            _lib.check(L.sfp_run_steps_timed(self._run, 1, ms, _stream_ptr()), "sfp_run_steps_timed")
            self._pos_dirty = True
            _lib.check(L.sfp_run_read_state(self._run, ctypes.byref(st), nbuf, _stream_ptr()), "read_state")
            self.kernel_launches += self._launches_per_step() + 1
            if st.error or (st.halted and not st.appends_pending):
                raise _lib.SFPError("timed step did not complete")
            if st.appends_pending:  # finish the step; its appends kernel was not timed
                resolve_pending(self._run, allp, lambda: self._update_run(counts=False))
                _lib.check(L.sfp_run_read_state(self._run, ctypes.byref(st), nbuf, _stream_ptr()), "read_state")
            else:
                out.append((float(ms[0]), float(ms[1]), float(ms[2])))
            for i, p in enumerate(allp):
                p.N_buffered = int(nbuf[i])
                p._touch()
        self.particle_steps = self._ps_base + int(st.particle_steps)
        self.step, self.t = int(st.step), float(st.t)
        for s in self.sims:
            s.step, s.t = self.step, self.t
        return out, before, [p.N_buffered for p in allp]

    def run_on_device(self, nstep: int):
        """Advance every member `nstep` steps, keeping all species on the device."""
        if self._run is None:
            self._begin()
        self._loop(nstep)

    def finish(self):
        """End a run_on_device() sequence: prune and return host arrays."""
        self._end()
        for p in self.species:
            p._prune()
            p._to_host()
        _release_cached_blocks()

    def start(self, nstep: int):
        """Advance every member `nstep` steps and return host arrays, like
        Simulation.start for each member."""
        self._begin()
        try:
            self._loop(nstep)
        finally:
            self._end()
        for p in self.species:
            p._prune()
            p._to_host()
        _release_cached_blocks()
