"""Simulation: the reference's step loop (sfparticles/simulation.py) driving
the fused B200 step.

``Simulation(*particles, dt, fields, print_every=100, t0=0.0,
photon_threshold=2.0)`` and ``start(nstep, total=None, call_back=None)``
behave as in the reference: species are classified into pushed, pair-creating
and radiating lists (simulation.py:62-71); every step evaluates fields at t,
generates QED events, appends photons then pairs, and pushes every pushed
particle (children included) from t to t+dt (simulation.py:102-144);
``start`` ends by pruning and returning host arrays (simulation.py:158-161).

Each step is a one-block bookkeeping launch followed by the massive kernel
(e+-: emission events; emitters marked, every other particle pushed), the
photon kernel (pair events; converted photons marked, the others pushed), a
one-block scan of both kinds of event counts and the appends kernel (photon
children, the emitters' recoil and push, e-/e+ children, all written in the
reference's order and pushed); steps between progress reports / callbacks
run back to back on the device, replayed from CUDA graphs, with no host
synchronisation.  No kernel overruns a buffer: the scan compares each
destination's room with the step's exact number of children before any is
written, and if one lacks room the step waits; the host grows that buffer
by the reference rule and resumes the step.  Between device chunks the host
grows destinations ahead of the append rates it has seen, so waits are rare.

Extra keyword arguments (no reference counterpart):
  seed        -- 64-bit key of the Philox streams (default: random);
  form        -- 'fp64' (plain float64, the reference arithmetic) or 'fp32';
  graph_chunk -- steps per captured CUDA graph (0 disables graphs);
  m_stages, min_blocks -- massive-kernel variant: depth of the copy ring
                 that streams e+- state into shared memory and minimum
                 resident blocks per SM (see autotune.py);
  p_stages, p_min_blocks -- photon-kernel variant: depth of the copy ring
                 that streams photon state into shared memory and minimum
                 resident blocks per SM;
  sampler     -- optical depth only: 'table' (the inverse-CDF table, as in
                 the reference) or 'mlp', the learned photon-energy sampler
                 (sfparticles_b200.mlp) evaluated on the tensor cores inside
                 the step;
  monitor     -- a callable monitor(sim), run at every print_every
                 boundary and at the end of start(); shard.JobDiagnostics
                 reduces the counters and the photon spectrum over the ranks
                 of a multi-GPU job there;
  engine      -- 'fused' (the persistent step kernels) or 'ops': the
                 reference's own step loop (simulation.py:102-144) over the
                 one-for-one kernels of the C-ABI (float64, materialised
                 fields, host-synchronised appends).  'ops' keys every
                 species' Philox stream by (seed, species index, step), like
                 the fused step, so both engines draw the same numbers.
"""
from __future__ import annotations

import ctypes
import os
from time import perf_counter_ns
from typing import Callable


from . import _lib, program, qed
from .fields import Fields
from .particles import Particles, _RR_CODE, _device, _random_seed, _stream_ptr

try:
    from tqdm.autonotebook import tqdm
except Exception:  # pragma: no cover
    tqdm = None


def resolve_pending(run, species, update):
    """Finish a step that stopped before writing its children: grow every
    species to the size the step needs (the reference's _extend rule,
    particles.py:487-500), hand the new buffers to the run and resume it."""
    L = _lib.load()
    need = (ctypes.c_int64 * len(species))()
    _lib.check(L.sfp_run_pending_need(run, need), "sfp_run_pending_need")
    for i, p in enumerate(species):
        if int(need[i]) > p.buffer_size:
            p._extend(int(need[i]) - p.N_buffered)
    update()
    _lib.check(L.sfp_run_resume(run, _stream_ptr()), "sfp_run_resume")


# a growth may always reach this many slots (about 60 MB per species), so a
# destination that starts empty does not grow in many small, halting steps
GROWTH_FLOOR = 1 << 20
# free slots a destination with appends is given at least (about 15 MB per
# species): append rates ramp up within a chunk as a beam enters a pulse,
# and small runs would otherwise stop for room again and again
MIN_ROOM = 1 << 18


def plan_chunk(species, rates, max_chunk, min_room=MIN_ROOM):
    """Size append destinations for the next chunk of device steps from the
    append rates seen so far (`rates`: id(species) -> particles per step),
    and return (grew, chunk).  A destination that cannot take a full chunk
    at 1.25x its rate (and at least `min_room` free slots) grows by the
    reference rule (particles.py:487-500), each growth capped at half its
    count (or GROWTH_FLOOR slots, whichever is more) so memory stays near
    its use; the chunk is shortened to what then fits.  Buffer sizes do not
    change results: they only decide how often a step waits for room."""
    grew = False
    chunk = max_chunk
    for p in species:
        r = rates.get(id(p), 0.0)
        if r <= 0.0:
            continue
        free = p.buffer_size - p.N_buffered
        want = max(int(r * max_chunk * 1.25) + 1, int(min_room))
        if free < want:
            extra = min(want, max(p.N_buffered // 2 + 1024, GROWTH_FLOOR))
            if free < extra:
                p._extend(extra)
                grew = True
            free = p.buffer_size - p.N_buffered
        chunk = min(chunk, max(1, int(free / (1.25 * r))))
    return grew, chunk


def _release_cached_blocks():
    """Return the device blocks that buffer growth outgrew to the driver, and
    the page-locked host blocks of earlier runs' copies that nothing holds any
    more (the caching host allocator keeps them otherwise, rounded up to a
    power of two).  Emptying the caches synchronises the device, so it is
    done once a run has ended, never between its chunks."""
    import torch
    if torch.cuda.is_available() and torch.cuda.is_initialized():
        torch.cuda.empty_cache()
        if hasattr(torch._C, "_host_emptyCache"):
            torch._C._host_emptyCache()


def attach_position_sync(owner, species):
    """A run stores its photons' positions as of its position epoch (the
    step kernels advance them in registers: photons fly straight).  Each
    photon species of the run gets a hook that writes them out before any
    read of x, y, z (Particles._sync_positions)."""
    owner._pos_dirty = False
    for p in species:
        if p.m == 0:
            p.__dict__["_pos_sync"] = owner._sync_positions


def detach_position_sync(species):
    for p in species:
        p.__dict__.pop("_pos_sync", None)


def sync_positions(owner, species):
    """sfp_run_sync_positions for a run that stepped since its last one."""
    run = getattr(owner, "_run", None)
    if run is None or not getattr(owner, "_pos_dirty", False):
        return
    owner._pos_dirty = False
    _lib.check(_lib.load().sfp_run_sync_positions(run, _stream_ptr()), "sfp_run_sync_positions")
    owner.kernel_launches = getattr(owner, "kernel_launches", 0) + 2
    for p in species:
        if p.m == 0:
            p._touch()


def observe_rates(species, before, steps, rates):
    """Update the append rates from the counts before and after `steps` steps."""
    if steps <= 0:
        return
    for p, n0 in zip(species, before):
        r = max(0, p.N_buffered - n0) / steps
        rates[id(p)] = max(r, 0.5 * rates.get(id(p), 0.0))


class Simulation(object):
    def __init__(self, *all_particles: Particles, dt: float, fields: Fields, print_every: int = 100, t0=0.0,
                 photon_threshold=2.0, seed: int = None, form: str = "fp64", graph_chunk: int = 64,
                 m_stages: int = 0, min_blocks: int = 0, p_stages: int = 0, p_min_blocks: int = 0,
                 engine: str = "fused", sampler: str = "table", monitor: Callable = None) -> None:
        self.all_particles = all_particles
        self.particles_push = []
        self.particles_bw = []
        self.particles_rad = []
        self.dt = dt
        self.fields = fields
        self.print_every = print_every
        self.photon_threshold = photon_threshold
        self.t = t0
        self.step = 0
        self.progress_bar = None
        self.seed = _random_seed() if seed is None else int(seed) & (2 ** 64 - 1)
        if form not in ("fp64", "fp32"):
            raise ValueError("form must be 'fp64' or 'fp32'")
        self.form = form
        # the step module reads the field parameters from its constant bank
        # (one instance per run); False: from global memory, the module
        # kind an Ensemble uses
        self._const_field = True
        if engine not in ("fused", "ops"):
            raise ValueError("engine must be 'fused' or 'ops'")
        if engine == "ops" and form != "fp64":
            raise ValueError("the 'ops' engine computes in float64 only")
        self.engine = engine
        if sampler not in ("table", "mlp"):
            raise ValueError("sampler must be 'table' or 'mlp'")
        if sampler == "mlp" and engine != "fused":
            raise ValueError("the learned photon-energy sampler runs in the fused engine")
        self.sampler = sampler
        self.graph_chunk = int(graph_chunk)
        self.monitor = monitor
        self.m_stages = int(m_stages)  # massive kernel: depth of the copy ring (0: the form's default)
        self.min_blocks = int(min_blocks)  # massive kernel: resident blocks per SM (0: default)
        self.p_stages = int(p_stages)  # photon kernel: depth of the copy ring (0: default)
        self.p_min_blocks = int(p_min_blocks)  # photon kernel: resident blocks per SM (0: default)
        self.particle_steps = 0  # sum over executed steps of all species' N_buffered
        self.kernel_launches = 0  # libsfp kernels launched by start()/run_on_device()
        self._run = None
        self._trajectories = []

        for p in all_particles:
            if p.bw:
                assert p.bw_electron_ref() in all_particles, f"{p.bw_electron_ref().name} not included in simulation."
                assert p.bw_positron_ref() in all_particles, f"{p.bw_positron_ref().name} not included in simulation."
                self.particles_bw.append(p)
            if p.radiating:
                assert p.photon_ref() in all_particles, f"{p.photon_ref().name} not included in simulation."
                self.particles_rad.append(p)
            if p.push:
                self.particles_push.append(p)
        ods = {p.uses_optical_depth for p in all_particles if p.radiating or p.bw}
        if len(ods) > 1:
            raise ValueError("all QED species of a simulation must use the same event method")
        self.qed_method = "od" if ods == {True} else "rs"
        if self.sampler == "mlp" and self.qed_method != "od":
            raise ValueError("the learned photon-energy sampler replaces the optical-depth table: "
                             "set SFPARTICLES_OPTICAL_DEPTH=1")
        from .autotune import DEFAULT
        dm, dp = DEFAULT[(self.form, self.qed_method)]
        if self.m_stages <= 0 or self.min_blocks <= 0:
            self.m_stages, self.min_blocks = dm
        if self.p_stages <= 0 or self.p_min_blocks <= 0:
            self.p_stages, self.p_min_blocks = dp

    def record(self, species: Particles, index, every: int = 1, attrs=None):
        """Record `attrs` of the buffer slots `index` of `species` after every
        `every`-th step, on the device (sfparticles_b200.trajectory); returns
        the Trajectory, whose numpy() gives the records."""
        from .trajectory import Trajectory
        assert species in self.all_particles, f"{species.name} not included in simulation."
        tr = Trajectory(species, index, every, attrs)
        self._trajectories.append(tr)
        return tr

    def _record(self):
        for tr in self._trajectories:
            if tr.due(self.step):
                tr.capture(self.step)

    # ------------------------------------------------------------------
    def _index(self, p):
        for i, q in enumerate(self.all_particles):
            if q is p:
                return i
        raise ValueError(f"{p.name} not in simulation")

    def _segments(self):
        """sfp_segment table of the species (one instance)."""
        segs = (_lib.Segment * len(self.all_particles))()
        channels = {}

        def channel(key):
            if key not in channels:
                if len(channels) >= 4:
                    raise ValueError("at most 4 distinct append destinations are supported")
                channels[key] = len(channels)
            return channels[key]

        for i, p in enumerate(self.all_particles):
            s = segs[i]
            for k in ("x", "y", "z", "ux", "uy", "uz"):
                setattr(s, k, p._d(k, sync=False).data_ptr())
            s.pruned = p._d("_to_be_pruned").data_ptr()
            spin = "sx" in p.attrs
            if spin:
                s.sx, s.sy, s.sz = (p._d(k).data_ptr() for k in ("sx", "sy", "sz"))
            s.tau = p._d("tau").data_ptr() if "tau" in p.attrs else None
            # the delta of this step's events, kept until their children are written
            s.delta = (p._d("pair_delta").data_ptr() if p.bw else
                       p._d("photon_delta").data_ptr() if p.radiating else None)
            s.capacity = p.buffer_size
            s.q = p.q
            s.ae = getattr(p, "ae", 0.0) if spin else 0.0
            s.massless = 1 if p.m == 0 else 0
            s.push = 1 if p.push else 0
            s.rr = _RR_CODE[p.RR]
            s.spin = 1 if spin else 0
            s.radiating = 1 if p.radiating else 0
            s.bw = 1 if p.bw else 0
            s.photon_dest = self._index(p.photon_ref()) if p.radiating else -1
            s.ele_dest = self._index(p.bw_electron_ref()) if p.bw else -1
            s.pos_dest = self._index(p.bw_positron_ref()) if p.bw else -1
            s.channel = 0
            if p.radiating:
                s.channel = channel(("ph", s.photon_dest))
            elif p.bw:
                s.channel = channel(("pair", s.ele_dest, s.pos_dest))
            s.instance = 0
            s.stream = i
        return segs

    def _destinations(self):
        """Species that receive children: photon and pair destinations."""
        d = {id(p.photon_ref()): p.photon_ref() for p in self.particles_rad}
        for p in self.particles_bw:
            d[id(p.bw_electron_ref())] = p.bw_electron_ref()
            d[id(p.bw_positron_ref())] = p.bw_positron_ref()
        return list(d.values())

    def reserve(self, nstep: int) -> bool:
        """Grow every append destination ahead of `nstep` device steps to
        twice the append rate observed so far (and at least MIN_ROOM free
        slots where appends were seen), so that those steps run without
        waiting for room and without growing (a run whose rate then doubles
        still waits and grows, as always).  Updates a live run; True if any
        buffer grew."""
        rates = self.__dict__.setdefault("_rates", {})
        grew = False
        for p in self._destinations():
            r = rates.get(id(p), 0.0)
            want = int(2.0 * r * int(nstep)) + 1024
            if r > 0.0:
                want = max(want, MIN_ROOM)
            if p.buffer_size - p.N_buffered < want:
                p._extend(want)
                grew = True
        if grew and getattr(self, "_run", None) is not None:
            self._update_run(self._run)
        return grew

    def _run_config(self):
        from .qed import device_tables
        dev = _device()
        cfg = _lib.RunConfig()
        cfg.dt = self.dt
        cfg.photon_threshold = self.photon_threshold
        cfg.t0 = self.t
        cfg.step0 = self.step
        cfg.qed = _lib.SFP_QED_OPTICAL_DEPTH if self.qed_method == "od" else _lib.SFP_QED_REJECTION
        cfg.form = _lib.SFP_FORM_FP32 if self.form == "fp32" else _lib.SFP_FORM_FP64
        cfg.m_stages = self.m_stages
        cfg.min_blocks = self.min_blocks
        cfg.p_stages = self.p_stages
        cfg.p_min_blocks = self.p_min_blocks
        if self.sampler == "mlp":
            from .mlp import PhotonSampler
            if getattr(self, "_mlp", None) is None:
                self._mlp = PhotonSampler.trained()
            cfg.mlp_params = self._mlp.params.data_ptr()
        if self.qed_method == "od":
            cfg.od_photon, cfg.od_pair = device_tables.od_tables(dev)
        else:
            cfg.rs = device_tables.rs_table(dev)
        return cfg

    # ------------------------------------------------------------------
    def start(self, nstep: int, total: int = None, call_back: Callable[[int], None] = None):
        """Run `nstep` steps (simulation.py:74-160)."""
        if total is None:
            total = nstep
        if self.progress_bar is None and self.print_every and tqdm is not None:
            self.progress_bar = tqdm(total=total, unit='step', smoothing=1)

        if self.engine == "ops":
            self._loop_ops(nstep, call_back)
        else:
            self._begin()
            try:
                self._loop(self._run, nstep, call_back)
            finally:
                self._end()
        if self.monitor is not None:
            self.monitor(self)
        for p in self.all_particles:
            p._prune()
            p._to_host()
        _release_cached_blocks()

    def _loop_ops(self, nstep, call_back):
        """The reference's step loop (simulation.py:102-144) over the per-op
        kernels: one launch per kernel per species, fields and events
        materialised in HBM, a host synchronisation per append."""
        for i, p in enumerate(self.all_particles):
            p._to_gpu()
            p.seed = self.seed
            p.rng_stream = i
        dt = self.dt
        for _ in range(int(nstep)):
            self.particle_steps += sum(p.N_buffered for p in self.all_particles)
            for p in self.particles_push:
                p._eval_field(self.fields, self.t)
            for p in self.particles_bw:
                p._calculate_chi()
                p._rng_step = self.step
                p._pair_event(dt)
            for p in self.particles_rad:
                p._calculate_chi()
                p._rng_step = self.step
                p._photon_event(dt)
                p._pick_hard_photon(self.photon_threshold)
            for p in self.particles_rad:
                p._create_photon(p.photon_ref())
            for p in self.particles_bw:
                p._create_pair(p.bw_electron_ref(), p.bw_positron_ref())
            for p in self.particles_push:
                p._push_position(0.5 * dt)
                p._eval_field(self.fields, self.t + 0.5 * dt)
                p._push_momentum(dt)
                p._push_position(0.5 * dt)
            if call_back:
                call_back(self.step)
            self.t += dt
            self.step += 1
            self._record()
            if self.print_every and self.step % self.print_every == 0:
                if self.progress_bar is not None:
                    self.progress_bar.update(self.print_every)
                if self.monitor is not None:
                    self.monitor(self)

    # -- device-resident driving (start() = _begin + _loop + _end + prune) --
    def _begin(self):
        """Move species to the device and create the fused-step run."""
        for p in self.all_particles:
            p._to_gpu()
            p._drop_scratch()
        mod = program.get_module(self.fields, form=self.form, qed=self.qed_method, single=self._const_field)
        params = self.fields.params_device(_device())
        inst = (_lib.Instance * 1)()
        inst[0].seed = self.seed
        inst[0].field_params = params.data_ptr()
        inst[0].first_seg = 0
        inst[0].n_seg = len(self.all_particles)
        segs = self._segments()
        nbuf = (ctypes.c_int64 * len(self.all_particles))(*[p.N_buffered for p in self.all_particles])
        cfg = self._run_config()
        # the step counter of the device restarts at self.step
        run = ctypes.c_void_p()
        _lib.call("sfp_run_create", mod.handle, ctypes.byref(cfg), 1, inst, len(self.all_particles), segs, nbuf,
                  ctypes.byref(run))
        self._run = run
        self._keep = (mod, params)
        self._ps_base = self.particle_steps  # the device counter restarts with the run
        attach_position_sync(self, self.all_particles)

    def _sync_positions(self):
        sync_positions(self, self.all_particles)

    def _end(self):
        run = getattr(self, "_run", None)
        if run is not None:
            self._sync_positions()
            detach_position_sync(self.all_particles)
            _lib.load().sfp_run_destroy(run)
        self._run = None
        self._keep = None

    def set_kernel(self, massive=None, photon=None):
        """Switch the kernel variants of a device-resident run: `massive` =
        (m_stages, min_blocks), `photon` = (p_stages, p_min_blocks); None
        keeps the current one."""
        if massive is not None:
            self.m_stages, self.min_blocks = int(massive[0]), int(massive[1])
        if photon is not None:
            self.p_stages, self.p_min_blocks = int(photon[0]), int(photon[1])
        if getattr(self, "_run", None) is not None:
            self._end()
            self._begin()

    def run_on_device(self, nstep: int):
        """Advance `nstep` steps keeping every species on the device (no
        prune, no host copies); call finish() to end like start()."""
        if getattr(self, "_run", None) is None:
            self._begin()
        self._loop(self._run, nstep, None)

    def finish(self):
        """End a run_on_device() sequence: prune and return host arrays."""
        self._end()
        for p in self.all_particles:
            p._prune()
            p._to_host()
        _release_cached_blocks()

    def time_step_kernel(self, nstep: int):
        """Advance `nstep` steps with eager launches and return, per step, the
        CUDA-event durations [ms] of its (massive, photon, scan + appends)
        kernels (recorded on the stream they run on; 0 for a kernel the run
        does not launch), with the buffered counts before and after.  A step
        that waited for room is finished untimed and not reported."""
        if getattr(self, "_run", None) is None:
            self._begin()
        before = [p.N_buffered for p in self.all_particles]
        out = []
        L = _lib.load()
        st = _lib.RunState()
        nbuf = (ctypes.c_int64 * len(self.all_particles))()
        for _ in range(int(nstep)):
            ms = (ctypes.c_float * 3)()
            _lib.check(L.sfp_run_steps_timed(self._run, 1, ms, _stream_ptr()), "sfp_run_steps_timed")
            self._pos_dirty = True
            _lib.check(L.sfp_run_read_state(self._run, ctypes.byref(st), nbuf, _stream_ptr()), "read_state")
            self.kernel_launches += self._launches_per_step() + 1
            if st.error or (st.halted and not st.appends_pending):
                raise _lib.SFPError("timed step did not complete")
            if st.appends_pending:  # finish the step; its appends kernel was not timed
                resolve_pending(self._run, self.all_particles, lambda: self._update_run(self._run, counts=False))
                _lib.check(L.sfp_run_read_state(self._run, ctypes.byref(st), nbuf, _stream_ptr()), "read_state")
            else:
                out.append((float(ms[0]), float(ms[1]), float(ms[2])))
            for i, p in enumerate(self.all_particles):
                p.N_buffered = int(nbuf[i])
                p._touch()
        self.particle_steps = self._ps_base + int(st.particle_steps)
        self.step = int(st.step)
        self.t = float(st.t)
        return out, before, [p.N_buffered for p in self.all_particles]

    def _launches_per_step(self):
        """libsfp kernels one step launches: bookkeeping + the massive and
        photon kernels that have species to work on + scan and appends when
        a species emits photons or creates pairs."""
        ps = self.all_particles
        return (1 + any(p.m != 0 for p in ps) + any(p.m == 0 for p in ps)
                + 2 * any(p.bw or p.radiating for p in ps))

    def _loop(self, run, nstep, call_back):
        L = _lib.load()
        n_seg = len(self.all_particles)
        nbuf = (ctypes.c_int64 * n_seg)()
        st = _lib.RunState()
        remaining = int(nstep)
        tic = perf_counter_ns()
        # A step that meets a full destination waits for the host and the rest
        # of the queued chunk is launched as no-op kernels: bound the chunk so
        # a wait wastes at most a few graphs (one host sync per chunk).
        max_chunk = 4 * self.graph_chunk if self.graph_chunk > 0 else 256
        rates = self.__dict__.setdefault("_rates", {})
        while remaining > 0:
            # plan for the chunk about to run; before any append rate is known
            # keep it to one graph, so a wait wastes little
            target = min(remaining, max_chunk if rates else (self.graph_chunk or 64))
            grew, fit = plan_chunk(self.all_particles, rates, target)
            chunk = min(target, fit)
            if call_back:
                chunk = 1
            if self.print_every:
                chunk = min(chunk, self.print_every - (self.step % self.print_every))
            for tr in self._trajectories:
                chunk = min(chunk, tr.steps_to_next(self.step))
            if grew:
                self._update_run(run)
            before = [p.N_buffered for p in self.all_particles]
            _lib.check(L.sfp_run_steps(run, chunk, self.graph_chunk if chunk >= self.graph_chunk else 0,
                                       _stream_ptr()), "sfp_run_steps")
            self._pos_dirty = True
            self.kernel_launches += self._launches_per_step() * chunk + 1
            done = self._sync_state(run, st, nbuf)
            halted = bool(st.halted)
            if halted:
                if st.appends_pending:
                    # finishing the stopped step completes it: count it
                    resolve_pending(run, self.all_particles, lambda: self._update_run(run, counts=False))
                    done += self._sync_state(run, st, nbuf)
                else:
                    _lib.check(L.sfp_run_clear_halt(run, _stream_ptr()), "sfp_run_clear_halt")
            remaining -= done
            if done:
                self._record()
            observe_rates(self.all_particles, before, done, rates)
            if done == 0 and not halted:
                raise _lib.SFPError("the step made no progress")
            if call_back and done:
                call_back(self.step - 1)
            if self.print_every is None or not done:
                continue
            elapsed = perf_counter_ns() - tic
            tic = perf_counter_ns()
            if self.step % self.print_every == 0 and self.progress_bar is not None:
                Ntotal = sum([p.Npart for p in self.all_particles])
                ns_per_particle = elapsed / max(Ntotal, 1) / max(done, 1)
                particle_num_str = ','.join([f"{p.Npart} {p.name}" for p in self.all_particles])
                self.progress_bar.set_postfix_str(f"{particle_num_str}, {ns_per_particle:.0f}ns/particle")
                self.progress_bar.update(self.print_every)
            if self.step % self.print_every == 0 and self.monitor is not None:
                self.monitor(self)

    def _sync_state(self, run, st, nbuf) -> int:
        """Read the run's state into the species; returns the steps completed
        since the last read."""
        _lib.check(_lib.load().sfp_run_read_state(run, ctypes.byref(st), nbuf, _stream_ptr()), "sfp_run_read_state")
        if st.error:
            raise _lib.SFPError(f"device error in the step kernel: {_lib.DEV_ERRORS.get(st.error, st.error)}")
        done = int(st.step) - self.step
        for i, p in enumerate(self.all_particles):
            p.N_buffered = int(nbuf[i])
            if done > 0:
                p._touch()
        self.particle_steps = self._ps_base + int(st.particle_steps)
        self.step = int(st.step)
        self.t = float(st.t)
        return done

    def _update_run(self, run, counts=True):
        segs = self._segments()
        n = len(self.all_particles)
        nbuf = (ctypes.c_int64 * n)(*[p.N_buffered for p in self.all_particles]) if counts else None
        _lib.call("sfp_run_update", run, n, segs, nbuf)
