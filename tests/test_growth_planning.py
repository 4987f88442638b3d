"""Buffer-growth planning of the device loop, on host species: the
reference's growth rule (particles.py:487-500) applied ahead of a chunk of
device steps from the observed append rates (simulation.plan_chunk,
observe_rates, Simulation.reserve).  The device checks each step's exact
number of children against the room before writing them; planning only
makes those waits rare."""
import numpy as np

import sfparticles_b200 as S
from sfparticles_b200.fields import static_field
from sfparticles_b200.simulation import GROWTH_FLOOR, MIN_ROOM, observe_rates, plan_chunk


def _species(n, name="pho"):
    m = 0 if name == "pho" else 1
    props = tuple(np.ones(n) for _ in range(6)) if m else tuple(np.ones(n) * (k + 1) for k in range(6))
    return S.Particles(name, 0 if m == 0 else -1, m, N=n, props=props)


def test_no_rate_no_growth_full_chunk():
    p = _species(100)
    assert plan_chunk([p], {}, 256) == (False, 256)
    assert p.buffer_size == 100


def test_growth_by_the_reference_rule_for_a_chunk():
    p = _species(1000)
    rates = {id(p): 10.0}
    grew, chunk = plan_chunk([p], rates, 256, min_room=0)
    # want 1.25 * 10 * 256 + 1 = 3201, below the cap: the reference rule grows by
    # N_buffered // 4 + N_new = 250 + 3201, and a full chunk fits
    assert grew and p.buffer_size == 1000 + 250 + 3201
    assert chunk == 256
    assert np.all(p._arr["_to_be_pruned"][1000:]) and np.all(p._arr["x"][1000:] == 0)
    assert np.array_equal(p._arr["ux"][:1000], np.full(1000, 4.0))


def test_growth_capped_at_half_the_count_or_the_floor():
    p = _species(1000)
    grew, chunk = plan_chunk([p], {id(p): 1e4}, 256, min_room=0)
    # want 3.2e6 + 1, capped at max(1000 // 2 + 1024, GROWTH_FLOOR) = 2^20
    assert grew and p.buffer_size == 1000 + 250 + GROWTH_FLOOR
    assert chunk == int((250 + GROWTH_FLOOR) / 12500.0)


def test_enough_room_keeps_the_buffers_and_bounds_the_chunk():
    p = _species(100)
    p._extend(5000)  # free room
    size = p.buffer_size
    grew, chunk = plan_chunk([p], {id(p): 4.0}, 256, min_room=0)
    assert not grew and p.buffer_size == size
    assert chunk == min(256, int((size - 100) / 5.0))


def test_a_capped_growth_shortens_the_chunk():
    """b's growth is capped at GROWTH_FLOOR, below a chunk's worth at its
    rate, so b sets the chunk; a has room for a full one."""
    a, b = _species(100), _species(100)
    a._extend(100_000)
    grew, chunk = plan_chunk([a, b], {id(a): 1.0, id(b): 5000.0}, 1000, min_room=0)
    assert grew and b.buffer_size == 100 + 25 + GROWTH_FLOOR
    assert chunk == int((b.buffer_size - 100) / 6250.0) < 1000


def test_a_destination_with_appends_gets_the_minimum_room():
    """A small rate still gets MIN_ROOM free slots (by the reference rule's
    growth), so a ramping rate does not stop a small run for room each
    chunk; a destination without appends is left alone."""
    p, q = _species(10), _species(10)
    grew, chunk = plan_chunk([p, q], {id(p): 0.5}, 256)
    assert grew and p.buffer_size - p.N_buffered == 10 // 4 + MIN_ROOM
    assert q.buffer_size == 10 and chunk == 256
    assert plan_chunk([p, q], {id(p): 0.5}, 256) == (False, 256)


def test_observed_rates_decay_by_half_at_most():
    p = _species(10)
    rates = {}
    observe_rates([p], [0], 5, rates)
    assert rates[id(p)] == 2.0
    observe_rates([p], [10], 5, rates)  # no appends: the rate halves
    assert rates[id(p)] == 1.0
    observe_rates([p], [10], 0, rates)  # no steps: unchanged
    assert rates[id(p)] == 1.0


def test_reserve_covers_a_window_at_twice_the_rate():
    """Simulation.reserve: room for a window of steps at twice the append
    rate seen, on destinations only; the window then plans one chunk."""
    ele = _species(500, "ele")
    pho = S.Particles("pho", 0, 0)
    ele.set_photon(pho)
    sim = S.Simulation(ele, pho, dt=1e-17, fields=static_field(), print_every=None)
    sim._rates = {id(pho): 40.0, id(ele): 0.0}
    size_e = ele.buffer_size
    assert sim.reserve(20)
    assert pho.buffer_size - pho.N_buffered >= 2 * 40 * 20
    assert ele.buffer_size == size_e  # nothing is appended to the electrons
    assert not sim.reserve(20)
    grew, chunk = plan_chunk([ele, pho], sim._rates, 20)
    assert not grew and chunk == 20


def test_destinations_are_photon_and_pair_targets():
    ele, pos = _species(10, "ele"), S.Particles("pos", 1, 1)
    pho = S.Particles("pho", 0, 0)
    ele.set_photon(pho)
    pho.set_pair(ele, pos)
    sim = S.Simulation(ele, pos, pho, dt=1e-17, fields=static_field(), print_every=None)
    assert {id(p) for p in sim._destinations()} == {id(pho), id(ele), id(pos)}
    sim2 = S.Simulation(_species(5, "ele"), dt=1e-17, fields=static_field(), print_every=None)
    assert sim2._destinations() == []
