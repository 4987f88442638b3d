"""Several ranks, one process each: the host side of a job split across GPUs,
run here as two gloo ranks on the CPU (sfparticles_b200/shard.py): the
split of a beam and of a batch of collisions, the Philox keys, and the
collectives -- job-wide counters and photon spectrum, slowest time and total
work."""
import os
import socket

import numpy as np

from sfparticles_b200 import shard


def test_split_counts_cover_the_beam_once():
    for total, world in ((10, 3), (7, 8), (1_000_003, 4), (0, 2)):
        parts = shard.split_counts(total, world)
        assert len(parts) == world and sum(n for _, n in parts) == total
        assert all(parts[r][0] + parts[r][1] == parts[r + 1][0] for r in range(world - 1))
        assert max(n for _, n in parts) - min(n for _, n in parts) <= 1


def test_assign_instances_balances_expected_work():
    rng = np.random.default_rng(0)
    costs = 10 ** rng.uniform(3, 6, 256)  # the batched workload's electron counts
    for world in (2, 4, 8):
        lists = shard.assign_instances(costs, world)
        assert sorted(i for lst in lists for i in lst) == list(range(256))
        assert all(lst == sorted(lst) for lst in lists)
        load = [costs[lst].sum() for lst in lists]
        assert max(load) <= sum(load) / world + costs.max()


def test_rank_seeds_differ():
    seeds = {shard.rank_seed(1000, r) for r in range(64)}
    assert len(seeds) == 64 and all(0 <= s < 2 ** 64 for s in seeds)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_species(rank):
    """Rank `rank`'s share of a job, host-resident product species: its slice
    of a beam of electrons, no positrons yet, and photons whose energies
    depend on the rank (some pruned, one below the spectrum's range)."""
    import sfparticles_b200 as S
    n = 600
    start, cnt = shard.split_counts(n, 2)[rank]
    rng = np.random.default_rng(3)
    g = 2000 * (1 + 0.01 * rng.normal(size=n))
    props = [np.full(n, 1e-6), np.zeros(n), np.zeros(n), np.sqrt(g * g - 1), np.zeros(n), np.zeros(n)]
    ele = S.Particles("ele", -1, 1, N=cnt, props=tuple(a[start:start + cnt] for a in props))
    pos = S.Particles("pos", 1, 1)
    m = 50 + 30 * rank
    e = 10 ** np.random.default_rng(10 + rank).uniform(0.0, 3.2, m)  # energies [m_e c^2], some below 2
    pho = S.Particles("pho", 0, 0, N=m, props=(np.zeros(m), np.zeros(m), np.zeros(m), e, np.zeros(m), np.zeros(m)))
    pr = np.zeros(m, dtype=bool)
    pr[::7] = True
    pho._to_be_pruned = pr
    return [ele, pos, pho], e[~pr]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        species, _ = _rank_species(rank)
        particle_steps = 1000.0 * (rank + 1)
        ms = 10.0 + rank  # stands in for a device time
        got = shard.reduce_job(ms, particle_steps)
        sums = shard.sum_over_ranks([rank + 1, 0.5 * species[2].N_buffered])
        diag = shard.reduce_diagnostics(species, particle_steps, bins=16, lo=2.0, hi=2500.0)

        class _Run:  # what a JobDiagnostics monitor reads from a Simulation
            all_particles, step = species, 40

        _Run.particle_steps = particle_steps
        mon = shard.JobDiagnostics(bins=16)
        mon(_Run)
        out[rank] = (got, sums, {k: (dict(v) if isinstance(v, dict) else (np.asarray(v).tolist()
                                 if not isinstance(v, tuple) else v)) for k, v in diag.items()},
                     mon.history[0][0], np.asarray(mon.history[0][1]["spectrum"]).tolist())
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_counters_spectrum_time_and_work():
    """Two ranks hold their halves of a job; one all-reduce gives every rank
    the job's buffered and alive counts, particle-steps and photon spectrum
    (the product's reduce_diagnostics on host-resident species), and
    reduce_job the slowest rank's time and the total work."""
    import torch.multiprocessing as mp
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")  # no fork of a process that already runs threads
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0, p.exitcode
        res = dict(out)
    # the expected job-wide values, from each rank's share built here
    shares = [_rank_species(r) for r in range(world)]
    energies = np.concatenate([e for _, e in shares])
    want_spec, _ = np.histogram(np.log10(energies), bins=16, range=(np.log10(2.0), np.log10(2500.0)))
    want_buf = {nm: sum(sp[i].N_buffered for sp, _ in shares) for i, nm in enumerate(("ele", "pos", "pho"))}
    want_alive = {nm: sum(sp[i].Npart for sp, _ in shares) for i, nm in enumerate(("ele", "pos", "pho"))}
    assert want_alive["pho"] < want_buf["pho"] and energies.min() < 2.0  # pruned and out-of-range photons
    for r in range(world):
        (ms, ps), sums, diag, mstep, mspec = res[r]
        assert ms == 11.0 and ps == 3000.0
        assert sums == [3.0, 0.5 * want_buf["pho"]]
        assert diag["buffered"] == want_buf and diag["alive"] == want_alive
        assert diag["particle_steps"] == 3000.0
        assert np.array_equal(np.asarray(diag["spectrum"]), want_spec)
        assert mstep == 40 and np.array_equal(np.asarray(mspec), want_spec)


def test_reduce_job_without_a_process_group_is_the_identity():
    assert shard.reduce_job(3.5, 42) == (3.5, 42.0)
    assert shard.sum_over_ranks([1, 2.5]) == [1.0, 2.5]
    species, e = _rank_species(0)
    d = shard.reduce_diagnostics(species, 7.0, bins=8)
    assert d["particle_steps"] == 7.0 and d["buffered"]["ele"] == 300 and d["spectrum"].sum() == np.sum(e >= 2.0)
