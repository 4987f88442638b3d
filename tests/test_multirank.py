"""Several ranks, one process each: the host side of a job split across GPUs,
run here as two gloo ranks on the CPU (sfparticles_b200/shard.py)."""
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


def _rank(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import oracle as orc
        from sfparticles_b200.qed import tables
        # rank r runs its slice of one beam on the CPU oracle with its own key
        n = 600
        start, cnt = shard.split_counts(n, world)[rank]
        rng = np.random.default_rng(3)
        g = 2000 * (1 + 0.01 * rng.normal(size=n))
        props = [np.full(n, 1e-6), np.zeros(n), np.zeros(n), np.sqrt(g * g - 1), np.zeros(n), np.zeros(n)]
        props = [a[start:start + cnt] for a in props]
        ele = orc.Species("ele", -1, 1, N=cnt, props=props)
        pho = orc.Species("pho", 0, 0)
        ele.set_photon(pho)
        iA, dA, _, zmax = tables.rs_tables()
        terms = orc.static_field(Bz=2e4)
        sim = orc.OracleSim([ele, pho], 1e-16, terms, ("rs", iA, dA), seed=shard.rank_seed(7, rank), z_max=zmax)
        sim.run(20)
        ms = 10.0 + rank  # stands in for a device time
        got = shard.reduce_job(ms, sim.particle_steps)
        sums = shard.sum_over_ranks([rank + 1, 0.5 * pho.N_buffered])
        out[rank] = (got, sim.particle_steps, pho.N_buffered, sums)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_time_and_work():
    """Two ranks run their halves of a beam; every rank gets the slowest
    rank's time and the job's total work."""
    import torch.multiprocessing as mp
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0, p.exitcode
        res = dict(out)
    total = sum(res[r][1] for r in range(world))
    photons = sum(res[r][2] for r in range(world))
    for r in range(world):
        (ms, ps), _, _, sums = res[r]
        assert ms == 11.0 and ps == total
        assert sums == [3.0, 0.5 * photons]
    assert res[0][1] > 0 and res[1][1] > 0


def test_reduce_job_without_a_process_group_is_the_identity():
    assert shard.reduce_job(3.5, 42) == (3.5, 42.0)
    assert shard.sum_over_ranks([1, 2.5]) == [1.0, 2.5]
