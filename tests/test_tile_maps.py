"""The step's tile maps and pair-prefix scan, restated from their index
arithmetic (sfparticles_b200/csrc/sfp_step.cuh: sfp_book_kernel,
sfp_super_info, sfp_pair_scan_kernel) and checked on the CPU against the
order the reference appends in: every particle in exactly one tile,
photon segments on super-tile boundaries so a super-tile never spans two
segments, and each super-tile's prefix equal to the pairs that the same
instance's earlier photon segments and tiles create on the same channel."""
import numpy as np
import pytest

SUPER = 64  # SFP_SUPER_TILE


def massive_map(n_buf, mseg, inst, mtile):
    """(mtile_start per massive segment + end, chain_first per segment)."""
    start, chain_first, acc, prev, chain = [], {}, 0, -1, 0
    for s in mseg:
        start.append(acc)
        if inst[s] != prev:
            prev, chain = inst[s], acc
        chain_first[s] = chain
        acc += (n_buf[s] + mtile - 1) // mtile
    return start + [acc], chain_first


def photon_map(n_buf, pseg, ptile):
    start, acc = [], 0
    for s in pseg:
        acc = (acc + SUPER - 1) // SUPER * SUPER
        start.append(acc)
        acc += (n_buf[s] + ptile - 1) // ptile
    return start + [acc]


def find_group_pos(start, n, tk):
    """sfp_find_group_pos: the last of start[0..n-1] at or below tk."""
    lo, hi = 0, n - 1
    while lo < hi:
        mid = (lo + hi + 1) >> 1
        if start[mid] <= tk:
            lo = mid
        else:
            hi = mid - 1
    return lo


def super_info(start, pseg, inst, s):
    """(segment, head): the segment of super-tile s and whether it starts
    its instance's chain (sfp_super_info: the segment of the previous
    super-tile belongs to another instance)."""
    def seg_of(tile):
        return pseg[find_group_pos(start, len(pseg), tile)]
    si = seg_of(s * SUPER)
    return si, s == 0 or inst[seg_of(s * SUPER - SUPER)] != inst[si]


@pytest.mark.parametrize("seed", range(6))
def test_tile_maps_and_pair_prefixes(seed):
    rng = np.random.default_rng(seed)
    n_inst = int(rng.integers(1, 5))
    segs = []  # (instance, massless, channel)
    for i in range(n_inst):
        for _ in range(int(rng.integers(1, 4))):
            segs.append((i, bool(rng.random() < 0.5), int(rng.integers(0, 4))))
    inst = [s[0] for s in segs]
    n_buf = [int(rng.choice([0, 1, 31, 1023, 1024, 1025, int(rng.integers(0, 300_000))])) for _ in segs]
    mseg = [k for k, s in enumerate(segs) if not s[1]]
    pseg = [k for k, s in enumerate(segs) if s[1]]

    mstart, chain_first = massive_map(n_buf, mseg, inst, 512)
    for j, s in enumerate(mseg):  # each particle in one tile, tiles contiguous per segment
        assert mstart[j + 1] - mstart[j] == -(-n_buf[s] // 512)
        first = next(k for k in mseg if inst[k] == inst[s])
        assert chain_first[s] == mstart[mseg.index(first)]

    ptile = 1024
    pstart = photon_map(n_buf, pseg, ptile)
    own_tiles = [-(-n_buf[s] // ptile) for s in pseg]  # the rest up to the next start is padding
    for j, s in enumerate(pseg):
        assert pstart[j] % SUPER == 0 and pstart[j] + own_tiles[j] <= pstart[j + 1]
    assert pstart[-1] == pstart[-2] + own_tiles[-1] if pseg else True
    n_tiles = pstart[-1]
    if not pseg or n_tiles == 0:
        return
    # events per photon tile (padding tiles between segments hold none)
    cnt = np.zeros(n_tiles, dtype=np.int64)
    owner = np.full(n_tiles, -1)
    for j, s in enumerate(pseg):
        a, b = pstart[j], pstart[j] + own_tiles[j]
        cnt[a:b] = rng.integers(0, 50, b - a)
        owner[a:b] = s
    n_super = -(-n_tiles // SUPER)
    sup = np.add.reduceat(cnt, np.arange(0, n_tiles, SUPER))
    for s in range(n_super):  # a super-tile never spans two segments
        own = set(owner[s * SUPER:(s + 1) * SUPER]) - {-1}
        assert len(own) <= 1
    # the scan's prefixes, restated: segmented by instance, per channel
    pre = np.zeros(n_super, dtype=np.int64)
    run = {}
    for s in range(n_super):
        si, head = super_info(pstart, pseg, inst, s)
        if head:
            run = {}
        ch = segs[si][2]
        pre[s] = run.get(ch, 0)
        run[ch] = run.get(ch, 0) + sup[s]
    # the reference's order: an instance's photon segments in order, tiles in index order
    for s in range(n_super):
        si, _ = super_info(pstart, pseg, inst, s)
        ch, i = segs[si][2], inst[si]
        want = sum(int(cnt[t]) for t in range(s * SUPER) if owner[t] >= 0 and inst[owner[t]] == i
                   and segs[owner[t]][2] == ch)
        assert pre[s] == want, (s, pre[s], want)
