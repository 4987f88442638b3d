"""The step's tile maps, event scan and children's slots, restated from
their index arithmetic (sfparticles_b200/csrc/sfp_step.cuh: sfp_group_plan,
sfp_group_map, sfp_super_info, sfp_scan_group, marks16, sfp_append_tile;
sfp_capi.cu: tiles_for) and checked on the CPU against the order the
reference appends in: every particle in exactly one tile, segments on
super-tile boundaries so a super-tile never spans two segments, each
super-tile's prefix equal to the children that the same instance's earlier
segments and tiles create on the same channel, a tile's marked particles
gathered in index order, and the step's tile length (32 to 1024 by the
population) always fitting the tile counters."""
import numpy as np
import pytest

SUPER = 64  # SFP_SUPER_TILE
TILE = 1024  # SFP_TILE_MAX
TILE_MIN, TILE_TARGET = 32, 4096  # SFP_TILE_MIN, SFP_TILE_TARGET
TILES = [32, 64, 128, 256, 512, 1024]
MARK = 2    # SFP_MARK


def group_map(n_buf, segs, tile=TILE):
    """sfp_group_map: each segment's first tile, at a multiple of SUPER."""
    start, acc = [], 0
    for s in segs:
        acc = (acc + SUPER - 1) // SUPER * SUPER
        start.append(acc)
        acc += (n_buf[s] + tile - 1) // tile
    return start + [acc]


def tiles_for(capacity, segs):
    """sfp_capi.cu tiles_for: the tile counters a group is given."""
    t = sum((capacity[s] + TILE - 1) // TILE + SUPER for s in segs)
    return max(t, TILE_TARGET + len(segs) * (SUPER + 1)) + 1


def group_plan(n_buf, segs, max_tiles):
    """sfp_group_plan: the shortest power-of-two tile from 32 with at most
    TILE_TARGET tiles of population, longer while the map overflows."""
    n = sum(n_buf[s] for s in segs)
    tile = TILE_MIN
    while tile < TILE and tile * TILE_TARGET < n:
        tile <<= 1
    start = group_map(n_buf, segs, tile)
    while start[-1] > max_tiles and tile < TILE:
        tile <<= 1
        start = group_map(n_buf, segs, tile)
    return tile, start


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


def super_info(start, segs, inst, s):
    """(segment, head): the segment of super-tile s and whether it starts
    its instance's chain (the segment of the previous super-tile belongs to
    another instance)."""
    def seg_of(tile):
        return segs[find_group_pos(start, len(segs), tile)]
    si = seg_of(s * SUPER)
    return si, s == 0 or inst[seg_of(s * SUPER - SUPER)] != inst[si]


def scan(start, segs, inst, channel, sup):
    """sfp_scan_group's prefixes: segmented by instance, per channel."""
    pre = np.zeros(len(sup), dtype=np.int64)
    run = {}
    for s in range(len(sup)):
        si, head = super_info(start, segs, inst, s)
        if head:
            run = {}
        ch = channel[si]
        pre[s] = run.get(ch, 0)
        run[ch] = run.get(ch, 0) + sup[s]
    return pre


def check_group(rng, n_buf, segs, inst, channel, tile=TILE):
    start = group_map(n_buf, segs, tile)
    own_tiles = [-(-n_buf[s] // tile) for s in segs]  # the rest up to the next start is padding
    for j, s in enumerate(segs):
        assert start[j] % SUPER == 0 and start[j] + own_tiles[j] <= start[j + 1]
    if not segs or start[-1] == 0:
        return
    assert start[-1] == start[-2] + own_tiles[-1]
    n_tiles = start[-1]
    cnt = np.zeros(n_tiles, dtype=np.int64)
    owner = np.full(n_tiles, -1)
    for j, s in enumerate(segs):
        a, b = start[j], start[j] + own_tiles[j]
        cnt[a:b] = rng.integers(0, 50, b - a)
        owner[a:b] = s
    for s in range(-(-n_tiles // SUPER)):  # a super-tile never spans two segments
        assert len(set(owner[s * SUPER:(s + 1) * SUPER]) - {-1}) <= 1
    sup = np.add.reduceat(cnt, np.arange(0, n_tiles, SUPER))
    pre = scan(start, segs, inst, channel, sup)
    # a tile's first child: super-tile prefix + earlier tiles of the super-tile
    # (sfp_append_tile) == the reference's order: an instance's segments in
    # order, tiles in index order, per channel
    for tile in range(n_tiles):
        if owner[tile] < 0:
            continue
        s = tile // SUPER
        first = pre[s] + cnt[s * SUPER:tile].sum()
        si = owner[tile]
        want = sum(int(cnt[t]) for t in range(tile) if owner[t] >= 0 and inst[owner[t]] == inst[si]
                   and channel[owner[t]] == channel[si])
        assert first == want, (tile, first, want)


@pytest.mark.parametrize("tile", [32, 256, 1024])
@pytest.mark.parametrize("seed", range(6))
def test_tile_maps_and_prefixes_of_both_groups(seed, tile):
    rng = np.random.default_rng(seed)
    n_inst = int(rng.integers(1, 5))
    segs = []  # (instance, massless, channel)
    for i in range(n_inst):
        for _ in range(int(rng.integers(1, 4))):
            segs.append((i, bool(rng.random() < 0.5), int(rng.integers(0, 4))))
    inst = [s[0] for s in segs]
    channel = [s[2] for s in segs]
    n_buf = [int(rng.choice([0, 1, 31, 1023, 1024, 1025, int(rng.integers(0, 300_000))])) for _ in segs]
    mseg = [k for k, s in enumerate(segs) if not s[1]]
    pseg = [k for k, s in enumerate(segs) if s[1]]
    check_group(rng, n_buf, mseg, inst, channel, tile)  # photon children of the massive group
    check_group(rng, n_buf, pseg, inst, channel, tile)  # pair children of the photon group


@pytest.mark.parametrize("seed", range(8))
def test_the_step_tile_fits_the_counters(seed):
    """For populations up to the capacities, the planned tile's map fits the
    counters sized by tiles_for, the tile is the rule's (no fallback to a
    longer one is ever needed), and a large population keeps 1024."""
    rng = np.random.default_rng(100 + seed)
    n_seg = int(rng.integers(1, 7))
    segs = list(range(n_seg))
    cap = [int(rng.choice([0, 1, 1000, 1 << 18, int(rng.integers(1, 1 << 24))])) for _ in segs]
    max_tiles = tiles_for(cap, segs)
    for _ in range(50):
        n_buf = [int(rng.integers(0, c + 1)) for c in cap]
        tile, start = group_plan(n_buf, segs, max_tiles)
        assert tile in TILES and start[-1] <= max_tiles
        n = sum(n_buf)
        want = TILE_MIN
        while want < TILE and want * TILE_TARGET < n:
            want <<= 1
        assert tile == want
        if n > TILE * TILE_TARGET // 2:
            assert tile == TILE
        if tile < TILE:  # a short tile only where the population leaves warps idle at 1024
            assert n <= tile * TILE_TARGET


def vcmpeq4(a, b):
    """__vcmpeq4: 0xff in each byte where the bytes of a and b are equal."""
    r = 0
    for q in range(4):
        if (a >> (8 * q)) & 0xFF == (b >> (8 * q)) & 0xFF:
            r |= 0xFF << (8 * q)
    return r


def marks16(words):
    k = MARK * 0x01010101
    m = 0
    for q, w in enumerate(words):
        c = vcmpeq4(w, k)
        m |= (((c >> 7) & 1) | ((c >> 14) & 2) | ((c >> 21) & 4) | ((c >> 28) & 8)) << (4 * q)
    return m


@pytest.mark.parametrize("seed", range(4))
def test_marks16_finds_the_marked_bytes(seed):
    rng = np.random.default_rng(seed)
    for _ in range(200):
        b = rng.choice([0, 1, MARK], size=16, p=[0.6, 0.2, 0.2]).astype(np.uint8)
        words = [int(x) for x in b.view("<u4")]
        want = sum(1 << i for i in range(16) if b[i] == MARK)
        assert marks16(words) == want


@pytest.mark.parametrize("tile", [32, 128, 1024])
@pytest.mark.parametrize("left,frac", [(1024, 0.1), (1024, 1.0), (1000, 0.3), (513, 0.5), (17, 0.9), (1, 1.0)])
def test_appends_gather_marks_in_index_order(left, frac, tile):
    """sfp_append_tile's gather: lane q of a pass covers flags 16q..16q+15 of
    the pass's 512; each lane writes its marks at the warp's exclusive prefix
    of mark counts; passes stop once the tile's count is reached.  Flags are
    read up to the tile's end (min(N, base + tile)): a tile shorter than a
    pass never reads the next tile's marks, which are planted here."""
    rng = np.random.default_rng(left)
    flags = np.where(rng.random(2 * TILE) < frac, MARK, rng.choice([0, 1], 2 * TILE)).astype(np.uint8)
    flags[left:TILE] = 0  # past the segment's end
    lim = min(left, tile)
    c = int((flags[:lim] == MARK).sum())
    lst = [None] * TILE
    n = 0
    for q0 in range(0, tile, 512):
        if n >= c:
            break
        counts, masks = [], []
        for lane in range(32):
            e0 = q0 + 16 * lane
            if e0 + 16 <= lim:
                m = marks16([int(x) for x in flags[e0:e0 + 16].view("<u4")])
            else:
                m = sum(1 << b for b in range(16) if e0 + b < lim and flags[e0 + b] == MARK)
            masks.append(m)
            counts.append(bin(m).count("1"))
        incl = np.cumsum(counts)
        for lane in range(32):
            w = n + incl[lane] - counts[lane]
            m = masks[lane]
            while m:
                b = (m & -m).bit_length() - 1
                m &= m - 1
                lst[w] = q0 + 16 * lane + b
                w += 1
        n += int(incl[-1])
    assert n == c
    assert lst[:n] == list(np.flatnonzero(flags[:lim] == MARK))
