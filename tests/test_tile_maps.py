"""The step's tile maps, event scan and children's slots, restated from
their index arithmetic (sfparticles_b200/csrc/sfp_step.cuh: sfp_group_map,
sfp_super_info, sfp_scan_group, marks16, sfp_append_tile) and checked on
the CPU against the order the reference appends in: every particle in
exactly one tile, segments on super-tile boundaries so a super-tile never
spans two segments, each super-tile's prefix equal to the children that the
same instance's earlier segments and tiles create on the same channel, and
a tile's marked particles gathered in index order."""
import numpy as np
import pytest

SUPER = 64  # SFP_SUPER_TILE
TILE = 1024  # 32 * SFP_WSUB
MARK = 2    # SFP_MARK


def group_map(n_buf, segs, tile=TILE):
    """sfp_group_map: each segment's first tile, at a multiple of SUPER."""
    start, acc = [], 0
    for s in segs:
        acc = (acc + SUPER - 1) // SUPER * SUPER
        start.append(acc)
        acc += (n_buf[s] + tile - 1) // tile
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


def check_group(rng, n_buf, segs, inst, channel):
    start = group_map(n_buf, segs)
    own_tiles = [-(-n_buf[s] // TILE) for s in segs]  # the rest up to the next start is padding
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


@pytest.mark.parametrize("seed", range(6))
def test_tile_maps_and_prefixes_of_both_groups(seed):
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
    check_group(rng, n_buf, mseg, inst, channel)  # photon children of the massive group
    check_group(rng, n_buf, pseg, inst, channel)  # pair children of the photon group


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


@pytest.mark.parametrize("left,frac", [(1024, 0.1), (1024, 1.0), (1000, 0.3), (513, 0.5), (17, 0.9), (1, 1.0)])
def test_appends_gather_marks_in_index_order(left, frac):
    """sfp_append_tile's gather: lane q of a pass covers flags 16q..16q+15 of
    the pass's 512; each lane writes its marks at the warp's exclusive prefix
    of mark counts; passes stop once the tile's count is reached."""
    rng = np.random.default_rng(left)
    flags = np.where(rng.random(TILE) < frac, MARK, rng.choice([0, 1], TILE)).astype(np.uint8)
    flags[left:] = 0  # not part of the segment
    c = int((flags[:left] == MARK).sum())
    lst = [None] * TILE
    n = 0
    for q0 in range(0, TILE, 512):
        if n >= c:
            break
        counts, masks = [], []
        for lane in range(32):
            e0 = q0 + 16 * lane
            if e0 + 16 <= left:
                m = marks16([int(x) for x in flags[e0:e0 + 16].view("<u4")])
            else:
                m = sum(1 << b for b in range(16) if e0 + b < left and flags[e0 + b] == MARK)
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
    assert lst[:n] == list(np.flatnonzero(flags[:left] == MARK))
