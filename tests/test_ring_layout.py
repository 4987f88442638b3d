"""The copy ring of the massive and photon kernels, restated from its index
arithmetic (sfparticles_b200/csrc/sfp_step.cuh: sfp_ring_issue and the
reads of sfp_massive_tile / sfp_photon_body) and checked on the CPU: every
staged double and flag of a sub-step lands where the compute loop reads it,
exactly once, full 16-byte copies stay inside their arrays, and short copies
cover exactly the particles that exist.  Layouts: 6 components (x..uz), 7
(+ optical depth), 9 (+ spin), 10 (both)."""
import numpy as np
import pytest



def issue(nc, sub, left):
    """(dst byte offset, slot, first element, bytes) of each lane's copy of
    one sub-step; slot nc is the flags array, elements counted from the
    tile's first photon."""
    ncopy = nc * 16 + 2
    full = left >= (sub + 1) * 32
    out = []
    for lane in range(32):
        for k in range((ncopy + 31) // 32):
            c = lane + 32 * k
            if c < nc * 16:
                e = sub * 32 + 2 * (c & 15)
                nb = 16 if full else (16 if left - e >= 2 else (8 if left - e == 1 else 0))
                out.append((c * 16, c >> 4, e, nb))
            elif c < ncopy:
                e = sub * 32 + 16 * (c - nc * 16)
                nb = 16 if full else (16 if left - e >= 16 else max(left - e, 0))
                out.append((c * 16, nc, e, nb))
    return out


@pytest.mark.parametrize("tile", [32, 256, 1024])
@pytest.mark.parametrize("nc", [6, 7, 9, 10])
@pytest.mark.parametrize("left", [1024, 1000, 33, 32, 31, 17, 16, 1])
def test_every_staged_value_lands_where_it_is_read(nc, left, tile):
    """Sub-steps 0..tile/32-1 of a tile (32 to 1024 particles, a multiple of
    32 from the segment's start, so its base stays 16-byte aligned)."""
    stage = nc * 32 * 8 + 32  # sfp_ring<NC>::STAGE_BYTES
    for sub in range(tile // 32):
        owner = np.full(stage, -1, dtype=np.int64)  # which (slot, element) fills each byte
        for dst, slot, e, nb in issue(nc, sub, left):
            assert dst % 16 == 0 and dst + 16 <= stage
            if slot < nc:
                assert e % 2 == 0  # 16-byte aligned source for a tile base at a multiple of 32
                for b in range(nb):  # 8-byte elements e, e+1
                    assert owner[dst + b] == -1  # no byte is written twice
                    owner[dst + b] = slot * 1_000_000 + e + b // 8
                assert nb in (0, 8, 16) and e + nb // 8 <= max(left, e)
            else:
                assert e % 16 == 0
                for b in range(nb):
                    assert owner[dst + b] == -1
                    owner[dst + b] = nc * 1_000_000 + e + b
                assert e + nb <= max(left, e)
        for lane in range(32):  # the compute loop's reads: sd[32 comp + lane], stg[256 nc + lane]
            e = sub * 32 + lane
            if e >= left:
                continue  # not alive: nothing read
            for comp in range(nc):
                off = 8 * (32 * comp + lane)
                assert (owner[off:off + 8] == comp * 1_000_000 + e).all(), (comp, e)
            assert owner[256 * nc + lane] == nc * 1_000_000 + e
