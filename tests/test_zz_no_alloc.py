"""sfp_find_event_index_noalloc (find_event_index with the library's own
fixed scratch, no allocation) against the workspace entry point
sfp_find_event_index and against torch.nonzero, through the C-ABI.

Indices are integers: the bar is exact equality.  The file is named to be
collected last, so it also runs after every other GPU test in the same
process; run alone, its first call is the one that sets the scratch up.
"""
import ctypes

import pytest

from gpu_helpers import cuda_or_skip

pytestmark = pytest.mark.gpu

MAX_N = 1 << 28  # SFP_FEI_NOALLOC_MAX_N


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _events(n, density, gen):
    import torch
    return (torch.rand(n, device="cuda", generator=gen) < density).to(torch.uint8)


def _with_workspace(L, ev, n_event, stream):
    """Indices from the existing entry point (caller workspace)."""
    import torch
    from sfparticles_b200 import _lib
    n = ev.numel()
    ws = torch.empty(max(int(L.sfp_find_event_index_workspace(n)), 8), dtype=torch.uint8, device="cuda")
    out = torch.full((max(n_event, 1),), -1, dtype=torch.int64, device="cuda")
    _lib.check(L.sfp_find_event_index(_p(ev), n_event, n, _p(out), _p(ws), ws.numel(), stream),
               "sfp_find_event_index")
    return out[:n_event]


def test_noalloc_matches_workspace_entry_on_two_calls_in_a_row():
    cuda_or_skip()
    import torch
    from sfparticles_b200 import _lib
    L = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    gen = torch.Generator(device="cuda").manual_seed(20240601)
    # a large ragged mask, then a small one: the second call leaves most of
    # the scratch as the first call wrote it, which must not matter
    cases = [(10_000_019, 0.3), (4097, 0.5)]
    evs = [_events(n, d, gen) for n, d in cases]
    n_events = [int(e.sum().item()) for e in evs]
    outs = [torch.full((max(k, 1),), -1, dtype=torch.int64, device="cuda") for k in n_events]
    # set-up call (N = 0): looks up the scratch address, loading the module if needed;
    # then one small call, so that the kernels' code is loaded before memory is measured
    _lib.check(L.sfp_find_event_index_noalloc(_p(evs[0]), 0, 0, _p(outs[0]), stream), "set-up")
    warm = torch.empty(max(n_events[1], 1), dtype=torch.int64, device="cuda")
    _lib.check(L.sfp_find_event_index_noalloc(_p(evs[1]), n_events[1], evs[1].numel(), _p(warm), stream), "warm")
    torch.cuda.synchronize()
    free0, alloc0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_allocated()
    for ev, k, out in zip(evs, n_events, outs):  # two calls in a row, one stream, no sync between
        _lib.check(L.sfp_find_event_index_noalloc(_p(ev), k, ev.numel(), _p(out), stream),
                   "sfp_find_event_index_noalloc")
    torch.cuda.synchronize()
    free1, alloc1 = torch.cuda.mem_get_info()[0], torch.cuda.memory_allocated()
    # nothing was allocated: neither through torch nor from the driver
    assert alloc1 == alloc0, (alloc0, alloc1)
    assert free1 == free0, (free0, free1)
    for ev, k, out in zip(evs, n_events, outs):
        ref = _with_workspace(L, ev, k, stream)
        truth = torch.nonzero(ev).flatten()
        assert k > 0 and out[:k].shape == ref.shape == truth.shape
        assert torch.equal(out[:k], ref), "no-alloc and workspace entry points differ"
        assert torch.equal(out[:k], truth)


def test_noalloc_at_the_maximum_size_and_repeated():
    """N = 2^28 exactly (sparse events), twice: same result both times."""
    cuda_or_skip()
    import torch
    from sfparticles_b200 import _lib
    L = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    gen = torch.Generator(device="cuda").manual_seed(7)
    ev = _events(MAX_N, 1e-3, gen)
    k = int(ev.sum().item())
    a = torch.empty(k, dtype=torch.int64, device="cuda")
    b = torch.empty(k, dtype=torch.int64, device="cuda")
    _lib.check(L.sfp_find_event_index_noalloc(_p(ev), k, MAX_N, _p(a), stream), "noalloc")
    _lib.check(L.sfp_find_event_index_noalloc(_p(ev), k, MAX_N, _p(b), stream), "noalloc")
    ref = _with_workspace(L, ev, k, stream)
    torch.cuda.synchronize()
    assert torch.equal(a, ref) and torch.equal(b, ref)


def test_noalloc_rejects_sizes_beyond_the_maximum_and_accepts_empty():
    cuda_or_skip()
    import torch
    from sfparticles_b200 import _lib
    L = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ev = torch.zeros(16, dtype=torch.uint8, device="cuda")
    out = torch.full((4,), -1, dtype=torch.int64, device="cuda")
    # rejected on the host before any device work
    rc = L.sfp_find_event_index_noalloc(_p(ev), 1, MAX_N + 1, _p(out), stream)
    assert rc == -1  # SFP_EINVAL
    assert b"exceeds the maximum" in L.sfp_last_error()
    # empty inputs: nothing to do, nothing written
    assert L.sfp_find_event_index_noalloc(_p(ev), 0, 16, _p(out), stream) == 0
    assert L.sfp_find_event_index_noalloc(_p(ev), 0, 0, _p(out), stream) == 0
    torch.cuda.synchronize()
    assert bool((out == -1).all())
