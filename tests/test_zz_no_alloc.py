"""gw_superstep_static: the superstep for callers that cannot allocate device
memory (a framework whose caching allocator owns the free memory, a serving
loop that must not stall on an allocation's device-wide synchronisation).

It must give exactly what the allocating engine gives for the same superstep
(gw_run in blocked mode, stopped after one block execution): the same visit
counts and, per destination block, the same walks in the same order.  Two
calls in a row check that the shared scratch array left behind by one call
does not leak into the next.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _reference_superstep(gw, G, rule, seed):
    """The allocating engine: one block execution of gw_run's blocked mode."""
    G.walks_clear()
    cur = np.arange(G.nv, dtype=np.uint32)
    G.add_walks_at(cur)
    walknum, _ = G.walks_count()
    b = int(np.argmax(walknum))  # prob = 0: chooseBlock takes the block with the most walks
    p = gw.params(rule, gw.SINK_VERTEX_COUNT, 10, seed=seed, mode=gw.MODE_BLOCKED, prob=0.0,
                  max_supersteps=1)
    st = G.run(p)
    assert st.supersteps == 1
    moved = {}
    for d in range(G.nblocks):
        pool = G.read_pool(d)
        moved[d] = pool[int(walknum[d]):] if d != b else pool
    assert len(moved[b]) == 0
    return b, p, G.read_counts(), moved


def _static_superstep(gw, G, p, b, stream=None):
    """One gw_superstep_static call on `stream` (a torch stream; None = the
    default stream), then gw_sync on that stream, which also reports the
    device status word."""
    import torch
    lo, hi = int(G.blocks[b]), int(G.blocks[b + 1])
    v = torch.arange(lo, hi, dtype=torch.int64, device="cuda")
    walks = torch.stack([v, v, v, torch.zeros_like(v)], 1).to(torch.int32).contiguous()
    n = hi - lo
    counts = torch.zeros(G.nv, dtype=torch.int32, device="cuda")
    moved = torch.full((max(n, 1), 4), -1, dtype=torch.int32, device="cuda")
    offsets = torch.zeros(G.nblocks + 1, dtype=torch.int32, device="cuda")
    minhop = torch.zeros(G.nblocks, dtype=torch.int32, device="cuda")
    lib = gw.load()
    torch.cuda.synchronize()  # the inputs above were written on torch's stream
    sh = None if stream is None else stream.cuda_stream
    status = lib.gw_superstep_static(G.handle, ctypes.byref(p), b, walks.data_ptr(), n, counts.data_ptr(),
                                     moved.data_ptr(), offsets.data_ptr(), minhop.data_ptr(), sh)
    gw._lib.check(status, G.handle)
    G.sync(sh)
    return (counts.cpu().numpy().view(np.uint32), moved.cpu().numpy().view(np.uint32),
            offsets.cpu().numpy().view(np.uint32), minhop.cpu().numpy().view(np.uint32))


def test_superstep_static_matches_blocked_engine(cuda_device):
    import graphwalker_b200 as gw
    with gw.Graph.rmat(14, 16, seed=6, blocksize_kb=64) as G:
        assert 1 < G.nblocks <= 256
        for rule, seed in ((gw.RULE_JUMP, 77), (gw.RULE_STOP, 78)):  # two calls in a row
            b, p, ref_counts, ref_moved = _reference_superstep(gw, G, rule, seed)
            counts, moved, offsets, minhop = _static_superstep(gw, G, p, b)
            assert np.array_equal(counts, ref_counts)
            assert offsets[0] == 0
            for d in range(G.nblocks):
                got = moved[offsets[d]:offsets[d + 1]]
                assert np.array_equal(got, ref_moved[d]), f"destination block {d}"
                exp_min = int(ref_moved[d][:, 3].min()) if len(ref_moved[d]) else 0xFFFFFFFF
                assert int(minhop[d]) == exp_min
            assert offsets[G.nblocks] == sum(len(m) for m in ref_moved.values())


def test_superstep_static_rejects_sizes_beyond_its_limit(cuda_device):
    import graphwalker_b200 as gw
    from graphwalker_b200._lib import GW_E_INVALID
    with gw.Graph.rmat(10, 4, seed=2, blocksize_kb=8) as G:
        p = gw.params(gw.RULE_JUMP, gw.SINK_VERTEX_COUNT, 10, mode=gw.MODE_BLOCKED)
        lib = gw.load()
        status = lib.gw_superstep_static(G.handle, ctypes.byref(p), 0, 16, (1 << 20) + 1, 16, 16, 16, 16, None)
        assert status == GW_E_INVALID
        assert b"at most" in lib.gw_last_error(G.handle)


def test_superstep_static_empty_call_and_side_stream(cuda_device):
    """An empty call (n = 0, no walk buffers) still writes every output: the
    offsets all 0 and every block's min hop "no walk" (0xffffffff), whatever
    the arrays held and whatever the previous call left in the scratch.  A
    call on a side stream, synchronised through gw_sync on that stream, gives
    the default-stream call's results."""
    import torch

    import graphwalker_b200 as gw
    with gw.Graph.rmat(14, 16, seed=6, blocksize_kb=64) as G:
        b, p, ref_counts, ref_moved = _reference_superstep(gw, G, gw.RULE_JUMP, 91)
        default = _static_superstep(gw, G, p, b)  # leaves this superstep in the scratch
        offsets = torch.full((G.nblocks + 1,), 7, dtype=torch.int32, device="cuda")
        minhop = torch.full((G.nblocks,), 5, dtype=torch.int32, device="cuda")
        counts = torch.full((G.nv,), 3, dtype=torch.int32, device="cuda")  # the count sink still needs its array
        torch.cuda.synchronize()
        lib = gw.load()
        gw._lib.check(lib.gw_superstep_static(G.handle, ctypes.byref(p), b, None, 0, counts.data_ptr(), None,
                                              offsets.data_ptr(), minhop.data_ptr(), None), G.handle)
        G.sync()
        assert np.all(counts.cpu().numpy() == 3)  # no walk, no visit
        assert np.all(offsets.cpu().numpy() == 0)
        assert np.all(minhop.cpu().numpy().view(np.uint32) == 0xFFFFFFFF)
        side = torch.cuda.Stream()
        got = _static_superstep(gw, G, p, b, stream=side)
        for x, y in zip(got, default):
            assert np.array_equal(x, y)
        assert np.array_equal(got[0], ref_counts)
