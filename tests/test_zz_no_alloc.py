"""The allocation-free LBVH build (ipcb_lbvh_build_noalloc) against the
regular build (ipcb_lbvh_build), through the C ABI (gpu).

The no-alloc entry point exists for callers that cannot call cudaMalloc
while a step runs: its scratch is a static device array shared by all calls,
so this test runs two builds in a row on different boxes (the second must not
see the first one's scratch) and checks that sizes above the static limit are
refused before anything is launched.  It is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest
import torch

from ipc_warp_b200 import _native as N

pytestmark = pytest.mark.gpu


def _bound(n, device):
    mem = torch.empty(N.size("ipcb_lbvh_bytes", n), dtype=torch.uint8, device=device)
    bvh = N.Lbvh()
    N.call("ipcb_lbvh_bind", ctypes.byref(bvh), N.ptr(mem), n)
    return bvh, mem


def _arrays(bvh, mem, n):
    def view(addr, count, dtype):
        off = addr - mem.data_ptr()
        size = count * torch.tensor([], dtype=dtype).element_size()
        return mem[off:off + size].view(dtype).cpu().numpy()

    parent = view(bvh.parent, 2 * n, torch.int32)
    # written parent entries: internal nodes 1..n-2 (the root has none) and the n leaves
    written = np.concatenate([parent[1:max(n - 1, 1)], parent[n:2 * n]]) if n > 1 else parent[:0]
    # nodes compared as raw bits: their w lanes hold integer child codes
    return (view(bvh.nodes, 16 * max(n - 1, 1), torch.int32), view(bvh.sorted, n, torch.int32), written)


@pytest.mark.parametrize("sizes", [(50_000, 1_000), (3, 262_144)])
def test_noalloc_build_matches_regular_build_twice(cuda, sizes):
    rng = np.random.default_rng(sizes[0])
    stream = N.stream_handle()
    for n in sizes:  # two calls in a row on the shared static scratch
        c = rng.uniform(-1, 1, size=(n, 3)).astype(np.float32)
        ext = rng.uniform(0, 0.02, size=(n, 3)).astype(np.float32)
        lo = torch.tensor(c - ext, device=cuda)
        hi = torch.tensor(c + ext, device=cuda)

        ref, ref_mem = _bound(n, cuda)
        ws = torch.empty(N.size("ipcb_lbvh_build_workspace", n), dtype=torch.uint8, device=cuda)
        N.call("ipcb_lbvh_build", ctypes.byref(ref), N.ptr(lo), N.ptr(hi), n, N.ptr(ws), ws.numel(), stream)

        got, got_mem = _bound(n, cuda)
        rc = N.lib().ipcb_lbvh_build_noalloc(ctypes.byref(got), N.ptr(lo), N.ptr(hi), n, stream)
        assert rc == 0, N.lib().ipcb_last_error()
        torch.cuda.synchronize()
        assert got.n == ref.n == n
        for a, b in zip(_arrays(got, got_mem, n), _arrays(ref, ref_mem, n)):
            assert np.array_equal(a, b)


def test_noalloc_rejects_sizes_above_the_static_limit(cuda):
    limit = 1 << 18
    assert N.lib().ipcb_lbvh_build_noalloc_scratch_bytes() >= N.size("ipcb_lbvh_build_workspace", limit)
    bvh, _ = _bound(1, cuda)
    rc = N.lib().ipcb_lbvh_build_noalloc(ctypes.byref(bvh), None, None, limit + 1, N.stream_handle())
    assert rc == 1
    assert b"IPCB_LBVH_NOALLOC_MAX_PRIMS" in N.lib().ipcb_last_error()


@pytest.mark.parametrize("n", [0, 1])
def test_noalloc_tiny_sizes_match_regular_build(cuda, n):
    stream = N.stream_handle()
    lo = torch.tensor([[0.0, 0.0, 0.0]], device=cuda)
    hi = torch.tensor([[1.0, 1.0, 1.0]], device=cuda)
    ref, ref_mem = _bound(1, cuda)
    ws = torch.empty(N.size("ipcb_lbvh_build_workspace", 1), dtype=torch.uint8, device=cuda)
    N.call("ipcb_lbvh_build", ctypes.byref(ref), N.ptr(lo), N.ptr(hi), n, N.ptr(ws), ws.numel(), stream)
    got, got_mem = _bound(1, cuda)
    rc = N.lib().ipcb_lbvh_build_noalloc(ctypes.byref(got), N.ptr(lo), N.ptr(hi), n, stream)
    assert rc == 0, N.lib().ipcb_last_error()
    torch.cuda.synchronize()
    assert got.n == ref.n == n
    if n == 1:
        assert np.array_equal(_arrays(got, got_mem, 1)[1], _arrays(ref, ref_mem, 1)[1])


def test_noalloc_rejects_negative_n_and_small_capacity(cuda):
    bvh, _ = _bound(4, cuda)
    lo = torch.zeros((8, 3), device=cuda)
    hi = torch.ones((8, 3), device=cuda)
    rc = N.lib().ipcb_lbvh_build_noalloc(ctypes.byref(bvh), N.ptr(lo), N.ptr(hi), -1, N.stream_handle())
    assert rc == 1 and b"negative" in N.lib().ipcb_last_error()
    rc = N.lib().ipcb_lbvh_build_noalloc(ctypes.byref(bvh), N.ptr(lo), N.ptr(hi), 8, N.stream_handle())
    assert rc == 1 and b"capacity" in N.lib().ipcb_last_error()
    assert bvh.n == 0  # a refused call leaves the hierarchy as it was
    # the allocating build reports its own argument errors the same way
    ws = torch.empty(N.size("ipcb_lbvh_build_workspace", 8), dtype=torch.uint8, device=cuda)
    rc = N.lib().ipcb_lbvh_build(ctypes.byref(bvh), N.ptr(lo), N.ptr(hi), 8, N.ptr(ws), ws.numel(),
                                 N.stream_handle())
    assert rc == 1 and b"capacity" in N.lib().ipcb_last_error()
