"""Device radix sort and LBVH structure (gpu)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [0, 1, 2, 7, 2048, 2049, 100_003])
@pytest.mark.parametrize("bits", [8, 30, 32])
def test_sort_u32_stable(cuda, n, bits):
    from ipc_warp_b200.lbvh import sort_pairs

    rng = np.random.default_rng(n + bits)
    hi = (1 << bits) if bits < 32 else (1 << 31)
    keys = rng.integers(0, min(hi, max(n // 3, 2)), size=n).astype(np.int64)
    if bits == 32 and n:
        keys[::5] |= 1 << 31  # exercise the top bit
    k = torch.tensor(keys.astype(np.uint32).view(np.int32), device=cuda)
    v = torch.arange(n, dtype=torch.int32, device=cuda)
    sort_pairs(k, v, bits)
    ku = k.cpu().numpy().view(np.uint32)
    masked = keys.astype(np.uint64) & np.uint64((1 << bits) - 1)
    ref = np.argsort(masked, kind="stable")
    assert np.array_equal(v.cpu().numpy(), ref)
    assert np.array_equal(ku.astype(np.uint64) & np.uint64((1 << bits) - 1), masked[ref])


@pytest.mark.parametrize("n", [1, 3, 50_000])
def test_sort_u64(cuda, n):
    from ipc_warp_b200.lbvh import sort_pairs

    rng = np.random.default_rng(n)
    keys = rng.integers(0, 1 << 40, size=n, dtype=np.int64)
    keys[::7] = keys[0]
    k = torch.tensor(keys, device=cuda)
    v = torch.arange(n, dtype=torch.int32, device=cuda)
    sort_pairs(k, v, 41)
    ref = np.argsort(keys, kind="stable")
    assert np.array_equal(v.cpu().numpy(), ref)
    assert np.array_equal(k.cpu().numpy(), keys[ref])


def _check_tree(bvh, lo, hi):
    """Every leaf reached exactly once; every child slot box is the exact
    union of the leaf boxes below it."""
    n = lo.shape[0]
    nodes = bvh.nodes.cpu().numpy()
    seen = np.zeros(n, dtype=np.int64)

    def code(v):
        return int(np.float32(v).view(np.int32))

    def visit(node):
        ls = []
        for side in (0, 1):
            c = code(nodes[node, 2 * side, 3])
            blo, bhi = nodes[node, 2 * side, :3], nodes[node, 2 * side + 1, :3]
            if c < 0:
                prim = ~c
                seen[prim] += 1
                sub = [prim]
            else:
                sub = visit(c)
            assert np.array_equal(blo, lo[sub].min(axis=0)), (node, side)
            assert np.array_equal(bhi, hi[sub].max(axis=0)), (node, side)
            ls += sub
        return ls

    if n >= 2:
        visit(0)
        assert np.all(seen == 1)
    _check_wide(bvh, lo, hi)


def _check_wide(bvh, lo, hi):
    """4-wide view: from wide node 0 every leaf is reached exactly once, each
    slot box is the union of the leaves below it, and each slot's last rank
    is the largest Morton rank below it, the slot covering a contiguous rank
    range (what the pruned self-queries rely on)."""
    import torch

    n = lo.shape[0]
    m = max(n - 1, 1)
    W = bvh._view(bvh.c.wide, 32 * m, torch.float32).view(m, 8, 4).cpu().numpy()
    Wi = W.view(np.int32)
    rank = np.empty(n, dtype=np.int64)
    rank[bvh.sorted.cpu().numpy()] = np.arange(n)
    seen = np.zeros(n, dtype=np.int64)

    def visit(node):
        leaves = []
        for k in range(4):
            blo = np.array([W[node, 0, k], W[node, 1, k], W[node, 2, k]])
            bhi = np.array([W[node, 3, k], W[node, 4, k], W[node, 5, k]])
            c = int(Wi[node, 6, k])
            if blo[0] > bhi[0]:  # empty slot
                continue
            if c < 0:
                seen[~c] += 1
                sub = [~c]
            else:
                sub = visit(c)
            assert np.array_equal(blo, lo[sub].min(axis=0)) and np.array_equal(bhi, hi[sub].max(axis=0))
            r = np.sort(rank[sub])
            assert int(Wi[node, 7, k]) == r[-1] and r[-1] - r[0] == len(r) - 1
            leaves += sub
        return leaves

    visit(0)
    assert np.all(seen == 1)


@pytest.mark.parametrize("n", [2, 3, 17, 4096])
def test_lbvh_structure_and_refit(cuda, n):
    from ipc_warp_b200.lbvh import Bvh

    rng = np.random.default_rng(n)
    c = rng.uniform(-1, 1, size=(n, 3)).astype(np.float32)
    if n > 10:
        c[5] = c[4]  # duplicate Morton code
    ext = rng.uniform(0, 0.05, size=(n, 3)).astype(np.float32)
    lo, hi = c - ext, c + ext
    tl, th = torch.tensor(lo, device=cuda), torch.tensor(hi, device=cuda)
    bvh = Bvh(tl, th)
    torch.cuda.synchronize()
    assert sorted(bvh.sorted.cpu().numpy().tolist()) == list(range(n))
    _check_tree(bvh, lo, hi)
    # refit with moved boxes keeps topology and recomputes unions; twice to
    # check the arrival counters were reset
    for step in range(2):
        d = rng.normal(scale=0.01, size=(n, 3)).astype(np.float32)
        lo2, hi2 = lo + d, hi + d
        tl.copy_(torch.tensor(lo2))
        th.copy_(torch.tensor(hi2))
        bvh.refit()
        torch.cuda.synchronize()
        _check_tree(bvh, lo2, hi2)


def test_lbvh_single_leaf(cuda):
    from ipc_warp_b200.lbvh import Bvh

    lo = torch.tensor([[0.0, 0.0, 0.0]], device=cuda)
    hi = torch.tensor([[1.0, 1.0, 1.0]], device=cuda)
    bvh = Bvh(lo, hi)
    nodes = bvh.nodes.cpu().numpy()
    assert np.array_equal(nodes[0, 0, :3], [0, 0, 0]) and np.array_equal(nodes[0, 1, :3], [1, 1, 1])
    assert int(np.float32(nodes[0, 0, 3]).view(np.int32)) == ~0
