"""CPU oracle of the learned preconditioner (test infrastructure only; the
product never imports this module).

The network is a message-passing net over the 3x3-block sparsity graph of a
Newton matrix A (n block rows, the edges are the stored blocks, self loops
included, sorted by (row, column)).  It outputs, on the lower pattern of A,
the row directions H of a block lower-triangular factorised sparse
approximate inverse (FSAI): H_ii = I and H_ij = (rho_i out_ij - I) A^_ij,
with A^ = S A S (S = diag(A)^-1/2 per scalar), out_ij the head output read as
a 3x3 matrix and rho_i a coupling gate (``coupling``).  Each block row is then
normalised exactly: with T_ij = sum_k H_ik A^_kj and M_i = sum_j T_ij H_ij^T
= H_i A^ H_i^T, G^_i = L_i H_i where L_i = chol(M_i)^-1, so that every
diagonal block of G^ A^ G^T is the identity, and M^-1 = S G^T G^ S
preconditions A.  For such a factor the Kaporin condition number reduces to

  loss = (1 / N) sum_i log det M_i,  N = 3 n,     dloss/dH_ij = (2 / N) M_i^-1 T_ij,

minimised over H by training (the FSAI functional).  The reference has no
learned component (its solve is cg or cuDSS LDLT,
time_integrator_base.py:470-507); this module restates the algorithm of
ipc_warp_b200/csrc/mpnn.cu in float64 with the same bfloat16 rounding points,
so that the device kernels can be checked value by value.

Rounding points (as the kernels): inputs x, y, the weights used in the
products, and the stored activations h, e, m, u and the aggregate a are
bfloat16; products accumulate in float; biases are float; H and G^ are float.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

WIDTH = 64
IN_DIM = 16
LAYERS = 4


ROUND = True  # set False for finite-difference checks of the backward pass


def bf16(a):
    """Round float values to bfloat16 (nearest even), returned as float64."""
    if not ROUND:
        return np.asarray(a, dtype=np.float64)
    a32 = np.ascontiguousarray(a, dtype=np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)
    return out.astype(np.float64)


def relu(a):
    return np.maximum(a, 0.0)


@dataclass
class Graph:
    n: int
    offsets: np.ndarray  # (n+1,)
    cols: np.ndarray     # (E,)
    rows: np.ndarray     # (E,)
    rev: np.ndarray      # (E,) index of (j, i)
    lower: np.ndarray    # (L,) edge indices with col <= row, in edge order
    diag: np.ndarray     # (n,) edge index of (i, i)


def graph(offsets, cols) -> Graph:
    offsets = np.asarray(offsets, np.int64)
    cols = np.asarray(cols, np.int64)
    n = len(offsets) - 1
    rows = np.repeat(np.arange(n), np.diff(offsets))
    key = rows * n + cols
    order = {int(k): e for e, k in enumerate(key)}
    rev = np.array([order[int(c) * n + int(r)] for r, c in zip(rows, cols)], np.int64)
    lower = np.nonzero(cols <= rows)[0]
    diag = np.array([order[i * n + i] for i in range(n)], np.int64)
    return Graph(n, offsets, cols, rows, rev, lower, diag)


def scaled(g: Graph, vals):
    """A^ = S A S, S = diag(A)^-1/2 per scalar dof; returns (A^ blocks, s)."""
    vals = np.asarray(vals, np.float64).reshape(-1, 3, 3)
    d = np.stack([vals[g.diag][:, a, a] for a in range(3)], axis=1)  # (n, 3)
    s = 1.0 / np.sqrt(d)
    Ah = vals * s[g.rows][:, :, None] * s[g.cols][:, None, :]
    return Ah, s


def features(g: Graph, Ah):
    """Node inputs x (n, 16) and edge inputs y (E, 16), bfloat16."""
    deg = np.diff(g.offsets).astype(np.float64)
    fro = np.sqrt((Ah * Ah).sum(axis=(1, 2)))
    off = np.where(g.cols != g.rows, fro, 0.0)
    rowsum = np.zeros(g.n)
    np.add.at(rowsum, g.rows, off)
    x = np.zeros((g.n, IN_DIM))
    x[:, :9] = Ah[g.diag].reshape(-1, 9)
    x[:, 9] = np.log1p(deg)
    x[:, 10] = rowsum
    y = np.zeros((len(g.cols), IN_DIM))
    y[:, :9] = Ah.reshape(-1, 9)
    y[:, 9] = fro
    y[:, 10] = (g.cols == g.rows).astype(np.float64)
    return bf16(x), bf16(y)


def init_params(seed=0, zero_head=True):
    """Weights (in, out) with biases; the output head starts at zero, so that
    the initial directions are first-order FSAI (H_ij = -A^_ij)."""
    rng = np.random.default_rng(seed)

    def lin(i, o, scale=None):
        s = np.sqrt(2.0 / i) if scale is None else scale
        return rng.normal(scale=s, size=(i, o)), np.zeros(o)

    p = {}
    p["W_hin"], p["b_hin"] = lin(IN_DIM, WIDTH)
    p["W_ein"], p["b_ein"] = lin(IN_DIM, WIDTH)
    for l in range(LAYERS):
        p[f"W1_{l}"], p[f"b1_{l}"] = lin(3 * WIDTH, WIDTH)
        p[f"W2_{l}"], p[f"b2_{l}"] = lin(2 * WIDTH, WIDTH)
    p["W_off"], p["b_off"] = lin(WIDTH, 9, scale=0.0 if zero_head else 0.05)
    return p


PARAM_ORDER = (["W_hin", "b_hin", "W_ein", "b_ein"]
               + [f"{k}_{l}" for l in range(LAYERS) for k in ("W1", "b1", "W2", "b2")]
               + ["W_off", "b_off"])


def forward(g: Graph, x, y, p, keep=False, Ah=None):
    """Row directions H on the lower edges (L, 3, 3): H_ii = I and
    H_ij = (rho_i out - I) A^_ij (Ah: float32 values as the kernels read
    them); with keep=True also the stored activations for the backward
    pass."""
    W = {k: (bf16(v) if k.startswith("W") else v) for k, v in p.items()}
    deg = np.diff(g.offsets).astype(np.float64)
    h = bf16(relu(x @ W["W_hin"] + W["b_hin"]))
    e = bf16(relu(y @ W["W_ein"] + W["b_ein"]))
    tape = []
    for l in range(LAYERS):
        X = np.concatenate([h[g.rows], h[g.cols], e], axis=1)
        m = bf16(relu(X @ W[f"W1_{l}"] + W[f"b1_{l}"]))
        agg = np.zeros((g.n, WIDTH))
        np.add.at(agg, g.rows, m)
        a = bf16(agg / deg[:, None])
        Xn = np.concatenate([h, a], axis=1)
        u = bf16(relu(Xn @ W[f"W2_{l}"] + W[f"b2_{l}"]))
        tape.append((h, e, m, a, u))
        e = bf16(e + m)
        h = bf16(h + u)
    el = e[g.lower]
    is_diag = g.cols[g.lower] == g.rows[g.lower]
    Al = _lower_blocks(g, Ah)
    rho = coupling(x)[g.rows[g.lower]]
    P_off = (el @ W["W_off"] + W["b_off"]).reshape(-1, 3, 3) * rho[:, None, None] - np.eye(3)
    H = np.where(is_diag[:, None, None], np.eye(3), P_off @ Al)
    if keep:
        return H, dict(tape=tape, h=h, e=e, W=W, is_diag=is_diag, Al=Al, rho=rho)
    return H


def _lower_blocks(g: Graph, Ah):
    """A^ of the lower blocks as float32 values (identity blocks where A^ is
    not given)."""
    if Ah is None:
        return np.tile(np.eye(3), (len(g.lower), 1, 1))
    return np.asarray(Ah, np.float32).reshape(-1, 3, 3)[g.lower].astype(np.float64)


def head_output_grad(dH, is_diag, Al, rho):
    """Gradient w.r.t. the head outputs (L, 9) from the gradient w.r.t. H:
    rho_i dH A^T off the diagonal (H_ij = (rho_i out - I) A^_ij), 0 on it."""
    dout = np.asarray(dH, np.float64).reshape(-1, 3, 3).copy()
    dout[~is_diag] = dout[~is_diag] @ np.transpose(Al[~is_diag], (0, 2, 1))
    dout *= rho[:, None, None]
    dout[is_diag] = 0.0
    return dout.reshape(-1, 9)


def coupling(x):
    """rho_i = c / (1 + c), c = sum_j |A^_ij|_F over the off-diagonal blocks
    of row i (node feature 10, bf16): a row without coupling keeps its
    first-order directions whatever the head outputs."""
    c = np.asarray(x, np.float64)[:, 10]
    return c / (1.0 + c)


def random_spd(nb, seed, band=5, couplings=3):
    """A symmetric positive definite block matrix with a banded random pattern
    (diagonal plus PSD pair couplings), as (offsets, cols, vals)."""
    rng = np.random.default_rng(seed)
    blocks = {}

    def add(i, j, B):
        blocks[(i, j)] = blocks.get((i, j), 0.0) + B

    for i in range(nb):
        add(i, i, np.eye(3) * (0.5 + rng.uniform()) + np.diag(rng.uniform(0, 2, 3)))
        if i == 0:
            continue
        for j in rng.choice(np.arange(max(0, i - band), i), size=min(i, couplings), replace=False):
            B = rng.normal(size=(3, 3))
            Gm = B @ B.T
            add(i, i, Gm)
            add(int(j), int(j), Gm)
            add(i, int(j), -0.9 * Gm)
            add(int(j), i, -0.9 * Gm)
    keys = sorted(blocks)
    offsets = np.zeros(nb + 1, np.int64)
    for (i, _) in keys:
        offsets[i + 1] += 1
    offsets = np.cumsum(offsets)
    cols = np.array([j for (_, j) in keys], np.int64)
    vals = np.stack([blocks[k] for k in keys])
    return offsets, cols, vals


def _lower_rows(g: Graph):
    rows = [[] for _ in range(g.n)]
    for s, e in enumerate(g.lower):
        rows[int(g.rows[e])].append((int(g.cols[e]), s))
    return rows


def products(g: Graph, Ah, H):
    """T_ij = sum_{k <= i} H_ik A^_kj on the lower pattern (L, 3, 3)."""
    full = {(int(r), int(c)): e for e, (r, c) in enumerate(zip(g.rows, g.cols))}
    T = np.zeros_like(H)
    for i, row in enumerate(_lower_rows(g)):
        for (j, sj) in row:
            acc = np.zeros((3, 3))
            for (k, sk) in row:
                e = full.get((k, j))
                if e is not None:
                    acc += H[sk] @ Ah[e]
            T[sj] = acc
    return T


def normalize(g: Graph, Ah, H):
    """G^ = L H row by row with L_i = chol(M_i)^-1, M_i = sum_j T_ij H_ij^T;
    returns (G, loss, dH): loss = (1/N) sum_i log det M_i and its gradient
    w.r.t. the off-diagonal H_ij, (2/N) M_i^-1 T_ij."""
    T = products(g, Ah, H)
    N = 3 * g.n
    G = np.zeros_like(H)
    dH = np.zeros_like(H)
    loss = 0.0
    for i, row in enumerate(_lower_rows(g)):
        M = sum(T[s] @ H[s].T for (_, s) in row)
        M = 0.5 * (M + M.T)
        C = np.linalg.cholesky(M)
        Li = np.linalg.inv(C)
        Mi = np.linalg.inv(M)
        loss += np.linalg.slogdet(M)[1]
        for (j, s) in row:
            G[s] = Li @ H[s]
            if j != i:
                dH[s] = (2.0 / N) * Mi @ T[s]
    return G, loss / N, dH


def kaporin(g: Graph, Ah, G):
    """log(tr(G A^ G^T) / N) - (2/N) sum_i log|det G_ii| of any factor G."""
    T = products(g, Ah, G)
    N = 3 * g.n
    tr = float((T * G).sum())
    logdet = 0.0
    for i, row in enumerate(_lower_rows(g)):
        for (j, s) in row:
            if j == i:
                logdet += np.linalg.slogdet(G[s])[1]
    return np.log(tr / N) - (2.0 / N) * logdet


def backward(g: Graph, x, y, p, dH, cache):
    """Gradients of sum(dH * H) w.r.t. every parameter (dict), in float64,
    with the forward's rounding points held fixed."""
    W = cache["W"]
    deg = np.diff(g.offsets).astype(np.float64)
    is_diag = cache["is_diag"]
    grads = {k: np.zeros_like(v) for k, v in p.items()}
    dout = head_output_grad(dH, is_diag, cache["Al"], cache["rho"])
    el = cache["e"][g.lower]
    grads["W_off"] = el.T @ dout
    grads["b_off"] = dout.sum(axis=0)
    de = np.zeros((len(g.cols), WIDTH))
    de[g.lower] = dout @ W["W_off"].T
    dh = np.zeros((g.n, WIDTH))
    for l in reversed(range(LAYERS)):
        h, e, m, a, u = cache["tape"][l]
        # h_out = h + u ; e_out = e + m
        du = dh * (u > 0)
        Xn = np.concatenate([h, a], axis=1)
        grads[f"W2_{l}"] = Xn.T @ du
        grads[f"b2_{l}"] = du.sum(axis=0)
        dXn = du @ W[f"W2_{l}"].T
        dh_in = dh + dXn[:, :WIDTH]
        da = dXn[:, WIDTH:]
        dm = de + (da / deg[:, None])[g.rows]
        dmp = dm * (m > 0)
        X = np.concatenate([h[g.rows], h[g.cols], e], axis=1)
        grads[f"W1_{l}"] = X.T @ dmp
        grads[f"b1_{l}"] = dmp.sum(axis=0)
        dX = dmp @ W[f"W1_{l}"].T
        np.add.at(dh_in, g.rows, dX[:, :WIDTH])
        np.add.at(dh_in, g.cols, dX[:, WIDTH:2 * WIDTH])
        de = de + dX[:, 2 * WIDTH:]
        dh = dh_in
    h0 = bf16(relu(x @ W["W_hin"] + W["b_hin"]))
    e0 = bf16(relu(y @ W["W_ein"] + W["b_ein"]))
    dh0 = dh * (h0 > 0)
    de0 = de * (e0 > 0)
    grads["W_hin"] = x.T @ dh0
    grads["b_hin"] = dh0.sum(axis=0)
    grads["W_ein"] = y.T @ de0
    grads["b_ein"] = de0.sum(axis=0)
    return grads


def apply_preconditioner(g: Graph, G, s, r):
    """z = S G^T G S r for r (n, 3)."""
    t = s * r
    y = np.zeros_like(t)
    for k, e in enumerate(g.lower):
        i, j = int(g.rows[e]), int(g.cols[e])
        y[i] += G[k] @ t[j]
    z = np.zeros_like(t)
    for k, e in enumerate(g.lower):
        i, j = int(g.rows[e]), int(g.cols[e])
        z[j] += G[k].T @ y[i]
    return s * z
