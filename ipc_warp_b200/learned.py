"""Learned preconditioner for the Newton PCG solve: a message-passing net
over the 3x3-block graph of the Newton matrix predicts a factorised sparse
approximate inverse (FSAI) ``M^-1 = S G^T G S`` on the lower block pattern
(include/ipcb.h, ipc_warp_b200/csrc/mpnn.cu).

The reference solves the Newton system with cg or cuDSS LDLT
(time_integrator_base.py:470-507); this preconditioner replaces the
identity/diagonal one inside PCG, and the direct solve stays the fallback and
judge (``newton.FEMContactSolver``).  Training is unsupervised: the Kaporin
condition number of ``G A G^T`` (exactly computable on the pattern of G) is
minimised with Adam, on Newton systems the simulator itself produces; the
forward and backward passes run in the package's tcgen05 kernels.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N
from .bsr import BsrMatrix

WIDTH, IN_DIM, LAYERS = 64, 16, 4


def _param_sizes():
    """(name, shape) in the master-vector order of the kernels."""
    out = [("W_hin", (IN_DIM, WIDTH)), ("b_hin", (WIDTH,)), ("W_ein", (IN_DIM, WIDTH)), ("b_ein", (WIDTH,))]
    for l in range(LAYERS):
        out += [(f"W1_{l}", (3 * WIDTH, WIDTH)), (f"b1_{l}", (WIDTH,)), (f"W2_{l}", (2 * WIDTH, WIDTH)),
                (f"b2_{l}", (WIDTH,))]
    out += [("W_off", (WIDTH, 9)), ("b_off", (9,))]
    return out


PARAMS = _param_sizes()
PARAM_COUNT = sum(int(np.prod(s)) for _, s in PARAMS)


def flatten(params: dict) -> np.ndarray:
    return np.concatenate([np.asarray(params[k], np.float64).reshape(-1) for k, _ in PARAMS]).astype(np.float32)


def unflatten(vec) -> dict:
    vec = np.asarray(vec)
    out, o = {}, 0
    for k, s in PARAMS:
        n = int(np.prod(s))
        out[k] = vec[o:o + n].reshape(s)
        o += n
    return out


def init_params(seed: int = 0) -> np.ndarray:
    """He-initialised trunk, zero output heads (the net starts as first-order
    FSAI, G^_ij = -A^_ij)."""
    rng = np.random.default_rng(seed)
    p = {}
    for k, s in PARAMS:
        if k.startswith("b") or k == "W_off":
            p[k] = np.zeros(s)
        else:
            p[k] = rng.normal(scale=math.sqrt(2.0 / s[0]), size=s)
    return flatten(p)


class Pool:
    """Device buffers reused by name across factor builds, so that a build in
    the Newton loop allocates nothing once the sizes have been seen (a new
    allocation can synchronise the device) and the PCG's captured graph keeps
    its pointers.  A buffer handed out again invalidates its previous user."""

    def __init__(self):
        self._bufs = {}

    def get(self, name: str, shape, dtype, device) -> torch.Tensor:
        shape = tuple(int(v) for v in shape)
        t = self._bufs.get(name)
        if t is None or t.dtype != dtype or t.device != torch.device(device) or t.numel() < math.prod(shape):
            t = torch.empty(max(math.prod(shape), 1), dtype=dtype, device=device)
            self._bufs[name] = t
        return t[:math.prod(shape)].view(shape)


def _alloc(pool: Pool | None, name: str, shape, dtype, device) -> torch.Tensor:
    if pool is None:
        return torch.empty(shape, dtype=dtype, device=device)
    return pool.get(name, shape, dtype, device)


class Graph:
    """rows / rev / diag / lower of a canonical BSR pattern (device)."""

    def __init__(self, A: BsrMatrix, nnz: int | None = None, pool: Pool | None = None):
        self.n = A.nrow
        self.nnz = A.nnz_sync() if nnz is None else int(nnz)
        if (self.nnz + self.n) % 2:
            raise ValueError("pattern is not structurally symmetric")
        self.n_lower = (self.nnz + self.n) // 2
        dev = A.device
        self.offsets = A.offsets
        self.columns = A.columns
        self.rows = _alloc(pool, "g.rows", (self.nnz,), torch.int32, dev)
        self.rev = _alloc(pool, "g.rev", (self.nnz,), torch.int32, dev)
        self.diag = _alloc(pool, "g.diag", (self.n,), torch.int32, dev)
        self.lower = _alloc(pool, "g.lower", (self.n_lower,), torch.int32, dev)
        i32 = dict(dtype=torch.int32, device=dev)
        self.c = N.Graph(self.n, self.nnz, self.n_lower, N.ptr(self.offsets), N.ptr(self.columns), N.ptr(self.rows),
                         N.ptr(self.rev), N.ptr(self.diag), N.ptr(self.lower))
        status = torch.zeros(1, **i32)
        ws = _alloc(pool, "g.ws", (N.size("ipcb_mpnn_graph_workspace", self.n),), torch.uint8, dev)
        N.call("ipcb_mpnn_graph", ctypes.byref(self.c), N.ptr(status), N.ptr(ws), ws.numel(), N.stream_handle())
        if int(status.item()) & 16:
            raise ValueError("pattern is not symmetric or lacks a diagonal block")


class Net:
    """FP32 master parameters and their BF16 operand copies."""

    def __init__(self, params: np.ndarray | None = None, device="cuda", seed: int = 0):
        assert N.lib().ipcb_mpnn_param_count() == PARAM_COUNT
        vec = init_params(seed) if params is None else np.asarray(params, np.float32)
        self.device = torch.device(device)
        self.params = torch.tensor(vec, dtype=torch.float32, device=self.device)
        self.packed = torch.empty(N.lib().ipcb_mpnn_packed_count(), dtype=torch.bfloat16, device=self.device)
        self.pack()

    def pack(self):
        N.call("ipcb_mpnn_pack", N.ptr(self.params), N.ptr(self.packed), N.stream_handle())

    def save(self, path: str):
        np.save(path, self.params.cpu().numpy())

    @staticmethod
    def load(path: str, device="cuda") -> "Net":
        return Net(np.load(path), device=device)


@dataclass
class System:
    """One Newton matrix prepared for the net."""
    A: BsrMatrix
    graph: Graph
    scale: torch.Tensor  # float32 (n, 3)
    ahat: torch.Tensor   # float32 (nnz, 9)
    x: torch.Tensor      # bf16 (n, 16)
    y: torch.Tensor      # bf16 (nnz, 16)

    @staticmethod
    def from_bsr(A: BsrMatrix, graph: Graph | None = None, pool: Pool | None = None,
                 status: torch.Tensor | None = None) -> "System":
        """With ``status`` given, the feature status is ORed into it and not
        read here (the caller reads it once)."""
        g = graph if graph is not None else Graph(A, pool=pool)
        dev = A.device
        scale = _alloc(pool, "s.scale", (g.n, 3), torch.float32, dev)
        ahat = _alloc(pool, "s.ahat", (g.nnz, 9), torch.float32, dev)
        x = _alloc(pool, "s.x", (g.n, IN_DIM), torch.bfloat16, dev)
        y = _alloc(pool, "s.y", (g.nnz, IN_DIM), torch.bfloat16, dev)
        st = torch.zeros(1, dtype=torch.int32, device=dev) if status is None else status
        N.call("ipcb_mpnn_features", ctypes.byref(g.c), int(A.dtype == torch.float64), N.ptr(A.values), N.ptr(scale),
               N.ptr(ahat), N.ptr(x), N.ptr(y), N.ptr(st), N.stream_handle())
        if status is None and int(st.item()) & 16:
            raise ValueError("non-positive diagonal entry")
        return System(A, g, scale, ahat, x, y)


class _Tape:
    def __init__(self, g: Graph, training: bool, dev, pool: Pool | None = None):
        bf = torch.bfloat16
        nh = LAYERS + 1 if training else 2
        self.h = _alloc(pool, "t.h", (nh, g.n, WIDTH), bf, dev)
        self.e = _alloc(pool, "t.e", (nh, g.nnz, WIDTH), bf, dev)
        self.m = _alloc(pool, "t.m", (LAYERS if training else 1, g.nnz, WIDTH), bf, dev)
        self.a = _alloc(pool, "t.a", (LAYERS if training else 1, g.n, WIDTH), bf, dev)
        self.u = _alloc(pool, "t.u", (LAYERS, g.n, WIDTH), bf, dev) if training else None
        self.proj = _alloc(pool, "t.proj", (g.n, 2 * WIDTH), torch.float32, dev)
        opt = lambda t: N.ptr(t) if t is not None else None
        self.c = N.Tape(N.ptr(self.h), N.ptr(self.e), N.ptr(self.m), N.ptr(self.a), opt(self.u), N.ptr(self.proj),
                        int(training))


def forward(net: Net, sysm: System, training: bool = False, pool: Pool | None = None,
            status: torch.Tensor | None = None):
    """Row directions H (float32 (nnz, 3, 3), valid on the lower blocks) and
    the tape.  With ``status`` given, the kernel status is ORed into it and
    not read here."""
    g = sysm.graph
    dev = sysm.A.device
    tape = _Tape(g, training, dev, pool)
    H = _alloc(pool, "H", (g.nnz, 3, 3), torch.float32, dev).zero_()
    st = torch.zeros(1, dtype=torch.int32, device=dev) if status is None else status
    N.call("ipcb_mpnn_forward", ctypes.byref(g.c), N.ptr(net.packed), N.ptr(net.params), N.ptr(sysm.ahat),
           N.ptr(sysm.x), N.ptr(sysm.y), ctypes.byref(tape.c), N.ptr(H), N.ptr(st), N.stream_handle())
    if status is None and int(st.item()):
        raise RuntimeError(f"mpnn forward status {int(st.item())}")
    return H, tape


@dataclass
class Normalized:
    G: torch.Tensor     # float32 (nnz, 3, 3): the factor on the lower blocks
    T: torch.Tensor     # float32 (nnz, 9): T_ij = sum_k H_ik A^_kj
    minv: torch.Tensor  # float32 (n, 9): M_i^-1
    loss: float         # (1/N) sum_i log det M_i
    status: int


def normalize(sysm: System, H: torch.Tensor, pool: Pool | None = None,
              status: torch.Tensor | None = None) -> Normalized:
    """Exact row normalisation G^_i = chol(M_i)^-1 H_i and the FSAI loss.
    With ``status`` given, nothing is read back (loss and status are left
    on the device: ``loss`` is then NaN)."""
    g = sysm.graph
    dev = H.device
    G = _alloc(pool, "G", tuple(H.shape), torch.float32, dev).zero_()
    T = _alloc(pool, "T", (g.nnz, 9), torch.float32, dev)
    minv = _alloc(pool, "minv", (g.n, 9), torch.float32, dev)
    acc = torch.zeros(1, dtype=torch.float64, device=dev)
    st = torch.zeros(1, dtype=torch.int32, device=dev) if status is None else status
    N.call("ipcb_fsai_normalize", ctypes.byref(g.c), N.ptr(sysm.ahat), N.ptr(H), N.ptr(T), N.ptr(minv), N.ptr(G),
           N.ptr(acc), N.ptr(st), N.stream_handle())
    if status is not None:
        return Normalized(G, T, minv, float("nan"), 0)
    return Normalized(G, T, minv, float(acc.item()) / (3 * g.n), int(st.item()))


def loss_grad(sysm: System, nz: Normalized, weight: float = 1.0) -> torch.Tensor:
    """Gradient of weight x loss w.r.t. the head outputs (bf16 (L, 64))."""
    g = sysm.graph
    dG = torch.empty((g.n_lower, 64), dtype=torch.bfloat16, device=nz.G.device)
    N.call("ipcb_mpnn_loss_grad", ctypes.byref(g.c), N.ptr(sysm.ahat), N.ptr(sysm.x), N.ptr(nz.T), N.ptr(nz.minv),
           N.ptr(dG), float(weight), N.stream_handle())
    return dG


def backward(net: Net, sysm: System, tape: _Tape, dG: torch.Tensor, grad: torch.Tensor):
    """Parameter gradients of sum(dG * head outputs), added to grad."""
    g = sysm.graph
    dev = dG.device
    ws = torch.empty(N.size("ipcb_mpnn_backward_workspace", g.n, g.nnz, g.n_lower), dtype=torch.uint8, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    N.call("ipcb_mpnn_backward", ctypes.byref(g.c), N.ptr(net.packed), N.ptr(net.params), N.ptr(sysm.x),
           N.ptr(sysm.y), ctypes.byref(tape.c), N.ptr(dG), N.ptr(grad), N.ptr(status), N.ptr(ws), ws.numel(),
           N.stream_handle())
    if int(status.item()):
        raise RuntimeError(f"mpnn backward status {int(status.item())}")


class Trainer:
    """Adam on the Kaporin loss over a list of systems.  The gradient is
    clipped to norm ``clip`` and a step whose loss or gradient is not finite
    is skipped: one very stiff system in a batch can otherwise throw the
    parameters far enough that the net collapses to the diagonal."""

    def __init__(self, net: Net, lr: float = 1e-3, betas=(0.9, 0.999), eps: float = 1e-8, clip: float = 1.0):
        self.net = net
        self.lr, self.betas, self.eps = lr, betas, eps
        self.clip = float(clip)
        self.skipped = 0
        z = lambda: torch.zeros_like(net.params)
        self.m, self.v, self.grad = z(), z(), z()
        self.t = 0

    def step(self, batch: list[System]) -> float:
        self.grad.zero_()
        total = 0.0
        for sysm in batch:
            H, tape = forward(self.net, sysm, training=True)
            nz = normalize(sysm, H)
            dG = loss_grad(sysm, nz, weight=1.0 / len(batch))
            backward(self.net, sysm, tape, dG, self.grad)
            total += nz.loss / len(batch)
        gn = float(self.grad.norm())
        if not (math.isfinite(gn) and math.isfinite(total)):
            self.skipped += 1
            return total
        if self.clip > 0 and gn > self.clip:
            self.grad.mul_(self.clip / gn)
        self.t += 1
        N.call("ipcb_adam", self.net.params.numel(), N.ptr(self.net.params), N.ptr(self.grad), N.ptr(self.m),
               N.ptr(self.v), float(self.lr), float(self.betas[0]), float(self.betas[1]), float(self.eps), self.t,
               N.stream_handle())
        self.net.pack()
        return total


class LearnedFactor:
    """The FSAI factor of one Newton matrix in the form DevicePcg applies
    (bf16 blocks, upper slots mirrored)."""
    kind = 1

    def __init__(self, net: Net, A: BsrMatrix, pool: Pool | None = None):
        """``pool``: buffers shared with earlier factors (which this build
        invalidates); the build then allocates nothing once sizes repeat and
        reads the device twice (the matrix size and one status word)."""
        # own copy of the pattern: the factor may outlive this matrix (reuse
        # across Newton iterations), whose buffers a later assembly overwrites
        nnz = A.nnz_sync()
        dev = A.device
        B = BsrMatrix.__new__(BsrMatrix)
        B.nrow, B.ncol, B.dtype, B.device = A.nrow, A.ncol, A.dtype, dev
        B.offsets = _alloc(pool, "B.offsets", (A.nrow + 1,), torch.int32, dev)
        B.columns = _alloc(pool, "B.columns", (max(nnz, 1),), torch.int32, dev)
        B.values = _alloc(pool, "B.values", (max(nnz, 1), 3, 3), A.dtype, dev)
        B.nnz_dev = _alloc(pool, "B.nnz", (1,), torch.int32, dev)
        B.offsets.copy_(A.offsets)
        B.columns[:nnz].copy_(A.columns[:nnz])
        B.values[:nnz].copy_(A.values[:nnz])
        B.nnz_dev.copy_(A.nnz_dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.sysm = System.from_bsr(B, Graph(B, nnz=nnz, pool=pool), pool=pool, status=status)
        H, _ = forward(net, self.sysm, pool=pool, status=status)
        self.G = normalize(self.sysm, H, pool=pool, status=status).G
        self.gh = _alloc(pool, "gh", (self.sysm.graph.nnz, 9), torch.bfloat16, dev)
        N.call("ipcb_fsai_mirror", ctypes.byref(self.sysm.graph.c), N.ptr(self.G), N.ptr(self.gh),
               N.stream_handle())
        st = int(status.item())
        if st & 16:
            raise ValueError("non-positive diagonal entry in the Newton matrix")
        if st:
            raise RuntimeError(f"learned factor status {st:#x}")

    def fill(self, P):
        g = self.sysm.graph
        P.g_offsets, P.g_columns = N.ptr(g.offsets), N.ptr(g.columns)
        P.diag = N.ptr(g.diag)
        P.g = N.ptr(self.gh)
        P.scale = N.ptr(self.sysm.scale)


class LearnedPreconditioner:
    """z = S G^T G S r for the PCG of newton.py: ``LearnedPreconditioner(net)``
    is a factory (called with the Newton matrix) like ``BlockJacobi``."""

    def __init__(self, net: Net):
        self.net = net

    def __call__(self, A: BsrMatrix) -> "_Apply":
        sysm = System.from_bsr(A)
        H, _ = forward(self.net, sysm)
        return _Apply(sysm, normalize(sysm, H).G, A.dtype)


class _Apply:
    def __init__(self, sysm: System, G: torch.Tensor, dtype):
        self.sysm, self.G, self.dtype = sysm, G, dtype
        self.tmp = torch.empty((sysm.graph.n, 3), dtype=dtype, device=G.device)

    def __call__(self, r: torch.Tensor) -> torch.Tensor:
        z = torch.empty_like(r)
        N.call("ipcb_fsai_apply", ctypes.byref(self.sysm.graph.c), N.ptr(self.G), N.ptr(self.sysm.scale),
               int(self.dtype == torch.float64), N.ptr(r), N.ptr(self.tmp), N.ptr(z), N.stream_handle())
        return z


DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "mpnn_fsai.npy")
