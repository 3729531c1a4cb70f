"""Synthetic scenes for the contact pipeline (host-side numpy, not timed).

The reference loads its meshes from `.tobj`/`.obj` files through libigl
(fem/geometry.py:165-276); the scenes the benchmarks name are not shipped with
it, so they are generated here from seeded parameters.  The output follows the
reference `Soup` layout (fem/geometry.py:165-171):

* ``x``          float[V,3]  world positions (``soup.x_transformed``)
* ``xcs``        float[V,3]  rest positions
* ``edges``      int32[2E]   flat surface edges (igl.edges of the surface faces)
* ``triangles``  int32[3T]   flat outward-oriented surface triangles
* ``body``       int32[V]    body index per vertex
* ``tets``       int32[n_tets,4]

Hex cells are split into 5 tetrahedra with the split mirrored on alternating
cells so that neighbouring cells share face diagonals.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# Corner (dx, dy, dz) bits of a hex cell.
_CORNERS = np.array([[i & 1, (i >> 1) & 1, (i >> 2) & 1] for i in range(8)], dtype=np.int64)


def _corner_id(bits):
    return bits[0] | (bits[1] << 1) | (bits[2] << 2)


def _five_tet_split(parity: int):
    """Return the 5 tets (as corner ids) of a hex cell.

    parity 0: centre tet on the even corners {000,110,101,011};
    parity 1: centre tet on the odd corners {100,010,001,111}.
    Each remaining tet joins one corner of the other class with its 3
    axis neighbours.
    """
    even = [0b000, 0b011, 0b101, 0b110]
    odd = [0b001, 0b010, 0b100, 0b111]
    centre, tips = (even, odd) if parity == 0 else (odd, even)
    tets = [list(centre)]
    for t in tips:
        nb = [t ^ 1, t ^ 2, t ^ 4]
        tets.append([t] + nb)
    return tets


@dataclass
class Mesh:
    x: np.ndarray
    tets: np.ndarray
    triangles: np.ndarray  # [T,3]
    edges: np.ndarray      # [E,2]


def hex_grid_tets(nx: int, ny: int, nz: int, size=(1.0, 1.0, 1.0)) -> Mesh:
    """Tetrahedralised box with (nx,ny,nz) cells spanning [0,size]."""
    sx, sy, sz = size
    gx, gy, gz = np.meshgrid(
        np.linspace(0.0, sx, nx + 1), np.linspace(0.0, sy, ny + 1), np.linspace(0.0, sz, nz + 1),
        indexing="ij",
    )
    x = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1)

    def vid(i, j, k):
        return (i * (ny + 1) + j) * (nz + 1) + k

    tets = []
    splits = [_five_tet_split(0), _five_tet_split(1)]
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                cid = [vid(i + b[0], j + b[1], k + b[2]) for b in _CORNERS]
                for t in splits[(i + j + k) & 1]:
                    tets.append([cid[c] for c in t])
    tets = np.asarray(tets, dtype=np.int64)
    # orient every tet positively
    a, b, c, d = (x[tets[:, q]] for q in range(4))
    vol = np.einsum("ij,ij->i", np.cross(b - a, c - a), d - a)
    flip = vol < 0
    tets[flip, 1], tets[flip, 2] = tets[flip, 2].copy(), tets[flip, 1].copy()
    tris = boundary_faces(tets)
    edges = surface_edges(tris)
    return Mesh(x=x, tets=tets, triangles=tris, edges=edges)


def boundary_faces(tets: np.ndarray) -> np.ndarray:
    """Faces used by exactly one tet, oriented with outward normals
    (positive tets: face opposite vertex q is wound away from it)."""
    # faces of a positively oriented tet (a,b,c,d), outward
    local = np.array([[1, 2, 3], [0, 3, 2], [0, 1, 3], [0, 2, 1]])
    faces = tets[:, local].reshape(-1, 3)
    key = np.sort(faces, axis=1)
    _, inv, cnt = np.unique(key, axis=0, return_inverse=True, return_counts=True)
    return faces[cnt[inv.ravel()] == 1].astype(np.int64)


def surface_edges(tris: np.ndarray) -> np.ndarray:
    e = np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [2, 0]]])
    e = np.sort(e, axis=1)
    return np.unique(e, axis=0).astype(np.int64)


def rot_z(deg: float) -> np.ndarray:
    t = np.deg2rad(deg)
    c, s = np.cos(t), np.sin(t)
    return np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])


@dataclass
class Scene:
    name: str
    x: np.ndarray
    xcs: np.ndarray
    edges: np.ndarray
    triangles: np.ndarray
    body: np.ndarray
    tets: np.ndarray
    dhat: float
    kappa: float
    meta: dict = field(default_factory=dict)

    @property
    def n_verts(self):
        return self.x.shape[0]

    @property
    def n_edges(self):
        return self.edges.shape[0] // 2

    @property
    def n_tris(self):
        return self.triangles.shape[0] // 3

    @property
    def thickness(self):
        """The reference's ``_thickness``: dhat = l0 = 2 * _thickness (contact.py:180)."""
        return 0.5 * self.dhat


def assemble(meshes, name, dhat, kappa, meta=None) -> Scene:
    xs, es, ts, bs, tets = [], [], [], [], []
    off = 0
    for b, m in enumerate(meshes):
        xs.append(m.x)
        es.append(m.edges + off)
        ts.append(m.triangles + off)
        tets.append(m.tets + off)
        bs.append(np.full(m.x.shape[0], b, dtype=np.int32))
        off += m.x.shape[0]
    x = np.concatenate(xs)
    return Scene(
        name=name,
        x=x.copy(),
        xcs=x.copy(),
        edges=np.concatenate(es).astype(np.int32).ravel(),
        triangles=np.concatenate(ts).astype(np.int32).ravel(),
        body=np.concatenate(bs).astype(np.int32),
        tets=np.concatenate(tets).astype(np.int32),
        dhat=float(dhat),
        kappa=float(kappa),
        meta=meta or {},
    )


def two_cubes(n: int = 8, gap: float = 1e-3, angle_deg: float = 15.0, jitter: float = 1e-5,
              seed: int = 0, dhat: float = 1e-3, kappa: float = 1e4, tilt_deg: float = 0.0) -> Scene:
    """Two tetrahedralised unit cubes; the upper one is rotated about z (then
    tilted about x by ``tilt_deg``) and its lowest vertex sits ``gap`` above
    the lower cube's top face (y-up)."""
    rng = np.random.default_rng(seed)
    lo = hex_grid_tets(n, n, n)
    up = hex_grid_tets(n, n, n)
    c = np.array([0.5, 0.5, 0.5])
    t = np.radians(tilt_deg)
    rot_x = np.array([[1.0, 0.0, 0.0], [0.0, np.cos(t), -np.sin(t)], [0.0, np.sin(t), np.cos(t)]])
    up.x = (up.x - c) @ (rot_x @ rot_z(angle_deg)).T + c
    up.x[:, 1] += 1.0 + gap - up.x[:, 1].min()
    sc = assemble([lo, up], f"two_cubes_{n}", dhat, kappa, {"gap": gap, "angle_deg": angle_deg})
    sc.x += rng.uniform(-jitter, jitter, size=sc.x.shape)
    sc.xcs = sc.x.copy()
    return sc


def rod_bundle(n_rods_side: int = 4, cells=(4, 4, 256), width: float = 0.1, spacing: float = 1.2,
               gap_over_dhat: float | None = None, jitter_over_dhat: float = 0.05, seed: int = 1,
               dhat_over_width: float = 1e-3, kappa: float = 1e4) -> Scene:
    """``n_rods_side``^2 parallel square rods (cells[0] x cells[1] x cells[2] hex
    cells, 5 tets/cell) along z.  By default they sit at ``spacing`` x width
    centre distance, as in the rod-twist setup.  With ``gap_over_dhat`` the
    bundle is packed so that facing rod surfaces are ``gap_over_dhat * dhat``
    apart: the wound contact state of the twist, where every facing pair of
    rod sides is inside the barrier.  Alternate rods are shifted along the
    axis by 0.37 cells so grids are not aligned."""
    rng = np.random.default_rng(seed)
    cx, cy, cz = cells
    length = width * cz / cx
    dhat = dhat_over_width * width
    meshes = []
    pitch = spacing * width if gap_over_dhat is None else width + gap_over_dhat * dhat
    cell = width / cx
    for a in range(n_rods_side):
        for b in range(n_rods_side):
            m = hex_grid_tets(cx, cy, cz, size=(width, width, length))
            m.x = m.x + np.array([a * pitch, b * pitch, 0.37 * cell * ((a + b) & 1)])
            meshes.append(m)
    sc = assemble(meshes, f"rods_{n_rods_side}x{n_rods_side}_{cx}x{cy}x{cz}", dhat, kappa,
                  {"width": width, "pitch": pitch})
    sc.x += rng.uniform(-jitter_over_dhat * dhat, jitter_over_dhat * dhat, size=sc.x.shape)
    sc.xcs = sc.x.copy()
    return sc


def twist_bundle(sc: Scene, theta: float) -> np.ndarray:
    """Positions of a rod bundle (rods along z) whose cross-sections are turned
    rigidly about the bundle axis by theta * (2 (z - z0) / L - 1): a wound
    state of the rod twist in which facing rod sides keep their gap."""
    x = sc.xcs.copy()
    c = x[:, :2].mean(axis=0)
    z = x[:, 2]
    th = theta * (2.0 * (z - z.min()) / (z.max() - z.min()) - 1.0)
    d = x[:, :2] - c
    x[:, 0] = c[0] + np.cos(th) * d[:, 0] - np.sin(th) * d[:, 1]
    x[:, 1] = c[1] + np.sin(th) * d[:, 0] + np.cos(th) * d[:, 1]
    return x


def twist_targets(sc: Scene, omega: float):
    """Clamped ends of the rod twist: returns (fixed mask, targets(t)); the
    z-min end turns by +omega t and the z-max end by -omega t about the
    bundle axis."""
    x = sc.xcs
    c = x[:, :2].mean(axis=0)
    lo = x[:, 2] <= x[:, 2].min() + 1e-9
    hi = x[:, 2] >= x[:, 2].max() - 1e-9

    def at(t):
        tgt = x.copy()
        for mask, sgn in ((lo, 1.0), (hi, -1.0)):
            a = sgn * omega * t
            ca, sa = np.cos(a), np.sin(a)
            d = x[mask, :2] - c
            tgt[mask, 0] = c[0] + ca * d[:, 0] - sa * d[:, 1]
            tgt[mask, 1] = c[1] + sa * d[:, 0] + ca * d[:, 1]
        return tgt

    return lo | hi, at


# ------------------------------------------------------------ affine bodies
def icosphere(subdiv: int = 2, radius: float = 0.5):
    """Closed triangle sphere (outward faces): a regular icosahedron whose
    faces are split in four ``subdiv`` times, vertices pushed to the sphere.
    subdiv 4 gives 2562 vertices / 5120 triangles."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    verts = [np.asarray(p, np.float64) / np.linalg.norm(p) for p in v]
    faces = [tuple(x) for x in f]
    for _ in range(subdiv):
        mid = {}

        def midpoint(a, b):
            key = (min(a, b), max(a, b))
            if key not in mid:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                mid[key] = len(verts) - 1
            return mid[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return radius * np.array(verts), np.array(faces, dtype=np.int64)


def box_surface(n=(4, 4, 4), size=(1.0, 1.0, 1.0)):
    """Closed triangulated box surface (outward faces, surface vertices only),
    n cells per side, corner at the origin."""
    m = hex_grid_tets(*n, size=size)
    tris = m.triangles
    used = np.unique(tris)
    remap = np.full(m.x.shape[0], -1, np.int64)
    remap[used] = np.arange(len(used))
    return m.x[used].copy(), remap[tris]


def transform(rotation_deg=(0.0, 0.0, 0.0), position=(0.0, 0.0, 0.0)) -> np.ndarray:
    """4x4 rigid transform: rotations about x, then y, then z (degrees), then
    the translation."""
    rx, ry, rz = np.radians(rotation_deg)
    cx, sx, cy, sy, cz, sz = np.cos(rx), np.sin(rx), np.cos(ry), np.sin(ry), np.cos(rz), np.sin(rz)
    Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    T = np.eye(4)
    T[:3, :3] = Rz @ Ry @ Rx
    T[:3, 3] = position
    return T


def abd_balls(n_side: int = 2, layers: int = 1, subdiv: int = 2, radius: float = 0.5, gap: float = 2e-3,
              drop: float = 1e-3, seed: int = 0, ground_cells: int = 8) -> dict:
    """Affine-body scene: ``n_side`` x ``n_side`` x ``layers`` icospheres in a
    stacked grid (neighbours ``gap`` apart, randomly turned), the lowest
    layer ``drop`` above a fixed box slab.  Keyword arguments of
    :class:`AffineBodyDynamics` (meshes, transforms, fixed_bodies, gravity)."""
    rng = np.random.default_rng(seed)
    ball = icosphere(subdiv, radius)
    pitch = 2.0 * radius + gap
    meshes, transforms = [], []
    for k in range(layers):
        for i in range(n_side):
            for j in range(n_side):
                meshes.append(ball)
                pos = (i * pitch, radius + drop + k * pitch, j * pitch)
                transforms.append(transform(rng.uniform(0, 360, 3), pos))
    width = n_side * pitch + 2.0 * radius
    slab = box_surface((ground_cells, 1, ground_cells), (width, 0.2, width))
    meshes.append(slab)
    transforms.append(transform(position=(-1.5 * radius, -0.2, -1.5 * radius)))
    return dict(meshes=meshes, transforms=transforms, fixed_bodies=[len(meshes) - 1], gravity=(0.0, -9.8, 0.0))


# ------------------------------------------------------------ screw and nut
def iso_thread_radius(s, major: float, pitch: float):
    """Radius of a 60-degree ISO metric thread profile at thread phase s
    (turns; the profile repeats every unit of s): crest flat of pitch/8 at the
    major radius (centred on s = 0), flanks at 30 degrees from the radial
    direction over 5 pitch/16 each, root flat of pitch/4; depth 5/8 of the
    sharp-V height sqrt(3)/2 pitch."""
    u = np.mod(np.asarray(s, np.float64), 1.0)
    depth = 5.0 / 16.0 * np.sqrt(3.0) * pitch
    r = np.full(u.shape, major)
    down = (u >= 1 / 16) & (u < 6 / 16)
    r[down] = major - depth * (u[down] - 1 / 16) / (5 / 16)
    r[(u >= 6 / 16) & (u < 10 / 16)] = major - depth
    up = (u >= 10 / 16) & (u < 15 / 16)
    r[up] = major - depth * (15 / 16 - u[up]) / (5 / 16)
    return r


def helical_tube(n_rho: int, n_theta: int, per_pitch: int, turns: int, pitch: float, r_in, r_out,
                 theta0: float = 0.0) -> Mesh:
    """Tetrahedralised tube on a helical grid: vertex (i, j, k) at angle
    theta_j = theta0 + 2 pi j / n_theta, thread phase s_k = k / per_pitch,
    height z = pitch (s_k + theta_j / 2 pi) and radius interpolated between
    r_in(s) and r_out(s) by i / n_rho, so grid lines along k follow the
    helix and every profile corner at a multiple of 1/per_pitch is a grid
    line.  Around the axis, column n_theta - 1 joins column 0 one turn up
    (k + per_pitch); cells whose neighbour would lie past the last turn are
    left out (the ends are helical ramps).  Cells are split into 5 tets with
    the split alternating in (i + j + k), which matches across the seam when
    n_theta - per_pitch is even."""
    assert (n_theta - per_pitch) % 2 == 0, "the 5-tet split needs n_theta - per_pitch even"
    ns = per_pitch * turns
    k = np.arange(ns + 1)
    sk = k / per_pitch
    ri, ro = np.broadcast_to(r_in(sk), sk.shape), np.broadcast_to(r_out(sk), sk.shape)
    I, J, K = np.meshgrid(np.arange(n_rho + 1), np.arange(n_theta), k, indexing="ij")
    rad = ri[K] + (ro[K] - ri[K]) * (I / n_rho)
    th = theta0 + 2.0 * np.pi * J / n_theta
    z = pitch * (K / per_pitch + th / (2.0 * np.pi))
    x = np.stack([rad * np.cos(th), rad * np.sin(th), z], axis=-1).reshape(-1, 3)

    def vid(i, j, kk):
        return (i * n_theta + j) * (ns + 1) + kk

    ci, cj, ck = np.meshgrid(np.arange(n_rho), np.arange(n_theta), np.arange(ns), indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()
    corners = []
    keep = np.ones(ci.shape, bool)
    for b in _CORNERS:
        j = cj + b[1]
        kk = ck + b[2]
        wrap = j == n_theta
        j = np.where(wrap, 0, j)
        kk = np.where(wrap, kk + per_pitch, kk)
        keep &= kk <= ns
        corners.append(vid(ci + b[0], j, kk))
    corners = np.stack(corners, axis=1)[keep]
    parity = ((ci + cj + ck) & 1)[keep]
    tets = []
    for par in (0, 1):
        cs = corners[parity == par]
        for t in _five_tet_split(par):
            tets.append(cs[:, t])
    tets = np.concatenate(tets).astype(np.int64)
    a, b_, c, d = (x[tets[:, q]] for q in range(4))
    vol = np.einsum("ij,ij->i", np.cross(b_ - a, c - a), d - a)
    flip = vol < 0
    tets[flip, 1], tets[flip, 2] = tets[flip, 2].copy(), tets[flip, 1].copy()
    used = np.unique(tets)
    remap = np.full(x.shape[0], -1, np.int64)
    remap[used] = np.arange(used.size)
    x, tets = x[used], remap[tets]
    tris = boundary_faces_fast(tets)
    return Mesh(x=x, tets=tets, triangles=tris, edges=surface_edges_fast(tris))


def boundary_faces_fast(tets: np.ndarray) -> np.ndarray:
    """boundary_faces with a packed 63-bit key per face (vertex ids < 2^21)."""
    local = np.array([[1, 2, 3], [0, 3, 2], [0, 1, 3], [0, 2, 1]])
    faces = tets[:, local].reshape(-1, 3)
    assert faces.max() < (1 << 21)
    srt = np.sort(faces, axis=1).astype(np.int64)
    key = (srt[:, 0] << 42) | (srt[:, 1] << 21) | srt[:, 2]
    order = np.argsort(key, kind="stable")
    ks = key[order]
    first = np.r_[True, ks[1:] != ks[:-1]]
    start = np.flatnonzero(first)
    cnt = np.diff(np.r_[start, ks.size])
    single = order[start[cnt == 1]]
    return faces[np.sort(single)].astype(np.int64)


def surface_edges_fast(tris: np.ndarray) -> np.ndarray:
    e = np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [2, 0]]])
    e = np.sort(e, axis=1).astype(np.int64)
    key = np.unique((e[:, 0] << 21) | e[:, 1])
    return np.stack([key >> 21, key & ((1 << 21) - 1)], axis=1)


def screw_and_nut(n_theta: int = 640, per_pitch: int = 16, turns: int = 12, n_rho: int = 2, major: float = 1.0,
                  pitch: float = 0.1, hole: float = 0.5, nut_outer: float = 1.5, clearance: float = 1e-4,
                  dhat: float = 5e-5, load_gap_over_dhat: float = 0.4, kappa: float = 1e4,
                  seed: int = 4) -> Scene:
    """Bolt and nut of a 60-degree ISO thread (pitch 0.1 of the 1.0 major
    radius, 12 turns) on the same helical grid (``helical_tube``): the bolt a
    tube from radius ``hole`` to the thread profile, the nut a tube from the
    profile plus the radial clearance (1e-4 radius) to ``nut_outer``.  A
    radial clearance c leaves c sin(30 deg) = c/2 between facing flanks; the
    nut is then pushed along the axis onto one flank so that flank's gap is
    ``load_gap_over_dhat`` dhat (the loaded state of a nut driven onto the
    bolt), which puts the whole loaded flank inside the barrier.  The nut's
    grid is turned half a column about the axis so its edges cross the
    bolt's.  Defaults: 640 columns around, 16 rows a pitch, 2 cells through
    the wall: about 0.5M surface triangles and 1.23M tets per body.  Bolt
    (body 0) is the affine body and the nut (body 1) the FEM body of the
    screw-and-nut configuration."""
    rng = np.random.default_rng(seed)
    prof = lambda s: iso_thread_radius(s, major, pitch)  # noqa: E731
    bolt = helical_tube(n_rho, n_theta, per_pitch, turns, pitch, lambda s: np.full_like(s, hole), prof)
    half = np.pi / n_theta
    nut = helical_tube(n_rho, n_theta, per_pitch, turns, pitch, lambda s: prof(s) + clearance,
                       lambda s: np.full_like(s, nut_outer), theta0=half)
    # both flanks are c/2 from the bolt's; the axial push closes one of them
    flank_gap = 0.5 * clearance
    push = (flank_gap - load_gap_over_dhat * dhat) / np.cos(np.pi / 6)
    nut.x[:, 2] -= push
    sc = assemble([bolt, nut], f"screw_nut_{n_theta}x{per_pitch * turns}x{n_rho}", dhat, kappa,
                  {"pitch": pitch, "major": major, "clearance": clearance, "push": push, "n_theta": n_theta,
                   "per_pitch": per_pitch, "turns": turns})
    sc.x += rng.uniform(-1e-7, 1e-7, size=sc.x.shape)
    sc.xcs = sc.x.copy()
    return sc


def screw_direction(sc: Scene, omega: float = 4.0, dt: float = 2e-3, seed: int = 5) -> np.ndarray:
    """Newton direction of the driven nut (x1 = x - dx): one step of the
    nut turning at ``omega`` about the axis while held axially, so its
    loaded flank advances into the bolt's by pitch omega dt / 2 pi; small
    seeded noise on every vertex."""
    rng = np.random.default_rng(seed)
    x = sc.x
    nut = sc.body == 1
    a = omega * dt
    c, s_ = np.cos(a), np.sin(a)
    x1 = x.copy()
    x1[nut, 0] = c * x[nut, 0] - s_ * x[nut, 1]
    x1[nut, 1] = s_ * x[nut, 0] + c * x[nut, 1]
    dx = x - x1
    dx += rng.normal(scale=0.05 * sc.dhat, size=dx.shape)
    return dx


# --------------------------------------------- mixed affine + FEM wrecking balls
@dataclass
class MixedScene:
    """Deformable tet bodies and affine bodies in one scene.

    ``fem``: the tet bodies as a :class:`Scene` (vertices, tets, surface, body
    ids).  ``bodies``: per affine body its world vertices (n, 3) and
    outward faces (m, 3); ``fixed_bodies`` never move (the ground).
    ``pins``: body -> (world point on the body at rest, world target,
    stiffness), a pendulum rod as a quadratic penalty.  ``velocities``:
    body -> (linear, angular) initial velocity."""
    name: str
    fem: Scene
    bodies: list
    fixed_bodies: list
    pins: dict
    velocities: dict
    dhat: float
    kappa: float
    meta: dict = field(default_factory=dict)


def ground_grid(quads: int, extent: float, origin=(0.0, 0.0, 0.0)):
    """A flat square of quads x quads quads (2 triangles each) spanning
    [0, extent]^2 in x-z at height origin[1], faces pointing up (+y)."""
    n = quads + 1
    g = np.linspace(0.0, extent, n)
    X, Z = np.meshgrid(g, g, indexing="ij")
    v = np.column_stack([X.ravel(), np.zeros(n * n), Z.ravel()]) + np.asarray(origin, np.float64)
    i, j = np.meshgrid(np.arange(quads), np.arange(quads), indexing="ij")
    a = (i * n + j).ravel()
    b, c, d = a + n, a + n + 1, a + 1
    # (a, d, c) and (a, c, b): counter-clockwise seen from +y
    f = np.concatenate([np.column_stack([a, d, c]), np.column_stack([a, c, b])])
    return v, f.astype(np.int64)


def wrecking_balls(n_balls: int = 64, subdiv: int = 4, radius: float = 0.5, rope: float = 1.0,
                   max_angle_deg: float = 60.0, stack=(2, 2, 2), cube_cells: int = 4, cube_size: float = 0.25,
                   ground_quads: int = 100, station: float = 3.0, dhat: float = 1e-3, kappa: float = 1e12,
                   pin_stiffness: float = 1e9, seed: int = 0) -> MixedScene:
    """Batched affine + FEM wrecking balls: ``n_balls`` affine icospheres
    (subdiv 4: 2562 vertices, 5120 triangles; radius 0.5) on pendulum pins,
    each released from rest at a seeded angle uniform in [0, max_angle_deg]
    towards a stack of FEM cubes (``stack`` cubes of cube_cells^3 hex cells,
    5 tets/cell; 64 balls x 2x2x2 = 512 cubes) that rests on a fixed ground
    of ground_quads^2 quads.  Each ball has its own station on a square
    grid ``station`` apart; at the bottom of its swing the ball's centre is
    ``radius + 0.05`` above the ground and 0.01 in front of its stack.
    Neighbouring cubes and the lowest layer and the ground start 1.5 dhat
    apart, inside the barrier."""
    rng = np.random.default_rng(seed)
    side = int(np.ceil(np.sqrt(n_balls)))
    gap = 1.5 * dhat
    ball_v, ball_f = icosphere(subdiv, radius)
    cubes, bodies, pins, velocities = [], [], {}, {}
    sx, sy, sz = stack
    pitch = cube_size + gap
    for k in range(n_balls):
        cx, cz = (k // side) * station + 0.5 * station, (k % side) * station + 0.5 * station
        low = radius + 0.05
        pivot = np.array([cx, low + rope, cz])
        th = np.radians(rng.uniform(0.0, max_angle_deg))
        centre = pivot + rope * np.array([-np.sin(th), -np.cos(th), 0.0])
        R = transform(rng.uniform(0, 360, 3))[:3, :3]
        bodies.append((ball_v @ R.T + centre, ball_f.copy()))
        pins[k] = (pivot.copy(), pivot.copy(), float(pin_stiffness))
        x0 = cx + radius + 0.01
        for a in range(sx):
            for b in range(sy):
                for c in range(sz):
                    m = hex_grid_tets(cube_cells, cube_cells, cube_cells, size=(cube_size,) * 3)
                    m.x = m.x + np.array([x0 + a * pitch, gap + b * pitch, cz - 0.5 * sz * pitch + c * pitch])
                    cubes.append(m)
    extent = side * station
    bodies.append(ground_grid(ground_quads, extent))
    fem = assemble(cubes, "wrecking_cubes", dhat, kappa)
    return MixedScene(name=f"wrecking_balls_{n_balls}", fem=fem, bodies=bodies, fixed_bodies=[len(bodies) - 1],
                      pins=pins, velocities=velocities, dhat=float(dhat), kappa=float(kappa),
                      meta={"radius": radius, "rope": rope, "cube_size": cube_size, "stack": tuple(stack),
                            "ground_quads": ground_quads})


def mixed_touching(subdiv: int = 1, radius: float = 0.5, cube_cells: int = 2, cube_size: float = 1.0,
                   dhat: float = 1e-3, gap_over_dhat: float = 0.6, kappa: float = 1e8, ground_quads: int = 4,
                   pin_stiffness: float = 1e6) -> MixedScene:
    """A small mixed scene with every kind of body pair inside the barrier:
    two affine balls side by side, a FEM cube beside the first, all resting
    on a fixed ground, every facing gap ``gap_over_dhat`` dhat (measured
    between the meshes' extreme vertices).  Ball 0 hangs on a pin at its
    top.  Body pairs: ball-ball, ball-cube, ball-ground, cube-ground."""
    g = gap_over_dhat * dhat
    v, f = icosphere(subdiv, radius)
    lo = v.min(axis=0)
    hi = v.max(axis=0)
    a = v - np.array([0.0, lo[1] - g, 0.0])                 # resting g above y = 0
    b = a + np.array([hi[0] - lo[0] + g, 0.0, 0.0])          # g to the right of ball 0
    cube = hex_grid_tets(cube_cells, cube_cells, cube_cells, size=(cube_size,) * 3)
    cube.x = cube.x + np.array([a[:, 0].min() - g - cube_size, g, -0.5 * cube_size])
    span = 4.0 * (radius + cube_size)
    ground = ground_grid(ground_quads, span, origin=(-0.5 * span, 0.0, -0.5 * span))
    fem = assemble([cube], "touching_cube", dhat, kappa)
    top = a.mean(axis=0) + np.array([0.0, radius, 0.0])
    return MixedScene(name="mixed_touching", fem=fem, bodies=[(a, f.copy()), (b, f.copy()), ground],
                      fixed_bodies=[2], pins={0: (top, top.copy(), float(pin_stiffness))}, velocities={},
                      dhat=float(dhat), kappa=float(kappa), meta={})
