"""Seeded synthetic meshes and query sets for the distance-field workloads.

No public dataset is involved: every mesh and query set is generated here from a seed. All meshes
are indexed triangle lists in ssdf's layout -- SoA vertex coordinates ``sx, sy, sz`` and int32
vertex indices ``s0, s1, s2`` per triangle -- with right-handed (outward) orientation where the
surface is closed.

Workloads (sizes as used by the benchmark and the tests):

* ``icosphere``: unit icosahedron subdivided 4x (2,562 vertices / 5,120 triangles), each vertex
  moved along its normal by ``0.02 * U(-1, 1)``; queried on a cell-centred 64^3 grid over its
  bounding box padded by 0.2.
* ``torus_knot_tube``: a tube of radius 0.15 swept along a (2,3) torus knot (major radius 1,
  minor 0.4), 1,024 path samples x 64 around = 131,072 triangles, closed, coordinates jittered by
  ``N(0, 1e-4)``; queried on a 256^3 node grid over its bounding box padded by 0.25.
* ``beam_lattice``: 20,000 rectangular beams of 12 triangles (240,000 triangles), centres
  ``U[0,1]^3``, axes uniform on the sphere, lengths ``U(0.1, 0.4)``, square sections
  ``U(0.005, 0.02)``; queried at 8M uniform points in ``[-0.1, 1.1]^3`` plus a 512^3 grid.
* ``voxel_staircase``: the watertight, non-convex lattice-cell surface whose faces lie on grid
  planes, the sign fixture of ssdf's tests/sample_sdf_bvh_test.cpp:19-97 (restated here).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Mesh:
    """Indexed triangle surface: vertices (nv, 3) float64, triangles (nt, 3) int32."""

    vertices: np.ndarray
    triangles: np.ndarray

    @property
    def nv(self) -> int:
        return int(self.vertices.shape[0])

    @property
    def nt(self) -> int:
        return int(self.triangles.shape[0])

    def coords(self, dtype=np.float64):
        v = self.vertices.astype(dtype, copy=False)
        return tuple(np.ascontiguousarray(v[:, d]) for d in range(3))

    def indices(self):
        t = self.triangles.astype(np.int32, copy=False)
        return tuple(np.ascontiguousarray(t[:, d]) for d in range(3))

    def bbox(self):
        return self.vertices.min(axis=0), self.vertices.max(axis=0)

    def diagonal(self) -> float:
        lo, hi = self.bbox()
        return float(np.linalg.norm(hi - lo))

    def signed_volume(self) -> float:
        v = self.vertices[self.triangles]
        return float(np.einsum("ij,ij->i", v[:, 0], np.cross(v[:, 1], v[:, 2])).sum() / 6.0)


@dataclass
class Grid:
    """ssdf's node grid: n = (nx, ny, nz) nodes from lo to hi inclusive, x fastest."""

    n: tuple
    lo: tuple
    hi: tuple

    @property
    def size(self) -> int:
        return int(self.n[0]) * int(self.n[1]) * int(self.n[2])

    @staticmethod
    def padded_nodes(mesh: Mesh, n: int, pad: float) -> "Grid":
        lo, hi = mesh.bbox()
        return Grid((n, n, n), tuple(float(v) for v in lo - pad), tuple(float(v) for v in hi + pad))

    @staticmethod
    def cell_centred(mesh: Mesh, n: int, pad: float) -> "Grid":
        """n^3 cell centres of the padded box, as ssdf's node grid over [min + h/2, max - h/2]."""
        lo, hi = mesh.bbox()
        lo, hi = lo - pad, hi + pad
        h = (hi - lo) / n
        return Grid((n, n, n), tuple(float(v) for v in lo + h / 2), tuple(float(v) for v in hi - h / 2))


# ----------------------------------------------------------------------------------------------
# Meshes
# ----------------------------------------------------------------------------------------------

def _icosahedron():
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t],
                  [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4],
                  [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
                  [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    return v / np.linalg.norm(v, axis=1, keepdims=True), f


def _subdivide(v, f):
    edges = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
    key = np.sort(edges, axis=1)
    uniq, inv = np.unique(key[:, 0] * (len(v) + 1) + key[:, 1], return_inverse=True)
    a, b = uniq // (len(v) + 1), uniq % (len(v) + 1)
    mid = (v[a] + v[b]) / 2.0
    mid /= np.linalg.norm(mid, axis=1, keepdims=True)
    nf = len(f)
    m = inv.reshape(3, nf) + len(v)
    ab, bc, ca = m[0], m[1], m[2]
    f0, f1, f2 = f[:, 0], f[:, 1], f[:, 2]
    nfaces = np.concatenate([np.stack([f0, ab, ca], 1), np.stack([f1, bc, ab], 1), np.stack([f2, ca, bc], 1),
                             np.stack([ab, bc, ca], 1)])
    return np.concatenate([v, mid]), nfaces


def icosphere(subdivisions: int = 4, radius: float = 1.0, displacement: float = 0.02, seed: int = 1,
              center=(0.0, 0.0, 0.0)) -> Mesh:
    v, f = _icosahedron()
    for _ in range(subdivisions):
        v, f = _subdivide(v, f)
    rng = np.random.default_rng(seed)
    r = radius * (1.0 + displacement * rng.uniform(-1.0, 1.0, size=len(v)))
    v = v * r[:, None] + np.asarray(center, dtype=np.float64)
    return Mesh(v, f.astype(np.int32))


def torus_knot_tube(p: int = 2, q: int = 3, major: float = 1.0, minor: float = 0.4, tube: float = 0.15,
                    nu: int = 1024, nv: int = 64, jitter: float = 1e-4, seed: int = 2) -> Mesh:
    """Closed tube around a (p, q) torus knot, Frenet frame (periodic: the knot's curvature never vanishes)."""
    t = np.arange(nu) * (2.0 * np.pi / nu)

    def curve(s):
        rr = major + minor * np.cos(q * s)
        return np.stack([rr * np.cos(p * s), rr * np.sin(p * s), minor * np.sin(q * s)], axis=1)

    eps = 1e-4
    c = curve(t)
    d1 = (curve(t + eps) - curve(t - eps)) / (2 * eps)
    d2 = (curve(t + eps) - 2 * c + curve(t - eps)) / (eps * eps)
    T = d1 / np.linalg.norm(d1, axis=1, keepdims=True)
    B = np.cross(d1, d2)
    B /= np.linalg.norm(B, axis=1, keepdims=True)
    N = np.cross(B, T)
    th = np.arange(nv) * (2.0 * np.pi / nv)
    ring = np.cos(th)[None, :, None] * N[:, None, :] + np.sin(th)[None, :, None] * B[:, None, :]
    verts = (c[:, None, :] + tube * ring).reshape(-1, 3)
    rng = np.random.default_rng(seed)
    verts = verts + rng.normal(0.0, jitter, size=verts.shape)
    i = np.arange(nu)[:, None]
    j = np.arange(nv)[None, :]
    a = i * nv + j
    b = i * nv + (j + 1) % nv
    c1 = ((i + 1) % nu) * nv + j
    d = ((i + 1) % nu) * nv + (j + 1) % nv
    tri = np.concatenate([np.stack([a, b, c1], -1).reshape(-1, 3), np.stack([b, d, c1], -1).reshape(-1, 3)])
    m = Mesh(verts, tri.astype(np.int32))
    if m.signed_volume() < 0:
        m = Mesh(verts, tri[:, [0, 2, 1]].astype(np.int32))
    return m


def _box_triangles():
    # corners indexed by bits (x, y, z); two outward triangles per face
    return np.array([[0, 2, 3], [0, 3, 1],  # -x
                     [4, 5, 7], [4, 7, 6],  # +x
                     [0, 1, 5], [0, 5, 4],  # -y
                     [2, 6, 7], [2, 7, 3],  # +y
                     [0, 4, 6], [0, 6, 2],  # -z
                     [1, 3, 7], [1, 7, 5]], dtype=np.int64)  # +z


def beam_lattice(nbeams: int = 20000, seed: int = 3) -> Mesh:
    """Union of rectangular beams (12 triangles each), overlapping, not watertight as a whole."""
    rng = np.random.default_rng(seed)
    centre = rng.uniform(0.0, 1.0, size=(nbeams, 3))
    axis = rng.normal(size=(nbeams, 3))
    axis /= np.linalg.norm(axis, axis=1, keepdims=True)
    length = rng.uniform(0.1, 0.4, size=nbeams)
    side = rng.uniform(0.005, 0.02, size=nbeams)
    helper = np.where(np.abs(axis[:, :1]) < 0.9, np.array([[1.0, 0, 0]]), np.array([[0, 1.0, 0]]))
    u = np.cross(axis, helper)
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    w = np.cross(axis, u)
    bits = np.array([[(k >> 2) & 1, (k >> 1) & 1, k & 1] for k in range(8)], dtype=np.float64) - 0.5
    # local frame (u, w, axis) is right-handed, so the canonical box's outward faces stay outward
    verts = (centre[:, None, :] + bits[None, :, 0:1] * side[:, None, None] * u[:, None, :]
             + bits[None, :, 1:2] * side[:, None, None] * w[:, None, :]
             + bits[None, :, 2:3] * length[:, None, None] * axis[:, None, :]).reshape(-1, 3)
    tri = (_box_triangles()[None, :, :] + 8 * np.arange(nbeams)[:, None, None]).reshape(-1, 3)
    if Mesh(verts[:8], tri[:12]).signed_volume() < 0:  # keep every beam outward-oriented
        tri = tri[:, [0, 2, 1]]
    return Mesh(verts, tri.astype(np.int32))


def torus(major: float = 1.0, minor: float = 0.3, nu: int = 64, nv: int = 32, jitter: float = 0.0,
          seed: int = 4, center=(0.0, 0.0, 0.0)) -> Mesh:
    u = np.arange(nu) * (2 * np.pi / nu)
    v = np.arange(nv) * (2 * np.pi / nv)
    uu, vv = np.meshgrid(u, v, indexing="ij")
    rr = major + minor * np.cos(vv)
    verts = np.stack([rr * np.cos(uu), rr * np.sin(uu), minor * np.sin(vv)], -1).reshape(-1, 3)
    rng = np.random.default_rng(seed)
    verts = verts + jitter * minor * rng.uniform(-1.0, 1.0, size=verts.shape) + np.asarray(center)
    i = np.arange(nu)[:, None]
    j = np.arange(nv)[None, :]
    a = i * nv + j
    b = ((i + 1) % nu) * nv + j
    c = i * nv + (j + 1) % nv
    d = ((i + 1) % nu) * nv + (j + 1) % nv
    tri = np.concatenate([np.stack([a, b, d], -1).reshape(-1, 3), np.stack([a, d, c], -1).reshape(-1, 3)])
    m = Mesh(verts, tri.astype(np.int32))
    if m.signed_volume() < 0:
        m = Mesh(verts, tri[:, [0, 2, 1]].astype(np.int32))
    return m


def voxel_staircase(ncell: int = 4, h: float = 0.25):
    """Boundary faces of the lattice cells (i <= j, 1 <= k <= 2) of an ncell^3 lattice, two outward
    triangles per face (ssdf tests/sample_sdf_bvh_test.cpp:19-90, restated). Returns the mesh, the
    axis-aligned face rectangles (lo, hi) for the exact distance and the filled() predicate."""

    def filled(i, j, k):
        if i < 0 or j < 0 or k < 0 or i >= ncell or j >= ncell or k >= ncell:
            return False
        return i <= j and 1 <= k <= 2

    m = ncell + 1
    vid = lambda i, j, k: i + m * (j + m * k)  # noqa: E731
    verts = np.array([[i * h, j * h, k * h] for k in range(m) for j in range(m) for i in range(m)])
    tris, rects = [], []
    for k in range(ncell):
        for j in range(ncell):
            for i in range(ncell):
                if not filled(i, j, k):
                    continue
                for axis in range(3):
                    for sign in (-1, 1):
                        nb = [i, j, k]
                        nb[axis] += sign
                        if filled(*nb):
                            continue
                        u, v = (axis + 1) % 3, (axis + 2) % 3
                        c = [[i, j, k] for _ in range(4)]
                        for qq in range(4):
                            c[qq][axis] += 1 if sign > 0 else 0
                        c[1][u] += 1
                        c[2][u] += 1
                        c[2][v] += 1
                        c[3][v] += 1
                        order = [0, 1, 2, 3] if sign > 0 else [0, 3, 2, 1]
                        a, b, d, e = (vid(*c[o]) for o in order)
                        tris += [[a, b, d], [a, d, e]]
                        lo = [min(c[0][dd], c[2][dd]) * h for dd in range(3)]
                        hi = [max(c[0][dd], c[2][dd]) * h for dd in range(3)]
                        rects.append((lo, hi))
    mesh = Mesh(verts.astype(np.float64), np.array(tris, dtype=np.int32))
    return mesh, np.array([r[0] for r in rects]), np.array([r[1] for r in rects]), filled


def random_soup(ntri: int, seed: int = 0, scale: float = 1.0) -> Mesh:
    """Disjoint random triangles with coordinates U(-scale, scale)."""
    rng = np.random.default_rng(seed)
    v = rng.uniform(-scale, scale, size=(3 * ntri, 3))
    return Mesh(v, np.arange(3 * ntri, dtype=np.int32).reshape(-1, 3))


def uniform_points(n: int, lo, hi, seed: int = 5) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, size=(n, 3)).T.copy()


def multi_mesh_set(count: int = 256, tri_lo: float = 1e3, tri_hi: float = 2e5, side_lo: float = 32,
                   side_hi: float = 160, seed: int = 7):
    """Uneven batch: seeded icospheres / tori, triangle count and grid side log-uniform."""
    rng = np.random.default_rng(seed)
    out = []
    for m in range(count):
        target = float(np.exp(rng.uniform(np.log(tri_lo), np.log(tri_hi))))
        side = int(round(np.exp(rng.uniform(np.log(side_lo), np.log(side_hi)))))
        centre = rng.uniform(-2.0, 2.0, size=3)
        if rng.uniform() < 0.5:
            sub = int(np.clip(np.floor(np.log(target / 20.0) / np.log(4.0)), 2, 6))  # 320 .. 81,920
            mesh = icosphere(sub, radius=float(rng.uniform(0.3, 1.0)), displacement=0.01,
                             seed=int(rng.integers(1 << 30)), center=centre)
        else:
            nu = max(8, int(round(np.sqrt(target / 2.0 * 4.0))))
            nv = max(4, int(round(target / 2.0 / nu)))
            mesh = torus(major=float(rng.uniform(0.5, 1.0)), minor=float(rng.uniform(0.1, 0.3)), nu=nu, nv=nv,
                         jitter=0.01, seed=int(rng.integers(1 << 30)), center=centre)
        out.append((mesh, Grid.padded_nodes(mesh, side, 0.1 * mesh.diagonal())))
    return out
