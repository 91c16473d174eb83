"""Pins the CPU oracle (oracle/) before anything is checked against it.

* against the golden vectors of the reference's own tests (tests/golden/reference_tests.json,
  regenerated from ssdf's sources by tests/golden/make_golden.py);
* against the reference's own edf / edf_celllist outputs on seeded workload samples
  (tests/golden/*_sample.npz), bitwise;
* against the reference compiled from its sources (oracle/_ref) on fresh random inputs, when
  that build is present;
* against the analytic signed distance of the voxel staircase (the sign fixture of ssdf's
  tests/sample_sdf_bvh_test.cpp), restated.
"""

import ctypes
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN, golden_mesh, load_golden_json
from ssdf_b200 import workloads as W


def test_golden_single_triangle_float():
    g = load_golden_json()["ssdf_test"]
    mesh = golden_mesh(g, np.float32)
    pts = np.array([g["x"], g["y"], g["z"]], dtype=np.float32)
    out = oracle.edf(pts, mesh, out=np.full(5, g["out_init"], np.float32), dtype=np.float32)
    assert np.array_equal(out, np.array(g["edf_select"], np.float32))
    assert np.all(np.abs(out - np.array(g["brute"], np.float32)) < g["tolerance"])


def test_golden_brute_force_double():
    g = load_golden_json()["ssdf_brute_force"]
    mesh = golden_mesh(g)
    pts = np.array([g["x"], g["y"], g["z"]])
    out = oracle.edf(pts, mesh, out=np.full(20, g["out_init"]))
    for key in ("edf", "edf_select", "brute"):
        assert np.array_equal(out, np.array(g[key])), key


def test_golden_point_aabb():
    g = load_golden_json()["point_aabb"]
    box = g["box"]
    for x, y, z, e, r in zip(g["x"], g["y"], g["z"], g["expected"], g["reference"]):
        v = oracle.lib().oracle_point_aabb_distance_squared_d(x, y, z, *box)
        assert v == r and abs(v - e) <= g["tolerance"]


def test_golden_box_sdf():
    g = load_golden_json()["box_sdf"]
    box = g["box"]
    for x, y, z, e, r in zip(g["x"], g["y"], g["z"], g["expected"], g["reference"]):
        v = oracle.lib().oracle_point_aabb_signed_distance_d(x, y, z, *box)
        assert v == r and abs(v - e) <= g["tolerance"]


@pytest.mark.parametrize("name", ["icosphere", "torus_knot", "beam_lattice"])
def test_workload_samples_bitwise(name):
    mesh = {"icosphere": W.icosphere, "torus_knot": W.torus_knot_tube, "beam_lattice": W.beam_lattice}[name]()
    z = np.load(os.path.join(GOLDEN, f"{name}_sample.npz"))
    for key in z.files:
        if key in ("ids", "points"):
            continue
        dt = np.float64 if key.endswith("_d") else np.float32
        got = oracle.edf(z["points"].astype(dt), mesh, dtype=dt)
        assert np.array_equal(got, z[key]), key


def test_sample_points_are_the_grid_nodes():
    z = np.load(os.path.join(GOLDEN, "icosphere_sample.npz"))
    mesh = W.icosphere()
    q = oracle.grid_points(W.Grid.cell_centred(mesh, 64, 0.2))
    assert np.array_equal(q[:, z["ids"]], z["points"])


needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference CPU library not built here")


@needs_ref
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_against_reference_random(dtype):
    rng = np.random.default_rng(42)
    mesh = W.random_soup(300, seed=3)
    pts = rng.uniform(-1.5, 1.5, size=(3, 500))
    init = np.where(rng.uniform(size=500) < 0.2, 0.05, np.finfo(dtype).max).astype(dtype)
    mine = oracle.edf(pts.astype(dtype), mesh, out=init, dtype=dtype)
    for which in ("edf", "celllist", "select"):
        ref = oracle.ref_edf(pts.astype(dtype), mesh, out=init, dtype=dtype, which=which)
        assert np.array_equal(mine, ref), which


def same(a, b):
    return a == b or (np.isnan(a) and np.isnan(b))


@needs_ref
def test_point_triangle_kernels_against_reference():
    rng = np.random.default_rng(7)
    lib, ref = oracle.lib(), oracle.ref()
    import ctypes as C

    for k in range(4000):
        v = rng.uniform(-1, 1, size=12)
        if k % 4 == 1:  # degenerate: collinear / coincident vertices
            v[6:9] = v[3:6] if k % 8 == 1 else 0.5 * (v[3:6] + v[6:9] * 0 + v[3:6])
        if k % 4 == 2:  # point on a vertex / edge
            v[0:3] = v[3:6] if k % 8 == 2 else 0.5 * (v[3:6] + v[6:9])
        args = [float(a) for a in v]
        # degenerate triangles can give NaN (0/0 in the face region) in both: compare NaN-aware
        assert same(lib.oracle_point_triangle_dist_sq_d(*args), ref.ref_point_triangle_dist_sq_d(*args))
        f = [float(np.float32(a)) for a in v]
        assert same(lib.oracle_point_triangle_dist_sq_f(*f), ref.ref_point_triangle_dist_sq_f(*f))
        a = [C.c_double() for _ in range(3)]
        b = [C.c_double() for _ in range(3)]
        lib.oracle_point_triangle_closest_point_d(*args, *[C.byref(t) for t in a])
        ref.ref_point_triangle_closest_point_d(*args, *[C.byref(t) for t in b])
        assert all(same(x.value, y.value) for x, y in zip(a, b))


def test_tie_rule_lowest_index():
    base = W.random_soup(4, seed=1)
    v = base.vertices
    t = np.concatenate([base.triangles, base.triangles[[2, 0]]])  # triangles 4, 5 duplicate 2, 0
    mesh = W.Mesh(v, t.astype(np.int32))
    pts = np.random.default_rng(2).uniform(-1, 1, size=(3, 200))
    _, tri = oracle.edf(pts, mesh, with_index=True)
    assert not np.any(tri >= 4)


def test_staircase_sign_and_distance():
    """The sign KAT of ssdf's tests/sample_sdf_bvh_test.cpp:92-132, on the oracle."""
    mesh, lo, hi, filled = W.voxel_staircase()
    n = 5 * 6 + 1
    grid = W.Grid((n, n, n), (-0.25,) * 3, (1.25,) * 3)
    q = oracle.grid_points(grid, dtype=np.float32)
    sd, _ = oracle.sdf_points(q, mesh)
    p = q.T
    d2 = np.full(p.shape[0], np.inf)
    for a, b in zip(lo, hi):
        c = np.clip(p, a, b)
        d2 = np.minimum(d2, ((p - c) ** 2).sum(1))
    d = np.sqrt(d2)
    cell = np.floor(p / 0.25).astype(int)
    inside = np.array([filled(*c) for c in cell])
    keep = d >= 1e-6
    assert np.sum((sd[keep] < 0) != inside[keep]) == 0
    assert np.max(np.abs(np.abs(sd[keep]) - d[keep])) < 1e-5


def test_sign_of_closed_surfaces():
    for mesh in (W.icosphere(), W.torus(nu=48, nv=24)):
        lo, hi = mesh.bbox()
        pts = W.uniform_points(3000, lo - 0.3, hi + 0.3, seed=9)
        sd, _ = oracle.sdf_points(pts, mesh)
        # winding-number inside test (solid angle sum) as an independent check
        v = mesh.vertices[mesh.triangles]
        p = pts.T[:, None, None, :]
        r = v[None] - p
        ln = np.linalg.norm(r, axis=-1)
        num = np.einsum("ijk,ijk->ij", r[:, :, 0], np.cross(r[:, :, 1], r[:, :, 2]))
        den = (ln[:, :, 0] * ln[:, :, 1] * ln[:, :, 2] + np.einsum("ijk,ijk->ij", r[:, :, 0], r[:, :, 1]) * ln[:, :, 2]
               + np.einsum("ijk,ijk->ij", r[:, :, 1], r[:, :, 2]) * ln[:, :, 0]
               + np.einsum("ijk,ijk->ij", r[:, :, 2], r[:, :, 0]) * ln[:, :, 1])
        wind = 2 * np.arctan2(num, den).sum(1) / (4 * np.pi)
        inside = wind > 0.5
        far = np.abs(sd) > 1e-3
        assert np.sum((sd[far] < 0) != inside[far]) == 0


def test_pseudonormals_manifold_edges():
    mesh = W.icosphere(2)
    fn, en, vn = oracle.pseudonormals(mesh)
    fn = fn.reshape(-1, 3)
    en = en.reshape(-1, 3, 3)
    assert np.allclose(np.linalg.norm(fn, axis=1), 1.0)
    # every edge of a closed manifold: sum of its two faces' normals, identical from both sides
    t = mesh.triangles
    for f in range(0, len(t), 7):
        for e in range(3):
            a, b = t[f, e], t[f, (e + 1) % 3]
            g = np.where(((t == b) | (t == a)).sum(1) == 2)[0]
            g = g[g != f][0]
            assert np.allclose(en[f, e], fn[f] + fn[g], atol=0, rtol=0) or np.array_equal(en[f, e], fn[g] + fn[f])
    assert np.all(np.linalg.norm(vn.reshape(-1, 3), axis=1) > 0)


def _box_points(n, seed, dtype):
    """Points inside, outside, on faces and on edges of a box spanning [-1, 2] x [0, 3] x [-2, 1]."""
    rng = np.random.default_rng(seed)
    p = rng.uniform(-3.0, 4.0, size=(3, n))
    p[:, : n // 4] = np.round(p[:, : n // 4])  # exact face / edge / corner coordinates
    return p.astype(dtype)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_box_helpers_golden_and_reference(dtype):
    g = load_golden_json()["box_sdf"]
    pts = np.array([g["x"], g["y"], g["z"]], dtype=np.float64)
    if dtype == np.float64:
        assert np.array_equal(oracle.all_points_aabb_signed_distance(pts, g["box"]), np.array(g["reference"]))
    if not oracle.ref_available():
        pytest.skip("the reference was not compiled here")
    p = _box_points(4099, 7, dtype)
    b = oracle.compute_aabb(p, dtype)
    assert np.array_equal(b, oracle.compute_aabb(p, dtype, reference=True))
    assert np.array_equal(b, np.array([p[0].min(), p[0].max(), p[1].min(), p[1].max(), p[2].min(), p[2].max()]))
    box = np.array([-1, 2, 0, 3, -2, 1], dtype=dtype)
    d = oracle.all_points_aabb_signed_distance(p, box, dtype)
    assert np.array_equal(d, oracle.all_points_aabb_signed_distance(p, box, dtype, reference=True))


# ---- closest primitive within a radius (serial/bvh/bvh.cpp:367-832) ----------------------------

def test_golden_quad_closest_point():
    g = load_golden_json()["quad_closest"]
    rows = np.array(g["rows"]).reshape(-1, 15)
    for k, name in enumerate(g["names"]):
        s, t = oracle.quad_closest_st(rows[k, :3], rows[k, 3:])
        assert (s, t) == tuple(g["reference"][2 * k: 2 * k + 2]), name
        assert abs(s - g["expected"][2 * k]) < g["tolerance"] and abs(t - g["expected"][2 * k + 1]) < g["tolerance"]
    tri = g["triangle"]
    assert oracle.triangle_barycentric(tri[:3], tri[3:]) == tuple(g["triangle_reference"])


def _random_quads(rng, n, dtype):
    base = rng.uniform(-1, 1, size=(n, 1, 3))
    quads = base + rng.uniform(-0.5, 0.5, size=(n, 4, 3))
    quads[: n // 8, 3] = quads[: n // 8, 2]  # a repeated corner
    quads[n // 8: n // 4] = quads[n // 8: n // 4, :1] + np.linspace(0, 1, 4)[None, :, None] * rng.normal(size=(n // 8, 1, 3))
    quads[n // 4: n // 3, :, 2] = 0.25  # planar
    return quads.astype(dtype)


@needs_ref
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_quad_and_barycentric_against_reference(dtype):
    """The restated primitives equal the reference's own templates bit for bit on random, planar,
    collinear and repeated-corner inputs."""
    rng = np.random.default_rng(17)
    quads = _random_quads(rng, 800, dtype)
    pts = rng.uniform(-2, 2, size=(800, 3)).astype(dtype)
    for p, q in zip(pts, quads):
        assert oracle.quad_closest_st(p, q, dtype) == oracle.quad_closest_st(p, q, dtype, reference=True)
        tri = q[:3]
        a, b = oracle.triangle_barycentric(p, tri, dtype), oracle.triangle_barycentric(p, tri, dtype, reference=True)
        assert a == b or all((x == y) or (np.isnan(x) and np.isnan(y)) for x, y in zip(a, b))


def _brute_within(points, quads_or_tris, verts, r2, skip_self):
    """Independent float restatement of the per-point loop, on top of the pinned primitives."""
    n = points.shape[1]
    out = []
    for pid in range(n):
        q = points[:, pid].astype(np.float32)
        best, bt = np.float32(r2[pid]), -1
        for e, idx in enumerate(quads_or_tris):
            if skip_self and pid in idx:
                continue
            c = verts[:, idx].T.astype(np.float32)
            if len(idx) == 4:
                s, t = oracle.quad_closest_st(q, c, np.float32)
                s, t = np.float32(s), np.float32(t)
                w = [(1 - s) * (1 - t), s * (1 - t), s * t, (1 - s) * t]
                cp = ((c[0] * w[0] + c[1] * w[1]) + c[2] * w[2]) + c[3] * w[3]
            else:
                o = [ctypes.c_float() for _ in range(3)]
                oracle.lib().oracle_point_triangle_closest_point_f(*q, *c.reshape(9), *[ctypes.byref(v) for v in o])
                cp = np.array([v.value for v in o], np.float32)
            d = q - cp
            d2 = np.float32(np.float32(d[0] * d[0] + d[1] * d[1]) + d[2] * d[2])
            if d2 != np.inf and (d2 < best or (d2 == best and bt < 0)):
                best, bt = d2, e
        out.append((bt, best))
    return out


@pytest.mark.parametrize("quads", [False, True])
def test_within_radius_oracle_semantics(quads):
    rng = np.random.default_rng(3 + quads)
    verts = rng.uniform(0, 1, size=(3, 40))
    k = 4 if quads else 3
    elems = [rng.choice(40, size=k, replace=False) for _ in range(30)]
    pts = verts[:, :25] + rng.normal(0, 0.05, size=(3, 25))
    pts[:, 20:] = verts[:, 20:25]  # on corners: skip_self matters
    r2 = np.where(np.arange(25) % 3 == 0, 1e-4, 0.05)
    r2[5] = np.inf
    r2[6] = -1.0
    for skip in (False, True):
        got = oracle.within_radius(pts.astype(np.float32), [np.array([e[j] for e in elems]) for j in range(k)],
                                   verts.astype(np.float32), r2.astype(np.float32), skip_self=skip,
                                   gdtype=np.float32)
        want = _brute_within(pts, elems, verts, r2.astype(np.float32), skip)
        assert [int(t) for t in got[0]] == [w[0] for w in want]
        assert np.array_equal(got[1], np.array([w[1] for w in want], np.float32))
        none = got[0] < 0
        assert np.all(got[2][none] == 0) and np.all(got[3][none] == 0) and np.all(got[4][none] == 0)
        assert got[1][6] == -1.0 and got[0][6] == -1
    # stride 0: one radius for every point; the local variant carries the same index and distance
    a = oracle.within_radius(pts, [np.array([e[j] for e in elems]) for j in range(k)], verts, np.array([0.01]),
                             stride=0)
    b = oracle.within_radius(pts, [np.array([e[j] for e in elems]) for j in range(k)], verts, np.array([0.01]),
                             stride=0, local=True)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    if quads:
        assert np.all((b[2] >= 0) & (b[2] <= 1) & (b[3] >= 0) & (b[3] <= 1))


# The reference's own known answers for the candidate contact pairs
# (tests/potential_contact_triangles_bvh_test.cpp:14-78, tests/potential_contact_quads_bvh_test.cpp:21-60).
PC_TRIANGLES = dict(x=[0, 1, 0, .2, .8, .2, -.5, 3, 4, 3], y=[0, 0, 1, .2, .2, .8, 1.5, 0, 0, 1],
                    z=[0, 0, 0, .1, .1, .1, 0, 0, 0, 0], e=[[0, 3, 0, 7], [1, 5, 2, 8], [2, 4, 6, 9]],
                    ptr=[0, 1, 2, 2, 2], contacts=[(0, 1), (1, 0)])
PC_QUADS = dict(x=[0, 1, 1, 0, 0, 1, 1, 0, 3, 4, 4, 3, 3, 4, 4, 3, 8, 9, 9, 8],
                y=[0, 0, 1, 1, 0, 0, 1, 1, 0, 0, 1, 1, 0, 0, 1, 1, 0, 0, 1, 1],
                z=[0, 0, 0, 0, .2, .2, .2, .2, 0, 0, .5, 0, .6, .6, 1.1, .6, 0, 0, 0, 0],
                e=[[0, 4, 8, 12, 16], [1, 7, 9, 15, 17], [2, 6, 10, 14, 18], [3, 5, 11, 13, 19]],
                ptr=[0, 1, 2, 3, 4, 4], contacts=[(0, 1), (1, 0), (2, 3), (3, 2)])


@pytest.mark.parametrize("case", [PC_TRIANGLES, PC_QUADS])
def test_potential_contact_known_answers(case):
    for dt in (np.float32, np.float64):
        ptr, idx = oracle.potential_contact(case["e"], (case["x"], case["y"], case["z"]), 0.3, dt)
        assert list(ptr) == case["ptr"]
        for e, c in case["contacts"]:
            assert c in idx[ptr[e]:ptr[e + 1]]
