"""GPU parity of the closest-primitive-within-a-radius queries (closest_within_radius_bvh,
_local_bvh, _quads_bvh, _quads_local_bvh) against the oracle's brute force: primitive index,
squared distance and closest point or local coordinates bit for bit, for the three (G, T) type
pairs, per-point and shared radii, self-contact skipping, point sets large enough to be visited in
Morton order, empty inputs, and radii that are negative, zero, NaN or infinite."""

import numpy as np
import pytest

import oracle
import ssdf_b200 as S
from ssdf_b200 import workloads as W
from test_gpu_golden import env

pytestmark = pytest.mark.gpu

TYPES = [(np.float32, np.float32), (np.float32, np.float64), (np.float64, np.float64)]


def quad_surface(nu=48, nv=24, seed=0):
    """A warped torus of nu x nv quads, jittered, with a few degenerate and concave quads."""
    rng = np.random.default_rng(seed)
    u, v = np.meshgrid(np.linspace(0, 2 * np.pi, nu, endpoint=False), np.linspace(0, 2 * np.pi, nv, endpoint=False),
                       indexing="ij")
    r = 0.3 + 0.05 * np.sin(3 * u)
    p = np.stack([(1 + r * np.cos(v)) * np.cos(u), (1 + r * np.cos(v)) * np.sin(u), r * np.sin(v)], 0)
    p = p.reshape(3, -1) + rng.normal(0, 0.004, size=(3, nu * nv))
    i, j = np.meshgrid(np.arange(nu), np.arange(nv), indexing="ij")
    vid = lambda a, b: (a % nu) * nv + (b % nv)  # noqa: E731
    q = [vid(i, j).ravel(), vid(i + 1, j).ravel(), vid(i + 1, j + 1).ravel(), vid(i, j + 1).ravel()]
    q = [a.astype(np.int32) for a in q]
    q[3][::97] = q[2][::97]  # a repeated corner: a triangle
    q[2][5::89] = q[0][5::89]  # a folded quad
    return q, p


def near_points(verts, n, spread, seed):
    rng = np.random.default_rng(seed)
    verts = np.asarray(verts)
    base = verts[:, rng.integers(0, verts.shape[1], n)]
    return base + rng.normal(0, spread, size=(3, n))


def check(got, want, name):
    assert np.array_equal(got[0], want[0]), name + ": primitive"
    for k in range(1, len(want)):
        assert np.array_equal(got[k], want[k], equal_nan=True), f"{name}: output {k}"


@pytest.mark.parametrize("gdt,tdt", TYPES)
@pytest.mark.parametrize("local", [False, True])
def test_triangles(gdt, tdt, local):
    mesh = W.torus_knot_tube(nu=192, nv=24)
    verts, elems = mesh.coords(), mesh.indices()
    pts = near_points(verts, 3000, 0.02, seed=1)
    rng = np.random.default_rng(2)
    r2 = rng.uniform(0, 0.03, 3000) ** 2
    r2[::11] = np.inf
    r2[1::53] = -1.0
    r2[2::59] = 0.0
    r2[3::61] = np.nan
    args = (pts.astype(gdt), elems, tuple(a.astype(gdt) for a in verts), r2.astype(tdt))
    got = S.closest_within_radius(*args, local=local, gdtype=gdt, tdtype=tdt)
    want = oracle.within_radius(*args, local=local, gdtype=gdt, tdtype=tdt)
    check(got, want, f"{gdt.__name__}/{tdt.__name__} local={local}")
    assert (got[0] >= 0).sum() > 1000


@pytest.mark.parametrize("gdt,tdt", TYPES)
@pytest.mark.parametrize("local", [False, True])
def test_quads(gdt, tdt, local):
    q, verts = quad_surface()
    pts = near_points(verts, 3000, 0.03, seed=3)
    r2 = np.full(3000, 0.04 ** 2)
    r2[::7] = np.inf
    args = (pts.astype(gdt), q, tuple(a.astype(gdt) for a in verts), r2.astype(tdt))
    got = S.closest_within_radius(*args, local=local, gdtype=gdt, tdtype=tdt)
    want = oracle.within_radius(*args, local=local, gdtype=gdt, tdtype=tdt)
    check(got, want, f"quads {gdt.__name__}/{tdt.__name__} local={local}")
    assert (got[0] >= 0).sum() > 1000


@pytest.mark.parametrize("quads", [False, True])
def test_self_contact_and_shared_radius(quads):
    """Points are the mesh's own vertices (node-to-surface contact): skip_self drops the primitives
    around each point; one radius for all (stride 0)."""
    if quads:
        elems, verts = quad_surface(32, 16, seed=5)
    else:
        mesh = W.torus(nu=64, nv=32, jitter=0.01)
        elems, verts = mesh.indices(), mesh.coords()
    for skip in (False, True):
        for local in (False, True):
            args = (verts, elems, verts, np.array([0.05 ** 2]))
            got = S.closest_within_radius(*args, stride=0, skip_self=skip, local=local)
            want = oracle.within_radius(*args, stride=0, skip_self=skip, local=local)
            check(got, want, f"skip={skip} local={local}")
            if not skip:
                assert np.all(got[1] == 0)  # every vertex lies on its own primitives


@pytest.mark.parametrize("quads", [False, True])
def test_morton_order_and_large_sets(quads):
    if quads:
        elems, verts = quad_surface(96, 48, seed=7)
    else:
        mesh = W.icosphere(4)
        elems, verts = mesh.indices(), mesh.coords()
    pts = near_points(verts, 20000, 0.05, seed=8)
    r2 = np.full(20000, 0.06 ** 2)
    with env(SSDF_B200_SORT_POINTS=0):
        a = S.closest_within_radius(pts, elems, verts, r2)
    b = S.closest_within_radius(pts, elems, verts, r2)
    check(a, b, "sorted vs input order")
    ids = np.arange(0, 20000, 7)
    want = oracle.within_radius(pts[:, ids], elems, verts, r2[ids])
    check(tuple(x[ids] for x in b), want, "oracle sample")


def test_empty_and_invalid():
    pts = np.random.default_rng(0).uniform(size=(3, 50))
    empty = [np.zeros(0, np.int32)] * 3
    r2 = np.linspace(-1, 1, 50)
    got = S.closest_within_radius(pts, empty, np.zeros((3, 0)), r2)
    assert np.all(got[0] == -1) and np.array_equal(got[1], r2.astype(np.float32).astype(np.float64))
    assert all(np.all(g == 0) for g in got[2:])
    mesh = W.icosphere(1)
    out = S.closest_within_radius(np.zeros((3, 0)), mesh.indices(), mesh.coords(), np.zeros(0))
    assert len(out[0]) == 0
    bad = [a.copy() for a in mesh.indices()]
    bad[1][3] = mesh.nv
    with pytest.raises(S.SsdfError) as e:
        S.closest_within_radius(pts, bad, mesh.coords(), np.ones(50))
    assert e.value.status == S.SSDF_ERR_INVALID_ARGUMENT


# ---- candidate contact pairs (potential_contact_triangles_bvh / _quads_bvh) ---------------------

from test_oracle import PC_QUADS, PC_TRIANGLES  # noqa: E402


@pytest.mark.parametrize("case", [PC_TRIANGLES, PC_QUADS])
@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_potential_contact_known_answers(case, dt):
    ptr, idx = S.potential_contact(case["e"], (case["x"], case["y"], case["z"]), 0.3, dt)
    assert list(ptr) == case["ptr"]
    for e, c in case["contacts"]:
        assert c in idx[ptr[e]:ptr[e + 1]]


def sorted_rows(ptr, idx):
    return np.concatenate([np.sort(idx[ptr[i]:ptr[i + 1]]) for i in range(len(ptr) - 1)] + [np.zeros(0, idx.dtype)])


def small_soup(n, size, seed):
    rng = np.random.default_rng(seed)
    v = rng.uniform(0, 1, size=(n, 1, 3)) + rng.uniform(-size, size, size=(n, 3, 3))
    return W.Mesh(v.reshape(-1, 3), np.arange(3 * n, dtype=np.int32).reshape(-1, 3))


def contact_cases():
    soup = small_soup(3000, 0.03, seed=2)
    torus = W.torus(nu=64, nv=32, jitter=0.01)
    q, qv = quad_surface(48, 24, seed=9)
    return [("soup", soup.indices(), soup.coords(), 0.02), ("torus", torus.indices(), torus.coords(), 0.05),
            ("quads", q, tuple(qv), 0.03), ("quads-wide", q, tuple(qv), 0.4)]


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_potential_contact_equals_brute_force(dt):
    for name, elems, verts, ext in contact_cases():
        ptr, idx = S.potential_contact(elems, verts, ext, dt)
        wptr, widx = oracle.potential_contact(elems, verts, ext, dt)
        assert np.array_equal(ptr, wptr), name
        assert np.array_equal(sorted_rows(ptr, idx), widx), name
        ptr2, idx2 = S.potential_contact(elems, verts, ext, dt)
        assert np.array_equal(idx2, idx), name  # the same order on the same input
        assert ptr[-1] > 0, name  # the cases do have contacts


def test_potential_contact_empty_and_invalid():
    ptr, idx = S.potential_contact([np.zeros(0, np.int32)] * 3, (np.zeros(0),) * 3, 0.1)
    assert list(ptr) == [0] and len(idx) == 0
    mesh = W.icosphere(1)
    bad = [a.copy() for a in mesh.indices()]
    bad[2][0] = -1
    with pytest.raises(S.SsdfError):
        S.potential_contact(bad, mesh.coords(), 0.1)
