"""GPU edge cases: empty and ragged inputs, degenerate and duplicate triangles, ties, points on
the surface, far-from-origin coordinates, leaf sizes, invalid indices (rejected on the host,
before any device work), determinism."""

import numpy as np
import pytest

import oracle
import ssdf_b200 as S
from ssdf_b200 import workloads as W
from test_gpu_golden import env

pytestmark = pytest.mark.gpu

ALL_UNSIGNED = ("edf", "celllist", "bvh_f32x", "bvh_f64")


def run_unsigned(method, pts, mesh, out=None):
    if method == "edf":
        return S.edf(pts, mesh, out=out)
    if method == "celllist":
        return S.edf_celllist(pts, mesh, out=out)
    with env(SSDF_B200_PRECISION=method.split("_")[1]):
        return S.edf_index(pts, mesh, out=out)[0]


def test_empty_mesh_leaves_out_untouched():
    empty = W.Mesh(np.zeros((0, 3)), np.zeros((0, 3), np.int32))
    pts = np.random.default_rng(0).uniform(size=(3, 10))
    init = np.arange(10, dtype=np.float64)
    for m in ALL_UNSIGNED:
        assert np.array_equal(run_unsigned(m, pts, empty, out=init), init)
    assert np.array_equal(S.edf_select(pts, empty, out=init), init)
    g = W.Grid((3, 3, 3), (0, 0, 0), (1, 1, 1))
    assert np.array_equal(S.sample_sqedf_bvh(empty, g, out=np.ones(27)), np.ones(27))


def test_no_points():
    mesh = W.icosphere(1)
    for m in ALL_UNSIGNED:
        assert run_unsigned(m, np.zeros((3, 0)), mesh).shape == (0,)


@pytest.mark.parametrize("n", [(1, 1, 1), (7, 3, 5), (1, 9, 2), (33, 1, 1)])
def test_ragged_grids(n):
    mesh = W.icosphere(2)
    g = W.Grid(n, (-1.4, -1.3, -1.2), (1.1, 1.2, 1.3))
    q = oracle.grid_points(g)
    want, wtri = oracle.sdf_points(q, mesh)
    got, gtri = S.sample_sdf_bvh(mesh, g, with_index=True)
    assert np.array_equal(got, want) and np.array_equal(gtri, wtri)


def test_degenerate_and_duplicate_triangles():
    rng = np.random.default_rng(3)
    soup = W.random_soup(60, seed=4)
    v = soup.vertices.copy()
    t = soup.triangles.copy()
    t[5] = [t[5, 0], t[5, 0], t[5, 0]]          # a point
    t[9] = [t[9, 0], t[9, 1], t[9, 1]]          # a segment
    v[t[13, 2]] = 0.5 * (v[t[13, 0]] + v[t[13, 1]])  # collinear
    t = np.concatenate([t, t[[20, 3, 40]]])     # duplicates of 20, 3, 40 at the end
    mesh = W.Mesh(v, t.astype(np.int32))
    pts = rng.uniform(-1.2, 1.2, size=(3, 3000))
    want, wtri = oracle.edf(pts, mesh, with_index=True)
    for m in ALL_UNSIGNED:
        assert np.array_equal(run_unsigned(m, pts, mesh), want), m
    for prec in ("f32x", "f64"):
        with env(SSDF_B200_PRECISION=prec):
            _, tri = S.edf_index(pts, mesh)
        assert np.array_equal(tri, wtri), prec
    assert not np.any(wtri >= 60)
    wf = oracle.edf(pts.astype(np.float32), mesh, dtype=np.float32)
    assert np.array_equal(S.edf_bvh(pts.astype(np.float32), mesh, gdtype=np.float32), wf)
    assert np.array_equal(S.edf(pts.astype(np.float32), mesh, dtype=np.float32), wf)


def test_points_on_vertices_and_edges():
    mesh = W.icosphere(2)
    v = mesh.vertices
    t = mesh.triangles
    on = np.concatenate([v[:200], 0.5 * (v[t[:200, 0]] + v[t[:200, 1]]), v[t[:200]].mean(1)]).T
    want, wtri = oracle.edf(on, mesh, with_index=True)
    for m in ALL_UNSIGNED:
        assert np.array_equal(run_unsigned(m, on, mesh), want), m
    got, gtri = S.edf_index(on, mesh)
    assert np.array_equal(gtri, wtri)
    sd, _ = S.sdf_points(on, mesh)
    osd, _ = oracle.sdf_points(on, mesh)
    assert np.array_equal(sd, osd)


@pytest.mark.parametrize("offset", [1e3, -2.5e4])
def test_far_from_origin(offset):
    mesh = W.torus(nu=40, nv=20, jitter=0.02)
    mesh = W.Mesh(mesh.vertices + offset, mesh.triangles)
    lo, hi = mesh.bbox()
    pts = W.uniform_points(5000, lo - 0.3, hi + 0.3, seed=8)
    want, wtri = oracle.sdf_points(pts, mesh)
    got, gtri = S.sdf_points(pts, mesh)
    assert np.array_equal(got, want) and np.array_equal(gtri, wtri)


@pytest.mark.parametrize("leaf", [1, 2, 3, 8, 16])
def test_leaf_sizes(leaf):
    mesh = W.torus_knot_tube(nu=128, nv=16)
    g = W.Grid.padded_nodes(mesh, 24, 0.25)
    want, wtri = oracle.sdf_points(oracle.grid_points(g), mesh)
    with env(SSDF_B200_LEAF=leaf):
        got, gtri = S.sample_sdf_bvh(mesh, g, with_index=True)
    assert np.array_equal(got, want) and np.array_equal(gtri, wtri)


@pytest.mark.parametrize("leaf", [1, 4, 8])
def test_treelet_refinement(leaf):
    """SAH treelet refinement rearranges the tree; the values cannot change."""
    mesh = W.torus_knot_tube(nu=256, nv=16)
    g = W.Grid.padded_nodes(mesh, 24, 0.25)
    want, wtri = oracle.sdf_points(oracle.grid_points(g), mesh)
    for arity in (2, 4):
        with env(SSDF_B200_LEAF=leaf, SSDF_B200_TREELET=1, SSDF_B200_ARITY=arity):
            got, gtri = S.sample_sdf_bvh(mesh, g, with_index=True)
        assert np.array_equal(got, want) and np.array_equal(gtri, wtri)
    plain = S.DeviceMesh(mesh, leaf_size=leaf, treelet=False).stats()
    tuned = S.DeviceMesh(mesh, leaf_size=leaf, treelet=True).stats()
    assert tuned["leaves"] > 0 and tuned["depth"] < 64 and plain["leaves"] > 0


def test_invalid_indices_are_rejected():
    mesh = W.icosphere(1)
    bad = W.Mesh(mesh.vertices, np.where(mesh.triangles == 5, mesh.nv + 3, mesh.triangles).astype(np.int32))
    pts = np.zeros((3, 4))
    for fn in (S.edf, S.edf_celllist, S.edf_bvh, S.edf_select):
        with pytest.raises(S.SsdfError) as e:
            fn(pts, bad)
        assert e.value.status == 1
    with pytest.raises(S.SsdfError):
        S.DeviceMesh(bad)


def test_deterministic():
    mesh = W.beam_lattice(2000)
    pts = W.uniform_points(100000, -0.1, 1.1, seed=2)
    a = S.edf_index(pts, mesh)
    b = S.edf_index(pts, mesh)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_nan_and_infinite_points():
    """Points with a NaN or infinite coordinate take part like the reference's loops take them: no
    comparison with NaN succeeds, so such a point keeps its incoming value, the others are exact; every
    method and precision agrees with the oracle, and the points around them are unaffected (sorted
    and unsorted lists)."""
    mesh = W.icosphere(2)
    rng = np.random.default_rng(9)
    for n in (300, 5000):
        pts = rng.uniform(-1.5, 1.5, size=(3, n))
        pts[0, ::37] = np.nan
        pts[1, 5::41] = np.inf
        pts[2, 7::43] = -np.inf
        init = np.where(np.arange(n) % 5 == 0, 0.3, np.finfo(np.float64).max)
        want, wtri = oracle.edf(pts, mesh, out=init, with_index=True)
        for method in ALL_UNSIGNED:
            got = run_unsigned(method, pts, mesh, out=init)
            assert np.array_equal(got, want, equal_nan=True), (method, n)
        with env(SSDF_B200_PRECISION="f64"):
            g64, t64 = S.edf_index(pts, mesh, out=init)
        assert np.array_equal(g64, want, equal_nan=True) and np.array_equal(t64, np.where(wtri >= 0, wtri, -1))
