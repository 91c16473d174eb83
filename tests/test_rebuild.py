"""The level-set path (serial/bvh/sdf_rebuild.cpp): marching tetrahedra, cubic refinement, the banded
rebuild and the rounding of edges.

The reference's sdf_rebuild.cpp includes cuBQL and cannot be compiled here, so the oracle
(oracle/ssdf_oracle_rebuild*.c) is pinned by the analytic checks of the reference's own
tests/round_sdf_test.cpp, restated: a tilted plane rebuilt to float rounding, a cubic reproduced by
the refinement, and (GPU, larger grids) the rounded box converging with the spacing. The GPU path is
then checked bitwise against the oracle: the soup (order and vertices), the refined field, and the
rebuilt and rounded distances.
"""

import numpy as np
import pytest

import oracle


def cube(n):
    return (n, n, n), (-0.5, -0.5, -0.5), (1.0 / (n - 1),) * 3


def points(n, o, h, dtype=np.float32):
    """Sample positions o + i h in double from G's o and h (x fastest)."""
    o = np.asarray(o, dtype=dtype).astype(np.float64)
    h = np.asarray(h, dtype=dtype).astype(np.float64)
    k, j, i = np.meshgrid(*[np.arange(v) for v in n[::-1]], indexing="ij")
    return np.stack([o[0] + i.ravel() * h[0], o[1] + j.ravel() * h[1], o[2] + k.ravel() * h[2]])


def round_box(p, b, r):
    q = np.abs(p) - np.asarray(b)[:, None] + r
    return np.sqrt((np.maximum(q, 0) ** 2).sum(0)) + np.minimum(q.max(0), 0) - r


NRM, C0 = np.array([0.48, 0.6, 0.64]), 0.05


def plane_field(n, o, h):
    p = points(n, o, h)
    return p, (NRM @ p - C0).astype(np.float32)


def plane_error(p, out, h, band):
    s = NRM @ p - C0
    inside = np.all(np.abs(p - s * NRM[:, None]) < 0.5 - np.asarray(h)[:, None], axis=0) & (np.abs(s) <= band)
    return np.max(np.abs(out.astype(np.float64) - s)[inside])


# ---- CPU: the oracle against the reference test's analytic expectations ---------------------------

def test_oracle_tilted_plane():
    n, o, h = cube(21)
    p, f = plane_field(n, o, h)
    out = oracle.rebuild_sdf(n, o, h, f, 0.0, 0.2, dtype=np.float32)
    assert plane_error(p, out, h, 0.2) < 1e-6


def test_oracle_refine_reproduces_a_cubic():
    n, o, h = cube(9)
    cubic = lambda q: q[0] ** 3 - 2 * q[1] ** 2 + q[0] * q[1] * q[2] + 0.5 * q[2] - 0.1  # noqa: E731
    f = cubic(points(n, o, h)).astype(np.float32)
    m = 3
    fine = oracle.refine_field(n, f, m, np.float32)
    fn = tuple((v - 1) * m + 1 for v in n)
    fh = tuple(np.float32(np.float64(np.float32(v)) / m) for v in h)
    q = points(fn, o, fh)
    idx = np.arange(fine.size).reshape(fn[::-1])[m:-m, m:-m, m:-m].ravel()
    assert np.max(np.abs(fine[idx].astype(np.float64) - cubic(q[:, idx]))) < 1e-6


def test_oracle_soup_closes_a_sphere():
    n, o, h = cube(13)
    p = points(n, o, h, np.float64)
    f = np.sqrt((p ** 2).sum(0)) - 0.31
    s = oracle.level_set_triangles(n, o, h, f, 0.0)
    v = s.reshape(3, -1, 3)
    a, b, c = v[:, :, 0], v[:, :, 1], v[:, :, 2]
    assert np.all(np.abs(np.sqrt((s ** 2).sum(0)) - 0.31) < 0.5 * h[0])  # vertices on the sphere
    # the triangles (unoriented, as the reference's) cover the sphere once: their area is its area
    area = 0.5 * np.linalg.norm(np.cross(b - a, c - a, axis=0), axis=0).sum()
    assert abs(area - 4 * np.pi * 0.31 ** 2) < 0.05 * 4 * np.pi * 0.31 ** 2


# ---- GPU: bitwise the oracle, and the reference test's convergence ---------------------------------

def grid(n, o, h, dtype):
    import ssdf_b200 as S

    return S.GridGeometry(n, o, h, dtype)


def blob(n, o, h, dtype):
    """A field with exact zeros at samples (degenerate crossings) and non-cubic grid extents."""
    p = points(n, o, h, dtype)
    f = np.minimum(np.sqrt(((p - 0.1) ** 2).sum(0)) - 0.3, p[0] + 0.25)
    f[::37] = 0.0
    return f.astype(dtype)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("n", [(9, 13, 11), (24, 24, 24)])
def test_soup_bitwise(dtype, n):
    import ssdf_b200 as S

    o, h = (-0.55, -0.5, -0.45), (1.1 / (n[0] - 1), 1.0 / (n[1] - 1), 0.9 / (n[2] - 1))
    f = blob(n, o, h, dtype)
    for level in (0.0, 0.05):
        got = S.level_set_triangles(grid(n, o, h, dtype), f, level)
        want = oracle.level_set_triangles(n, o, h, f, level, dtype)
        assert got.shape == want.shape and got.shape[1] > 0
        assert np.array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_refine_bitwise(dtype):
    import ssdf_b200 as S

    n, o, h = (7, 9, 8), (-0.5, -0.4, -0.3), (0.1, 0.1, 0.1)
    f = blob(n, o, h, dtype)
    for m in (1, 2, 3):
        assert np.array_equal(S.refine_field(grid(n, o, h, dtype), f, m), oracle.refine_field(n, f, m, dtype))


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("stride", [1, 2])
def test_rebuild_bitwise(dtype, stride):
    import ssdf_b200 as S

    n, o, h = (21, 19, 17), (-0.5, -0.45, -0.4), (0.05, 0.05, 0.05)
    f = blob(n, o, h, dtype)
    for level, band in ((0.0, 0.15), (0.03, 0.5)):
        got = S.rebuild_sdf(grid(n, o, h, dtype), f, level, band, stride)
        want = oracle.rebuild_sdf(n, o, h, f, level, band, stride, dtype)
        assert np.array_equal(got, want)
    # no level set inside the grid: +-band everywhere, unsearched
    got = S.rebuild_sdf(grid(n, o, h, dtype), np.full(f.size, 2.0, dtype), 0.0, 0.1, stride)
    assert np.all(got == dtype(0.1))


@pytest.mark.gpu
def test_round_bitwise():
    import ssdf_b200 as S

    n, o, h = cube(21)
    p = points(n, o, h)
    f = (-round_box(p, (0.3, 0.25, 0.2), 0)).astype(np.float32)
    for op, cl, stride in ((True, True, 1), (True, False, 2), (False, True, 1)):
        got, f0 = S.round_sdf(grid(n, o, h, np.float32), f, 0.08, 0.3, op, cl, stride, with_f0=True)
        want, w0 = oracle.round_sdf(n, o, h, f, 0.08, 0.3, op, cl, stride, np.float32)
        assert np.array_equal(f0, w0)
        assert np.array_equal(got, want)


@pytest.mark.gpu
def test_tilted_plane():
    """tests/round_sdf_test.cpp's tilted plane at its size (33^3), on the GPU."""
    import ssdf_b200 as S

    n, o, h = cube(33)
    p, f = plane_field(n, o, h)
    out = S.rebuild_sdf(grid(n, o, h, np.float32), f, 0.0, 0.2)
    assert plane_error(p, out, h, 0.2) < 1e-6


def rounded_box_error(n, sign, stride, refine=1, self_check=False):
    import ssdf_b200 as S

    b, r = (0.3, 0.25, 0.2), 0.08
    gn, go, gh = cube(n)
    g = grid(gn, go, gh, np.float32)
    f = (-sign * round_box(points(gn, go, gh), b, 0)).astype(np.float32)
    if refine > 1:
        f = S.refine_field(g, f, refine)
        g = g.refined(refine)
    out = S.round_sdf(g, f, r, 0.3, True, True, stride if refine == 1 else refine)
    og = g.strided(stride if refine == 1 else refine)
    q = points(og.n, og.o, og.h) if refine == 1 else points(gn, go, gh)  # refined: the coarse samples
    exact = -sign * round_box(q, b, r)
    near = np.abs(exact) <= r
    err = np.max(np.abs(out.astype(np.float64) - exact)[near])
    if not self_check:
        return err
    again = S.rebuild_sdf(og, out, 0.0, 0.3)
    return err, np.max(np.abs(again.astype(np.float64) - out)[near])


@pytest.mark.gpu
@pytest.mark.parametrize("sign", [1.0, -1.0])
def test_rounded_box_converges(sign):
    """tests/round_sdf_test.cpp's rounded box: opening the box and closing its complement, at
    h = 1/40, 1/80, 1/160, written strided and refined, with its thresholds."""
    e1, s1 = rounded_box_error(41, sign, 1, self_check=True)
    e2, s2 = rounded_box_error(81, sign, 1, self_check=True)
    e3, s3 = rounded_box_error(161, sign, 1, self_check=True)
    es = rounded_box_error(81, sign, 2)
    er = rounded_box_error(41, sign, 1, refine=2)
    assert e1 < 1.0 / 40 and e2 < 0.6 / 80 and e3 < 0.25 / 160
    assert e2 < 0.6 * e1 and e3 < 0.6 * e2
    assert s1 < 0.1 / 40 and s2 < 0.35 * s1 and s3 < 0.35 * s2
    assert es <= 1.01 * e2
    assert er < 0.6 * e1
