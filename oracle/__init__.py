"""CPU oracle for ssdf's closest-point distance path -- TEST INFRASTRUCTURE ONLY.

This package is the checker: only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline leg import it. The product (``ssdf_b200``) never imports, links or falls back to it.

Two CPU libraries sit behind it, both built by ``oracle/Makefile``:

* ``liboracle.so`` -- the C restatement in ``ssdf_oracle.c`` (see its header for the reference
  lines each function follows), always present once built;
* ``_ref/libssdf_ref.so`` -- zulianp/ssdf's own CPU code (``serial/ssdf.cpp`` + ``ssdf.hpp``)
  compiled from its sources, with ``ref_harness.cpp`` exporting ``edf`` and ``edf_celllist``.
  It exists only where the reference sources were present at build time (it then travels with
  the repository snapshot as a built file).
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libssdf_ref.so")
# where the reference's sources are (read only; SSDF_REFERENCE_SRC overrides the default)
REF_SRC = os.environ.get("SSDF_REFERENCE_SRC", "/root/reference")

_pd = C.c_ssize_t
_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


def build(ref_src: str | None = None) -> None:
    """Compile liboracle.so, and the reference's CPU library when its sources are present."""
    src = ref_src or REF_SRC
    targets = ["oracle"]
    if os.path.isdir(os.path.join(src, "serial")):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, f"REF={src}", *targets], check=True)


def _load(path: str) -> C.CDLL:
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built (run `make -C oracle`)")
    return C.CDLL(path)


_lib = None
_ref = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        _lib = _load(ORACLE_SO)
        for suf, fptr, ft in (("_d", _dp, C.c_double), ("_f", _fp, C.c_float)):
            f = getattr(_lib, "oracle_point_triangle_dist_sq" + suf)
            f.restype = ft
            f.argtypes = [ft] * 12
            f = getattr(_lib, "oracle_point_triangle_closest_point" + suf)
            f.restype = None
            f.argtypes = [ft] * 12 + [fptr] * 3
            for n in ("oracle_point_aabb_distance_squared", "oracle_point_aabb_signed_distance"):
                f = getattr(_lib, n + suf)
                f.restype = ft
                f.argtypes = [ft] * 9
            f = getattr(_lib, "oracle_edf" + suf)
            f.restype = C.c_int
            f.argtypes = [_pd, fptr, fptr, fptr, _pd, _ip, _ip, _ip, _pd, fptr, fptr, fptr, fptr, _ip]
            f = getattr(_lib, "oracle_compute_aabb" + suf)
            f.restype = None
            f.argtypes = [_pd, fptr, fptr, fptr, fptr]
            f = getattr(_lib, "oracle_all_points_aabb_signed_distance" + suf)
            f.restype = None
            f.argtypes = [_pd, fptr, fptr, fptr, fptr, fptr]
            f = getattr(_lib, "oracle_grid_points" + suf)
            f.restype = None
            f.argtypes = [_pd, _pd, _pd] + [ft] * 6 + [_dp, _dp, _dp]
        for suf, fptr, ft in (("_d", _dp, C.c_double), ("_f", _fp, C.c_float)):
            n3 = C.POINTER(C.c_ssize_t)
            f = getattr(_lib, "oracle_level_set_triangles" + suf)
            f.restype = C.c_ssize_t
            f.argtypes = [n3, fptr, fptr, fptr, ft, fptr, fptr, fptr]
            f = getattr(_lib, "oracle_refine_field" + suf)
            f.restype = None
            f.argtypes = [n3, fptr, C.c_ssize_t, fptr]
            f = getattr(_lib, "oracle_rebuild_sdf" + suf)
            f.restype = None
            f.argtypes = [n3, fptr, fptr, fptr, ft, ft, C.c_ssize_t, fptr]
        _lib.oracle_pseudonormals_d.restype = C.c_int
        _lib.oracle_pseudonormals_d.argtypes = [_pd, _ip, _ip, _ip, _pd, _dp, _dp, _dp, _dp, _dp, _dp]
        _lib.oracle_sdf_points_d.restype = C.c_int
        _lib.oracle_sdf_points_d.argtypes = [_pd, _dp, _dp, _dp, _pd, _ip, _ip, _ip, _pd, _dp, _dp, _dp,
                                             _dp, _dp, _dp, _dp, _ip]
        _lib.oracle_closest_point_d.restype = C.c_int
        _lib.oracle_closest_point_d.argtypes = [_pd, _dp, _dp, _dp, _pd, _ip, _ip, _ip, _pd, _dp, _dp, _dp,
                                                _dp, _dp, _dp, _dp, _ip]
        for suf, (gp, tp) in (("_ff", (_fp, _fp)), ("_fd", (_fp, _dp)), ("_dd", (_dp, _dp))):
            f = getattr(_lib, "oracle_within_radius" + suf)
            f.restype = C.c_int
            f.argtypes = [_pd, gp, gp, gp, _pd, _ip, _ip, _ip, _ip, gp, gp, gp, _pd, tp, C.c_int, C.c_int, _ip,
                          tp, tp, tp, tp]
        for suf, fptr, ft in (("_d", _dp, C.c_double), ("_f", _fp, C.c_float)):
            f = getattr(_lib, "oracle_point_to_quad_closest_point" + suf)
            f.restype = None
            f.argtypes = [ft] * 15 + [fptr, fptr]
            f = getattr(_lib, "oracle_point_triangle_barycentric" + suf)
            f.restype = ft
            f.argtypes = [ft] * 12 + [fptr] * 3
        _lib.oracle_potential_contact.restype = C.c_ssize_t
        _lib.oracle_potential_contact.argtypes = [_pd, _ip, _ip, _ip, _ip, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                                  C.c_float, C.c_float, C.POINTER(C.c_ssize_t), _ip, _pd]
        _lib.oracle_sqedf_points_d.restype = C.c_int
        _lib.oracle_sqedf_points_d.argtypes = [_pd, _dp, _dp, _dp, _pd, _ip, _ip, _ip, _pd, _dp, _dp, _dp, _dp]
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref() -> C.CDLL:
    """The reference's own CPU library (raises if it was not built)."""
    global _ref
    if _ref is None:
        _ref = _load(REF_SO)
        for suf, fptr in (("_d", _dp), ("_f", _fp)):
            for n in ("ref_edf", "ref_edf_celllist", "ssdf_edf"):
                f = getattr(_ref, n + suf)
                f.restype = C.c_int
                f.argtypes = [_pd, fptr, fptr, fptr, _pd, _ip, _ip, _ip, _pd, fptr, fptr, fptr, fptr]
        _ref.ref_point_triangle_dist_sq_d.restype = C.c_double
        _ref.ref_point_triangle_dist_sq_d.argtypes = [C.c_double] * 12
        _ref.ref_point_triangle_dist_sq_f.restype = C.c_float
        _ref.ref_point_triangle_dist_sq_f.argtypes = [C.c_float] * 12
        _ref.ref_point_triangle_closest_point_d.restype = None
        _ref.ref_point_triangle_closest_point_d.argtypes = [C.c_double] * 12 + [_dp] * 3
        for n in ("ref_point_aabb_distance_squared_d", "ref_point_aabb_signed_distance_d"):
            getattr(_ref, n).restype = C.c_double
            getattr(_ref, n).argtypes = [C.c_double] * 9
        for suf, fptr in (("_d", _dp), ("_f", _fp)):
            f = getattr(_ref, "ref_compute_aabb" + suf)
            f.restype = None
            f.argtypes = [_pd, fptr, fptr, fptr, fptr]
            f = getattr(_ref, "ref_all_points_aabb_signed_distance" + suf)
            f.restype = None
            f.argtypes = [_pd, fptr, fptr, fptr, fptr, fptr]
        for suf, fptr, ft in (("_d", _dp, C.c_double), ("_f", _fp, C.c_float)):
            f = getattr(_ref, "ref_point_to_quad_closest_point" + suf)
            f.restype = None
            f.argtypes = [fptr, fptr, fptr]
            f = getattr(_ref, "ref_point_triangle_barycentric" + suf)
            f.restype = ft
            f.argtypes = [ft] * 12 + [fptr]
        _ref.ref_set_quiet.restype = None
        _ref.ref_set_quiet.argtypes = [C.c_int]
        _ref.ref_set_quiet(1)
    return _ref


# ----------------------------------------------------------------------------------------------
# numpy conveniences
# ----------------------------------------------------------------------------------------------

def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def _real(dtype):
    return (C.c_double, "_d") if np.dtype(dtype) == np.float64 else (C.c_float, "_f")


def _mesh_args(mesh, dtype):
    ct, _ = _real(dtype)
    sx, sy, sz = (np.ascontiguousarray(a, dtype=dtype) for a in mesh.coords())
    s0, s1, s2 = (np.ascontiguousarray(a, dtype=np.int32) for a in mesh.indices())
    keep = (sx, sy, sz, s0, s1, s2)
    return keep, [len(s0), _ptr(s0, C.c_int), _ptr(s1, C.c_int), _ptr(s2, C.c_int), len(sx),
                  _ptr(sx, ct), _ptr(sy, ct), _ptr(sz, ct)]


def edf(points, mesh, out=None, dtype=np.float64, with_index=False):
    """Brute-force edf value (and closest triangle) at points (3, n) -- the oracle's restatement."""
    ct, suf = _real(dtype)
    x, y, z = (np.ascontiguousarray(a, dtype=dtype) for a in points)
    n = len(x)
    o = np.full(n, np.finfo(dtype).max, dtype=dtype) if out is None else np.array(out, dtype=dtype, copy=True)
    tri = np.full(n, -1, dtype=np.int32)
    keep, margs = _mesh_args(mesh, dtype)
    rc = getattr(lib(), "oracle_edf" + suf)(n, _ptr(x, ct), _ptr(y, ct), _ptr(z, ct), *margs, _ptr(o, ct),
                                            _ptr(tri, C.c_int))
    assert rc == 0
    return (o, tri) if with_index else o


def ref_edf(points, mesh, out=None, dtype=np.float64, which="edf"):
    """The reference's own edf / edf_celllist / ssdf_edf (edf_select) on the CPU."""
    ct, suf = _real(dtype)
    x, y, z = (np.ascontiguousarray(a, dtype=dtype) for a in points)
    n = len(x)
    o = np.full(n, np.finfo(dtype).max, dtype=dtype) if out is None else np.array(out, dtype=dtype, copy=True)
    keep, margs = _mesh_args(mesh, dtype)
    fn = {"edf": "ref_edf", "celllist": "ref_edf_celllist", "select": "ssdf_edf"}[which]
    rc = getattr(ref(), fn + suf)(n, _ptr(x, ct), _ptr(y, ct), _ptr(z, ct), *margs, _ptr(o, ct))
    assert rc == 0
    return o


def pseudonormals(mesh):
    sx, sy, sz = (np.ascontiguousarray(a, dtype=np.float64) for a in mesh.coords())
    s0, s1, s2 = (np.ascontiguousarray(a, dtype=np.int32) for a in mesh.indices())
    nt, nv = len(s0), len(sx)
    fn = np.zeros(3 * nt)
    en = np.zeros(9 * nt)
    vn = np.zeros(3 * nv)
    rc = lib().oracle_pseudonormals_d(nt, _ptr(s0, C.c_int), _ptr(s1, C.c_int), _ptr(s2, C.c_int), nv,
                                      _ptr(sx, C.c_double), _ptr(sy, C.c_double), _ptr(sz, C.c_double),
                                      _ptr(fn, C.c_double), _ptr(en, C.c_double), _ptr(vn, C.c_double))
    assert rc == 0
    return fn, en, vn


def sdf_points(points, mesh, normals=None):
    """Signed double distance and closest triangle at double points (3, n)."""
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in points)
    n = len(x)
    fn, en, vn = normals if normals is not None else pseudonormals(mesh)
    out = np.zeros(n)
    tri = np.zeros(n, dtype=np.int32)
    keep, margs = _mesh_args(mesh, np.float64)
    rc = lib().oracle_sdf_points_d(n, _ptr(x, C.c_double), _ptr(y, C.c_double), _ptr(z, C.c_double), *margs,
                                   _ptr(fn, C.c_double), _ptr(en, C.c_double), _ptr(vn, C.c_double),
                                   _ptr(out, C.c_double), _ptr(tri, C.c_int))
    assert rc == 0
    return out, tri


def closest_point(points, mesh, outd=None):
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in points)
    n = len(x)
    d = np.full(n, np.finfo(np.float64).max) if outd is None else np.array(outd, dtype=np.float64, copy=True)
    ox, oy, oz = np.zeros(n), np.zeros(n), np.zeros(n)
    tri = np.full(n, -1, dtype=np.int32)
    keep, margs = _mesh_args(mesh, np.float64)
    rc = lib().oracle_closest_point_d(n, _ptr(x, C.c_double), _ptr(y, C.c_double), _ptr(z, C.c_double), *margs,
                                      _ptr(d, C.c_double), _ptr(ox, C.c_double), _ptr(oy, C.c_double),
                                      _ptr(oz, C.c_double), _ptr(tri, C.c_int))
    assert rc == 0
    return d, ox, oy, oz, tri


def sqedf_points(points, mesh, out=None):
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in points)
    n = len(x)
    o = np.full(n, np.finfo(np.float64).max) if out is None else np.array(out, dtype=np.float64, copy=True)
    keep, margs = _mesh_args(mesh, np.float64)
    rc = lib().oracle_sqedf_points_d(n, _ptr(x, C.c_double), _ptr(y, C.c_double), _ptr(z, C.c_double), *margs,
                                     _ptr(o, C.c_double))
    assert rc == 0
    return o


def grid_points(grid, dtype=np.float64):
    """Node-grid coordinates (3, nx*ny*nz) in the reference's G precision, widened to double."""
    ct, suf = _real(dtype)
    nx, ny, nz = grid.n
    n = nx * ny * nz
    q = np.zeros((3, n))
    lo = [ct(v) for v in grid.lo]
    hi = [ct(v) for v in grid.hi]
    getattr(lib(), "oracle_grid_points" + suf)(nx, ny, nz, *lo, *hi, _ptr(q[0], C.c_double),
                                               _ptr(q[1], C.c_double), _ptr(q[2], C.c_double))
    return q


def compute_aabb(points, dtype=np.float64, reference=False):
    """(xmin, xmax, ymin, ymax, zmin, zmax) of the points converted to dtype -- the oracle's
    restatement of ssdf::compute_aabb, or (reference=True) the reference's own template."""
    ct, suf = _real(dtype)
    x, y, z = (np.ascontiguousarray(a, dtype=dtype) for a in points)
    b = np.empty(6, dtype=dtype)
    fn = ("ref_compute_aabb" if reference else "oracle_compute_aabb") + suf
    getattr(ref() if reference else lib(), fn)(len(x), _ptr(x, ct), _ptr(y, ct), _ptr(z, ct), _ptr(b, ct))
    return b


def all_points_aabb_signed_distance(points, box, dtype=np.float64, reference=False):
    """Signed distance of each point (converted to dtype) to box (minx, maxx, miny, maxy, minz, maxz)."""
    ct, suf = _real(dtype)
    x, y, z = (np.ascontiguousarray(a, dtype=dtype) for a in points)
    b = np.ascontiguousarray(box, dtype=dtype)
    out = np.empty(len(x), dtype=dtype)
    fn = ("ref_all_points_aabb_signed_distance" if reference else "oracle_all_points_aabb_signed_distance") + suf
    getattr(ref() if reference else lib(), fn)(len(x), _ptr(x, ct), _ptr(y, ct), _ptr(z, ct), _ptr(b, ct),
                                               _ptr(out, ct))
    return out


# ---- level sets (serial/bvh/sdf_rebuild.cpp) -----------------------------------------------------

def _grid_args(n, o, h, dtype):
    ct, suf = _real(dtype)
    na = (C.c_ssize_t * 3)(*[int(v) for v in n])
    oa = np.ascontiguousarray(o, dtype=dtype)
    ha = np.ascontiguousarray(h, dtype=dtype)
    return ct, suf, na, oa, ha


def level_set_triangles(n, o, h, f, level, dtype=np.float64):
    """The oracle's marching-tetrahedra soup (3, 3 * ntri) of {f = level}."""
    ct, suf, na, oa, ha = _grid_args(n, o, h, dtype)
    fa = np.ascontiguousarray(f, dtype=dtype)
    fn = getattr(lib(), "oracle_level_set_triangles" + suf)
    nt = fn(na, _ptr(oa, ct), _ptr(ha, ct), _ptr(fa, ct), dtype(level), None, None, None)
    x, y, z = (np.empty(3 * nt, dtype=dtype) for _ in range(3))
    fn(na, _ptr(oa, ct), _ptr(ha, ct), _ptr(fa, ct), dtype(level), _ptr(x, ct), _ptr(y, ct), _ptr(z, ct))
    return np.stack([x, y, z])


def refine_field(n, f, factor, dtype=np.float64):
    ct, suf, na, _, _ = _grid_args(n, (0, 0, 0), (0, 0, 0), dtype)
    fa = np.ascontiguousarray(f, dtype=dtype)
    rn = [(int(v) - 1) * factor + 1 for v in n]
    fine = np.empty(rn[0] * rn[1] * rn[2], dtype=dtype)
    getattr(lib(), "oracle_refine_field" + suf)(na, _ptr(fa, ct), int(factor), _ptr(fine, ct))
    return fine


def rebuild_sdf(n, o, h, f, level, band, stride=1, dtype=np.float64):
    ct, suf, na, oa, ha = _grid_args(n, o, h, dtype)
    fa = np.ascontiguousarray(f, dtype=dtype)
    on = [(int(v) - 1) // stride + 1 for v in n]
    out = np.empty(on[0] * on[1] * on[2], dtype=dtype)
    getattr(lib(), "oracle_rebuild_sdf" + suf)(na, _ptr(oa, ct), _ptr(ha, ct), _ptr(fa, ct), dtype(level),
                                               dtype(band), int(stride), _ptr(out, ct))
    return out


def round_sdf(n, o, h, f, radius, band, open=True, close=True, stride=1, dtype=np.float64):
    """serial/bvh/sdf_rebuild.cpp:300-336 composed from the oracle's rebuilds (shifts in REAL)."""
    t = np.dtype(dtype).type
    r0 = rebuild_sdf(n, o, h, f, 0, band, 1, dtype)
    cur = r0
    if open:
        cur = (rebuild_sdf(n, o, h, cur, radius, band, 1, dtype) + t(radius)).astype(dtype)
    if close:
        cur = (rebuild_sdf(n, o, h, cur, -t(radius), band, 1, dtype) - t(radius)).astype(dtype)
    return rebuild_sdf(n, o, h, cur, 0, band, stride, dtype), r0


# ----------------------------------------------------------------------------------------------
# closest primitive within a radius (serial/bvh/bvh.cpp:367-832)
# ----------------------------------------------------------------------------------------------

def quad_closest_st(p, quad, dtype=np.float64, reference=False):
    """(s, t) of point p on the quad (4 x 3 corners): point_to_quad_closest_point
    (serial/edf/edf.hpp:388-489), the restatement or (reference=True) the reference's own."""
    ct, suf = _real(dtype)
    p = np.asarray(p, dtype=dtype)
    v = np.asarray(quad, dtype=dtype).reshape(12)
    if reference:
        st = np.zeros(2, dtype=dtype)
        getattr(ref(), "ref_point_to_quad_closest_point" + suf)(_ptr(np.ascontiguousarray(p), ct), _ptr(np.ascontiguousarray(v), ct),
                                                       _ptr(st, ct))
        return float(st[0]), float(st[1])
    s, t = ct(), ct()
    getattr(lib(), "oracle_point_to_quad_closest_point" + suf)(*[ct(float(a)) for a in p], *[ct(float(a)) for a in v],
                                                      C.byref(s), C.byref(t))
    return s.value, t.value


def triangle_barycentric(q, tri, dtype=np.float64, reference=False):
    """(d2, wa, wb, wc): point_triangle_barycentric (serial/edf/edf.hpp:251-386)."""
    ct, suf = _real(dtype)
    args = [ct(float(a)) for a in np.asarray(q, dtype=dtype)] + [ct(float(a)) for a in np.asarray(tri, dtype=dtype).reshape(9)]
    w = np.zeros(3, dtype=dtype)
    if reference:
        d2 = getattr(ref(), "ref_point_triangle_barycentric" + suf)(*args, _ptr(w, ct))
        return d2, float(w[0]), float(w[1]), float(w[2])
    wa, wb, wc = ct(), ct(), ct()
    d2 = getattr(lib(), "oracle_point_triangle_barycentric" + suf)(*args, C.byref(wa), C.byref(wb), C.byref(wc))
    return d2, wa.value, wb.value, wc.value


def within_radius(points, elements, vertices, radius_squared, stride=1, skip_self=False, local=False,
                  gdtype=np.float64, tdtype=None):
    """Brute-force closest primitive within a radius: closest_within_radius_bvh (elements = 3
    index arrays, triangles) or closest_within_radius_quads_bvh (4 arrays, quads), with local=True
    their _local_ variants. Returns (outtri, out_sqr_dist, o0, o1[, o2])."""
    tdtype = gdtype if tdtype is None else tdtype
    suf = {(np.float32, np.float32): "_ff", (np.float32, np.float64): "_fd",
           (np.float64, np.float64): "_dd"}[(np.dtype(gdtype).type, np.dtype(tdtype).type)]
    gct = C.c_float if np.dtype(gdtype) == np.float32 else C.c_double
    tct = C.c_float if np.dtype(tdtype) == np.float32 else C.c_double
    x, y, z = (np.ascontiguousarray(a, dtype=gdtype) for a in points)
    sx, sy, sz = (np.ascontiguousarray(a, dtype=gdtype) for a in vertices)
    idx = [np.ascontiguousarray(a, dtype=np.int32) for a in elements]
    quads = len(idx) == 4
    r2 = np.ascontiguousarray(radius_squared, dtype=tdtype)
    n = len(x)
    outtri = np.empty(n, dtype=np.int32)
    outs = [np.empty(n, dtype=tdtype) for _ in range(4)]
    getattr(lib(), "oracle_within_radius" + suf)(n, _ptr(x, gct), _ptr(y, gct), _ptr(z, gct), len(idx[0]),
                                        *[_ptr(a, C.c_int) for a in idx[:3]],
                                        _ptr(idx[3], C.c_int) if quads else None,
                                        _ptr(sx, gct), _ptr(sy, gct), _ptr(sz, gct), int(stride), _ptr(r2, tct),
                                        int(bool(skip_self)), int(bool(local)), _ptr(outtri, C.c_int),
                                        *[_ptr(a, tct) for a in outs])
    return (outtri, outs[0], outs[1], outs[2]) if local else (outtri, *outs)


def potential_contact(elements, vertices, extrusion, dtype=np.float64):
    """Brute-force candidate contact pairs (potential_contact_triangles_bvh / _quads_bvh,
    serial/bvh/bvh.cpp:834-1196): (pc_ptr int64, idx int32), rows ascending."""
    sx, sy, sz = (np.ascontiguousarray(a, dtype=dtype) for a in vertices)
    idx = [np.ascontiguousarray(a, dtype=np.int32) for a in elements]
    n = len(idx[0])
    t = np.dtype(dtype).type
    ext = float(np.float32(extrusion))
    inner = float(np.float32(t(0.1) * t(extrusion)))
    ptr = np.zeros(n + 1, dtype=np.int64)
    pp = ptr.ctypes.data_as(C.POINTER(C.c_ssize_t))
    args = [n, *[_ptr(a, C.c_int) for a in idx[:3]], _ptr(idx[3], C.c_int) if len(idx) == 4 else None,
            sx.ctypes.data, sy.ctypes.data, sz.ctypes.data, int(np.dtype(dtype) == np.float64), ext, inner, pp]
    total = lib().oracle_potential_contact(*args, None, 0)
    out = np.zeros(max(total, 1), dtype=np.int32)
    lib().oracle_potential_contact(*args, _ptr(out, C.c_int), total)
    return ptr, out[:total]
