"""ssdf_b200.capi -- ctypes binding of the CUDA library's C ABI.

A ctypes binding over the C ABI of ``ssdf_b200/_lib/libssdf_b200.so`` (declared in
``include/ssdf_b200.h``). Every call runs the CUDA library: there is no CPU path, and importing
this package raises if the library is not built (``python -m ssdf_b200.build``).

Two layers:

* drop-in functions over host (numpy) arrays, one per reference entry point --
  :func:`edf_select` (``ssdf_edf_f/_d``), :func:`edf`, :func:`edf_celllist`, :func:`edf_bvh`,
  :func:`closest_point_bvh`, :func:`sample_sqedf_bvh`, :func:`sample_sdf_bvh` -- plus the additive
  :func:`edf_index`, :func:`sdf_points`;
* :class:`DeviceMesh`: a mesh and its BVH resident on the GPU, queried with device buffers
  (torch tensors or raw pointers) on a caller-chosen stream.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("SSDF_B200_LIBRARY") or os.path.join(HERE, "_lib", "libssdf_b200.so")

SSDF_OK = 0
SSDF_ERR_INVALID_ARGUMENT, SSDF_ERR_OUT_OF_MEMORY, SSDF_ERR_CUDA, SSDF_ERR_NOT_SUPPORTED, SSDF_ERR_INTERNAL = 1, 2, 3, 4, 5
SSDF_ERR_BUSY = 6
F32, F64 = 0, 1
PREC_F32, PREC_F64, PREC_F32_FIXUP = 0, 1, 2
OUT_EDF, OUT_SQEDF, OUT_SDF, OUT_CLOSEST = 0, 1, 2, 3

_pd = C.c_ssize_t
_vp = C.c_void_p
_ip = C.POINTER(C.c_int)


class SsdfError(RuntimeError):
    def __init__(self, status: int, fn: str, message: str):
        super().__init__(f"{fn} -> {_status_name(status)}: {message}")
        self.status = status


class BuildOpts(C.Structure):
    _fields_ = [("leaf_size", C.c_int), ("keep_fp64", C.c_int), ("normals", C.c_int), ("treelet_opt", C.c_int)]


class QueryOpts(C.Structure):
    _fields_ = [("precision", C.c_int), ("output", C.c_int), ("coord_type", C.c_int), ("out_type", C.c_int),
                ("reserved", C.c_int * 4)]


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build the CUDA library first (python -m ssdf_b200.build)")
    return C.CDLL(LIB_PATH)


lib = _load()


def _sig(name, args, res=C.c_int):
    f = getattr(lib, name)
    f.argtypes = args
    f.restype = res
    return f


_sig("ssdf_status_string", [C.c_int], C.c_char_p)
_sig("ssdf_last_error", [], C.c_char_p)
_sig("ssdf_b200_version", [], C.c_char_p)

_EDF = [_pd, _vp, _vp, _vp, _pd, _ip, _ip, _ip, _pd, _vp, _vp, _vp, _vp]
_GRID = [_pd, _ip, _ip, _ip, _pd, _vp, _vp, _vp, _pd, _pd, _pd]
for _n in ("ssdf_edf_f", "ssdf_edf_d", "ssdf_b200_edf_ff", "ssdf_b200_edf_dd", "ssdf_b200_edf_celllist_ff",
           "ssdf_b200_edf_celllist_dd", "ssdf_b200_edf_bvh_ff", "ssdf_b200_edf_bvh_fd", "ssdf_b200_edf_bvh_dd"):
    _sig(_n, _EDF)
for _n in ("ssdf_b200_edf_index_dd", "ssdf_b200_edf_index_ff", "ssdf_b200_sdf_points_dd"):
    _sig(_n, _EDF + [_ip])
for _n in ("ssdf_b200_closest_point_bvh_ff", "ssdf_b200_closest_point_bvh_fd", "ssdf_b200_closest_point_bvh_dd"):
    _sig(_n, _EDF + [_vp, _vp, _vp, _ip])
_sig("ssdf_b200_sample_sqedf_bvh_ff", _GRID + [C.c_float] * 6 + [_vp])
_sig("ssdf_b200_sample_sdf_bvh_ff", _GRID + [C.c_float] * 6 + [_vp])
_sig("ssdf_b200_sample_sqedf_bvh_dd", _GRID + [C.c_double] * 6 + [_vp])
_sig("ssdf_b200_sample_sdf_bvh_dd", _GRID + [C.c_double] * 6 + [_vp])
_sig("ssdf_b200_sample_sdf_index_bvh_dd", _GRID + [C.c_double] * 6 + [_vp, _ip])
_sig("ssdf_mesh_create", [C.POINTER(_vp), _pd, _ip, _ip, _ip, _pd, _vp, _vp, _vp, C.c_int, C.c_int,
                          C.POINTER(BuildOpts), _vp])
_sig("ssdf_mesh_destroy", [_vp])
_sig("ssdf_mesh_destroy_async", [_vp, _vp])
_sig("ssdf_mesh_stats", [_vp] + [C.POINTER(C.c_int64)] * 4)
_sig("ssdf_mesh_filter_info", [_vp, C.POINTER(C.c_float), C.POINTER(C.c_int), C.POINTER(C.c_int64)])
_sig("ssdf_grown_box", [_pd, _vp, _vp, _vp, _vp, C.c_int, C.c_int, _vp, _vp])
_sig("ssdf_triangles_meeting_boxes", [_pd, _vp, _vp, _vp, _pd, _vp, _vp, _vp, C.c_int, C.c_int, _vp, _vp,
                                      C.c_longlong, C.POINTER(C.c_longlong), _vp])
for _n in ("ssdf_pedf_nccl", "ssdf_pedf_update_nccl"):
    _sig(_n, [_vp, _pd, _vp, _vp, _vp, _pd, _vp, _vp, _vp, _pd, _vp, _vp, _vp, C.c_int, C.c_int, _vp, _vp])
_sig("ssdf_edf_device", [C.c_int, _pd, _vp, _vp, _vp, _pd, _vp, _vp, _vp, _pd, _vp, _vp, _vp, C.c_int, _vp, _vp, _vp])
_sig("ssdf_query_points", [_vp, _pd, _vp, _vp, _vp, _vp, _ip, _vp, _vp, _vp, C.POINTER(QueryOpts), _vp])
_sig("ssdf_query_grid", [_vp, _pd, _pd, _pd, C.POINTER(C.c_double * 3), C.POINTER(C.c_double * 3), _vp, _ip,
                         C.POINTER(QueryOpts), _vp])
_sig("ssdf_last_query_counts", [C.POINTER(C.c_int64)] * 4)
_sig("ssdf_b200_fma_peak", [C.c_int, C.POINTER(C.c_double)])
_sig("ssdf_batch_create", [C.POINTER(_vp), C.c_int, C.c_int, C.c_int, C.c_int])
_sig("ssdf_batch_destroy", [_vp])
_sig("ssdf_batch_reserve", [_vp, C.c_longlong, _vp])
_sig("ssdf_batch_clear", [_vp])
_sig("ssdf_batch_size", [_vp])
_sig("ssdf_batch_add_grid", [_vp, _vp, _pd, _pd, _pd, C.POINTER(C.c_double * 3), C.POINTER(C.c_double * 3), _vp, _ip,
                             C.POINTER(QueryOpts)])
_sig("ssdf_batch_add_grid_slab", [_vp, _vp, _pd, _pd, _pd, C.POINTER(C.c_double * 3), C.POINTER(C.c_double * 3), _pd,
                                  _pd, _vp, _ip, C.POINTER(QueryOpts)])
_sig("ssdf_batch_add_points", [_vp, _vp, _pd, _vp, _vp, _vp, _vp, _ip, C.POINTER(QueryOpts)])
_sig("ssdf_batch_run", [_vp, C.c_int, _vp])
_sig("ssdf_batch_last_blocks", [_vp], C.c_longlong)
_sig("ssdf_query_grid_noalloc", [_vp, _pd, _pd, _pd, C.POINTER(C.c_double * 3), C.POINTER(C.c_double * 3), _vp, _ip,
                                 C.POINTER(QueryOpts), _vp])
_sig("ssdf_query_grid_noalloc_max", [], C.c_longlong)
for _g, _gc in (("f", C.c_float), ("d", C.c_double)):
    for _t, _tc in (("f", C.c_float), ("d", C.c_double)):
        _sig(f"ssdf_b200_compute_aabb_{_g}{_t}", [_pd, _vp, _vp, _vp] + [C.POINTER(_tc)] * 6)
        _sig(f"ssdf_b200_all_points_aabb_signed_distance_{_g}{_t}", [_pd, _vp, _vp, _vp] + [_tc] * 6 + [_vp])
_sig("ssdf_points_aabb", [_pd, _vp, _vp, _vp, C.c_int, C.c_int, _vp, _vp])
for _g, _gc in (("f", C.c_float), ("d", C.c_double)):
    _sig(f"ssdf_b200_points_inside_bvh_{_g}", _EDF[:-1] + [_vp])
    _sig(f"ssdf_b200_sample_inside_bvh_{_g}", _GRID + [_gc] * 6 + [_vp])
for _g, _gc in (("ff", C.c_float), ("dd", C.c_double)):
    _GP = [C.POINTER(C.c_ssize_t * 3), C.POINTER(_gc * 3), C.POINTER(_gc * 3), _vp]
    _sig(f"ssdf_b200_level_set_triangles_{_g}", _GP + [_gc, _pd, _vp, _vp, _vp, C.POINTER(C.c_ssize_t)])
    _sig(f"ssdf_b200_rebuild_sdf_{_g}", _GP + [_gc, _gc, _pd, _vp])
    _sig(f"ssdf_b200_refine_field_{_g}", _GP + [_pd, _vp])
    _sig(f"ssdf_b200_round_sdf_{_g}", _GP + [_gc, _gc, C.c_int, C.c_int, _pd, _vp, _vp])
for _g in ("ff", "fd", "dd"):
    _sig(f"ssdf_b200_closest_within_radius_bvh_{_g}", _EDF[:-1] + [_pd, _vp, _ip] + [_vp] * 4 + [C.c_int])
    _sig(f"ssdf_b200_closest_within_radius_local_bvh_{_g}", _EDF[:-1] + [_pd, _vp, _ip] + [_vp] * 3 + [C.c_int])
    _QE = [_pd, _vp, _vp, _vp, _pd, _ip, _ip, _ip, _ip, _pd, _vp, _vp, _vp]
    _sig(f"ssdf_b200_closest_within_radius_quads_bvh_{_g}", _QE + [_pd, _vp, _ip] + [_vp] * 4 + [C.c_int])
    _sig(f"ssdf_b200_closest_within_radius_quads_local_bvh_{_g}", _QE + [_pd, _vp, _ip] + [_vp] * 3 + [C.c_int])
for _g, _gc in (("ff", C.c_float), ("dd", C.c_double)):
    _PC = [_gc, C.POINTER(C.c_ssize_t), C.POINTER(_ip)]
    _sig(f"ssdf_b200_potential_contact_triangles_bvh_{_g}", [_pd, _ip, _ip, _ip, _pd, _vp, _vp, _vp] + _PC)
    _sig(f"ssdf_b200_potential_contact_quads_bvh_{_g}", [_pd, _ip, _ip, _ip, _ip, _pd, _vp, _vp, _vp] + _PC)
_sig("ssdf_b200_free", [_vp], None)
_sig("ssdf_points_aabb_signed_distance", [_pd, _vp, _vp, _vp, C.c_int, C.POINTER(C.c_double * 6), C.c_int, _vp,
                                          C.c_int, _vp])


class ServerOpts(C.Structure):
    _fields_ = [("memory_budget", C.c_size_t), ("max_batch_queries", C.c_int), ("max_batch_jobs", C.c_int),
                ("precision", C.c_int), ("leaf_size", C.c_int), ("slots", C.c_int),
                ("max_queued_queries", C.c_longlong), ("split_queries", C.c_int)]


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_longlong), ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("max_ms", C.c_double),
                ("queries", C.c_longlong), ("batches", C.c_longlong), ("evictions", C.c_longlong),
                ("builds", C.c_longlong), ("resident_bytes", C.c_longlong), ("resident_meshes", C.c_longlong),
                ("seconds", C.c_double), ("rejected", C.c_longlong)]


_dp_ = C.POINTER(C.c_double)


class Tuning(C.Structure):
    _fields_ = [("leaf_size", C.c_int), ("traversal", C.c_int), ("arity", C.c_int), ("ms", C.c_double)]


_sig("ssdf_autotune_grid", [_pd, _ip, _ip, _ip, _pd, _vp, _vp, _vp, _pd, _pd, _pd, C.POINTER(C.c_double * 3),
                            C.POINTER(C.c_double * 3), C.c_int, C.c_char_p, C.POINTER(Tuning)])
_sig("ssdf_server_create", [C.POINTER(_vp), C.POINTER(ServerOpts)])
_sig("ssdf_server_destroy", [_vp])
_sig("ssdf_server_add_mesh", [_vp, _pd, _ip, _ip, _ip, _pd, _vp, _vp, _vp, _ip])
_sig("ssdf_server_submit_points", [_vp, C.c_int, _pd, _vp, _vp, _vp, _vp, _ip, C.POINTER(C.c_longlong)])
_sig("ssdf_server_submit_grid", [_vp, C.c_int, _pd, _pd, _pd, C.POINTER(C.c_double * 3), C.POINTER(C.c_double * 3),
                                 _vp, _ip, C.POINTER(C.c_longlong)])
_sig("ssdf_server_wait", [_vp, C.c_longlong, C.c_double])
_sig("ssdf_server_stats", [_vp, C.POINTER(ServerStats)])
_sig("ssdf_server_reset_stats", [_vp])

EXPORTED = ["ssdf_status_string", "ssdf_last_error", "ssdf_b200_version", "ssdf_edf_f", "ssdf_edf_d",
            "ssdf_b200_edf_ff", "ssdf_b200_edf_dd", "ssdf_b200_edf_celllist_ff", "ssdf_b200_edf_celllist_dd",
            "ssdf_b200_edf_bvh_ff", "ssdf_b200_edf_bvh_fd", "ssdf_b200_edf_bvh_dd", "ssdf_b200_closest_point_bvh_ff",
            "ssdf_b200_closest_point_bvh_fd", "ssdf_b200_closest_point_bvh_dd", "ssdf_b200_sample_sqedf_bvh_ff", "ssdf_b200_sample_sqedf_bvh_dd",
            "ssdf_b200_sample_sdf_bvh_ff", "ssdf_b200_sample_sdf_bvh_dd", "ssdf_b200_edf_index_dd",
            "ssdf_b200_edf_index_ff", "ssdf_b200_sdf_points_dd", "ssdf_b200_sample_sdf_index_bvh_dd",
            "ssdf_mesh_create", "ssdf_mesh_destroy", "ssdf_mesh_stats", "ssdf_mesh_filter_info", "ssdf_edf_device", "ssdf_grown_box", "ssdf_triangles_meeting_boxes", "ssdf_pedf_nccl", "ssdf_pedf_update_nccl", "ssdf_query_points", "ssdf_query_grid",
            "ssdf_last_query_counts", "ssdf_b200_fma_peak", "ssdf_batch_create", "ssdf_batch_destroy", "ssdf_batch_clear",
            "ssdf_batch_size", "ssdf_batch_add_grid", "ssdf_batch_add_grid_slab", "ssdf_batch_add_points", "ssdf_batch_run",
            "ssdf_batch_last_blocks", "ssdf_query_grid_noalloc", "ssdf_query_grid_noalloc_max", "ssdf_server_create",
            "ssdf_server_destroy", "ssdf_server_add_mesh", "ssdf_server_submit_points", "ssdf_server_submit_grid",
            "ssdf_server_wait", "ssdf_server_stats", "ssdf_server_reset_stats", "ssdf_autotune_grid",
            "ssdf_points_aabb", "ssdf_points_aabb_signed_distance", "ssdf_batch_reserve", "ssdf_mesh_destroy_async",
            "ssdf_b200_points_inside_bvh_f", "ssdf_b200_points_inside_bvh_d", "ssdf_b200_sample_inside_bvh_f",
            "ssdf_b200_sample_inside_bvh_d"] + \
    [f"ssdf_b200_{k}_{g}{t}" for k in ("compute_aabb", "all_points_aabb_signed_distance") for g in "fd" for t in "fd"] + \
    [f"ssdf_b200_{k}_{g}" for k in ("level_set_triangles", "rebuild_sdf", "refine_field", "round_sdf") for g in ("ff", "dd")] + \
    [f"ssdf_b200_closest_within_radius_{k}_{g}" for k in ("bvh", "local_bvh", "quads_bvh", "quads_local_bvh")
     for g in ("ff", "fd", "dd")] + \
    [f"ssdf_b200_potential_contact_{k}_bvh_{g}" for k in ("triangles", "quads") for g in ("ff", "dd")] + \
    ["ssdf_b200_free"]


def _status_name(status: int) -> str:
    return lib.ssdf_status_string(status).decode()


def last_error() -> str:
    return lib.ssdf_last_error().decode()


def _check(status: int, fn: str) -> None:
    if status != SSDF_OK:
        raise SsdfError(status, fn, last_error())


def version() -> str:
    return lib.ssdf_b200_version().decode()


# ----------------------------------------------------------------------------------------------
# host (numpy) drop-in layer
# ----------------------------------------------------------------------------------------------

def _arr(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _p(a):
    return C.c_void_p(a.ctypes.data)


def _ipp(a):
    return a.ctypes.data_as(_ip)


def _suffix(dtype) -> str:
    return "d" if np.dtype(dtype) == np.float64 else "f"


class _HostMesh:
    def __init__(self, mesh, dtype):
        self.sx, self.sy, self.sz = (_arr(a, dtype) for a in mesh.coords())
        self.s0, self.s1, self.s2 = (_arr(a, np.int32) for a in mesh.indices())

    def args(self):
        return [len(self.s0), _ipp(self.s0), _ipp(self.s1), _ipp(self.s2), len(self.sx), _p(self.sx), _p(self.sy),
                _p(self.sz)]


def _points(points, dtype):
    x, y, z = (_arr(a, dtype) for a in points)
    return x, y, z


def _init_out(n, dtype, out):
    if out is None:
        return np.full(n, np.finfo(dtype).max, dtype=dtype)
    return np.array(out, dtype=dtype, copy=True)


def _edf_call(fn, points, mesh, out, gdtype, tdtype, extra=()):
    x, y, z = _points(points, gdtype)
    o = _init_out(len(x), tdtype, out)
    hm = _HostMesh(mesh, gdtype)
    _check(getattr(lib, fn)(len(x), _p(x), _p(y), _p(z), *hm.args(), _p(o), *extra), fn)
    return o


def edf_select(points, mesh, out=None, dtype=np.float64):
    """ssdf_edf_f / ssdf_edf_d: the reference's C ABI (environment-dispatched edf_select)."""
    return _edf_call("ssdf_edf_" + _suffix(dtype), points, mesh, out, dtype, dtype)


def edf(points, mesh, out=None, dtype=np.float64):
    """ssdf::edf<G, G, int>: GPU brute force, bitwise the reference's value."""
    s = _suffix(dtype)
    return _edf_call(f"ssdf_b200_edf_{s}{s}", points, mesh, out, dtype, dtype)


def edf_celllist(points, mesh, out=None, dtype=np.float64):
    """ssdf::edf_celllist<G, G, int>: GPU cell list, bitwise the reference's value."""
    s = _suffix(dtype)
    return _edf_call(f"ssdf_b200_edf_celllist_{s}{s}", points, mesh, out, dtype, dtype)


def edf_device(method, x, y, z, s0, s1, s2, sx, sy, sz, out, outtri=None, stream=None):
    """ssdf_edf_device: edf (method 0, brute force) or edf_celllist (1) on torch CUDA tensors; points,
    vertices and out of one float type, out in/out; returns when the query is done."""
    import torch

    ct = F64 if out.dtype == torch.float64 else F32
    _check(lib.ssdf_edf_device(int(method), x.numel(), _dptr(x), _dptr(y), _dptr(z), s0.numel(), _dptr(s0), _dptr(s1),
                               _dptr(s2), sx.numel(), _dptr(sx), _dptr(sy), _dptr(sz), ct, _dptr(out),
                               _dptr(outtri) if outtri is not None else None, _stream_handle(stream)),
           "ssdf_edf_device")


def grown_box(x, y, z, out, stream=None):
    """ssdf_grown_box on torch CUDA tensors: [min(p - r) x3, max(p + r) x3] in the coordinates' type."""
    import torch

    box = torch.empty(6, dtype=x.dtype, device=x.device)
    ct = F64 if x.dtype == torch.float64 else F32
    ot = F64 if out.dtype == torch.float64 else F32
    _check(lib.ssdf_grown_box(x.numel(), _dptr(x), _dptr(y), _dptr(z), _dptr(out), ct, ot, _dptr(box),
                              _stream_handle(stream)), "ssdf_grown_box")
    return box


def triangles_meeting_boxes(s0, s1, s2, sx, sy, sz, boxes, stream=None):
    """ssdf_triangles_meeting_boxes on torch CUDA tensors: (corners [m, 9], counts per box) for the
    boxes [k, 6], each box's triangles in triangle order, box after box."""
    import torch

    k = boxes.shape[0]
    boxes = boxes.contiguous()
    counts = (C.c_longlong * max(k, 1))()
    ct = F64 if sx.dtype == torch.float64 else F32
    args = (s0.numel(), _dptr(s0), _dptr(s1), _dptr(s2), sx.numel(), _dptr(sx), _dptr(sy), _dptr(sz), ct, k,
            _dptr(boxes))
    _check(lib.ssdf_triangles_meeting_boxes(*args, None, 0, counts, _stream_handle(stream)),
           "ssdf_triangles_meeting_boxes")
    total = sum(counts[i] for i in range(k))
    corners = torch.empty((total, 9), dtype=sx.dtype, device=sx.device)
    if total:
        _check(lib.ssdf_triangles_meeting_boxes(*args, _dptr(corners), total, counts, _stream_handle(stream)),
               "ssdf_triangles_meeting_boxes")
    return corners, [int(counts[i]) for i in range(k)]


def edf_bvh(points, mesh, out=None, gdtype=np.float64, tdtype=None):
    """ssdf::edf_bvh<G, T, int> over the device BVH."""
    tdtype = tdtype or gdtype
    return _edf_call(f"ssdf_b200_edf_bvh_{_suffix(gdtype)}{_suffix(tdtype)}", points, mesh, out, gdtype, tdtype)


def edf_index(points, mesh, out=None, dtype=np.float64):
    """Unsigned distance (in/out) and the closest triangle (-1 where nothing improved)."""
    x, y, z = _points(points, dtype)
    tri = np.full(len(x), -1, dtype=np.int32)
    s = _suffix(dtype)
    o = _edf_call(f"ssdf_b200_edf_index_{s}{s}", (x, y, z), mesh, out, dtype, dtype, extra=(_ipp(tri),))
    return o, tri


def sdf_points(points, mesh):
    """Signed distance (double) and closest triangle at a point list."""
    x, y, z = _points(points, np.float64)
    tri = np.full(len(x), -1, dtype=np.int32)
    o = _edf_call("ssdf_b200_sdf_points_dd", (x, y, z), mesh, np.zeros(len(x)), np.float64, np.float64,
                  extra=(_ipp(tri),))
    return o, tri


def closest_point_bvh(points, mesh, outd=None, dtype=np.float64, tdtype=None):
    """ssdf::closest_point_bvh<G, T>: (outd, outx, outy, outz, outtri), updated where closer than outd.
    dtype is G (points, mesh, closest point), tdtype T (distance; G by default)."""
    tdtype = dtype if tdtype is None else tdtype
    x, y, z = _points(points, dtype)
    n = len(x)
    d = _init_out(n, tdtype, outd)
    ox, oy, oz = np.zeros(n, dtype), np.zeros(n, dtype), np.zeros(n, dtype)
    tri = np.full(n, -1, dtype=np.int32)
    hm = _HostMesh(mesh, dtype)
    fn = f"ssdf_b200_closest_point_bvh_{_suffix(dtype)}{_suffix(tdtype)}"
    _check(getattr(lib, fn)(n, _p(x), _p(y), _p(z), *hm.args(), _p(d), _p(ox), _p(oy), _p(oz), _ipp(tri)), fn)
    return d, ox, oy, oz, tri


def closest_within_radius(points, elements, vertices, radius_squared, stride=1, skip_self=False, local=False,
                          gdtype=np.float64, tdtype=None):
    """ssdf::closest_within_radius_bvh / _local_bvh (elements = three index arrays, triangles) and
    _quads_bvh / _quads_local_bvh (four arrays, quads) on the GPU. Returns (outtri, out_sqr_dist,
    closest_x, closest_y, closest_z), or (outtri, out_sqr_dist, closest_s, closest_t) when local."""
    tdtype = gdtype if tdtype is None else tdtype
    x, y, z = _points(points, gdtype)
    sx, sy, sz = (_arr(a, gdtype) for a in vertices)
    idx = [_arr(a, np.int32) for a in elements]
    if len(idx) not in (3, 4):
        raise ValueError("elements: three (triangles) or four (quads) index arrays")
    r2 = _arr(radius_squared, tdtype)
    n = len(x)
    need = (stride * (n - 1) + 1) if n else 0
    if stride < 0 or len(r2) < need:
        raise ValueError(f"radius_squared holds {len(r2)} values; stride {stride} over {n} points needs {need}")
    outtri = np.empty(n, dtype=np.int32)
    outs = [np.empty(n, dtype=tdtype) for _ in range(3 if local else 4)]
    kind = ("quads_" if len(idx) == 4 else "") + ("local_" if local else "") + "bvh"
    fn = f"ssdf_b200_closest_within_radius_{kind}_{_suffix(gdtype)}{_suffix(tdtype)}"
    _check(getattr(lib, fn)(n, _p(x), _p(y), _p(z), len(idx[0]), *[_ipp(a) for a in idx], len(sx), _p(sx), _p(sy),
                            _p(sz), int(stride), _p(r2), _ipp(outtri), *[_p(a) for a in outs], int(bool(skip_self))),
           fn)
    return (outtri, *outs)


def potential_contact(elements, vertices, extrusion, dtype=np.float64):
    """ssdf::potential_contact_triangles_bvh (three index arrays) / potential_contact_quads_bvh (four)
    on the GPU: (pc_ptr int64 [n + 1], pc_idx int32 [pc_ptr[n]]), each row in the BVH walk's order."""
    sx, sy, sz = (_arr(a, dtype) for a in vertices)
    idx = [_arr(a, np.int32) for a in elements]
    if len(idx) not in (3, 4):
        raise ValueError("elements: three (triangles) or four (quads) index arrays")
    n = len(idx[0])
    ptr = np.full(n + 1, -7, dtype=np.int64)
    out = _ip()
    kind = "quads" if len(idx) == 4 else "triangles"
    fn = f"ssdf_b200_potential_contact_{kind}_bvh_{_suffix(dtype) * 2}"
    _check(getattr(lib, fn)(n, *[_ipp(a) for a in idx], len(sx), _p(sx), _p(sy), _p(sz), float(extrusion),
                            ptr.ctypes.data_as(C.POINTER(C.c_ssize_t)), C.byref(out)), fn)
    try:
        pairs = np.ctypeslib.as_array(out, shape=(int(ptr[n]),)).copy() if ptr[n] > 0 else np.zeros(0, np.int32)
    finally:
        lib.ssdf_b200_free(C.cast(out, _vp))
    return ptr, pairs


def points_inside_bvh(points, mesh, dtype=np.float64):
    """ssdf::points_inside_bvh on the GPU: uint8 flags, 1 inside the closed surface."""
    x, y, z = _points(points, dtype)
    out = np.empty(len(x), dtype=np.uint8)
    hm = _HostMesh(mesh, dtype)
    fn = f"ssdf_b200_points_inside_bvh_{_suffix(dtype)}"
    _check(getattr(lib, fn)(len(x), _p(x), _p(y), _p(z), *hm.args(), _p(out)), fn)
    return out


def sample_inside_bvh(mesh, grid, dtype=np.float64):
    """ssdf::sample_inside_bvh on the GPU: uint8 flags on the node grid."""
    hm = _HostMesh(mesh, dtype)
    out = np.empty(grid.size, dtype=np.uint8)
    fn = f"ssdf_b200_sample_inside_bvh_{_suffix(dtype)}"
    ct = C.c_double if np.dtype(dtype) == np.float64 else C.c_float
    nx, ny, nz = grid.n
    _check(getattr(lib, fn)(*hm.args(), nx, ny, nz, *[ct(v) for v in grid.lo], *[ct(v) for v in grid.hi], _p(out)), fn)
    return out


def compute_aabb(points, gdtype=np.float64, tdtype=None):
    """ssdf::compute_aabb<G, T> (serial/edf/edf.hpp:500-539) on the GPU: the bounding box of the points
    as (xmin, xmax, ymin, ymax, zmin, zmax) in T."""
    tdtype = gdtype if tdtype is None else tdtype
    x, y, z = _points(points, gdtype)
    tc = C.c_double if np.dtype(tdtype) == np.float64 else C.c_float
    v = [tc() for _ in range(6)]
    fn = f"ssdf_b200_compute_aabb_{_suffix(gdtype)}{_suffix(tdtype)}"
    _check(getattr(lib, fn)(len(x), _p(x), _p(y), _p(z), *[C.byref(a) for a in v]), fn)
    return tuple(np.dtype(tdtype).type(a.value) for a in v)


def all_points_aabb_signed_distance(points, box, gdtype=np.float64, tdtype=None):
    """ssdf::all_points_aabb_signed_distance<G, T> (serial/edf/edf.hpp:541-557) on the GPU: each point's
    signed distance to box = (minx, maxx, miny, maxy, minz, maxz), negative inside."""
    tdtype = gdtype if tdtype is None else tdtype
    x, y, z = _points(points, gdtype)
    out = np.empty(len(x), dtype=tdtype)
    fn = f"ssdf_b200_all_points_aabb_signed_distance_{_suffix(gdtype)}{_suffix(tdtype)}"
    _check(getattr(lib, fn)(len(x), _p(x), _p(y), _p(z), *[float(b) for b in box], _p(out)), fn)
    return out


class GridGeometry:
    """ssdf::GridGeometry<G> (serial/bvh/sdf_rebuild.hpp:10-21): n[d] samples at o[d] + i h[d], x fastest."""

    def __init__(self, n, o, h, dtype=np.float64):
        self.n = tuple(int(v) for v in n)
        self.dtype = np.dtype(dtype)
        self.o = tuple(self.dtype.type(v) for v in o)
        self.h = tuple(self.dtype.type(v) for v in h)

    @property
    def size(self):
        return self.n[0] * self.n[1] * self.n[2]

    def strided(self, stride):
        t = self.dtype.type
        return GridGeometry([(v - 1) // stride + 1 for v in self.n], self.o, [t(v * t(stride)) for v in self.h], self.dtype)

    def refined(self, factor):
        return GridGeometry([(v - 1) * factor + 1 for v in self.n], self.o,
                            [self.dtype.type(float(v) / float(factor)) for v in self.h], self.dtype)

    def _args(self):
        ct = C.c_double if self.dtype == np.float64 else C.c_float
        return [C.byref((C.c_ssize_t * 3)(*self.n)), C.byref((ct * 3)(*self.o)), C.byref((ct * 3)(*self.h))]

    def _suffix(self):
        return "dd" if self.dtype == np.float64 else "ff"


def level_set_triangles(grid: GridGeometry, f, level):
    """ssdf::level_set_triangles on the GPU: the triangle soup (3, 3 * ntri) of {f = level}."""
    fa = _arr(f, grid.dtype)
    fn = f"ssdf_b200_level_set_triangles_{grid._suffix()}"
    nt = C.c_ssize_t(0)
    _check(getattr(lib, fn)(*grid._args(), _p(fa), float(level), 0, None, None, None, C.byref(nt)), fn)
    x, y, z = (np.empty(3 * nt.value, dtype=grid.dtype) for _ in range(3))
    if nt.value:
        _check(getattr(lib, fn)(*grid._args(), _p(fa), float(level), nt.value, _p(x), _p(y), _p(z), C.byref(nt)), fn)
    return np.stack([x, y, z])


def rebuild_sdf(grid: GridGeometry, f, level, band, stride=1):
    """ssdf::rebuild_sdf on the GPU: signed distance to {f = level} within band on grid.strided(stride)."""
    fa = _arr(f, grid.dtype)
    out = np.empty(grid.strided(stride).size, dtype=grid.dtype)
    fn = f"ssdf_b200_rebuild_sdf_{grid._suffix()}"
    _check(getattr(lib, fn)(*grid._args(), _p(fa), float(level), float(band), int(stride), _p(out)), fn)
    return out


def refine_field(grid: GridGeometry, f, factor):
    """ssdf::refine_field on the GPU: f on grid.refined(factor), cubic along each axis in turn."""
    fa = _arr(f, grid.dtype)
    fine = np.empty(grid.refined(factor).size, dtype=grid.dtype)
    fn = f"ssdf_b200_refine_field_{grid._suffix()}"
    _check(getattr(lib, fn)(*grid._args(), _p(fa), int(factor), _p(fine)), fn)
    return fine


def round_sdf(grid: GridGeometry, f, radius, band, open=True, close=True, stride=1, with_f0=False):
    """ssdf::round_sdf on the GPU: the region f > 0 rounded by radius, its signed distance strided."""
    fa = _arr(f, grid.dtype)
    out = np.empty(grid.strided(stride).size, dtype=grid.dtype)
    f0 = np.empty(grid.size, dtype=grid.dtype) if with_f0 else None
    fn = f"ssdf_b200_round_sdf_{grid._suffix()}"
    _check(getattr(lib, fn)(*grid._args(), _p(fa), float(radius), float(band), int(open), int(close), int(stride),
                            _p(out), _p(f0) if with_f0 else None), fn)
    return (out, f0) if with_f0 else out


def _grid_call(fn, mesh, grid, out, dtype, extra=()):
    nx, ny, nz = (int(v) for v in grid.n)
    hm = _HostMesh(mesh, dtype)
    ct = C.c_double if np.dtype(dtype) == np.float64 else C.c_float
    bounds = [ct(v) for v in grid.lo] + [ct(v) for v in grid.hi]
    _check(getattr(lib, fn)(*hm.args(), nx, ny, nz, *bounds, _p(out), *extra), fn)
    return out


def sample_sqedf_bvh(mesh, grid, out=None, dtype=np.float64):
    """ssdf::sample_sqedf_bvh: squared distance on the node grid, min with the incoming out."""
    o = _init_out(grid.size, dtype, out)
    s = _suffix(dtype)
    return _grid_call(f"ssdf_b200_sample_sqedf_bvh_{s}{s}", mesh, grid, o, dtype)


def sample_sdf_bvh(mesh, grid, dtype=np.float64, with_index=False):
    """ssdf::sample_sdf_bvh: signed distance on the node grid (x fastest)."""
    o = np.zeros(grid.size, dtype=dtype)
    s = _suffix(dtype)
    if with_index:
        if s != "d":
            raise ValueError("the indexed grid sampler is double only")
        tri = np.full(grid.size, -1, dtype=np.int32)
        _grid_call("ssdf_b200_sample_sdf_index_bvh_dd", mesh, grid, o, dtype, extra=(_ipp(tri),))
        return o, tri
    return _grid_call(f"ssdf_b200_sample_sdf_bvh_{s}{s}", mesh, grid, o, dtype)


def fma_peak_tflops(f64: bool = False) -> float:
    """Measured FMA throughput of the current GPU (TFLOP/s)."""
    v = C.c_double()
    _check(lib.ssdf_b200_fma_peak(int(f64), C.byref(v)), "ssdf_b200_fma_peak")
    return v.value


def last_query_counts():
    v = [C.c_int64() for _ in range(4)]
    _check(lib.ssdf_last_query_counts(*[C.byref(a) for a in v]), "ssdf_last_query_counts")
    return dict(triangle_tests=v[0].value, box_tests=v[1].value, fixup_evaluations=v[2].value,
                fallback_queries=v[3].value)


# ----------------------------------------------------------------------------------------------
# device-resident meshes
# ----------------------------------------------------------------------------------------------

def _dptr(t) -> int:
    """Device pointer of a torch tensor (or an int pointer)."""
    if t is None:
        return None
    if isinstance(t, int):
        return t
    return t.data_ptr()


def _stream_handle(stream) -> int:
    if stream is None:
        return 0
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _dtype_code(t) -> int:
    import torch

    if t.dtype == torch.float64:
        return F64
    if t.dtype == torch.float32:
        return F32
    raise TypeError(f"unsupported dtype {t.dtype}")


def points_aabb_device(x, y, z, box6, stream=None):
    """Device form of compute_aabb: torch tensors x, y, z (one float dtype) in, the six extremes
    (xmin, xmax, ymin, ymax, zmin, zmax) written to the device tensor box6 (its dtype is T)."""
    _check(lib.ssdf_points_aabb(x.numel(), _dptr(x), _dptr(y), _dptr(z), _dtype_code(x), _dtype_code(box6),
                                _dptr(box6), _stream_handle(stream)), "ssdf_points_aabb")


def points_aabb_signed_distance_device(x, y, z, box, out, absolute=False, stream=None):
    """Device form of all_points_aabb_signed_distance: out (device, T) gets each point's signed (or,
    with absolute, unsigned) distance to box = (minx, maxx, miny, maxy, minz, maxz)."""
    b = (C.c_double * 6)(*[float(v) for v in box])
    _check(lib.ssdf_points_aabb_signed_distance(x.numel(), _dptr(x), _dptr(y), _dptr(z), _dtype_code(x), C.byref(b),
                                                int(bool(absolute)), _dptr(out), _dtype_code(out),
                                                _stream_handle(stream)), "ssdf_points_aabb_signed_distance")


RESIDENT_TREELET_ROUNDS = 3  # treelet rounds of a resident mesh's BVH (the library's default)


class DeviceMesh:
    """A mesh, its BVH and (optionally) pseudo-normals, resident on the current GPU. ``treelet``: rounds
    of SAH treelet refinement (True: the resident default, 3; False: none)."""

    def __init__(self, mesh, coord_dtype=np.float64, leaf_size=0, keep_fp64=True, normals=True, treelet=True,
                 stream=None):
        hm = _HostMesh(mesh, coord_dtype)
        self._h = C.c_void_p()
        rounds = RESIDENT_TREELET_ROUNDS if treelet is True else int(treelet)
        opts = BuildOpts(int(leaf_size), int(keep_fp64), int(normals), rounds)
        ct = F64 if np.dtype(coord_dtype) == np.float64 else F32
        _check(lib.ssdf_mesh_create(C.byref(self._h), *hm.args(), ct, 0, C.byref(opts), _stream_handle(stream)),
               "ssdf_mesh_create")
        self.nt = mesh.nt
        self.nv = mesh.nv

    @classmethod
    def from_device(cls, s0, s1, s2, sx, sy, sz, keep_fp64=True, normals=False, leaf_size=0, treelet=True,
                    stream=None):
        """A mesh from device arrays (torch CUDA tensors: int32 indices, one float dtype for the
        vertices), built without a host round trip."""
        self = cls.__new__(cls)
        self._h = C.c_void_p()
        opts = BuildOpts(int(leaf_size), int(keep_fp64), int(normals), int(treelet))
        _check(lib.ssdf_mesh_create(C.byref(self._h), s0.numel(), C.cast(C.c_void_p(_dptr(s0)), _ip),
                                    C.cast(C.c_void_p(_dptr(s1)), _ip), C.cast(C.c_void_p(_dptr(s2)), _ip),
                                    sx.numel(), _dptr(sx), _dptr(sy), _dptr(sz), _dtype_code(sx), 1, C.byref(opts),
                                    _stream_handle(stream)), "ssdf_mesh_create")
        self.nt = s0.numel()
        self.nv = sx.numel()
        return self

    def close(self):
        if self._h:
            lib.ssdf_mesh_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stats(self):
        v = [C.c_int64() for _ in range(4)]
        _check(lib.ssdf_mesh_stats(self._h, *[C.byref(a) for a in v]), "ssdf_mesh_stats")
        return dict(nodes=v[0].value, leaves=v[1].value, depth=v[2].value, bytes=v[3].value)

    def filter_info(self):
        """The fix-up path's view of the mesh: window width tau_rel, whether fix-up requests run the FP32
        filter (else the FP64 kernel), and how many triangles the filter sees through a proxy."""
        t, ok, n = C.c_float(), C.c_int(), C.c_int64()
        _check(lib.ssdf_mesh_filter_info(self._h, C.byref(t), C.byref(ok), C.byref(n)), "ssdf_mesh_filter_info")
        return dict(tau_rel=t.value, float_filter=bool(ok.value), slivers=n.value)

    def query_points(self, x, y, z, out, outtri=None, outx=None, outy=None, outz=None, precision=PREC_F32_FIXUP,
                     output=OUT_EDF, coord_type=F64, out_type=F64, stream=None):
        o = QueryOpts(precision, output, coord_type, out_type)
        tri = C.cast(C.c_void_p(_dptr(outtri)), _ip) if outtri is not None else None
        _check(lib.ssdf_query_points(self._h, int(x.numel() if hasattr(x, "numel") else len(x)), _dptr(x), _dptr(y),
                                     _dptr(z), _dptr(out), tri, _dptr(outx), _dptr(outy), _dptr(outz), C.byref(o),
                                     _stream_handle(stream)), "ssdf_query_points")

    def query_grid(self, grid, out, outtri=None, precision=PREC_F32_FIXUP, output=OUT_SDF, coord_type=F64,
                   out_type=F64, stream=None):
        o = QueryOpts(precision, output, coord_type, out_type)
        lo = (C.c_double * 3)(*grid.lo)
        hi = (C.c_double * 3)(*grid.hi)
        tri = C.cast(C.c_void_p(_dptr(outtri)), _ip) if outtri is not None else None
        nx, ny, nz = (int(v) for v in grid.n)
        _check(lib.ssdf_query_grid(self._h, nx, ny, nz, C.byref(lo), C.byref(hi), _dptr(out), tri, C.byref(o),
                                   _stream_handle(stream)), "ssdf_query_grid")


class Batch:
    """Many (resident mesh, query set) jobs run in one persistent launch, optionally as a CUDA graph."""

    def __init__(self, max_jobs, precision=PREC_F32_FIXUP, traversal=0, arity=0):
        self._h = C.c_void_p()
        self.precision = precision
        _check(lib.ssdf_batch_create(C.byref(self._h), int(max_jobs), int(precision), int(traversal), int(arity)),
               "ssdf_batch_create")
        self._keep = []

    def close(self):
        if self._h:
            lib.ssdf_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reserve(self, max_queries, stream=None):
        """Pre-size the fix-up overflow lists for runs of up to max_queries queries."""
        _check(lib.ssdf_batch_reserve(self._h, int(max_queries), _stream_handle(stream)), "ssdf_batch_reserve")

    def clear(self):
        _check(lib.ssdf_batch_clear(self._h), "ssdf_batch_clear")
        self._keep = []

    def __len__(self):
        return lib.ssdf_batch_size(self._h)

    def add_grid(self, mesh: "DeviceMesh", grid, out, outtri=None, output=OUT_SDF, coord_type=F64, out_type=F64):
        o = QueryOpts(self.precision, output, coord_type, out_type)
        lo = (C.c_double * 3)(*grid.lo)
        hi = (C.c_double * 3)(*grid.hi)
        tri = C.cast(C.c_void_p(_dptr(outtri)), _ip) if outtri is not None else None
        nx, ny, nz = (int(v) for v in grid.n)
        _check(lib.ssdf_batch_add_grid(self._h, mesh._h, nx, ny, nz, C.byref(lo), C.byref(hi), _dptr(out), tri,
                                       C.byref(o)), "ssdf_batch_add_grid")
        self._keep.append((mesh, out, outtri))

    def add_grid_slab(self, mesh: "DeviceMesh", grid, z0, nz, out, outtri=None, output=OUT_SDF, coord_type=F64,
                      out_type=F64):
        """The z-planes z0 .. z0 + nz - 1 of grid as one job, with the whole grid's node coordinates."""
        o = QueryOpts(self.precision, output, coord_type, out_type)
        lo = (C.c_double * 3)(*grid.lo)
        hi = (C.c_double * 3)(*grid.hi)
        tri = C.cast(C.c_void_p(_dptr(outtri)), _ip) if outtri is not None else None
        gx, gy, gz = (int(v) for v in grid.n)
        _check(lib.ssdf_batch_add_grid_slab(self._h, mesh._h, gx, gy, gz, C.byref(lo), C.byref(hi), int(z0), int(nz),
                                            _dptr(out), tri, C.byref(o)), "ssdf_batch_add_grid_slab")
        self._keep.append((mesh, out, outtri))

    def add_points(self, mesh: "DeviceMesh", x, y, z, out, outtri=None, output=OUT_SDF, coord_type=F64, out_type=F64):
        o = QueryOpts(self.precision, output, coord_type, out_type)
        tri = C.cast(C.c_void_p(_dptr(outtri)), _ip) if outtri is not None else None
        _check(lib.ssdf_batch_add_points(self._h, mesh._h, int(x.numel()), _dptr(x), _dptr(y), _dptr(z), _dptr(out),
                                         tri, C.byref(o)), "ssdf_batch_add_points")
        self._keep.append((mesh, x, y, z, out, outtri))

    def run(self, use_graph=True, stream=None):
        _check(lib.ssdf_batch_run(self._h, int(bool(use_graph)), _stream_handle(stream)), "ssdf_batch_run")

    def last_blocks(self) -> int:
        return int(lib.ssdf_batch_last_blocks(self._h))


class Server:
    """Continuous-batching request loop over resident meshes (host arrays in and out)."""

    def __init__(self, memory_budget=120 << 30, max_batch_queries=1 << 22, max_batch_jobs=64,
                 precision=PREC_F32_FIXUP, leaf_size=0, slots=0, max_queued_queries=0, split_queries=0):
        self._h = C.c_void_p()
        o = ServerOpts(int(memory_budget), int(max_batch_queries), int(max_batch_jobs), int(precision),
                       int(leaf_size), int(slots), int(max_queued_queries), int(split_queries))
        _check(lib.ssdf_server_create(C.byref(self._h), C.byref(o)), "ssdf_server_create")
        self._inflight = {}

    def close(self):
        if self._h:
            lib.ssdf_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_mesh(self, mesh) -> int:
        hm = _HostMesh(mesh, np.float64)
        mid = C.c_int()
        _check(lib.ssdf_server_add_mesh(self._h, *hm.args(), C.byref(mid)), "ssdf_server_add_mesh")
        return mid.value

    def submit_points(self, mesh_id, points):
        x, y, z = _points(points, np.float64)
        out = np.empty(len(x))
        tri = np.empty(len(x), dtype=np.int32)
        t = C.c_longlong()
        _check(lib.ssdf_server_submit_points(self._h, int(mesh_id), len(x), _p(x), _p(y), _p(z), _p(out), _ipp(tri),
                                             C.byref(t)), "ssdf_server_submit_points")
        self._inflight[t.value] = (x, y, z, out, tri)
        return t.value

    def submit_grid(self, mesh_id, grid):
        out = np.empty(grid.size)
        tri = np.empty(grid.size, dtype=np.int32)
        lo = (C.c_double * 3)(*grid.lo)
        hi = (C.c_double * 3)(*grid.hi)
        t = C.c_longlong()
        _check(lib.ssdf_server_submit_grid(self._h, int(mesh_id), *(int(v) for v in grid.n), C.byref(lo), C.byref(hi),
                                           _p(out), _ipp(tri), C.byref(t)), "ssdf_server_submit_grid")
        self._inflight[t.value] = (out, tri)
        return t.value

    def wait(self, ticket, timeout=120.0):
        _check(lib.ssdf_server_wait(self._h, int(ticket), float(timeout)), "ssdf_server_wait")
        arrays = self._inflight.pop(ticket)
        return arrays[-2], arrays[-1]

    def stats(self):
        st = ServerStats()
        _check(lib.ssdf_server_stats(self._h, C.byref(st)), "ssdf_server_stats")
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}

    def reset_stats(self):
        _check(lib.ssdf_server_reset_stats(self._h), "ssdf_server_reset_stats")


def autotune_grid(mesh, grid, precision=PREC_F32_FIXUP, cache_path=None):
    """Fastest (leaf_size, traversal, arity) for this mesh and grid; cached per size class."""
    hm = _HostMesh(mesh, np.float64)
    lo = (C.c_double * 3)(*grid.lo)
    hi = (C.c_double * 3)(*grid.hi)
    t = Tuning()
    path = cache_path.encode() if cache_path else None
    _check(lib.ssdf_autotune_grid(*hm.args(), *(int(v) for v in grid.n), C.byref(lo), C.byref(hi), int(precision),
                                  path, C.byref(t)), "ssdf_autotune_grid")
    return dict(leaf_size=t.leaf_size, traversal=t.traversal, arity=t.arity, ms=t.ms)

