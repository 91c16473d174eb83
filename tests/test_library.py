"""CPU checks of the boundary: the library builds, loads and exports every entry point that
include/ssdf_b200.h declares; status names; no compute call is made without a GPU."""

import os
import re

import pytest

from conftest import ROOT


def declared_functions():
    src = open(os.path.join(ROOT, "include", "ssdf_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ssdf_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    import ssdf_b200.capi as capi

    names = declared_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(capi.lib, n), n
        assert n in capi.EXPORTED, n


def test_status_strings():
    import ssdf_b200 as S

    assert S.lib.ssdf_status_string(0) == b"SSDF_OK"
    assert S.lib.ssdf_status_string(1) == b"SSDF_ERR_INVALID_ARGUMENT"
    assert S.version().startswith("ssdf_b200")


def test_cpp_header_compiles_against_c_abi(tmp_path):
    """include/ssdf.hpp (the C++ drop-in templates) compiles and links against the library."""
    import subprocess

    src = tmp_path / "use.cpp"
    src.write_text(
        '#include "bvh/sdf_rebuild.hpp"\n'
        '#include "ssdf.hpp"\n'
        "int main() {\n"
        "  double x[1] = {0}, y[1] = {0}, z[1] = {2}, sx[3] = {0, 1, 0}, sy[3] = {0, 0, 1}, sz[3] = {0, 0, 0};\n"
        "  int s0[1] = {0}, s1[1] = {1}, s2[1] = {2};\n"
        "  double out[1] = {1e300};\n"
        "  (void)ssdf::edf_select<double, double, int>(1, x, y, z, 1, s0, s1, s2, 3, sx, sy, sz, out);\n"
        "  (void)ssdf::edf<double, double, int>;\n"
        "  (void)ssdf::edf_celllist<float, float, int>;\n"
        "  (void)ssdf::edf_bvh<float, double, int>;\n"
        "  (void)ssdf::closest_point_bvh<double, double, int>;\n"
        "  (void)ssdf::closest_point_bvh<float, double, int>;\n"
        "  (void)ssdf::closest_point_bvh<float, float, int>;\n"
        "  (void)ssdf::edf_bvh<float, float, int>;\n"
        "  (void)ssdf::edf_bvh<double, double, int>;\n"
        "  (void)ssdf::sample_sdf_bvh<double, double, int>;\n"
        "  (void)ssdf::sample_sqedf_bvh<float, float, int>;\n"
        "  (void)ssdf::sample_sdf_bvh<float, float, int>;\n"
        "  (void)ssdf::sample_sqedf_bvh<double, double, int>;\n"
        "  (void)ssdf::compute_aabb<float, double>;\n"
        "  (void)ssdf::all_points_aabb_signed_distance<double, double>;\n"
        "  ssdf::GridGeometry<float> g{{4, 4, 4}, {0, 0, 0}, {0.5f, 0.5f, 0.5f}};\n"
        "  std::vector<float> vx, vy, vz;\n"
        "  (void)&ssdf::level_set_triangles<float, float>;\n"
        "  (void)ssdf::rebuild_sdf<double, double>;\n"
        "  (void)ssdf::refine_field<float, float>;\n"
        "  (void)ssdf::round_sdf<double, double>;\n"
        "  (void)g.strided(2).refined(2).size();\n"
        "  int q3[1] = {2}, tri[1];\n"
        "  double r2[1] = {1.0}, d2[1], cx[1], cy[1], cz[1];\n"
        "  float fx[1] = {0}, fy[1] = {0}, fz[1] = {2}, fsx[3] = {0, 1, 0}, fsy[3] = {0, 0, 1}, fsz[3] = {0, 0, 0};\n"
        "  (void)ssdf::closest_within_radius_bvh<double, double, int>(1, x, y, z, 1, s0, s1, s2, 3, sx, sy, sz, 1, r2,\n"
        "      tri, d2, cx, cy, cz);\n"
        "  (void)ssdf::closest_within_radius_local_bvh<float, double, int>(1, fx, fy, fz, 1, s0, s1, s2, 3, fsx, fsy,\n"
        "      fsz, 0, r2, tri, d2, cx, cy, true);\n"
        "  (void)ssdf::closest_within_radius_quads_bvh<float, double, int>(1, fx, fy, fz, 1, s0, s1, s2, q3, 3, fsx,\n"
        "      fsy, fsz, 1, r2, tri, d2, cx, cy, cz);\n"
        "  (void)ssdf::closest_within_radius_quads_local_bvh<double, double, int>(1, x, y, z, 1, s0, s1, s2, q3, 3, sx,\n"
        "      sy, sz, 1, r2, tri, d2, cx, cy);\n"
        "  ptrdiff_t pc[2]; int *pci = nullptr;\n"
        "  (void)ssdf::potential_contact_triangles_bvh<float, float, int, int>(1, s0, s1, s2, 3, fsx, fsy, fsz, 0.1f,\n"
        "      pc, &pci);\n"
        "  (void)ssdf::potential_contact_quads_bvh<double, double, int, int>(1, s0, s1, s2, q3, 3, sx, sy, sz, 0.1, pc,\n"
        "      &pci);\n"
        "  ssdf_b200_free(pci);\n"
        "  // every explicit instantiation of serial/bvh/bvh.cpp:1162-1981\n"
        "  (void)&ssdf::points_inside_bvh<float, int>;\n"
        "  (void)&ssdf::sample_inside_bvh<float, int>;\n"
        "  (void)&ssdf::sample_inside_bvh<double, int>;\n"
        "  (void)&ssdf::closest_within_radius_bvh<float, double, int>;\n"
        "  (void)&ssdf::closest_within_radius_bvh<float, float, int>;\n"
        "  (void)&ssdf::closest_within_radius_local_bvh<float, float, int>;\n"
        "  (void)&ssdf::closest_within_radius_local_bvh<double, double, int>;\n"
        "  (void)&ssdf::closest_within_radius_quads_bvh<float, float, int>;\n"
        "  (void)&ssdf::closest_within_radius_quads_bvh<double, double, int>;\n"
        "  (void)&ssdf::closest_within_radius_quads_local_bvh<float, float, int>;\n"
        "  (void)&ssdf::closest_within_radius_quads_local_bvh<float, double, int>;\n"
        "  (void)&ssdf::potential_contact_triangles_bvh<double, double, int, int>;\n"
        "  (void)&ssdf::potential_contact_quads_bvh<float, float, int, int>;\n"
        "  (void)&ssdf::sample_sdf_bvh<double, double, int>;\n"
        "  (void)&ssdf::sample_sqedf_bvh<float, float, int>;\n"
        "  return 0;\n}\n")
    lib = os.path.join(ROOT, "ssdf_b200", "_lib")
    res = subprocess.run(["g++", "-std=c++17", f"-I{ROOT}/include", str(src), "-o", str(tmp_path / "use"),
                          f"-L{lib}", "-lssdf_b200", f"-Wl,-rpath,{lib}"], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr


def test_distributed_header_compiles_against_c_abi(tmp_path):
    """include/ssdf_distributed.hpp (pedf / pedf_update over an NCCL communicator) compiles and links."""
    import subprocess

    src = tmp_path / "dist.cpp"
    src.write_text(
        '#include "ssdf_distributed.hpp"\n'
        "int main() {\n"
        "  (void)&ssdf::pedf<double, double, int>;\n"
        "  (void)&ssdf::pedf<float, double, int>;\n"
        "  (void)&ssdf::pedf_update<float, float, int>;\n"
        "  (void)&ssdf::pedf_update<double, double, int>;\n"
        "  return 0;\n}\n")
    lib = os.path.join(ROOT, "ssdf_b200", "_lib")
    res = subprocess.run(["g++", "-std=c++17", f"-I{ROOT}/include", "-I/usr/local/cuda/include", str(src), "-o",
                          str(tmp_path / "dist"), f"-L{lib}", "-lssdf_b200", f"-Wl,-rpath,{lib}"],
                         capture_output=True, text=True)
    assert res.returncode == 0, res.stderr


def test_build_imports_without_the_library():
    """``from ssdf_b200 import build`` (the first step of a fresh build) must not load the CUDA
    binding, which needs the library it is about to build."""
    import subprocess
    import sys

    code = ("import sys; from ssdf_b200 import build, workloads; "
            "assert 'ssdf_b200.capi' not in sys.modules, 'binding loaded'")
    res = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    # the binding module itself is reachable as an attribute on first use
    code = "import ssdf_b200 as S; assert S.capi.lib is not None; assert S.version() == S.capi.version()"
    res = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr


def test_radius_queries_validate_on_the_host():
    """closest_within_radius_*: bad indices and sizes are rejected before any device work, and an
    empty point set returns at once (neither needs a GPU)."""
    import numpy as np

    import ssdf_b200 as S

    pts = np.zeros((3, 4))
    verts = np.zeros((3, 3))
    tri = [np.array([0]), np.array([1]), np.array([3])]
    with pytest.raises(S.SsdfError) as e:
        S.closest_within_radius(pts, tri, verts, np.ones(4))
    assert e.value.status == S.SSDF_ERR_INVALID_ARGUMENT
    quad = [np.array([0]), np.array([1]), np.array([2]), np.array([-1])]
    with pytest.raises(S.SsdfError):
        S.closest_within_radius(pts, quad, verts, np.ones(4), local=True, gdtype=np.float32)
    out = S.closest_within_radius(np.zeros((3, 0)), [np.array([0]), np.array([1]), np.array([2])], verts, np.ones(0))
    assert len(out) == 5 and len(out[0]) == 0
    with pytest.raises(ValueError):
        S.closest_within_radius(pts, [np.array([0]), np.array([1]), np.array([2])], verts, np.ones(2))
    bad = [np.array([0]), np.array([1]), np.array([5])]
    with pytest.raises(S.SsdfError) as e:
        S.potential_contact(bad, verts, 0.1)
    assert e.value.status == S.SSDF_ERR_INVALID_ARGUMENT
