"""ssdf_b200 -- closest-point distance fields on one NVIDIA B200 (sm_100a).

The binding over the CUDA library lives in :mod:`ssdf_b200.capi` and is loaded on first use of
any of its names from this package (``ssdf_b200.edf_select(...)``, ``ssdf_b200.DeviceMesh``...):
it raises ImportError if ``_lib/libssdf_b200.so`` is not built -- there is no CPU path.
:mod:`ssdf_b200.build` (the nvcc build) and :mod:`ssdf_b200.workloads` (seeded synthetic inputs)
import without the library.
"""

from __future__ import annotations

import importlib

# submodules that import without the CUDA library (``from ssdf_b200 import build`` must work on a
# fresh checkout, before the library exists)
_LIBRARY_FREE = ("build", "workloads")


def __getattr__(name):
    if name.startswith("__"):
        raise AttributeError(name)
    if name in _LIBRARY_FREE:
        return importlib.import_module("." + name, __name__)
    capi = importlib.import_module(".capi", __name__)
    return capi if name == "capi" else getattr(capi, name)
