"""The C ABI library loads and exports every function include/pysweep_b200.h
declares (no device calls), and the host-side helpers mirror the reference."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    hdr = open(os.path.join(ROOT, "include", "pysweep_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(ps_[a-z_]+)\s*\(", hdr)))


def test_library_exports_header_symbols():
    from pysweep_b200 import _lib
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = _declared()
    assert names, "no declarations found"
    for n in names:
        assert hasattr(L, n), f"{n} declared but not exported"
    assert set(names) == set(_lib.exported_symbols())


def test_version_and_create_error_without_gpu_call():
    from pysweep_b200 import _lib
    L = _lib.lib()
    assert L.ps_version().startswith(b"pysweep_b200")
    # invalid arguments are rejected before any CUDA call
    h = ctypes.c_void_p()
    rc = L.ps_create(ctypes.byref(h), 0, 0, 1, 48, 48, 1, 1, 7)  # bs 7: not a multiple of 2*ops
    assert rc == -1
    assert b"blocksize" in L.ps_last_error(None)
    rc = L.ps_create(ctypes.byref(h), 0, 1, 4, 64, 64, 2, 1, 16)  # euler with its=1
    assert rc == -1


def test_plugin_constants_follow_set_globals():
    from pysweep_b200 import plugin_constants
    c = plugin_constants("heat", [0, 1, 0.1, 0.5, 0.5, 2.0, True])
    assert c == {"DT": 0.1, "DX": 0.5, "DY": 0.5, "ALPHA": 2.0, "SCHEME": True}
    c = plugin_constants("euler", [0, 1, 0.1, 0.5, 0.25, 1.4])
    assert c["GAM_M1"] == 1.4 - 1 and c["DTDX"] == 0.1 / 0.5 and c["DTDY"] == 0.1 / 0.25


def test_package_exports_the_documented_names():
    """The names the integration notes use are importable from the package."""
    import pysweep_b200
    for name in ("Solver", "Engine", "Batch", "plugin_constants", "PySweepError"):
        assert hasattr(pysweep_b200, name), name
    from pysweep_b200.adjoint import heat_solve  # noqa: F401
    from pysweep_b200.autotune import tune  # noqa: F401
    from pysweep_b200.distributed import SlabSolver  # noqa: F401
