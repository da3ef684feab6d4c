"""The drop-in Solver driven by the reference's own CPU plugin file.

When PYSWEEP_REFERENCE_PLUGINS names a directory holding the reference's
plugin modules (pysweep/equations/heat.py and its siblings; they are not part
of this repository), the Solver imports heat.py from there as `cpu:`, as the
reference's solver does (pysweep/core/solver.py:83-87), and its
set_globals(*globals, source_mod=...) sets the device constants through the
SourceModule stand-in (heat.py:33-46).  Modules that the plugin imports at
load time but that this image lacks (mpi4py, h5py, matplotlib, pycuda) are
stood in for by empty modules for the duration of the test; the plugin's CPU
step is not called.  The result must equal the run configured by the
repository's own restatement of the plugin, bitwise.
"""
import os
import sys
import types

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REF = os.environ.get("PYSWEEP_REFERENCE_PLUGINS", "")
HERE = os.path.dirname(os.path.abspath(__file__))


def _stub_missing(names):
    """Empty modules for the names that do not import; returns what to undo."""
    added = []
    for name in names:
        try:
            __import__(name)
        except Exception:
            mod = types.ModuleType(name)
            if name == "mpi4py":
                mod.rc = types.SimpleNamespace(recv_mprobe=False)
            if name == "matplotlib":
                mod.rc = lambda *a, **k: None
            sys.modules[name] = mod
            added.append(name)
            parent, _, child = name.rpartition(".")
            if parent in sys.modules:
                setattr(sys.modules[parent], child, mod)
    return added


@pytest.mark.skipif(not os.path.isfile(os.path.join(REF, "heat.py")),
                    reason="PYSWEEP_REFERENCE_PLUGINS not set")
@pytest.mark.parametrize("swept", [True, False])
def test_reference_heat_plugin_as_cpu_module(tmp_path, swept):
    import yaml

    from pysweep_b200 import Solver
    n = 64
    x = np.arange(n) / n
    ic = (np.sin(2 * np.pi * x)[:, None] * np.sin(2 * np.pi * x)[None, :])[None]
    dx = 1.0 / n
    g = [0.0, 60 * 0.2 * dx * dx, 0.2 * dx * dx, dx, dx, 1.0, True]
    saved = dict(sys.modules)
    added = _stub_missing(["h5py", "mpi4py", "mpi4py.MPI", "pycuda", "pycuda.driver",
                           "matplotlib", "matplotlib.pyplot", "matplotlib.cm",
                           "matplotlib.animation", "mpl_toolkits", "mpl_toolkits.mplot3d"])
    finals = {}
    try:
        for label, cpu in (("reference", os.path.join(REF, "heat.py")),
                           ("restated", os.path.join(os.path.dirname(HERE), "pysweep_b200",
                                                     "equations", "heat.py"))):
            y = tmp_path / f"{label}.yaml"
            y.write_text(yaml.dump({
                "swept": swept, "blocksize": 16, "intermediate_steps": 1, "operating_points": 1,
                "globals": g, "cpu": cpu, "gpu": "heat.cu", "share": 1.0,
                "write_output": False}))
            cwd = os.getcwd()
            os.chdir(tmp_path)
            try:
                s = Solver(ic, str(y))
                s()
            finally:
                os.chdir(cwd)
            finals[label] = s.final
    finally:
        for name in added:
            sys.modules.pop(name, None)
        for name in list(sys.modules):
            if name not in saved:
                sys.modules.pop(name, None)
    assert np.array_equal(finals["reference"], finals["restated"])
