"""pysweep_b200: a B200-native swept space-time solver for 2-D explicit PDEs.

The GPU share of a PySweep run (the UpPyramid, Y/X bridges, Octahedron and
DownPyramid phases and the standard decomposition) runs as hand-written
sm_100a CUDA kernels behind a C ABI (include/pysweep_b200.h); this package is
the Python side of that ABI and the drop-in ``Solver`` front-end.
"""
from ._lib import PySweepError  # noqa: F401
from .batch import Batch  # noqa: F401
from .engine import Engine, check_hook, plugin_constants  # noqa: F401

__version__ = "0.1.0"


def Solver(*args, **kwargs):  # noqa: N802 - mirrors pysweep.Solver
    from .solver import Solver as _S
    return _S(*args, **kwargs)
