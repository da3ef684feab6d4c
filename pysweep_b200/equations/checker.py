"""Checkerboard-averaging plugin (contract of pysweep/equations/checker.py:29-45)."""
import numpy

from pysweep_b200.solver import driver_shim as cuda

scheme = True


def set_globals(*args, source_mod=None):
    global dt, dx, dy, scheme
    t0, tf, dt, dx, dy, scheme = args
    if source_mod is not None:
        for key, val in zip(("DT", "DX", "DY"), args[2:5]):
            ckey, _ = source_mod.get_global(key)
            cuda.memcpy_htod(ckey, numpy.float64(val))
        ckey, _ = source_mod.get_global("SCHEME")
        cuda.memcpy_htod(ckey, numpy.intc(scheme))
