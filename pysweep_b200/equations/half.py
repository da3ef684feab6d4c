"""RK2 "/100" diffusion plugin (contract of pysweep/equations/half.py:35-39)."""
import numpy

from pysweep_b200.solver import driver_shim as cuda


def set_globals(*args, source_mod=None):
    global dt, dx, dy
    t0, tf, dt, dx, dy = args[:5]
    if source_mod is not None:
        for key, val in zip(("DT", "DX", "DY"), args[2:5]):
            ckey, _ = source_mod.get_global(key)
            cuda.memcpy_htod(ckey, numpy.float64(val))
