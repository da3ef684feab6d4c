"""CPU-side plugin modules for the built-in equations.

Each module keeps the plugin contract of the reference
(pysweep/equations/*.py): ``set_globals(*args, source_mod=None)`` stores the
CPU globals and, given a source module, copies the device constants through
``source_mod.get_global`` and ``cuda.memcpy_htod``.  The per-point CPU
``step`` is not needed here because every row runs on the GPU.
"""
