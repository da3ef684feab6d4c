"""Many independent fields advanced together (ps_batch_* of the C ABI).

    b = Batch("heat", sizes=[(128, 128), (512, 512)], its=1, blocksize=32)
    b.set_constants(0, {"DT": ..., "DX": ..., "ALPHA": ..., "SCHEME": True})
    b.set_state(0, field0); b.set_state(1, field1)
    b.run(levels)            # one launch per phase for all fields, from a CUDA graph
    out0 = b.get_state(0)
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import EQ

DEFAULT_OPS = {"heat": 1, "half": 1, "euler": 2}
DEFAULT_NV = {"heat": 1, "half": 1, "euler": 4}


def _chk(rc, h):
    _lib.check(rc, h, batch=True)


class Batch:
    def __init__(self, equation, sizes, nv=None, ops=None, its=1, blocksize=32, device=0):
        self.equation = equation
        self.nv = nv if nv is not None else DEFAULT_NV.get(equation, 1)
        self.ops = ops if ops is not None else DEFAULT_OPS.get(equation, 1)
        self.its = its
        self.sizes = [tuple(map(int, s)) for s in sizes]
        n = len(self.sizes)
        nx = (ctypes.c_int * n)(*[s[0] for s in self.sizes])
        ny = (ctypes.c_int * n)(*[s[1] for s in self.sizes])
        self._h = ctypes.c_void_p()
        _chk(_lib.lib().ps_batch_create(ctypes.byref(self._h), device, EQ[equation], n, nx, ny,
                                        self.nv, self.ops, its, blocksize), None)

    def __len__(self):
        return len(self.sizes)

    def set_global(self, index, name, value):
        if isinstance(value, (bool, np.bool_)):
            buf, n = ctypes.c_uint8(int(value)), 1
        elif isinstance(value, (int, np.integer)):
            buf, n = ctypes.c_int32(int(value)), 4
        else:
            buf, n = ctypes.c_double(float(value)), 8
        _chk(_lib.lib().ps_batch_set_global(self._h, index, name.encode(), ctypes.byref(buf), n),
             self._h)

    def set_constants(self, index, consts):
        for k, v in consts.items():
            self.set_global(index, k, v)

    def set_state(self, index, field):
        if hasattr(field, "is_cuda") and field.is_cuda:
            levels = field.numel() // (self.nv * self.sizes[index][0] * self.sizes[index][1])
            _chk(_lib.lib().ps_batch_set_state(self._h, index, ctypes.c_void_p(field.data_ptr()),
                                               levels, 1), self._h)
            return
        a = np.ascontiguousarray(field, dtype=np.float64)
        levels = a.size // (self.nv * self.sizes[index][0] * self.sizes[index][1])
        _chk(_lib.lib().ps_batch_set_state(self._h, index, a.ctypes.data_as(ctypes.c_void_p),
                                           levels, 0), self._h)

    def run(self, nlevels, graph=True):
        _chk(_lib.lib().ps_batch_run(self._h, int(nlevels), int(graph)), self._h)

    def get_state(self, index, level=0):
        nx, ny = self.sizes[index]
        a = np.empty((self.nv, nx, ny))
        _chk(_lib.lib().ps_batch_get_state(self._h, index, a.ctypes.data_as(ctypes.c_void_p),
                                           level, 0), self._h)
        return a

    def synchronize(self):
        _chk(_lib.lib().ps_batch_synchronize(self._h), self._h)

    @property
    def launches(self):
        return int(_lib.lib().ps_batch_launches(self._h))

    @property
    def units(self):
        return int(_lib.lib().ps_batch_units(self._h))

    def close(self):
        if self._h:
            _lib.lib().ps_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
