"""ctypes binding of libpysweep_b200.so (declarations: include/pysweep_b200.h).

The library must have been built (``python -m pysweep_b200.build``); there is
no CPU fallback, so a missing library is an error.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpysweep_b200.so")

PS_OK = 0
ERRORS = {
    -1: "invalid argument",
    -2: "CUDA error",
    -3: "out of device memory",
    -4: "device-side wait timed out",
    -5: "unsupported configuration",
    -6: "hook compilation failed",
    -7: "call out of order",
}
EQ = {"heat": 0, "euler": 1, "example": 2, "checker": 3, "half": 4, "heatvar": 6,
      "heatvar_adjoint": 7, "heatvar_adjoint_mu": 8}
MODE = {"swept": 0, "standard": 1}


class PySweepError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, 'error')} ({code}): {msg}")
        self.code = code


_lib = None

_SIGS = {
    "ps_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_int]),
    "ps_create_typed": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "ps_create_hook": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                      ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "ps_hook_check": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t]),
    "ps_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "ps_set_field": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "ps_set_global": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p,
                                     ctypes.c_size_t]),
    "ps_get_global": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p,
                                     ctypes.POINTER(ctypes.c_void_p),
                                     ctypes.POINTER(ctypes.c_size_t)]),
    "ps_set_global_handle": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_size_t]),
    "ps_get_global_value": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p,
                                           ctypes.POINTER(ctypes.c_double)]),
    "ps_configure": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int]),
    "ps_get_tiling": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_int)] * 4),
    "ps_set_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "ps_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int,
                              ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int]),
    "ps_get_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "ps_get_rows": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_void_p, ctypes.c_int]),
    "ps_set_rows": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_void_p, ctypes.c_int]),
    "ps_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "ps_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "ps_kernel_launches": (ctypes.c_int64, [ctypes.c_void_p]),
    "ps_profile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "ps_profile_read": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(ctypes.c_int64),
                                       ctypes.POINTER(ctypes.c_double)]),
    "ps_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "ps_version": (ctypes.c_char_p, []),
    "ps_heatvar_courant": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    "ps_heatvar_recompute": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p,
                                            ctypes.c_size_t]),
    "ps_heatvar_forward": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int64,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    "ps_heatvar_adjoint": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int64,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p,
                                          ctypes.c_size_t]),
    "ps_batch_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int]),
    "ps_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "ps_batch_set_global": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p,
                                           ctypes.c_void_p, ctypes.c_size_t]),
    "ps_batch_set_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                          ctypes.c_int, ctypes.c_int]),
    "ps_batch_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int]),
    "ps_batch_get_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                          ctypes.c_int, ctypes.c_int]),
    "ps_batch_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "ps_batch_launches": (ctypes.c_int64, [ctypes.c_void_p]),
    "ps_batch_units": (ctypes.c_int, [ctypes.c_void_p]),
    "ps_batch_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "ps_heat_swept_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_int, ctypes.c_int64,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
}


def exported_symbols():
    return sorted(_SIGS)


def lib():
    """Load the library (once).  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m pysweep_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc, handle=None, batch=False):
    if rc != PS_OK:
        f = lib().ps_batch_last_error if batch else lib().ps_last_error
        msg = f(handle)
        raise PySweepError(rc, msg.decode() if msg else "")
    return rc
