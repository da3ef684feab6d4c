"""Python handle on one device solver (a thin layer over the C ABI).

``Engine`` owns a ``ps_solver``: the device copy of one periodic field, the
buffers of the swept and standard decompositions, and a CUDA stream.  Host
arrays are numpy ``float64``; device arrays may be given as torch CUDA tensors
(their ``data_ptr`` is passed straight to the library).
"""
import ctypes
import os

import numpy as np

from . import _lib
from ._lib import EQ, MODE, check

DEFAULT_OPS = {"heat": 1, "half": 1, "euler": 2, "heatvar": 1, "heatvar_adjoint": 1,
               "heatvar_adjoint_mu": 1}
DEFAULT_NV = {"heat": 1, "half": 1, "euler": 4, "heatvar": 1, "heatvar_adjoint": 2,
              "heatvar_adjoint_mu": 1}


def _is_torch_cuda(x):
    return hasattr(x, "is_cuda") and hasattr(x, "data_ptr") and x.is_cuda


def _torch_stream(device):
    import torch
    return torch.cuda.current_stream(device)


DTYPES = {"float64": 0, "float32": 1}


def is_hook(equation):
    """Whether `equation` names a step hook (a .cu file) rather than a built-in."""
    return equation not in EQ and str(equation).endswith(".cu")


class Engine:
    """equation: a built-in name (heat, euler, example, checker, half), or the
    path of a plugin's .cu file whose ``__device__ step(shared_state, idx,
    globalTimeStep)`` is compiled at run time (NVRTC, sm_100a), as the
    reference's io.buildGPUSource builds it; ``hook_source`` passes the text
    instead (equation then only labels it).

    dtype: "float64" (default) or "float32" (the reference's `dtype:
    float32`: float32 fields, each level evaluated in float64 and rounded;
    heat with forward Euler only)."""

    def __init__(self, equation, nx, ny, nv=None, ops=None, its=1, blocksize=16, device=0,
                 dtype="float64", hook_source=None):
        hook = hook_source is not None or is_hook(equation)
        if not hook and equation not in EQ:
            raise ValueError(f"unknown equation {equation!r}; built-ins are {sorted(EQ)}, "
                             "or the path of a step hook's .cu file")
        self.equation = equation
        self.hook = hook
        self.nv = nv if nv is not None else DEFAULT_NV.get(equation, 1)
        self.ops = ops if ops is not None else DEFAULT_OPS.get(equation, 1)
        self.nx, self.ny, self.its, self.bs, self.device = nx, ny, its, blocksize, device
        self.dtype = np.dtype(dtype)
        if self.dtype.name not in DTYPES:
            raise ValueError(f"dtype {dtype!r}: float64 or float32")
        self._h = ctypes.c_void_p()
        self._stream = None  # cudaStream_t set by set_stream (None: the solver's own)
        L = _lib.lib()
        if hook:
            if self.dtype != np.float64:
                raise ValueError("step hooks run on float64 fields")
            if hook_source is None:
                with open(equation) as f:
                    hook_source = f.read()
            name = os.path.basename(str(equation))
            rc = L.ps_create_hook(ctypes.byref(self._h), device, hook_source.encode(),
                                  name.encode(), self.nv, nx, ny, self.ops, its, blocksize)
        else:
            rc = L.ps_create_typed(ctypes.byref(self._h), device, EQ[equation], self.nv, nx, ny,
                                   self.ops, its, blocksize, DTYPES[self.dtype.name])
        _lib.check(rc, None)
        self.shape = (self.nv, nx, ny)

    # -- constants ---------------------------------------------------------
    def set_global(self, name, value):
        """Set one plugin constant, typed like the value (float, int or bool);
        a step hook's constant receives it converted to its declared type."""
        if isinstance(value, (bool, np.bool_)):
            buf, n = ctypes.c_uint8(int(value)), 1
        elif isinstance(value, (int, np.integer)):
            buf, n = ctypes.c_int32(int(value)), 4
        else:
            buf, n = ctypes.c_double(float(value)), 8
        check(_lib.lib().ps_set_global(self._h, name.encode(), ctypes.byref(buf), n), self._h)

    def set_field(self, index, tensor):
        """Grid field `index` of a heatvar / heatvar_adjoint(_mu) engine (a
        device tensor kept alive by the caller while runs are queued; None
        clears it): 0 = courant numbers, 1 = the recomputed Laplacians, 2 = the
        mu-form adjoint's sum (ps_set_field)."""
        ptr = None if tensor is None else ctypes.c_void_p(tensor.data_ptr())
        check(_lib.lib().ps_set_field(self._h, index, ptr), self._h)

    def get_global(self, name):
        v = ctypes.c_double()
        check(_lib.lib().ps_get_global_value(self._h, name.encode(), ctypes.byref(v)), self._h)
        return v.value

    def global_handle(self, name):
        h = ctypes.c_void_p()
        n = ctypes.c_size_t()
        check(_lib.lib().ps_get_global(self._h, name.encode(), ctypes.byref(h), ctypes.byref(n)),
              self._h)
        return h.value, n.value

    def set_global_handle(self, handle, raw: bytes):
        buf = ctypes.create_string_buffer(raw, len(raw))
        check(_lib.lib().ps_set_global_handle(self._h, ctypes.c_void_p(handle), buf, len(raw)),
              self._h)

    def configure(self, h=0, nseg=0, chunk=0, threads=0):
        check(_lib.lib().ps_configure(self._h, h, nseg, chunk, threads), self._h)

    def tiling(self):
        """{"h", "nseg", "chunk", "mpss"}: levels per half-cycle, column blocks
        per band (the count the last swept run chose), chunk width, MPSS."""
        v = [ctypes.c_int() for _ in range(4)]
        check(_lib.lib().ps_get_tiling(self._h, *[ctypes.byref(x) for x in v]), self._h)
        return dict(zip(("h", "nseg", "chunk", "mpss"), (x.value for x in v)))

    # -- state -------------------------------------------------------------
    # Torch tensors are read and written on the solver's stream.  Unless that
    # stream is torch's current one, the solver first waits for work queued on
    # torch's stream (the tensor's producer) and, after writing into a
    # tensor, waits for its own copy before returning.
    def _shared_stream(self):
        return self._stream is not None and self._stream == _torch_stream(self.device).cuda_stream

    def _before_read(self):
        if not self._shared_stream():
            _torch_stream(self.device).synchronize()

    def _after_write(self):
        if not self._shared_stream():
            self.synchronize()

    def set_state(self, field):
        """Initial levels: one field (copied to every base level) or `its` fields."""
        if _is_torch_cuda(field):
            self._before_read()
            levels = field.numel() // (self.nv * self.nx * self.ny)
            check(_lib.lib().ps_set_state(self._h, ctypes.c_void_p(field.data_ptr()), levels, 1),
                  self._h)
            self._after_write()  # the tensor may be released once this returns
            return
        a = np.ascontiguousarray(field, dtype=self.dtype)
        levels = a.size // (self.nv * self.nx * self.ny)
        check(_lib.lib().ps_set_state(self._h, a.ctypes.data_as(ctypes.c_void_p), levels, 0),
              self._h)

    def get_state(self, level=0, out=None):
        if out is not None and _is_torch_cuda(out):
            self._before_read()
            check(_lib.lib().ps_get_state(self._h, ctypes.c_void_p(out.data_ptr()), level, 1),
                  self._h)
            self._after_write()
            return out
        a = out if out is not None else np.empty(self.shape, dtype=self.dtype)
        assert a.dtype == self.dtype and a.flags.c_contiguous
        check(_lib.lib().ps_get_state(self._h, a.ctypes.data_as(ctypes.c_void_p), level, 0),
              self._h)
        return a

    def get_rows(self, row0, nrows, level=0, out=None):
        """Rows [row0, row0+nrows) of base level `level` (0 = newest) as a
        (nv, nrows, ny) array, or into `out` (numpy or torch CUDA)."""
        if out is not None and _is_torch_cuda(out):
            self._before_read()
            check(_lib.lib().ps_get_rows(self._h, level, row0, nrows,
                                         ctypes.c_void_p(out.data_ptr()), 1), self._h)
            self._after_write()
            return out
        a = out if out is not None else np.empty((self.nv, nrows, self.ny), dtype=self.dtype)
        check(_lib.lib().ps_get_rows(self._h, level, row0, nrows,
                                     a.ctypes.data_as(ctypes.c_void_p), 0), self._h)
        return a

    def set_rows(self, row0, rows, level=0):
        """Overwrite rows [row0, row0+k) of base level `level` from a
        (nv, k, ny) array (numpy or torch CUDA)."""
        if _is_torch_cuda(rows):
            self._before_read()
            k = rows.numel() // (self.nv * self.ny)
            check(_lib.lib().ps_set_rows(self._h, level, row0, k,
                                         ctypes.c_void_p(rows.data_ptr()), 1), self._h)
            self._after_write()
            return
        a = np.ascontiguousarray(rows, dtype=self.dtype)
        k = a.size // (self.nv * self.ny)
        check(_lib.lib().ps_set_rows(self._h, level, row0, k, a.ctypes.data_as(ctypes.c_void_p), 0),
              self._h)

    def run(self, nlevels, mode="swept", gts0=1, frames=None, frame_every=1):
        """Advance `nlevels` levels.  frames: None, a host array or a device tensor of
        shape (k, nv, nx, ny) receiving every `frame_every`-th full step.  The
        run is queued on the solver's stream; device frames are complete after
        synchronize() (or at once for work queued later on the same stream)."""
        if frames is None:
            rc = _lib.lib().ps_run(self._h, MODE[mode], int(nlevels), gts0, None, 0, frame_every, 0)
        elif _is_torch_cuda(frames):
            rc = _lib.lib().ps_run(self._h, MODE[mode], int(nlevels), gts0,
                                   ctypes.c_void_p(frames.data_ptr()), frames.shape[0],
                                   frame_every, 1)
        else:
            assert frames.dtype == self.dtype and frames.flags.c_contiguous
            rc = _lib.lib().ps_run(self._h, MODE[mode], int(nlevels), gts0,
                                   frames.ctypes.data_as(ctypes.c_void_p), frames.shape[0],
                                   frame_every, 0)
        check(rc, self._h)

    def synchronize(self):
        check(_lib.lib().ps_synchronize(self._h), self._h)

    KINDS = ("prism", "ybridge", "gap", "octahedron", "standard")

    def profile(self, enable=True):
        """Bracket every following launch with CUDA events (resets the counters)."""
        check(_lib.lib().ps_profile(self._h, int(enable)), self._h)

    def profile_read(self):
        """{kind: (device ms, launches, algorithmic cell updates)} since profile()."""
        out = {}
        for i, k in enumerate(self.KINDS):
            ms, n, cells = ctypes.c_double(), ctypes.c_int64(), ctypes.c_double()
            check(_lib.lib().ps_profile_read(self._h, i, ctypes.byref(ms), ctypes.byref(n),
                                             ctypes.byref(cells)), self._h)
            out[k] = (ms.value, n.value, cells.value)
        return out

    def set_stream(self, stream_handle):
        check(_lib.lib().ps_set_stream(self._h, ctypes.c_void_p(stream_handle)), self._h)
        self._stream = stream_handle or None

    @property
    def launches(self):
        return int(_lib.lib().ps_kernel_launches(self._h))

    def close(self):
        if self._h:
            _lib.lib().ps_destroy(self._h)
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


def check_hook(source_or_path, nv=1, ops=1, its=1, name=None):
    """Compile a step hook without a device; returns "" or raises PySweepError
    with the compiler's log (the check io.buildGPUSource's SourceModule makes)."""
    src = source_or_path
    if str(source_or_path).endswith(".cu") and os.path.exists(str(source_or_path)):
        name = name or os.path.basename(str(source_or_path))
        with open(source_or_path) as f:
            src = f.read()
    log = ctypes.create_string_buffer(1 << 16)
    rc = _lib.lib().ps_hook_check(src.encode(), (name or "hook.cu").encode(), nv, ops, its, log,
                                  len(log))
    if rc != _lib.PS_OK:
        raise _lib.PySweepError(rc, log.value.decode())
    return log.value.decode()


def plugin_constants(equation, globals_):
    """The constants a plugin's set_globals copies to the device
    (pysweep/equations/heat.py:38-46, euler.py:25-31, example.py:40-48,
    checker.py:37-45, half.py:35-39)."""
    g = list(globals_)
    if equation == "heat":
        t0, tf, dt, dx, dy, alpha, scheme = g
        return {"DT": float(dt), "DX": float(dx), "DY": float(dy), "ALPHA": float(alpha),
                "SCHEME": bool(scheme)}
    if equation == "euler":
        t0, tf, dt, dx, dy, gamma = g
        return {"DT": float(dt), "DX": float(dx), "DY": float(dy), "GAMMA": float(gamma),
                "GAM_M1": float(gamma) - 1, "DTDX": float(dt) / float(dx),
                "DTDY": float(dt) / float(dy)}
    if equation in ("example", "checker"):
        t0, tf, dt, dx, dy, scheme = g
        return {"DT": float(dt), "DX": float(dx), "DY": float(dy), "SCHEME": bool(scheme)}
    if equation == "half":
        t0, tf, dt, dx, dy = g[:5]
        return {"DT": float(dt), "DX": float(dx), "DY": float(dy)}
    raise ValueError(equation)
