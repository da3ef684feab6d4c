"""CPU oracle for the swept space-time path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this package, and only as the checker (or, for the benchmark's
reference arm, as the timed CPU restatement of the reference algorithm).  The
product library never imports it.

``liboracle.so`` (built from ``oracle.c`` by ``make -C oracle``) restates the
reference's numpy arithmetic and its CPU swept decomposition; see the header of
``oracle.c`` for the file:line it follows.  This module mirrors the plugins'
``set_globals`` (pysweep/equations/heat.py:33-46, euler.py:19-31) to turn a
``globals`` list into the per-equation parameter vector, and the step-count
arithmetic of pysweep/core/solver.py:113-128.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
EQ = {"heat": 0, "euler": 1, "example": 2, "checker": 3, "half": 4}
NV = {"heat": 1, "euler": 4, "half": 1}

_lib = None


def build():
    subprocess.run(["make", "-C", HERE], check=True, capture_output=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        dp = ctypes.POINTER(ctypes.c_double)
        L.oracle_standard.restype = ctypes.c_long
        L.oracle_standard.argtypes = [ctypes.c_int, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, dp, dp, ctypes.c_long, ctypes.c_int, dp,
                                      ctypes.c_long, ctypes.c_int]
        L.oracle_swept.restype = ctypes.c_long
        L.oracle_swept.argtypes = [ctypes.c_int, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp,
                                   ctypes.c_long, dp, ctypes.c_int]
        L.oracle_max_threads.restype = ctypes.c_int
        L.oracle_heat_f32.restype = ctypes.c_long
        L.oracle_heat_f32.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.c_int, ctypes.c_int,
                                      ctypes.c_double, ctypes.c_long, ctypes.c_int]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


def params(eqn, globals_, nv=1, euler_square="pow"):
    """Per-equation constants, computed the way each plugin's set_globals does."""
    g = list(globals_)
    if eqn == "heat":
        t0, tf, dt, dx, dy, alpha, scheme = g
        courant = alpha * dt / dx / dx  # heat.py:37
        return np.array([courant, 1.0 if scheme else 0.0])
    if eqn == "euler":
        t0, tf, dt, dx, dy, gamma = g
        dtdx = dtdy = dt / dx  # euler.py:23
        return np.array([dtdx, dtdy, gamma, gamma - 1, 0.0 if euler_square == "pow" else 1.0])
    if eqn in ("example", "checker"):
        scheme = g[5]
        return np.array([1.0 if scheme else 0.0, float(nv)])
    if eqn == "half":
        return np.zeros(1)
    raise ValueError(eqn)


def step_data(globals_, bs, ops, its, swept=True):
    """pysweep/core/solver.py:113-128 -> (timeSteps, MPSS, maxGlobalSweptStep)."""
    ts = int((globals_[1] - globals_[0]) / globals_[2])
    if not swept:
        return ts, None, None
    mpss = bs // (2 * ops) - 1
    mgss = int(its * ts / mpss - 1)
    ts = int(mpss * (mgss + 1) / its + 1)
    return ts, mpss, mgss


def standard(eqn, ic, globals_, its, nlevels, gts0=1, nthreads=1, frames=True,
             euler_square="pow", prev=None):
    """Periodic level-by-level stepper.  Returns (frames, final, final_prev).

    frames[0] is ``ic``; frames[k] is the field after k full steps.
    """
    ic = np.ascontiguousarray(ic, dtype=np.float64)
    nv, nx, ny = ic.shape
    p = params(eqn, globals_, nv, euler_square)
    u = ic.copy()
    up = ic.copy() if prev is None else np.ascontiguousarray(prev, dtype=np.float64).copy()
    maxf = nlevels // its + 1 if frames else 0
    fr = np.empty((maxf,) + ic.shape) if frames else None
    got = lib().oracle_standard(EQ[eqn], _p(p), nv, nx, ny, its, _p(u), _p(up), nlevels, gts0,
                                _p(fr), maxf, nthreads)
    if got < 0:
        raise RuntimeError(f"oracle_standard failed: {got}")
    if frames:
        fr = np.concatenate([ic[None], fr[:got]])
    return fr, u, up


def swept(eqn, ic, globals_, its, ops, bs, max_gss=None, nthreads=1, frames=True,
          euler_square="pow"):
    """The reference CPU swept decomposition.  Returns (frames, final_level)."""
    ic = np.ascontiguousarray(ic, dtype=np.float64)
    nv, nx, ny = ic.shape
    p = params(eqn, globals_, nv, euler_square)
    if max_gss is None:
        _, _, max_gss = step_data(globals_, bs, ops, its, True)
    mpss = bs // (2 * ops) - 1
    nlev = mpss * (max_gss + 1)
    maxf = nlev // its + 2 if frames else 0
    fr = np.empty((maxf,) + ic.shape) if frames else None
    fin = np.empty_like(ic)
    got = lib().oracle_swept(EQ[eqn], _p(p), nv, nx, ny, its, ops, bs, max_gss, _p(ic), _p(fr),
                             maxf, _p(fin), nthreads)
    if got < 0:
        raise RuntimeError(f"oracle_swept failed: {got}")
    return (fr[:got] if frames else None), fin


def max_threads():
    return lib().oracle_max_threads()


def heat_f32(ic, globals_, nlevels, nthreads=1):
    """Forward-Euler heat with float32 storage: each level is evaluated in
    float64 (the plugin's courant is a float64 scalar) and rounded to float32,
    as the reference does with `dtype: float32`.  Returns the final field
    (float32)."""
    u = np.ascontiguousarray(ic, dtype=np.float32).copy()
    _, nx, ny = u.shape
    courant = params("heat", globals_)[0]
    got = lib().oracle_heat_f32(u.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), nx, ny,
                                courant, int(nlevels), nthreads)
    if got < 0:
        raise RuntimeError("oracle_heat_f32 failed")
    return u
