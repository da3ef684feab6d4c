"""Generate golden fixtures by running the reference's own CPU path (share = 0).

This script is the only code in the repository that imports the reference
(anthony-walker/pysweep).  It needs the reference checkout, so it runs only on
a development machine; its outputs (``*.npz`` next to this file) are the
fixtures the tests read.  Usage::

    python tests/golden/make_golden.py /path/to/pysweep-checkout

The reference imports mpi4py, h5py, pycuda, GPUtil and matplotlib at module
level and ``collections.Iterable`` (removed in Python 3.10).  None of these
are needed by the share = 0 swept/standard path, so they are replaced by
stubs: a single-rank MPI (``Sendrecv`` returns its input, shared windows are
``bytearray``-backed) and empty modules for the rest.  The solver is then
driven exactly as ``pysweep/tests/tests.py`` drives it (attributes set on a
``Solver`` object, then ``solver()``).

Frames are captured by wrapping ``pysweep.core.io.sweptWrite`` /
``standardWrite``: those functions select the completed time levels that the
(commented-out) HDF5 writer would store as ``data[cwt]``
(``pysweep/core/io.py:134-144`` and ``:186-208``); the wrapper stores exactly
those levels.  Frame 0 is the initial condition.
"""
import collections
import collections.abc
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


# ----------------------------------------------------------------- stubs ----
class _Group:
    def Incl(self, ranks):
        return self


class _Win:
    def __init__(self, nbytes):
        self.buf = bytearray(nbytes)

    def Shared_query(self, rank):
        return memoryview(self.buf), 1


class _Comm:
    group = _Group()

    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1

    def allgather(self, x):
        return [x]

    def scatter(self, x):
        return x[0] if x is not None else None

    def bcast(self, x):
        return x

    def Barrier(self):
        pass

    def Split(self, color):
        return self

    def Create_group(self, g):
        return self

    def Sendrecv(self, sendobj=None, dest=None, source=None):
        return sendobj


def _install_stubs():
    collections.Iterable = collections.abc.Iterable
    mpi = types.ModuleType("mpi4py")
    mpi.rc = types.SimpleNamespace(recv_mprobe=False)
    MPI = types.ModuleType("mpi4py.MPI")
    MPI.COMM_WORLD = _Comm()
    MPI.Get_processor_name = lambda: "node0"

    class Win:
        @staticmethod
        def Allocate_shared(nbytes, itemsize, comm=None):
            return _Win(max(int(nbytes), 1))

    MPI.Win = Win
    mpi.MPI = MPI
    sys.modules["mpi4py"] = mpi
    sys.modules["mpi4py.MPI"] = MPI
    for name in ("h5py", "GPUtil", "pycuda", "pycuda.driver",
                 "pycuda.compiler", "pycuda.autoinit"):
        sys.modules[name] = types.ModuleType(name)
    mpl = types.ModuleType("matplotlib")
    mpl.cm = types.ModuleType("matplotlib.cm")
    mpl.pyplot = types.ModuleType("matplotlib.pyplot")
    mpl.animation = types.ModuleType("matplotlib.animation")
    mpl.animation.animation = None
    mpl.rc = lambda *a, **k: None
    mpl.animation = types.SimpleNamespace()
    sys.modules["matplotlib"] = mpl
    sys.modules["matplotlib.pyplot"] = mpl.pyplot
    sys.modules["matplotlib.cm"] = mpl.cm
    sys.modules["matplotlib.animation"] = types.ModuleType("matplotlib.animation")
    sys.modules["matplotlib.animation"].animation = None
    sys.modules["matplotlib"].animation = sys.modules["matplotlib.animation"]
    tk = types.ModuleType("mpl_toolkits")
    tk.mplot3d = types.ModuleType("mpl_toolkits.mplot3d")
    sys.modules["mpl_toolkits"] = tk
    sys.modules["mpl_toolkits.mplot3d"] = tk.mplot3d


def _import_reference(refroot):
    _install_stubs()
    sys.path.insert(0, refroot)
    import pysweep  # noqa: F401  (reference package)
    import pysweep.core.io as io
    import pysweep.core.solver as solver_mod
    return pysweep, io, solver_mod


# --------------------------------------------------------------- capture ----
class _Capture:
    def __init__(self, io, solver_mod):
        self.frames = []
        self.io = io
        orig_swept, orig_std = io.sweptWrite, io.standardWrite

        def swept_write(cwt, solver):
            # levels selected by pysweep/core/io.py:137
            for i in range((solver.globalTimeStep + solver.subtraction) % solver.intermediate
                           + solver.intermediate,
                           solver.maxPyramidSize + solver.intermediate,
                           solver.intermediate):
                self.frames.append(np.array(solver.sharedArray[i], dtype=np.float64))
            return orig_swept(cwt, solver)

        def standard_write(cwt, solver):
            # level selected by pysweep/core/io.py:189-193
            if solver.globalTimeStep % solver.intermediate == 0:
                ops = solver.operating
                self.frames.append(np.array(
                    solver.sharedArray[solver.intermediate - 1, :, ops:-ops, ops:-ops],
                    dtype=np.float64))
            return orig_std(cwt, solver)

        io.sweptWrite = swept_write
        io.standardWrite = standard_write
        # functions.py imported io as a module object, so patching the module
        # attribute is enough.


def run_reference(pysweep, cap, eqn, ic, globals_, bs, ops, its, swept, dtype="float64"):
    eqdir = os.path.join(os.path.dirname(pysweep.__file__), "equations")
    cap.frames = []
    solver = pysweep.Solver(ic, None, sendWarning=False)
    solver.dtypeStr = dtype
    solver.dtype = np.dtype(dtype)
    solver.verbose = False
    solver.share = 0
    solver.simulation = swept
    solver.blocksize = (bs, bs, 1)
    solver.operating = ops
    solver.intermediate = its
    solver.globals = list(globals_)
    solver.setCPU(os.path.join(eqdir, eqn + ".py"))
    solver.setGPU(os.path.join(eqdir, eqn + ".cu"))
    solver.exid = []
    solver.output = "unused.hdf5"
    solver.loadCPUModule()
    cwd = os.getcwd()
    os.chdir("/tmp")  # cleanupProcesses appends to ./log.yaml
    try:
        solver()
    finally:
        os.chdir(cwd)
    # swept: data[0] is the initial condition and every sweptWrite call adds
    # completed levels; standard: the first standardWrite stores level 0
    # itself (pysweep/core/solver.py:184, io.py:189-193).
    head = [np.array(ic, dtype=np.float64)] if swept else []
    frames = np.stack(head + cap.frames)
    return frames, int(solver.arrayShape[0])


# ----------------------------------------------------------------- cases ----
def heat_ic(n):
    x = np.arange(n) / n
    return (np.sin(2 * np.pi * x)[:, None] * np.sin(2 * np.pi * x)[None, :])[None]


def euler_ic(pysweep, n):
    # pysweep/equations/euler.py:107-116 (getAnalyticalArray at t = 0)
    return pysweep.equations.euler.getAnalyticalArray(n, n, 0)


def half_ic(n):
    # pysweep/equations/half.py:56-60
    return (np.arange(n * n, dtype=np.float64) / 100).reshape(1, n, n)


def checker_ic(n):
    # pysweep/equations/checker.py:45-51
    d = np.zeros((1, n, n))
    d[:, 0::2, 0::2] = 1
    d[:, 1::2, 1::2] = 1
    return d


CASES = [
    # name, eqn, n, bs, ops, its, globals builder, steps
    ("heat_fe_n32_bs8", "heat", 32, 8, 1, 1, "heat_fe", 20),
    ("heat_fe_n48_bs12", "heat", 48, 12, 1, 1, "heat_fe", 23),
    ("heat_fe_n48_bs16", "heat", 48, 16, 1, 1, "heat_fe", 30),
    ("heat_rk2_n32_bs8", "heat", 32, 8, 1, 2, "heat_rk2", 12),
    ("heat_rk2_n48_bs12", "heat", 48, 12, 1, 2, "heat_rk2", 11),
    ("euler_n32_bs16", "euler", 32, 16, 2, 2, "euler", 8),
    ("euler_n24_bs12", "euler", 24, 12, 2, 2, "euler", 5),
    ("example_fe_n24_bs8", "example", 24, 8, 1, 1, "example_fe", 13),
    ("example_rk2_n24_bs8", "example", 24, 8, 2, 2, "example_rk2", 9),
    ("checker_one_n24_bs8", "checker", 24, 8, 1, 1, "checker_one", 10),
    ("checker_two_n24_bs8", "checker", 24, 8, 2, 2, "checker_two", 6),
    ("half_n24_bs8", "half", 24, 8, 1, 2, "half", 10),
]

# FP32 runs of the reference (yaml `dtype: float32`, io.py:72-73): the shared
# array and the frames are float32; the initial field is rounded to float32.
CASES_F32 = [
    ("heat_fe_f32_n64_bs16", "heat", 64, 16, 1, 1, "heat_fe", 37),
    ("heat_fe_f32_n128_bs32", "heat", 128, 32, 1, 1, "heat_fe", 45),
]


def make_globals(kind, n, steps):
    if kind in ("heat_fe", "heat_rk2"):
        dx = 1.0 / n
        alpha = 1.0
        dt = 0.2 * dx * dx / alpha
        return [0.0, steps * dt, dt, dx, dx, alpha, kind == "heat_fe"]
    if kind == "euler":
        dx = 10.0 / n
        dt = 0.1 * dx
        return [0.0, steps * dt, dt, dx, dx, 1.4]
    if kind in ("example_fe", "example_rk2", "checker_one", "checker_two"):
        fe = kind.endswith("fe") or kind.endswith("one")
        return [0.0, steps * 0.1, 0.1, 0.1, 0.1, fe]
    if kind == "half":
        return [0.0, steps * 0.1, 0.1, 0.1, 0.1]
    raise ValueError(kind)


def main(refroot):
    pysweep, io, solver_mod = _import_reference(refroot)
    cap = _Capture(io, solver_mod)
    for name, eqn, n, bs, ops, its, gkind, steps in CASES_F32:
        ic = heat_ic(n).astype(np.float32).astype(np.float64)
        g = make_globals(gkind, n, steps)
        out = {}
        for swept in (True, False):
            frames, nframes_ref = run_reference(pysweep, cap, eqn, ic, g, bs, ops, its, swept,
                                                dtype="float32")
            key = "swept" if swept else "standard"
            out[key] = frames
            out[key + "_array_shape0"] = np.int64(nframes_ref)
            print(f"{name:24s} {key:8s} frames={frames.shape[0]}", flush=True)
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"),
            eqn=eqn, n=n, bs=bs, ops=ops, its=its, globals=np.array(g, dtype=np.float64),
            ic=ic, dtype="float32", **out)
    for name, eqn, n, bs, ops, its, gkind, steps in CASES:
        if eqn == "heat":
            ic = heat_ic(n)
        elif eqn == "euler":
            ic = euler_ic(pysweep, n)
        elif eqn == "half":
            ic = half_ic(n)
        elif eqn == "checker":
            ic = checker_ic(n)
        else:
            ic = np.zeros((1, n, n))
        g = make_globals(gkind, n, steps)
        out = {}
        for swept in (True, False):
            frames, nframes_ref = run_reference(pysweep, cap, eqn, ic, g, bs, ops, its, swept)
            key = "swept" if swept else "standard"
            out[key] = frames
            out[key + "_array_shape0"] = np.int64(nframes_ref)
            print(f"{name:24s} {key:8s} frames={frames.shape[0]} "
                  f"(arrayShape[0]={nframes_ref})", flush=True)
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"),
            eqn=eqn, n=n, bs=bs, ops=ops, its=its, globals=np.array(g, dtype=np.float64),
            ic=np.asarray(ic, dtype=np.float64), **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_golden.py <path of the pysweep checkout>")
    main(sys.argv[1])
