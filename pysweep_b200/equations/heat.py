"""Heat equation plugin: constants, CPU step and analytic solution.

Contract of pysweep/equations/heat.py:33-46 (set_globals: t0, tf, dt, dx, dy,
alpha, scheme; device constants DT, DX, DY, ALPHA, SCHEME), the CPU step of
heat.py:21-64 (what the CPU rows of a run with share < 1 use) and the
decaying sine of heat.py:95-113.
"""
import numpy

from pysweep_b200.solver import driver_shim as cuda
from pysweep_b200.solver import write_field

scheme = True


def set_globals(*args, source_mod=None):
    global dt, dx, dy, alpha, scheme, courant
    t0, tf, dt, dx, dy, alpha, scheme = args
    courant = alpha * dt / dx / dx
    if source_mod is not None:
        for key, val in zip(("DT", "DX", "DY", "ALPHA"), args[2:6]):
            ckey, _ = source_mod.get_global(key)
            cuda.memcpy_htod(ckey, numpy.float64(val))
        ckey, _ = source_mod.get_global("SCHEME")
        cuda.memcpy_htod(ckey, numpy.intc(scheme))


def step(state, iidx, arrayTimeIndex, globalTimeStep):
    """One level at the cells `iidx` ((x, y) pairs) of the 4-D state
    [t, v, x, y]: level arrayTimeIndex + 1 from arrayTimeIndex (and, for the
    second Runge-Kutta stage, arrayTimeIndex - 1), forward Euler or two-stage
    Runge-Kutta by `scheme` (heat.py:21-31).  The cells are evaluated together
    as arrays, each in the per-cell operation order of heat.py:48-64, so every
    value equals the per-cell loop's; neighbours wrap around the state's x and
    y extent."""
    idx = numpy.asarray(iidx, dtype=numpy.intp).reshape(-1, 2)
    x, y = idx[:, 0], idx[:, 1]
    cur = state[arrayTimeIndex, 0]
    nx, ny = cur.shape
    c = cur[x, y]
    dxx = courant * (cur[(x + 1) % nx, y] - 2 * c + cur[x - 1, y])
    dyy = courant * (cur[x, (y + 1) % ny] - 2 * c + cur[x, y - 1])
    if scheme:
        state[arrayTimeIndex + 1, 0, x, y] = (dxx + dyy) + c
    else:
        coeff, back = (1, 1) if globalTimeStep % 2 == 0 else (0.5, 0)
        state[arrayTimeIndex + 1, 0, x, y] = coeff * (dxx + dyy) + state[arrayTimeIndex - back, 0, x, y]


def analytical(npx, npy, t, alpha=0.1):
    """sin(2 pi x) sin(2 pi y) exp(-8 pi^2 alpha t) on x_i = i/npx."""
    X = numpy.linspace(0, 1, npx, endpoint=False)
    Y = numpy.linspace(0, 1, npy, endpoint=False)
    u = numpy.sin(2 * numpy.pi * X)[:, None] * numpy.sin(2 * numpy.pi * Y)[None, :]
    return (u * numpy.exp(-8 * numpy.pi ** 2 * alpha * t))[None], X, Y


def analyticalEquation(x, y, t, alpha=0.1):
    """sin(2 pi x) sin(2 pi y) exp(-8 pi^2 alpha t) (pysweep/equations/heat.py:90-93)."""
    m = n = 2
    return (numpy.sin(m * numpy.pi * x) * numpy.sin(n * numpy.pi * y) *
            numpy.exp(-(m * m + n * n) * numpy.pi * numpy.pi * alpha * t))


def createInitialConditions(npx, npy, alpha=0.1, t=0, filename="heatConditions.hdf5"):
    """The initial field file of pysweep/equations/heat.py:66-88: dataset
    "data" of shape (1, npx, npy) on linspace(0, 1, n, endpoint=True).  HDF5
    through h5py when it is importable, else an .npz next to `filename`;
    returns the path written."""
    X = numpy.linspace(0, 1, npx, endpoint=True)
    Y = numpy.linspace(0, 1, npy, endpoint=True)
    data = analyticalEquation(X[:, None], Y[None, :], t, alpha=alpha)[None]
    return write_field(data, filename)
