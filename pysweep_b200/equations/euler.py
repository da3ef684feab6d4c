"""2-D Euler plugin: constants and the isentropic vortex.

Contract of pysweep/equations/euler.py:19-31 (set_globals: t0, tf, dt, dx, dy,
gamma; device constants DT, DX, DY, GAMMA, GAM_M1, DTDX, DTDY) and the
vortex of euler.py:63-116.
"""
import numpy

from pysweep_b200.solver import driver_shim as cuda
from pysweep_b200.solver import write_field

gamma = 1.4


def set_globals(*args, source_mod=None):
    global dtdx, dtdy, gamma, gM1
    t0, tf, dt, dx, dy, gamma = args
    dtdx = dtdy = dt / dx
    gM1 = gamma - 1
    if source_mod is not None:
        vals = args[2:] + (gamma - 1, dt / dx, dt / dy)
        for key, val in zip(("DT", "DX", "DY", "GAMMA", "GAM_M1", "DTDX", "DTDY"), vals):
            ckey, _ = source_mod.get_global(key)
            cuda.memcpy_htod(ckey, numpy.float64(val))


def vortex(x, y, t, gamma=1.4, alpha=numpy.pi / 4, strength=5.0):
    """Isentropic vortex (rho, rho u, rho v, E) with free stream rho = 1 and
    pressure 1/gamma, moving at Mach sqrt(2/gamma) along `alpha`."""
    mach = numpy.sqrt(2 / gamma)
    beta = mach * strength * numpy.sqrt(2) / 4 / numpy.pi * numpy.exp(0.5)
    c = numpy.sqrt(gamma)
    u0, v0 = mach * c * numpy.cos(alpha), mach * c * numpy.sin(alpha)
    dx0, dy0 = x - u0 * t, y - v0 * t
    om = beta * numpy.exp(-0.5 * (dx0 ** 2 + dy0 ** 2))
    du, dv = -dy0 * om, dx0 * om
    dT = -(gamma - 1) * om * om / 2
    rho = (1 + dT) ** (1 / (gamma - 1))
    u, v = u0 + du, v0 + dv
    P = 1 / gamma * (1 + dT) ** (gamma / (gamma - 1))
    return numpy.stack([rho, rho * u, rho * v, P / (gamma - 1) + 0.5 * rho * (u * u + v * v)])


def analytical_array(npx, npy, t, **kw):
    """The vortex on linspace(-5, 5, n, endpoint=False) in x and y."""
    x = numpy.linspace(-5, 5, npx, endpoint=False)
    y = numpy.linspace(-5, 5, npy, endpoint=False)
    X, Y = numpy.meshgrid(x, y, indexing="ij")
    return vortex(X, Y, t, **kw)


def analytical(x, y, t, gamma=1.4, alpha=numpy.pi / 4):
    """The vortex of pysweep/equations/euler.py:63-116 (strength 5)."""
    return vortex(x, y, t, gamma=gamma, alpha=alpha)


def createInitialConditions(npx, npy, t=0, gamma=1.4, filename="eulerConditions.hdf5"):
    """The initial field file of pysweep/equations/euler.py:33-56: dataset
    "data" of shape (4, npx, npy) on linspace(-5, 5, n, endpoint=True).  HDF5
    through h5py when it is importable, else an .npz next to `filename`;
    returns the path written."""
    X = numpy.linspace(-5, 5, npx, endpoint=True)
    Y = numpy.linspace(-5, 5, npy, endpoint=True)
    Xg, Yg = numpy.meshgrid(X, Y, indexing="ij")
    return write_field(analytical(Xg, Yg, t, gamma=gamma), filename)
