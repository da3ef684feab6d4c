"""Command line of pysweep_b200: `python -m pysweep_b200 -f heat --swept ...`.

The options, defaults and runs of the reference's command line
(pysweep/utils/commandline.py:117-144, runHeat :71-115, runEuler :26-69):
-f {heat, euler}, --swept, -b blocksize, -nx points per side, -nt time
steps, -s share, --clean, --ignore, -v.  Each run creates the example's
initial-condition file if it is missing, configures a Solver the way the
reference does (dx = domain/(nx-1), dt = 0.1 dx^2/alpha for heat and 0.1 dx
for Euler) and writes heatOutput / eulerOutput.  The reference's plotting
option (-p) draws matplotlib figures of the decomposition, which this
package does not provide; it is accepted and reported.
"""
import argparse
import os
import warnings

import numpy

from . import solver as _solver
from .equations import euler as _euler
from .equations import heat as _heat

EQN_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "equations")


def str2bool(v):
    if isinstance(v, bool):
        return v
    if v.lower() in ("yes", "true", "t", "y", "1"):
        return True
    if v.lower() in ("no", "false", "f", "n", "0"):
        return False
    raise argparse.ArgumentTypeError("Boolean value expected as string.")


def adjust_array_size(args):
    """Round the points per side up to a multiple of the blocksize (commandline.py:22-26)."""
    remainder = args.spacesteps % args.blocksize
    if remainder != 0:
        args.spacesteps += args.blocksize - remainder
        warnings.warn(f"Adjusting array size to fit blocksize. New array size is {args.spacesteps}.")


def _existing(filename):
    base, _ = os.path.splitext(filename)
    for p in (filename, base + ".npz"):
        if os.path.isfile(p):
            return p
    return None


def _configure(s, args, globals_, operating, intermediate, eqn, output):
    s.globals = globals_
    s.dtypeStr = "float64"
    s.dtype = numpy.dtype(s.dtypeStr)
    s.verbose = False
    s.operating = operating
    s.intermediate = intermediate
    s.share = args.share
    s.simulation = bool(args.swept)
    s.blocksize = (args.blocksize, args.blocksize, 1)
    s.setCPU(os.path.join(EQN_PATH, eqn + ".py"))
    s.setGPU(os.path.join(EQN_PATH, eqn + ".cu"))
    s.exid = []
    s.output = output
    s.loadCPUModule()


def _finish(s, args, remove_output):
    if args.verbose:
        print(s)
    s()
    if args.clean and remove_output:
        base, _ = os.path.splitext(s.output)
        for p in (s.output, base + ".npz"):
            if os.path.isfile(p):
                os.remove(p)
    return s


def run_heat(args):
    if args.ignore:
        warnings.filterwarnings("ignore")
    adjust_array_size(args)
    alpha = 1
    dx = 1 / (args.spacesteps - 1)
    dt = float(0.1 * dx ** 2 / alpha)
    filename = f"heatConditions{args.spacesteps}.hdf5"
    path = _existing(filename) or _heat.createInitialConditions(
        args.spacesteps, args.spacesteps, filename=filename, alpha=alpha)
    s = _solver.Solver(initialConditions=path, sendWarning=not args.ignore)
    _configure(s, args, [0, dt * args.timesteps, dt, dx, dx, alpha, True], 1, 1, "heat",
               "heatOutput.hdf5")
    return _finish(s, args, remove_output=True)


def run_euler(args):
    if args.ignore:
        warnings.filterwarnings("ignore")
    adjust_array_size(args)
    gamma = 1.4
    dx = 10 / (args.spacesteps - 1)
    dt = 0.1 * dx
    filename = f"eulerConditions{args.spacesteps}.hdf5"
    path = _existing(filename) or _euler.createInitialConditions(
        args.spacesteps, args.spacesteps, filename=filename, gamma=gamma)
    s = _solver.Solver(initialConditions=path, sendWarning=not args.ignore)
    _configure(s, args, [0, dt * args.timesteps, dt, dx, dx, gamma], 2, 2, "euler",
               "eulerOutput.hdf5")
    return _finish(s, args, remove_output=False)  # the reference keeps Euler's output


FUNCTIONS = {"euler": run_euler, "heat": run_heat}


def parser():
    p = argparse.ArgumentParser(prog="python -m pysweep_b200")
    p.add_argument("-f", "--function", nargs="?", default=None, choices=FUNCTIONS, type=str,
                   help="This specifies which function example to run.")
    p.add_argument("--swept", action="store_true", help="Set simulation type to swept.")
    p.add_argument("-b", "--blocksize", default=12, nargs="?", type=int,
                   help="blocksize, with mod(b, 2*k) == 0 for k points on each side")
    p.add_argument("-nx", "--spacesteps", default=24, nargs="?", type=int,
                   help="number of points in x and y (square domains)")
    p.add_argument("-nt", "--timesteps", default=10, nargs="?", type=int,
                   help="number of time steps")
    p.add_argument("-s", "--share", default=0.5, nargs="?", type=float,
                   help="GPU share, 0 to 1 (every row runs on the GPU here)")
    p.add_argument("--clean", action="store_true", help="Remove the results afterwards.")
    p.add_argument("--ignore", action="store_true", help="Ignore warnings.")
    p.add_argument("-v", "--verbose", action="store_true", help="Print the simulation setup.")
    p.add_argument("-p", "--plot", nargs="+", type=str,
                   help="The reference's decomposition figures (not provided here).")
    return p


def main(argv=None):
    args = parser().parse_args(argv)
    if args.plot:
        warnings.warn("pysweep_b200 does not draw the reference's decomposition figures "
                      f"({', '.join(args.plot)}).")
    if args.function is not None:
        return FUNCTIONS[args.function](args)
    return None
