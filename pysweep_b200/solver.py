"""Drop-in replacement for ``pysweep.Solver`` (pysweep/core/solver.py).

    solver = pysweep_b200.Solver(initialConditions, "input.yaml")
    solver()

The yaml keys, their defaults and the attributes a script may set directly
are those of pysweep/core/io.py:35-75 (``swept``, ``verbose``,
``intermediate_steps``, ``operating_points``, ``blocksize``, ``share``,
``exid``, ``globals``, ``cpu``, ``gpu``, ``filename``, ``dtype``).  The time
step arithmetic is the reference's (solver.py:113-128): a swept run computes
``MPSS*(maxGlobalSweptStep+1)`` levels and stores ``timeSteps`` frames, a
standard run stores ``timeSteps+1`` frames.

What runs where: with ``share`` 1 every row runs on the GPU through the CUDA
swept (or standard) kernels.  With ``share`` below 1 the first
ceil(share * nx / bs) block rows run on the GPU and the others on the host,
stepped by the CPU plugin's own numpy ``step`` as the reference's CPU ranks
step them, with the edge strips exchanged after every half-cycle
(share.SplitSolver; the reference's MajorSplit, process.py:131-176); the
effective share after that rounding is recorded.  A plugin without a numpy
``step`` (or float32 fields, or a hook file without the .cu suffix) runs every
row on the GPU, with a warning: the computed values do not depend on the
split.

The CPU plugin (``cpu:``) keeps its contract: its ``set_globals(*globals,
source_mod=...)`` is called with a module object whose ``get_global(name)``
and the ``cuda.memcpy_htod`` it uses set the device constants, exactly as
with a PyCUDA SourceModule (pysweep/equations/heat.py:38-46).  The GPU hook
(``gpu:``) names the step function: the file names of the reference's
plugins (heat.cu, euler.cu, example.cu, checker.cu, half.cu) and the bare
names select the built-in sm_100a kernels (their arithmetic follows the numpy
plugins operation by operation); any other ``.cu`` file, or any file at all
with the extra yaml key ``compile_hook: true``, is compiled at run time with
NVRTC for sm_100a, as io.buildGPUSource (io.py:146-155) builds it with
PyCUDA, and its ``__device__ step`` runs inside the swept and standard
kernels.

Output: the reference's HDF5 layout (io.py:78-90): datasets ``blocksize``,
``share``, ``exid``, ``globals``, ``clocktime`` and ``data[t, v, x, y]``.
h5py is used when importable; otherwise the same datasets go to an ``.npz``
file next to the requested name.  ``output_every`` (extra yaml key, default 1)
keeps every k-th frame, ``write_output: false`` skips the file.
"""
import importlib.util
import os
import time
import types
import warnings
from datetime import datetime

import numpy as np
import yaml

from .engine import Engine, plugin_constants
from .share import SplitSolver, gpu_rows

BUILTIN = ("heat", "euler", "example", "checker", "half")
NV = {"heat": 1, "half": 1, "euler": 4}


# ----------------------------------------------------- SourceModule stand-in
class GlobalRef:
    """What ``source_mod.get_global(name)[0]`` returns: a device constant."""

    def __init__(self, module, name):
        self.module, self.name = module, name


class SourceModuleShim:
    """Duck type of pycuda.compiler.SourceModule for the plugins' set_globals."""

    def __init__(self):
        self.values = {}
        self.engine = None

    def get_global(self, name):
        if self.engine is not None and self.engine.hook:
            _, size = self.engine.global_handle(name)  # the hook's declared size
        else:
            size = 4 if name == "SCHEME" else 8
        return GlobalRef(self, name), size

    def apply(self, engine):
        self.engine = engine
        for k, v in self.values.items():
            engine.set_global(k, v)


def memcpy_htod(dst, src):
    """pycuda.driver.memcpy_htod for GlobalRef destinations."""
    if not isinstance(dst, GlobalRef):
        raise TypeError("memcpy_htod: destination is not a pysweep_b200 constant")
    if isinstance(src, (bytes, bytearray)):
        val = int.from_bytes(bytes(src), "little") if src else 0
    else:
        a = np.asarray(src)
        if a.dtype.kind == "f":
            val = float(a)
        elif a.dtype.kind == "b":
            val = bool(a)
        else:
            val = int(a)
    dst.module.values[dst.name] = val
    if dst.module.engine is not None:
        dst.module.engine.set_global(dst.name, val)


driver_shim = types.SimpleNamespace(memcpy_htod=memcpy_htod)


# ------------------------------------------------------------------ Solver
class Solver:
    def __init__(self, initialConditions=None, yamlFileName=None, sendWarning=True):
        self.moments = [time.time()]
        self.rank = 0
        self.clusterMasterBool = True
        self.nodeMasterBool = True
        self.gpuBool = True
        self.assignInitialConditions(initialConditions, sendWarning=sendWarning)
        # defaults of io.yamlManager
        self.simulation = True
        self.verbose = False
        self.intermediate = 1
        self.operating = 1
        self.blocksize = (32, 32, 1)
        self.share = 0.9
        self.exid = []
        self.globals = []
        self.cpu = self.cpuStr = ""
        self.gpu = self.gpuStr = ""
        self.output = "output.hdf5"
        self.dtypeStr = "float64"
        self.dtype = np.dtype("float64")
        self.output_every = 1
        self.write_output = True
        self.device = 0
        self.tiling = {}
        self.compile_hook = False
        if yamlFileName is not None:
            self.yamlFileName = yamlFileName
            self._read_yaml()
        elif sendWarning:
            warnings.warn("yaml not specified, requires manual input.")

    # -- configuration -----------------------------------------------------
    def _read_yaml(self):
        with open(self.yamlFileName) as f:
            y = yaml.load(f, Loader=yaml.FullLoader) or {}
        get = lambda k, d: y[k] if k in y else d  # noqa: E731
        self.simulation = get("swept", True)
        self.verbose = get("verbose", False)
        self.intermediate = get("intermediate_steps", 1)
        self.operating = get("operating_points", 1)
        bs = get("blocksize", 32)
        assert bs % (2 * self.operating) == 0, (
            "Invalid blocksize, blocksize must satisfy BS = 2*ops*k and the architectural "
            "limit where k is any integer factor.")
        self.blocksize = (bs, bs, 1)
        self.share = get("share", 0.9)
        self.exid = get("exid", [])
        self.globals = get("globals", [])
        self.cpuStr = self.cpu = get("cpu", "")
        self.gpuStr = self.gpu = get("gpu", "")
        self.output = get("filename", "output.hdf5")
        self.dtypeStr = get("dtype", "float64")
        self.dtype = np.dtype(self.dtypeStr)
        self.output_every = int(get("output_every", 1))
        self.write_output = bool(get("write_output", True))
        self.tiling = get("tiling", {}) or {}
        self.compile_hook = bool(get("compile_hook", False))
        if self.cpu:
            self.loadCPUModule()

    def setGPU(self, gpu):
        self.gpu = self.gpuStr = gpu

    def setCPU(self, cpu):
        self.cpu = self.cpuStr = cpu

    def loadCPUModule(self):
        """Import the CPU plugin from its path (solver.py:83-87)."""
        if isinstance(self.cpu, types.ModuleType):
            return
        path = os.path.abspath(self.cpu)
        spec = importlib.util.spec_from_file_location("module.step", path)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.cuda = driver_shim  # set_globals calls cuda.memcpy_htod
        self.cpu = mod

    def assignInitialConditions(self, initialConditions, sendWarning=True):
        """An array (nv, nx, ny), or a file holding dataset ``data`` (solver.py:89-101)."""
        if isinstance(initialConditions, str):
            self.initialConditions = _read_data(initialConditions)
            self.arrayShape = self.initialConditions.shape
        elif initialConditions is not None:
            self.initialConditions = np.asarray(initialConditions, dtype=np.float64)
            self.arrayShape = self.initialConditions.shape
        elif sendWarning:
            warnings.warn("Initial condition not provided, requires manual assignment with "
                          "assignInitialConditionsFunction.")

    def equation(self):
        """The built-in step function's name, or the path of the hook to compile."""
        name = os.path.splitext(os.path.basename(str(self.gpu)))[0]
        if name in BUILTIN and not self.compile_hook:
            return name
        path = str(self.gpu)
        if not os.path.isfile(path):
            raise FileNotFoundError(
                f"GPU hook {self.gpu!r}: not a file (built-in step functions are {BUILTIN})")
        return path if path.endswith(".cu") else (path, "hook")

    def createTimeStepData(self):
        """pysweep/core/solver.py:113-128."""
        g = self.globals
        self.timeSteps = int((g[1] - g[0]) / g[2])
        if self.simulation:
            self.maxPyramidSize = self.blocksize[0] // (2 * self.operating) - 1
            self.maxGlobalSweptStep = int(self.intermediate * self.timeSteps / self.maxPyramidSize - 1)
            self.timeSteps = int(self.maxPyramidSize * (self.maxGlobalSweptStep + 1) / self.intermediate + 1)
            self.maxOctSize = 2 * self.maxPyramidSize
            self.levels = self.maxPyramidSize * (self.maxGlobalSweptStep + 1)
            self.nframes = self.timeSteps
        else:
            # standardSolve computes intermediate*(timeSteps+1) levels and stores
            # levels 0..timeSteps (solver.py:185, io.py:189-193)
            self.levels = self.intermediate * (self.timeSteps + 1)
            self.nframes = self.timeSteps + 1

    # -- run ---------------------------------------------------------------
    def __call__(self, start=0, stop=-1):
        self.moments.append(time.time())
        eqn = self.equation()
        # float32 fields (yaml `dtype: float32`) stay float32 on the device
        fdt = np.dtype(np.float32) if self.dtype == np.float32 else np.dtype(np.float64)
        ic = np.asarray(self.initialConditions, dtype=fdt)
        if ic.ndim == 2:
            ic = ic[None]
        nv, nx, ny = ic.shape
        self.createTimeStepData()
        self.moments.append(time.time())
        hook_src = None
        if isinstance(eqn, tuple):  # a hook file without the .cu suffix
            with open(eqn[0]) as f:
                hook_src = f.read()
            eqn = eqn[0]
        # share < 1: the first rows on the GPU, the rest stepped on the host by
        # the CPU plugin's own `step` (pysweep/core/process.py:131-176)
        split = None
        has_step = isinstance(self.cpu, types.ModuleType) and hasattr(self.cpu, "step")
        if self.share < 1 and not (has_step and fdt == np.float64 and hook_src is None):
            warnings.warn(f"share={self.share}: the CPU plugin has no numpy step for float64 "
                          "rows, so all rows run on the GPU (results do not depend on the split)")
        elif self.share < 1 and gpu_rows(nx, self.blocksize[0], self.share) < nx:
            # (when ceil(share * block rows) covers every block row, all rows
            # run on the GPU, as in the reference)
            split = SplitSolver(eqn, nx, ny, self.share, cpu_module=self.cpu, nv=nv,
                                ops=self.operating, its=self.intermediate,
                                blocksize=self.blocksize[0], device=self.device,
                                h=self.tiling.get("h", 0), nseg=self.tiling.get("nseg", 0))
        self.effective_share = split.share if split else 1.0
        if split:
            self.engine = split.gpu.eng
        else:
            self.engine = Engine(eqn, nx, ny, nv=nv, ops=self.operating, its=self.intermediate,
                                 blocksize=self.blocksize[0], device=self.device,
                                 dtype=fdt.name, hook_source=hook_src)
            if self.tiling:
                self.engine.configure(**self.tiling)
        src = SourceModuleShim()
        if self.engine.hook:
            src.engine = self.engine  # sizes and values go straight to the hook's constants
        if isinstance(self.cpu, types.ModuleType) and hasattr(self.cpu, "set_globals"):
            self.cpu.set_globals(*self.globals, source_mod=src)
            if not src.values and not self.engine.hook:  # the plugin set only CPU globals
                src.values = plugin_constants(eqn, self.globals)
        elif not self.engine.hook:
            src.values = plugin_constants(eqn, self.globals)
        src.apply(self.engine)
        (split or self.engine).set_state(ic)
        self.moments.append(time.time())
        every = max(1, self.output_every)
        # frames beyond the initial condition at full steps 1..nframes-1
        nkeep = (self.nframes - 1) // every
        frames = (np.empty((nkeep,) + ic.shape, dtype=fdt) if (self.write_output and nkeep)
                  else None)
        mode = "swept" if self.simulation else "standard"
        if split:  # every cell's arithmetic is the same in either decomposition
            split.run(self.levels, frames=frames, frame_every=every)
        else:
            self.engine.run(self.levels, mode=mode, frames=frames, frame_every=every)
        self.engine.synchronize()
        self.moments.append(time.time())
        self.final = split.get_state() if split else self.engine.get_state()
        if frames is not None:
            self.data = np.concatenate([ic[None], frames])
        else:
            self.data = ic[None]
        self.arrayShape = (self.nframes,) + ic.shape
        if self.write_output:
            self._write(self.data, self.moments[-1] - self.moments[0])
        (split or self.engine).close()
        clock = self.moments[stop] - self.moments[start]
        _update_log(self, clock)
        if self.verbose:
            print(f"Done in {self.moments[-1] - self.moments[0]} seconds...")

    def _write(self, data, clocktime):
        payload = {"blocksize": np.array([self.blocksize[0]]),
                   "share": np.array([self.effective_share]),
                   "exid": np.array(self.exid), "globals": np.array(self.globals, dtype=float),
                   "clocktime": np.array([clocktime]), "data": data.astype(self.dtype)}
        try:
            import h5py
        except ImportError:
            h5py = None
        if h5py is not None:
            with h5py.File(self.output, "w") as f:
                for k, v in payload.items():
                    f.create_dataset(k, data=v)
        else:
            base, _ = os.path.splitext(self.output)
            np.savez(base + ".npz", **payload)

    def __str__(self):
        s = "\nPysweep simulation properties:\n"
        s += f"\tsimulation type: {'swept' if self.simulation else 'standard'}\n"
        s += f"\tgpu source: {self.gpuStr}\n\tcpu source: {self.cpuStr}\n"
        s += f"\toutput file: {self.output}\n\tverbose: {self.verbose}\n"
        s += f"\tArray shape: {getattr(self, 'arrayShape', None)}\n\tdtype: {self.dtype}\n"
        s += f"\tshare: {self.share}\n\tblocksize: {self.blocksize[0]}\n"
        s += f"\tstencil size: {int(self.operating * 2 + 1)}\n"
        s += f"\tintermediate time steps: {self.intermediate}\n"
        if self.globals:
            s += "\ttime data (t0,tf,dt): ({},{},{})\n".format(*self.globals[:3])
        return s

    def compactPrint(self):
        moment = self.moments[-1] - self.moments[0] if self.moments else None
        print(("swept: " if self.simulation else "standard: ") +
              f"{self.blocksize[0]}, {self.share}, {self.intermediate}, {self.operating}, "
              f"{getattr(self, 'timeSteps', None)}, {moment}")


def write_field(data, filename):
    """Write an initial field as dataset "data": HDF5 when h5py is importable,
    otherwise an .npz with the same dataset name next to `filename`.  Returns
    the path written (readable by Solver(initialConditions=path))."""
    try:
        import h5py
    except ImportError:
        h5py = None
    if h5py is not None:
        with h5py.File(filename, "w") as f:
            f.create_dataset("data", data=data)
        return filename
    base, _ = os.path.splitext(filename)
    np.savez(base + ".npz", data=data)
    return base + ".npz"


def _read_data(path):
    if path.endswith(".npy"):
        return np.load(path)
    if path.endswith(".npz"):
        return np.load(path)["data"]
    import h5py  # noqa: WPS433 - only HDF5 inputs need it
    with h5py.File(path, "r") as f:
        return np.array(f["data"])


def _update_log(solver, clocktime, path="log.yaml"):
    """Append the run to ./log.yaml with the reference's keys (io.py:10-27)."""
    entry = {datetime.now().strftime("%m/%d/%Y-%H:%M:%S"): {
        "runtime": float(clocktime), "swept": bool(solver.simulation),
        "blocksize": int(solver.blocksize[0]),
        "share": float(getattr(solver, "effective_share", 1.0)), "cpu": str(solver.cpuStr),
        "array_shape": [int(x) for x in solver.arrayShape],
        "time_per_step": float(clocktime / max(solver.arrayShape[0] - 1, 1))}}
    prev = {}
    if os.path.isfile(path):
        with open(path) as f:
            prev = yaml.load(f, Loader=yaml.FullLoader) or {}
    prev.update(entry)
    with open(path, "w") as f:
        yaml.dump(prev, f)
