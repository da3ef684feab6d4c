"""A run split between the GPU and the host: the yaml `share` below 1.

The reference gives the first ceil(share * nx / bs) block rows of the grid to
its GPUs and the remaining rows to its CPU ranks (pysweep/core/process.py:
131-176, MajorSplit), which step them with the plugin's own numpy `step`
(pysweep/core/block.py:45-62, setupCPUSwept), and swaps the edge strips after
every phase group (pysweep/core/functions.py:90-123).  SplitSolver does the
same with two windows of the row-slab decomposition of distributed.py:

* the GPU rows [0, R) in an Engine window of R + bs rows (the swept kernels);
* the host rows [R, nx) in a window of nx - R + bs rows that the CPU plugin's
  `step(state, iidx, arrayTimeIndex, globalTimeStep)` advances level by level
  over every cell of the window, as the reference's CPU ranks do;

each window is periodic in itself, a half-cycle of H <= MPSS levels corrupts
at most OPS*H < bs/2 rows at its ends (its halo), and after every half-cycle
the first and last bs/2 rows of each part, for every base level, are copied
into the other window's halos (device <-> host copies of the strips).  The
GPU half-cycle is queued first and runs while the host steps its rows.  Every
cell is computed by the same arithmetic as in a run of the whole grid, so the
result equals it bitwise when the plugin's `step` follows the same operation
order as the GPU kernels (the reference's and this package's heat plugins do).
"""
import math

import numpy as np

from .distributed import EngineWindow


class PluginWindow:
    """Host rows stepped by a CPU plugin's `step` (EngineWindow's methods).

    The state is the reference's 4-D [t, v, x, y] array with three time
    slots (previous, current, next); each level calls step(state, iidx, 1,
    globalTimeStep) on every cell and shifts the slots."""

    def __init__(self, module, nxw, ny, nv, its):
        if not hasattr(module, "step"):
            raise ValueError("the CPU plugin has no step(state, iidx, arrayTimeIndex, "
                             "globalTimeStep) for the host rows of share < 1")
        self.mod, self.nv, self.ny, self.its = module, nv, ny, its
        self.state = np.zeros((3, nv, nxw, ny))
        xs, ys = np.meshgrid(np.arange(nxw), np.arange(ny), indexing="ij")
        self.iidx = np.stack([xs.ravel(), ys.ravel()], axis=1)  # (x, y) rows

    def set_global(self, name, value):
        pass  # the plugin's module globals are set by its set_globals

    def set_window(self, field):
        f = np.asarray(field, dtype=np.float64)
        if f.ndim == 4:  # oldest level first
            self.state[0], self.state[1] = f[0], f[-1]
        else:
            self.state[0] = f
            self.state[1] = f

    def run(self, nlevels, gts0):
        for k in range(nlevels):
            self.mod.step(self.state, self.iidx, 1, gts0 + k)
            self.state[0] = self.state[1]
            self.state[1] = self.state[2]

    def level(self, level):
        return self.state[1] if level == 0 else self.state[0]

    def get_rows(self, row0, nrows, level):
        return self.level(level)[:, row0:row0 + nrows].copy()

    def set_rows(self, row0, rows, level):
        self.level(level)[:, row0:row0 + rows.shape[1]] = rows

    def synchronize(self):
        pass

    def close(self):
        pass


def gpu_rows(nx, bs, share):
    """Rows of the GPU part: ceil(block rows * share) block rows
    (pysweep/core/process.py:146-148)."""
    return int(math.ceil(nx // bs * share)) * bs


class SplitSolver:
    """Swept solve of one periodic (nv, nx, ny) grid, the first
    gpu_rows(nx, bs, share) rows on the GPU, the rest on the host.
    `gpu_window` / `cpu_window` replace the two windows (tests)."""

    def __init__(self, equation, nx, ny, share, cpu_module=None, nv=1, ops=1, its=1,
                 blocksize=16, device=0, h=0, nseg=0, gpu_window=None, cpu_window=None):
        bs = blocksize
        if not 0 < share < 1:
            raise ValueError(f"share {share}: a split needs 0 < share < 1")
        self.R = gpu_rows(nx, bs, share)
        if not bs <= self.R <= nx - bs:
            raise ValueError(f"share {share} of {nx // bs} block rows leaves a part of less "
                             "than one block row")
        self.nx, self.ny, self.nv, self.ops, self.its, self.bs = nx, ny, nv, ops, its, bs
        self.share = self.R / nx  # effective share after rounding (process.py:148)
        self.hw = bs // 2
        mpss = bs // (2 * ops) - 1
        self.H = h or mpss
        if not 1 <= self.H <= mpss or ops * self.H >= self.hw:
            raise ValueError(f"levels per half-cycle must be in [1, {mpss}]")
        self.gpu = gpu_window if gpu_window is not None else EngineWindow(
            equation, self.R + bs, ny, nv, ops, its, bs, device, h, nseg)
        self.cpu = cpu_window if cpu_window is not None else PluginWindow(
            cpu_module, nx - self.R + bs, ny, nv, its)
        self.gts = 1

    def set_global(self, name, value):
        self.gpu.set_global(name, value)

    def _windows(self, f):
        """The two windows' rows of a (.., nx, ny) field: each part with bs/2
        rows of the other part above and below it (periodic)."""
        hw, R, nx = self.hw, self.R, self.nx
        g = (np.arange(-hw, R + hw)) % nx
        c = (np.arange(R - hw, nx + hw)) % nx
        return np.take(f, g, axis=-2), np.take(f, c, axis=-2)

    def set_state(self, field):
        """The initial field, (nv, nx, ny) or (its, nv, nx, ny)."""
        f = np.asarray(field, dtype=np.float64)
        g, c = self._windows(f)
        self.gpu.set_window(np.ascontiguousarray(g))
        self.cpu.set_window(np.ascontiguousarray(c))
        self.gts = 1

    def run(self, nlevels, gts0=None, frames=None, frame_every=1):
        """Advance `nlevels` levels, at most H levels between two strip
        exchanges on both parts (the GPU's queued first, the host's meanwhile).
        frames: None or an array (k, nv, nx, ny) receiving every
        frame_every-th full step, as Engine.run stores them; a half-cycle is
        cut at a frame's level (the halos' corruption depends only on the
        levels since the last exchange, so the cut changes no cell)."""
        if gts0 is not None:
            self.gts = gts0
        done = since = 0
        every = max(1, frame_every)
        while done < nlevels:
            h = min(self.H - since, nlevels - done)
            if frames is not None:  # stop at the next stored full step
                step_levels = self.its * every
                h = min(h, step_levels - done % step_levels)
            self.gpu.run(h, self.gts)   # asynchronous on the device
            self.cpu.run(h, self.gts)   # meanwhile on the host
            self.gts += h
            done += h
            since += h
            if frames is not None and done % (self.its * every) == 0:
                slot = done // (self.its * every) - 1
                if slot < len(frames):
                    frames[slot] = self.get_state()
            if since == self.H or done == nlevels:
                self._exchange()
                since = 0

    def _exchange(self):
        hw, R, C = self.hw, self.R, self.nx - self.R
        for level in range(self.its):
            g_first = self.gpu.get_rows(hw, hw, level)
            g_last = self.gpu.get_rows(R, hw, level)
            c_first = self.cpu.get_rows(hw, hw, level)
            c_last = self.cpu.get_rows(C, hw, level)
            self.gpu.set_rows(0, c_last, level)        # the rows above the GPU part
            self.gpu.set_rows(R + hw, c_first, level)  # and below it
            self.cpu.set_rows(0, g_last, level)
            self.cpu.set_rows(C + hw, g_first, level)

    def get_state(self, level=0):
        """The whole (nv, nx, ny) field of base level `level` (0 = newest)."""
        g = self.gpu.get_rows(self.hw, self.R, level)
        c = self.cpu.get_rows(self.hw, self.nx - self.R, level)
        return np.concatenate([np.asarray(g), np.asarray(c)], axis=-2)

    def synchronize(self):
        self.gpu.synchronize()

    def close(self):
        self.gpu.close()
        self.cpu.close()
