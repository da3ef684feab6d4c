"""One periodic grid split into row slabs over the ranks of a process group.

Rank r of P owns the global rows [r*R, (r+1)*R), R = nx / P (a multiple of the
blocksize), and solves them in a window of R + bs rows: its slab with a halo
of bs/2 rows above and below, treated by its own engine as one periodic grid.
A swept half-cycle advances H <= MPSS = bs/(2*OPS) - 1 levels, and one level
changes a cell only from neighbours at most OPS rows away.  The window's
wrap-around therefore corrupts at most OPS*H < bs/2 rows at either end during
a half-cycle, all of them in the halo, and the R slab rows come out exactly as
in a run of the whole grid (bitwise: the decomposition does not change any
cell's arithmetic).  After every half-cycle each rank sends the first and the
last bs/2 rows of its slab, for every base level, to the ranks above and below,
which write them into their halos: the path's one exchange step.  It is done
with point-to-point sends of torch.distributed (NCCL between GPUs; any backend
works, gloo stages through host memory).

Reference: the rows are split among ranks in pysweep/core/process.py:131-176
(MajorSplit), and after every phase group sendForward / sendBackward
(pysweep/core/functions.py:90-123) swap a `splitx`-row edge strip with the
neighbour ranks through MPI Sendrecv and shift the shared array by it.  Here
the swept kernels never leave the window, and only the halo strips move.
"""
import numpy as np

from .engine import DEFAULT_NV, DEFAULT_OPS, Engine

try:
    import torch
    import torch.distributed as dist
except ImportError:  # pragma: no cover - torch is part of the runtime here
    torch = dist = None


class EngineWindow:
    """The slab window on one GPU: an Engine over R + bs periodic rows."""

    def __init__(self, equation, nxw, ny, nv, ops, its, bs, device, h=0, nseg=0, on_device=False):
        self.eng = Engine(equation, nxw, ny, nv=nv, ops=ops, its=its, blocksize=bs, device=device)
        if h or nseg:
            self.eng.configure(h=h, nseg=nseg)
        self.on_device = on_device
        self.device = device
        self.nv, self.ny = nv, ny
        if torch is not None and torch.cuda.is_available():
            # the exchange runs on torch's current stream: queue the solver there too
            self.eng.set_stream(torch.cuda.current_stream(device).cuda_stream)

    def set_global(self, name, value):
        self.eng.set_global(name, value)

    def set_window(self, field):
        self.eng.set_state(field)

    def run(self, nlevels, gts0):
        self.eng.run(nlevels, "swept", gts0)

    def get_rows(self, row0, nrows, level):
        if self.on_device:
            out = torch.empty((self.nv, nrows, self.ny), dtype=torch.float64,
                              device=f"cuda:{self.device}")
            return self.eng.get_rows(row0, nrows, level, out=out)
        return self.eng.get_rows(row0, nrows, level)

    def set_rows(self, row0, rows, level):
        self.eng.set_rows(row0, rows, level)

    def synchronize(self):
        self.eng.synchronize()

    def close(self):
        self.eng.close()


def _world(group):
    if dist is not None and dist.is_available() and dist.is_initialized():
        return dist.get_world_size(group), dist.get_rank(group)
    return 1, 0


class SlabSolver:
    """Swept solve of one periodic (nv, nx, ny) grid on all ranks of `group`.

    Every rank constructs it with the same arguments (collective).  `window`
    replaces the per-rank engine by any object with the EngineWindow methods.
    """

    def __init__(self, equation, nx, ny, nv=None, ops=None, its=1, blocksize=16, h=0, nseg=0,
                 group=None, device=0, window=None):
        self.world, self.rank = _world(group)
        self.group = group
        bs = blocksize
        self.nv = nv if nv is not None else DEFAULT_NV.get(equation, 1)
        self.ops = ops if ops is not None else DEFAULT_OPS.get(equation, 1)
        if bs % (2 * self.ops) or nx % (self.world * bs):
            raise ValueError(f"nx={nx} must be a multiple of ranks*blocksize = "
                             f"{self.world}*{bs}, and blocksize of 2*ops")
        self.nx, self.ny, self.bs, self.its = nx, ny, bs, its
        self.rows = nx // self.world
        self.halo = bs // 2
        self.nxw = self.rows + 2 * self.halo
        mpss = bs // (2 * self.ops) - 1
        self.H = h or mpss
        if not 1 <= self.H <= mpss:
            raise ValueError(f"levels per half-cycle must be in [1, {mpss}]")
        assert self.ops * self.H < self.halo
        self.row0 = self.rank * self.rows
        self.backend = dist.get_backend(group) if self.world > 1 else None
        self.on_device = self.backend == "nccl"
        self.win = window if window is not None else EngineWindow(
            equation, self.nxw, ny, self.nv, self.ops, its, bs, device, h, nseg, self.on_device)
        self.gts = 1
        self.prev = (self.rank - 1) % self.world
        self.next = (self.rank + 1) % self.world
        if self.world > 1 and group is not None:
            self.prev = dist.get_global_rank(group, self.prev)
            self.next = dist.get_global_rank(group, self.next)

    # -- set-up ------------------------------------------------------------
    def set_global(self, name, value):
        self.win.set_global(name, value)

    def window_rows(self):
        """Global row of each window row."""
        return (self.row0 - self.halo + np.arange(self.nxw)) % self.nx

    def set_state(self, field):
        """The whole grid's initial field, (nv, nx, ny) or (its, nv, nx, ny),
        given on every rank; each keeps its window.  Collective, like
        set_slab (one halo exchange), so ranks may mix the two."""
        f = np.asarray(field, dtype=np.float64)
        self.win.set_window(np.ascontiguousarray(np.take(f, self.window_rows(), axis=-2)))
        self.gts = 1
        self._exchange()

    def set_slab(self, slab):
        """This rank's own (nv, R, ny) rows (numpy, or a torch CUDA tensor that
        stays on the device); the halos are filled by one exchange (collective)."""
        if torch is not None and torch.is_tensor(slab):
            win = torch.zeros(tuple(slab.shape[:-2]) + (self.nxw, self.ny), dtype=torch.float64,
                              device=slab.device)
            win[..., self.halo:self.halo + self.rows, :] = slab
        else:
            s = np.asarray(slab, dtype=np.float64)
            win = np.zeros(s.shape[:-2] + (self.nxw, self.ny))
            win[..., self.halo:self.halo + self.rows, :] = s
        self.win.set_window(win)
        self.gts = 1
        self._exchange()

    # -- time stepping -----------------------------------------------------
    def run(self, nlevels, gts0=None):
        """Advance `nlevels` levels: one swept half-cycle of at most H levels
        on every window, then the halo exchange, until done."""
        if gts0 is not None:
            self.gts = gts0
        done = 0
        while done < nlevels:
            h = min(self.H, nlevels - done)
            self.win.run(h, self.gts)
            self.gts += h
            done += h
            self._exchange()

    def _exchange(self):
        hw, R = self.halo, self.rows
        for level in range(self.its):
            first = self.win.get_rows(hw, hw, level)   # -> previous rank's bottom halo
            last = self.win.get_rows(R, hw, level)     # -> next rank's top halo
            if self.world == 1:
                self.win.set_rows(R + hw, first, level)
                self.win.set_rows(0, last, level)
                continue
            send_first, send_last = self._tensor(first), self._tensor(last)
            recv_bottom, recv_top = torch.empty_like(send_first), torch.empty_like(send_last)
            ops = [dist.P2POp(dist.isend, send_first, self.prev, self.group, 2 * level),
                   dist.P2POp(dist.irecv, recv_bottom, self.next, self.group, 2 * level),
                   dist.P2POp(dist.isend, send_last, self.next, self.group, 2 * level + 1),
                   dist.P2POp(dist.irecv, recv_top, self.prev, self.group, 2 * level + 1)]
            for req in dist.batch_isend_irecv(ops):
                req.wait()
            self.win.set_rows(R + hw, self._array(recv_bottom), level)
            self.win.set_rows(0, self._array(recv_top), level)

    def _tensor(self, rows):
        if torch.is_tensor(rows):
            return rows.contiguous()
        return torch.from_numpy(np.ascontiguousarray(rows))

    def _array(self, t):
        return t if self.on_device else t.numpy()

    # -- results -----------------------------------------------------------
    def get_slab(self, level=0):
        """This rank's (nv, R, ny) rows of base level `level` (0 = newest), on the host."""
        r = self.win.get_rows(self.halo, self.rows, level)
        return r.cpu().numpy() if torch is not None and torch.is_tensor(r) else np.asarray(r)

    def gather(self, level=0):
        """The whole (nv, nx, ny) field on every rank (collective)."""
        slab = self.get_slab(level)
        if self.world == 1:
            return slab
        t = torch.from_numpy(slab)
        if self.on_device:
            t = t.cuda()
        parts = [torch.empty_like(t) for _ in range(self.world)]
        dist.all_gather(parts, t, group=self.group)
        return np.concatenate([p.cpu().numpy() for p in parts], axis=-2)

    def synchronize(self):
        self.win.synchronize()

    def close(self):
        self.win.close()
