"""Row slabs on the GPU engine (pysweep_b200.distributed).

One rank: the slab window, its halo refresh through ps_get_rows/ps_set_rows
and the per-half-cycle runs must reproduce a single Engine run of the whole
grid bitwise.  Two ranks: two processes on the same GPU, each with its own
engine window, exchanging halo strips through gloo (host memory); the kernels
of the two processes never wait on one another.  The gathered field must
equal the oracle's run of the whole grid bitwise.
"""
import datetime
import os
import socket

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def heat_case(n, rows=None, seed=3):
    rng = np.random.default_rng(seed)
    rows = rows or n
    g = [0.0, 1.0, 0.2 / n / n, 1 / n, 1 / n, 1.0, True]
    return rng.standard_normal((1, rows, n)), g


def _engine_run(eq, ic, g, its, ops, bs, levels):
    from pysweep_b200 import Engine, plugin_constants
    nv, nx, ny = ic.shape
    with Engine(eq, nx, ny, nv=nv, ops=ops, its=its, blocksize=bs) as e:
        for k, v in plugin_constants(eq, g).items():
            e.set_global(k, v)
        e.set_state(ic)
        e.run(levels)
        return [e.get_state(level) for level in range(its)]


def _slab_run(eq, ic, g, its, ops, bs, levels, group=None, by_slab=False):
    from pysweep_b200 import plugin_constants
    from pysweep_b200.distributed import SlabSolver
    nv, nx, ny = ic.shape
    s = SlabSolver(eq, nx, ny, nv=nv, ops=ops, its=its, blocksize=bs, group=group)
    for k, v in plugin_constants(eq, g).items():
        s.set_global(k, v)
    if by_slab:
        s.set_slab(ic[:, s.row0:s.row0 + s.rows])
    else:
        s.set_state(ic)
    s.run(levels)
    out = [s.gather(level) for level in range(its)]
    s.close()
    return out


@pytest.mark.parametrize("bs,levels", [(32, 100), (16, 45)])
def test_one_rank_slab_matches_engine_heat(bs, levels):
    ic, g = heat_case(256)
    a = _slab_run("heat", ic, g, 1, 1, bs, levels)
    b = _engine_run("heat", ic, g, 1, 1, bs, levels)
    assert np.array_equal(a[0], b[0])


def test_one_rank_slab_matches_engine_euler():
    from pysweep_b200.equations.euler import analytical_array
    n = 128
    dx = 10.0 / n
    g = [0.0, 1.0, 0.1 * dx, dx, dx, 1.4]
    ic = analytical_array(n, n, 0.0)
    a = _slab_run("euler", ic, g, 2, 2, 16, 22, by_slab=True)
    b = _engine_run("euler", ic, g, 2, 2, 16, 22)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def _worker(rank, world, port, outdir):
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(0)
    # a short timeout turns a mismatched exchange into an error, not a hang
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ic, g = heat_case(128, rows=256, seed=5)
        got = _slab_run("heat", ic, g, 1, 1, 16, 60, by_slab=rank % 2 == 1)
        if rank == 0:
            np.save(os.path.join(outdir, "got.npy"), got[0])
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_ranks_on_one_gpu_through_gloo(tmp_path):
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    ic, g = heat_case(128, rows=256, seed=5)
    _, want, _ = oracle.standard("heat", ic, g, 1, 60, frames=False)
    assert np.array_equal(np.load(tmp_path / "got.npy"), want)
