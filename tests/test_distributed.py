"""Row-slab decomposition over ranks (pysweep_b200.distributed) on CPU.

Each rank's window is solved here by the oracle's periodic stepper instead of
the GPU engine, so the test exercises the driver itself: window placement,
half-cycle lengths, the halo exchange over gloo point-to-point messages (ring
neighbours, both base levels for two-stage schemes), level bookkeeping and
the gather.  The gathered field must equal one oracle run over the whole grid
bitwise.
"""
import datetime
import os
import socket

import numpy as np
import pytest

import oracle
from oracle_window import OracleWindow


def case(name):
    rng = np.random.default_rng(7)
    if name == "heat_fe":
        g = [0.0, 1.0, 0.2 / 64 / 64, 1 / 64, 1 / 64, 1.0, True]
        return dict(eq="heat", ic=rng.standard_normal((1, 64, 64)), g=g, its=1, ops=1, bs=16,
                    levels=40)
    if name == "heat_rk2":
        g = [0.0, 1.0, 0.1 / 64 / 64, 1 / 64, 1 / 64, 1.0, False]
        return dict(eq="heat", ic=rng.standard_normal((1, 64, 64)), g=g, its=2, ops=1, bs=16,
                    levels=31)
    if name == "heat_fe3":
        g = [0.0, 1.0, 0.2 / 96 / 96, 1 / 96, 1 / 96, 1.0, True]
        return dict(eq="heat", ic=rng.standard_normal((1, 96, 64)), g=g, its=1, ops=1, bs=16,
                    levels=23)
    if name == "euler":
        from pysweep_b200.equations.euler import analytical_array
        n = 64
        dx = 10.0 / n
        g = [0.0, 1.0, 0.1 * dx, dx, dx, 1.4]
        return dict(eq="euler", ic=analytical_array(n, n, 0.0), g=g, its=2, ops=2, bs=16,
                    levels=18)
    raise KeyError(name)


def solve_slabs(c, world, rank, group=None, by_slab=False):
    from pysweep_b200.distributed import SlabSolver
    nv, nx, ny = c["ic"].shape
    win = OracleWindow(c["eq"], c["g"], c["its"])
    s = SlabSolver(c["eq"], nx, ny, nv=nv, ops=c["ops"], its=c["its"], blocksize=c["bs"],
                   group=group, window=win)
    if by_slab:
        s.set_slab(c["ic"][:, s.row0:s.row0 + s.rows])
    else:
        s.set_state(c["ic"])
    s.run(c["levels"])
    return [s.gather(level) for level in range(c["its"])]


def expected(c):
    _, u, up = oracle.standard(c["eq"], c["ic"], c["g"], c["its"], c["levels"], frames=False)
    return [u, up][:c["its"]]


def _worker(rank, world, port, name, by_slab, outdir):
    import torch.distributed as dist
    # a short timeout turns a mismatched exchange into an error, not a hang
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        c = case(name)
        got = solve_slabs(c, world, rank, by_slab=by_slab)
        if rank == 0:
            np.save(os.path.join(outdir, "got.npy"), np.stack(got))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("name", ["heat_fe", "heat_rk2", "euler"])
def test_single_rank_matches_global_oracle(name):
    c = case(name)
    got = solve_slabs(c, 1, 0)
    for a, b in zip(got, expected(c)):
        assert np.array_equal(a, b)


@pytest.mark.timeout(300)
@pytest.mark.parametrize("name,world,by_slab", [("heat_fe", 2, False), ("heat_rk2", 2, True),
                                                ("euler", 2, False), ("heat_fe3", 3, True)])
def test_gloo_ranks_match_global_oracle(tmp_path, name, world, by_slab):
    import torch.multiprocessing as mp
    mp.start_processes(_worker, args=(world, _free_port(), name, by_slab, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    got = np.load(tmp_path / "got.npy")
    for a, b in zip(got, expected(case(name))):
        assert np.array_equal(a, b)


def test_rejects_slabs_that_are_not_whole_blocks():
    from pysweep_b200.distributed import SlabSolver
    with pytest.raises(ValueError):
        SlabSolver("heat", 72, 64, blocksize=16, window=OracleWindow("heat", [], 1))
