"""Batched instances: each field of a batch advances exactly as the same field
alone (bitwise), with and without CUDA-graph replay."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _heat_g(n, alpha):
    dx = 1.0 / n
    dt = 0.2 * dx * dx / alpha
    return [0.0, 1.0, dt, dx, dx, alpha, True]


def _single(eqn, ic, g, its, bs, nl):
    from pysweep_b200 import Engine, plugin_constants
    with Engine(eqn, ic.shape[1], ic.shape[2], nv=ic.shape[0], its=its, blocksize=bs) as e:
        for k, v in plugin_constants(eqn, g).items():
            e.set_global(k, v)
        e.set_state(ic)
        e.run(nl)
        return e.get_state()


@pytest.mark.parametrize("graph", [True, False])
def test_heat_batch_matches_single_instances(graph):
    from pysweep_b200 import plugin_constants
    from pysweep_b200.batch import Batch
    sizes = [128, 160, 224, 96, 256, 64]   # odd multiples of 32 included
    rng = np.random.default_rng(3)
    alphas = rng.uniform(0.5, 2.0, len(sizes))
    ics = [rng.standard_normal((1, n, n)) for n in sizes]
    nl = 37
    with Batch("heat", [(n, n) for n in sizes], its=1, blocksize=32) as b:
        for i, n in enumerate(sizes):
            b.set_constants(i, plugin_constants("heat", _heat_g(n, alphas[i])))
            b.set_state(i, ics[i])
        b.run(nl, graph=graph)
        b.run(nl, graph=graph)  # a second run continues from the first
        for i, n in enumerate(sizes):
            got = b.get_state(i)
            g = _heat_g(n, alphas[i])
            ref = _single("heat", ics[i], g, 1, 32, 2 * nl)
            assert np.array_equal(got, ref), f"instance {i} ({n}^2)"
            _, orc, _ = oracle.standard("heat", ics[i], g, 1, 2 * nl, frames=False)
            assert np.array_equal(got, orc)


def test_euler_batch_matches_single_instances():
    from pysweep_b200 import plugin_constants
    from pysweep_b200.batch import Batch
    from pysweep_b200.equations.euler import analytical_array
    sizes = [64, 96, 128]
    nl = 2 * 9
    ics, gs = [], []
    for i, n in enumerate(sizes):
        ics.append(analytical_array(n, n, 0.0, strength=1.0 + i))
        dx = 10.0 / n
        gs.append([0.0, 1.0, 0.1 * dx, dx, dx, 1.4])
    with Batch("euler", [(n, n) for n in sizes], its=2, blocksize=16) as b:
        for i in range(len(sizes)):
            b.set_constants(i, plugin_constants("euler", gs[i]))
            b.set_state(i, ics[i])
        b.run(nl)
        for i, n in enumerate(sizes):
            ref = _single("euler", ics[i], gs[i], 2, 16, nl)
            assert np.array_equal(b.get_state(i), ref)


@pytest.mark.parametrize("graph", [True, False])
def test_euler_batch_odd_runs_add_up_to_one_run(graph):
    """Two stages per step: the step function picks the stage by
    globalTimeStep % 2, so consecutive runs of odd length must continue the
    count (7 + 11 levels equal one run of 18)."""
    from pysweep_b200 import plugin_constants
    from pysweep_b200.batch import Batch
    from pysweep_b200.equations.euler import analytical_array
    sizes = [64, 96]
    ics, gs = [], []
    for i, n in enumerate(sizes):
        ics.append(analytical_array(n, n, 0.0, strength=2.0 + i))
        dx = 10.0 / n
        gs.append([0.0, 1.0, 0.1 * dx, dx, dx, 1.4])
    with Batch("euler", [(n, n) for n in sizes], its=2, blocksize=16) as b:
        for i in range(len(sizes)):
            b.set_constants(i, plugin_constants("euler", gs[i]))
            b.set_state(i, ics[i])
        b.run(7, graph=graph)
        b.run(11, graph=graph)
        for i, n in enumerate(sizes):
            ref = _single("euler", ics[i], gs[i], 2, 16, 18)
            got = b.get_state(i)
            assert np.array_equal(got, ref), f"instance {i}: {np.abs(got - ref).max()}"
        # a new state restarts that instance's count at globalTimeStep 1
        b.set_state(0, ics[0])
        b.set_state(1, ics[1])
        b.run(18, graph=graph)
        for i in range(len(sizes)):
            assert np.array_equal(b.get_state(i), _single("euler", ics[i], gs[i], 2, 16, 18))


def test_heat_batch_sizes_spanning_128_to_2048():
    """The batched range of the benchmark's instances (multiples of 32 in
    [128, 2048]): every instance bitwise equal to the oracle's standard run."""
    from pysweep_b200 import plugin_constants
    from pysweep_b200.batch import Batch
    sizes = [128, 2048, 544, 1056, 160, 1984]
    rng = np.random.default_rng(11)
    alphas = rng.uniform(0.5, 2.0, len(sizes))
    ics = [rng.standard_normal((1, n, n)) for n in sizes]
    nl = 30
    with Batch("heat", [(n, n) for n in sizes], its=1, blocksize=32) as b:
        for i, n in enumerate(sizes):
            b.set_constants(i, plugin_constants("heat", _heat_g(n, alphas[i])))
            b.set_state(i, ics[i])
        b.run(nl, graph=True)
        for i, n in enumerate(sizes):
            _, orc, _ = oracle.standard("heat", ics[i], _heat_g(n, alphas[i]), 1, nl, frames=False)
            assert np.array_equal(b.get_state(i), orc), f"instance {i} ({n}^2)"
