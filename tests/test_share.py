"""The CPU/GPU share split (pysweep_b200.share) on CPU.

The host part runs the heat plugin's own numpy step (what the reference's
CPU ranks run, pysweep/core/block.py:45-62); the GPU part is stood in for by
the oracle's window here (tests/test_gpu_share.py runs it on the GPU).  The
split follows the reference's row rounding (pysweep/core/process.py:146-148)
and must reproduce one oracle run of the whole grid bitwise, frames included.
"""
import numpy as np
import pytest

import oracle
from oracle_window import OracleWindow


def _heat(n, scheme):
    dx = 1.0 / n
    return [0.0, 1.0, (0.2 if scheme else 0.1) * dx * dx, dx, dx, 1.0, scheme]


@pytest.mark.parametrize("share,scheme,levels", [(0.5, True, 40), (0.75, True, 23),
                                                  (0.3, False, 31)])
def test_split_matches_whole_grid(share, scheme, levels):
    from pysweep_b200.equations import heat
    from pysweep_b200.share import SplitSolver, gpu_rows
    n, bs = 64, 16
    its = 1 if scheme else 2
    g = _heat(n, scheme)
    heat.set_globals(*g)
    ic = np.random.default_rng(5).standard_normal((1, n, n))
    s = SplitSolver("heat", n, n, share, cpu_module=heat, its=its, blocksize=bs,
                    gpu_window=OracleWindow("heat", g, its))
    assert s.R == gpu_rows(n, bs, share) and s.R % bs == 0 and 0 < s.R < n
    s.set_state(ic)
    frames = np.zeros((levels // its,) + ic.shape)
    s.run(levels, frames=frames)
    ref, fin, _ = oracle.standard("heat", ic, g, its, levels)
    assert np.array_equal(s.get_state(), fin)
    assert np.array_equal(frames, ref[1:1 + len(frames)])


def test_split_rows_and_errors():
    from pysweep_b200.equations import heat
    from pysweep_b200.share import SplitSolver, gpu_rows
    assert gpu_rows(384, 16, 0.9) == 352          # ceil(24 * 0.9) = 22 block rows
    assert gpu_rows(64, 16, 0.3) == 32            # ceil(1.2) = 2
    with pytest.raises(ValueError):               # the host part would be empty
        SplitSolver("heat", 64, 64, 0.99, cpu_module=heat, blocksize=16,
                    gpu_window=OracleWindow("heat", _heat(64, True), 1))
    with pytest.raises(ValueError):               # no CPU step in the plugin
        from pysweep_b200.equations import euler
        SplitSolver("euler", 64, 64, 0.5, cpu_module=euler, nv=4, ops=2, its=2, blocksize=16,
                    gpu_window=OracleWindow("euler", [0, 1, 0.01, 0.1, 0.1, 1.4], 2))
