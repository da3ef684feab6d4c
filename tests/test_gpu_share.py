"""The CPU/GPU share split on the GPU: Solver runs with share 0.5 and 0.75
(the first ceil(share * nx / bs) block rows on the GPU, the rest stepped on
the host by the heat plugin's numpy step, pysweep/core/process.py:131-176)
equal the whole-GPU run (share 1) bitwise, every frame included, and record
the effective share."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _solve(tmp_path, share, scheme, swept=True):
    import yaml

    from pysweep_b200 import Solver
    n = 64
    x = np.arange(n) / n
    ic = (np.sin(2 * np.pi * x)[:, None] * np.cos(4 * np.pi * x)[None, :])[None]
    dx = 1.0 / n
    dt = (0.2 if scheme else 0.1) * dx * dx
    its = 1 if scheme else 2
    y = tmp_path / f"s{share}.yaml"
    y.write_text(yaml.dump({
        "swept": swept, "blocksize": 16, "intermediate_steps": its, "operating_points": 1,
        "globals": [0.0, 45 * dt, dt, dx, dx, 1.0, scheme], "share": share,
        "cpu": os.path.join(ROOT, "pysweep_b200", "equations", "heat.py"), "gpu": "heat.cu",
        "filename": str(tmp_path / f"out{share}.hdf5")}))
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        s = Solver(ic, str(y))
        s()
    finally:
        os.chdir(cwd)
    return s


@pytest.mark.parametrize("scheme", [True, False])
@pytest.mark.parametrize("share", [0.5, 0.75])
def test_share_split_equals_whole_gpu_run(tmp_path, share, scheme):
    whole = _solve(tmp_path, 1.0, scheme)
    split = _solve(tmp_path, share, scheme)
    assert split.effective_share == np.ceil(4 * share) / 4 < 1
    assert whole.data.shape == split.data.shape
    assert np.array_equal(whole.data, split.data)
    assert np.array_equal(whole.final, split.final)


def test_share_split_standard_flag(tmp_path):
    """`swept: false` with a split: both parts keep every cell's arithmetic."""
    a = _solve(tmp_path, 1.0, True, swept=False)
    b = _solve(tmp_path, 0.5, True, swept=False)
    assert np.array_equal(a.data, b.data)
