"""The command line's options and initial-condition files (no GPU needed)."""
import numpy as np
import pytest

from pysweep_b200 import commandline
from pysweep_b200.equations import euler, heat
from pysweep_b200.solver import _read_data


def test_defaults_follow_the_reference():
    a = commandline.parser().parse_args([])
    # pysweep/utils/commandline.py:123-131
    assert (a.blocksize, a.spacesteps, a.timesteps, a.share) == (12, 24, 10, 0.5)
    assert not a.swept and a.function is None


def test_array_size_rounds_up_to_the_blocksize():
    a = commandline.parser().parse_args(["-b", "8", "-nx", "30"])
    with pytest.warns(UserWarning):
        commandline.adjust_array_size(a)
    assert a.spacesteps == 32


def test_initial_condition_files(tmp_path):
    p = heat.createInitialConditions(16, 12, alpha=1, filename=str(tmp_path / "h.hdf5"))
    d = _read_data(p)
    x = np.linspace(0, 1, 16, endpoint=True)[:, None]
    y = np.linspace(0, 1, 12, endpoint=True)[None, :]
    assert d.shape == (1, 16, 12)
    assert np.array_equal(d[0], np.sin(2 * np.pi * x) * np.sin(2 * np.pi * y) * np.exp(0.0))
    p = euler.createInitialConditions(8, 8, filename=str(tmp_path / "e.hdf5"))
    d = _read_data(p)
    assert d.shape == (4, 8, 8) and np.all(d[0] > 0)
