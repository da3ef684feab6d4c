"""The HDF5 branch of the writers and the reader, run against an in-memory
stand-in for h5py (h5py is not installed here): the datasets the reference
creates (pysweep/core/io.py:78-90: blocksize, share, exid, globals, clocktime
and data[t, v, x, y] of the run's dtype) and the initial-condition files of
the plugins (pysweep/equations/heat.py:66-88: one dataset "data")."""
import sys
import types

import numpy as np
import pytest


class _FakeH5:
    """h5py.File over a dict of {path: {name: array}}."""

    files = {}

    def __init__(self, path, mode="r", **kw):
        if mode == "w":
            _FakeH5.files[path] = {}
        elif path not in _FakeH5.files:
            raise OSError(path)
        self.ds = _FakeH5.files[path]

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def create_dataset(self, name, shape=None, dtype=None, data=None):
        a = np.array(data, dtype=dtype) if data is not None else np.zeros(shape, dtype=dtype)
        self.ds[name] = a
        return a

    def __getitem__(self, name):
        return self.ds[name]


@pytest.fixture
def fake_h5py(monkeypatch):
    mod = types.ModuleType("h5py")
    mod.File = _FakeH5
    _FakeH5.files = {}
    monkeypatch.setitem(sys.modules, "h5py", mod)
    return _FakeH5.files


def test_initial_condition_file_round_trip(fake_h5py, tmp_path):
    from pysweep_b200.equations import heat
    from pysweep_b200.solver import _read_data
    path = heat.createInitialConditions(16, 24, filename=str(tmp_path / "heatConditions.hdf5"))
    assert path.endswith(".hdf5") and set(fake_h5py[path]) == {"data"}
    d = _read_data(path)
    assert d.shape == (1, 16, 24) and d.dtype == np.float64
    assert np.array_equal(d, fake_h5py[path]["data"])


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_output_datasets_follow_the_reference(fake_h5py, tmp_path, dtype):
    from pysweep_b200.solver import Solver
    s = Solver.__new__(Solver)  # the writer needs only these attributes
    s.blocksize = (16, 16, 1)
    s.effective_share = 0.75
    s.exid = [1, 2]
    s.globals = [0.0, 0.1, 0.01, 0.1, 0.1, 1.0, True]
    s.dtype = np.dtype(dtype)
    s.output = str(tmp_path / "output.hdf5")
    data = np.random.default_rng(0).standard_normal((3, 1, 32, 32))
    s._write(data, 2.5)
    ds = fake_h5py[s.output]
    assert list(ds) == ["blocksize", "share", "exid", "globals", "clocktime", "data"]
    assert ds["blocksize"].shape == (1,) and ds["blocksize"][0] == 16
    assert ds["share"].shape == (1,) and ds["share"][0] == 0.75
    assert ds["exid"].shape == (2,) and list(ds["exid"]) == [1, 2]
    assert ds["globals"].shape == (7,) and ds["globals"][-1] == 1.0
    assert ds["clocktime"].shape == (1,) and ds["clocktime"][0] == 2.5
    assert ds["data"].shape == (3, 1, 32, 32) and ds["data"].dtype == np.dtype(dtype)
    assert np.array_equal(ds["data"], data.astype(dtype))
