"""The drop-in Solver front-end: yaml input, plugin set_globals routed to the
device constants, the reference's step rounding and frame layout."""
import glob
import os

import numpy as np
import pytest
import yaml

import oracle

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
EQDIR = os.path.join(os.path.dirname(HERE), "pysweep_b200", "equations")


@pytest.mark.parametrize("name", ["heat_fe_n48_bs12", "heat_rk2_n32_bs8", "euler_n32_bs16",
                                  "half_n24_bs8", "example_rk2_n24_bs8"])
@pytest.mark.parametrize("swept", [True, False])
def test_solver_yaml_matches_reference_frames(tmp_path, name, swept):
    import pysweep_b200
    d = np.load(os.path.join(HERE, "golden", name + ".npz"))
    eqn = str(d["eqn"])
    g = [float(x) for x in d["globals"]]
    if eqn in ("heat", "example", "checker"):
        g[-1] = bool(g[-1])
    cfg = {"swept": swept, "blocksize": int(d["bs"]), "share": 1,
           "intermediate_steps": int(d["its"]), "operating_points": int(d["ops"]),
           "globals": g, "cpu": os.path.join(EQDIR, eqn + ".py"), "gpu": eqn + ".cu",
           "filename": str(tmp_path / "out.hdf5"), "dtype": "float64"}
    yf = tmp_path / "in.yaml"
    yf.write_text(yaml.dump(cfg))
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        s = pysweep_b200.Solver(d["ic"], str(yf))
        s()
    finally:
        os.chdir(cwd)
    ref = d["swept" if swept else "standard"]
    assert s.data.shape == ref.shape
    if eqn == "euler":
        assert np.abs(s.data - ref).max() / np.abs(ref).max() < 1e-12
    else:
        assert np.array_equal(s.data, ref)
    out = glob.glob(str(tmp_path / "out.*"))
    assert out, "no output file written"
    assert (tmp_path / "log.yaml").exists()


def test_command_line_heat_runs_swept_and_standard(tmp_path, monkeypatch):
    """python -m pysweep_b200 -f heat [--swept] -b 8 -nx 32 -nt 12: the two
    decompositions give the same frames, equal to the oracle's."""
    from pysweep_b200 import commandline
    monkeypatch.chdir(tmp_path)
    runs = {}
    for swept in (True, False):
        argv = ["-f", "heat", "-b", "8", "-nx", "32", "-nt", "12", "--ignore"]
        s = commandline.main(argv + (["--swept"] if swept else []))
        runs[swept] = s.data
    assert np.array_equal(runs[True][-1], runs[False][-1])
    ic = s.initialConditions
    nlev = len(runs[False]) - 1
    _, want, _ = oracle.standard("heat", ic, s.globals, 1, nlev, frames=False)
    assert np.array_equal(runs[False][-1], want)


@pytest.mark.parametrize("name", ["heat_fe_f32_n64_bs16", "heat_fe_f32_n128_bs32"])
@pytest.mark.parametrize("swept", [True, False])
def test_solver_yaml_float32_matches_reference_standard_frames(tmp_path, name, swept):
    """`dtype: float32` in the yaml: float32 fields on the device, frames equal
    to the reference's float32 standard frames bitwise (both decompositions;
    the swept run keeps the reference's swept frame count)."""
    import pysweep_b200
    d = np.load(os.path.join(HERE, "golden", name + ".npz"))
    g = [float(x) for x in d["globals"]]
    g[-1] = bool(g[-1])
    cfg = {"swept": swept, "blocksize": int(d["bs"]), "share": 1, "intermediate_steps": 1,
           "operating_points": 1, "globals": g, "cpu": os.path.join(EQDIR, "heat.py"),
           "gpu": "heat.cu", "filename": str(tmp_path / "out.hdf5"), "dtype": "float32"}
    yf = tmp_path / "in.yaml"
    yf.write_text(yaml.dump(cfg))
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        s = pysweep_b200.Solver(d["ic"], str(yf))
        s()
    finally:
        os.chdir(cwd)
    assert s.data.dtype == np.float32 and s.final.dtype == np.float32
    ref = d["standard"]
    nf = len(d["swept"] if swept else ref)
    assert s.data.shape == (nf,) + ref.shape[1:]
    assert np.array_equal(s.data.astype(np.float64), ref[:nf])
