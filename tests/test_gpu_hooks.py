"""User step hooks compiled at run time (NVRTC, sm_100a) on the GPU.

The reference builds its kernels from the plugin's .cu file
(pysweep/core/io.py:146-155) and runs the plugin's __device__ step() inside
every phase (pysweep/core/pysweep.cu:25).  Here:

* hooks written in that plugin format with the numpy plugins' operation order
  (tests/hooks/*_numpy_order.cu) reproduce the reference's own golden frames
  bitwise, through the swept and the standard decomposition;
* a hook that is none of the reference's plugins (tests/hooks/wave4.cu: two
  variables, a five-point stencil, two stages) gives bitwise equal swept and
  standard results, and matches a numpy restatement of its arithmetic;
* the drop-in Solver runs a hook file named by `gpu:`;
* when the environment variable PYSWEEP_REFERENCE_HOOKS names a directory that
  holds the reference's own plugin .cu files, those compile unmodified and
  reproduce the golden frames (bitwise for example, checker and half, whose
  arithmetic is the numpy plugins'; heat.cu groups its products differently,
  so it is held to 1e-12).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
HOOKS = os.path.join(HERE, "hooks")
GOLDEN = os.path.join(HERE, "golden")

OWN = {  # golden fixture -> hook written in the numpy plugin's order
    "heat_fe_n32_bs8": "heat_numpy_order.cu",
    "heat_fe_n48_bs16": "heat_numpy_order.cu",
    "heat_rk2_n48_bs12": "heat_numpy_order.cu",
    "heat_rk2_n32_bs8": "heat_numpy_order.cu",
    "half_n24_bs8": "half_numpy_order.cu",
    "example_fe_n24_bs8": "example_numpy_order.cu",
    "example_rk2_n24_bs8": "example_numpy_order.cu",
    "checker_one_n24_bs8": "checker_numpy_order.cu",
    "checker_two_n24_bs8": "checker_numpy_order.cu",
}


def _hook_frames(path, fixture, mode, **tiling):
    from pysweep_b200 import Engine, plugin_constants
    d = np.load(os.path.join(GOLDEN, fixture + ".npz"))
    eqn, ic, g = str(d["eqn"]), d["ic"], list(d["globals"])
    ops, its, bs = int(d["ops"]), int(d["its"]), int(d["bs"])
    nlevels = (len(d[mode]) - 1) * its
    e = Engine(path, ic.shape[1], ic.shape[2], nv=ic.shape[0], ops=ops, its=its, blocksize=bs)
    assert e.hook
    for k, v in plugin_constants(eqn, g).items():  # every hook here declares these
        e.set_global(k, v)
    if tiling:
        e.configure(**tiling)
    e.set_state(ic)
    frames = np.zeros((nlevels // its,) + ic.shape)
    e.run(nlevels, mode=mode, frames=frames)
    e.close()
    return np.concatenate([ic[None], frames]), d[mode]


@pytest.mark.parametrize("fixture", sorted(OWN))
@pytest.mark.parametrize("mode", ["swept", "standard"])
def test_hooks_in_numpy_order_reproduce_golden_frames(fixture, mode):
    got, ref = _hook_frames(os.path.join(HOOKS, OWN[fixture]), fixture, mode)
    assert got.shape == ref.shape
    assert np.array_equal(got, ref), f"max difference {np.abs(got - ref).max()}"


def test_hook_tiling_changes_no_bit():
    path = os.path.join(HOOKS, "heat_numpy_order.cu")
    ref, _ = _hook_frames(path, "heat_fe_n48_bs16", "swept")
    for cfg in ({"h": 3}, {"nseg": 3}, {"chunk": 64}):
        got, _ = _hook_frames(path, "heat_fe_n48_bs16", "swept", **cfg)
        assert np.array_equal(got, ref), cfg


def test_hook_default_tiling_keeps_three_ctas_per_sm():
    """A one-variable hook at blocksize 32 defaults to 6 levels per
    half-cycle (the most whose stream tile, one linear slot per level, leaves
    room for three CTAs per SM), not MPSS = 15; both give the same bits."""
    import torch
    from pysweep_b200 import Engine, plugin_constants
    path = os.path.join(HOOKS, "heat_numpy_order.cu")
    n, nl = 256, 40
    ic = np.random.default_rng(5).standard_normal((1, n, n))
    dx = 1.0 / n
    g = [0.0, nl * 0.2 * dx * dx, 0.2 * dx * dx, dx, dx, 1.0, True]
    out = {}
    for h in (0, 15):
        e = Engine(path, n, n, blocksize=32)
        for k, v in plugin_constants("heat", g).items():
            e.set_global(k, v)
        if h:
            e.configure(h=h)
        else:
            assert e.tiling()["h"] == 6 and e.tiling()["mpss"] == 15
        e.set_state(ic)
        e.run(nl, mode="swept")
        out[h] = e.get_state()
        e.close()
    torch.cuda.synchronize()
    assert np.array_equal(out[0], out[15])


def _wave_numpy(u0, v0, a, dt, nlevels):
    """tests/hooks/wave4.cu restated on whole arrays, in the hook's order."""
    def d1(f, ax):
        return (-np.roll(f, -2, ax) + 8 * np.roll(f, -1, ax) - 8 * np.roll(f, 1, ax)
                + np.roll(f, 2, ax)) / 12
    prev = cur = (u0, v0)
    for gts in range(1, nlevels + 1):
        full = gts % 2 == 0
        coeff = 1.0 if full else 0.5
        base = prev if full else cur
        u, v = cur
        ru = -a * (d1(v, 0) + d1(v, 1))
        rv = -a * (d1(u, 0) + d1(u, 1))
        nxt = (base[0] + coeff * dt * ru, base[1] + coeff * dt * rv)
        prev, cur = cur, nxt
    return np.stack(cur)


@pytest.mark.parametrize("n,bs,cfg", [(96, 16, {}), (128, 32, {}), (128, 32, {"h": 5, "nseg": 2})])
def test_new_hook_swept_equals_standard_and_numpy(n, bs, cfg):
    from pysweep_b200 import Engine
    rng = np.random.default_rng(n + bs)
    ic = rng.standard_normal((2, n, n))
    a, dt, nl = 0.7, 0.05, 2 * 17
    out = {}
    for mode in ("swept", "standard"):
        e = Engine(os.path.join(HOOKS, "wave4.cu"), n, n, nv=2, ops=2, its=2, blocksize=bs)
        e.set_global("A", a)
        e.set_global("DT", dt)
        if mode == "swept" and cfg:
            e.configure(**cfg)
        e.set_state(ic)
        e.run(nl, mode=mode)
        out[mode] = e.get_state()
        e.close()
    assert np.array_equal(out["swept"], out["standard"])
    ref = _wave_numpy(ic[0], ic[1], a, dt, nl)
    assert np.abs(out["swept"] - ref).max() / np.abs(ref).max() < 1e-12


def test_solver_runs_a_hook_file(tmp_path):
    """The drop-in Solver with `gpu:` naming a hook file: the reference's heat
    globals through the repository's heat plugin (its set_globals sets the
    hook's constants by name), equal to the built-in heat kernels."""
    import yaml

    from pysweep_b200 import Solver
    n = 64
    x = np.arange(n) / n
    ic = (np.sin(2 * np.pi * x)[:, None] * np.sin(2 * np.pi * x)[None, :])[None]
    dx = 1.0 / n
    out = {}
    for gpu in (os.path.join(HOOKS, "heat_numpy_order.cu"), "heat.cu"):
        y = tmp_path / "in.yaml"
        y.write_text(yaml.dump({
            "swept": True, "blocksize": 16, "intermediate_steps": 1, "operating_points": 1,
            "globals": [0.0, 70 * 0.2 * dx * dx, 0.2 * dx * dx, dx, dx, 1.0, True],
            "cpu": os.path.join(os.path.dirname(HERE), "pysweep_b200", "equations", "heat.py"),
            "gpu": gpu, "filename": str(tmp_path / "out.hdf5"), "write_output": False}))
        cwd = os.getcwd()
        os.chdir(tmp_path)
        try:
            s = Solver(ic, str(y))
            s()
        finally:
            os.chdir(cwd)
        out[gpu] = s.final
    a, b = out.values()
    assert np.array_equal(a, b)


def test_hook_errors():
    from pysweep_b200 import Engine, PySweepError
    e = Engine(os.path.join(HOOKS, "heat_numpy_order.cu"), 32, 32, blocksize=8)
    with pytest.raises(PySweepError):
        e.set_global("NO_SUCH_CONSTANT", 1.0)
    with pytest.raises(PySweepError):
        e.set_global("TIMES", 3)  # framework constants belong to the engine
    e.close()
    with pytest.raises(PySweepError) as err:
        Engine("broken.cu", 32, 32, blocksize=8,
               hook_source="__device__ void step(double* s, int i, int g) { s[i] = nope; }")
    assert err.value.code == -6 and "broken.cu" in str(err.value)


REF = os.environ.get("PYSWEEP_REFERENCE_HOOKS", "")
REF_CASES = {  # reference plugin file -> fixtures, bitwise or relative bound
    "example.cu": (["example_fe_n24_bs8", "example_rk2_n24_bs8"], 0.0),
    "checker.cu": (["checker_one_n24_bs8", "checker_two_n24_bs8"], 0.0),
    "half.cu": (["half_n24_bs8"], 0.0),
    "heat.cu": (["heat_fe_n48_bs16", "heat_rk2_n48_bs12"], 1e-12),
}


@pytest.mark.skipif(not os.path.isdir(REF), reason="PYSWEEP_REFERENCE_HOOKS not set")
@pytest.mark.parametrize("name", sorted(REF_CASES))
@pytest.mark.parametrize("mode", ["swept", "standard"])
def test_reference_plugin_hooks_unmodified(name, mode):
    fixtures, tol = REF_CASES[name]
    for fx in fixtures:
        got, ref = _hook_frames(os.path.join(REF, name), fx, mode)
        err = np.abs(got - ref).max() / max(np.abs(ref).max(), 1e-300)
        assert (np.array_equal(got, ref) if tol == 0 else err < tol), f"{name} {fx}: {err}"
