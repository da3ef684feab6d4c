"""The CPU oracle against golden frames produced by the reference itself.

The fixtures (tests/golden/*.npz) were made by tests/golden/make_golden.py,
which runs the reference's CPU path (share = 0) for both decompositions.  These
tests pin the oracle before anything else is compared with it.
"""
import glob
import os

import numpy as np
import pytest

import oracle

ALL = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
GOLDEN = [p for p in ALL if "_f32_" not in p]  # float64 runs
GOLDEN_F32 = [p for p in ALL if "_f32_" in p]   # float32 runs (dtype: float32)


def _case(path):
    d = np.load(path)
    return (str(d["eqn"]), d["ic"], list(d["globals"]), int(d["its"]), int(d["ops"]),
            int(d["bs"]), d)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_reference_swept_equals_standard(path):
    """The reference's own two decompositions agree bitwise (decomposition invariance)."""
    d = np.load(path)
    k = min(len(d["swept"]), len(d["standard"]))
    assert np.array_equal(d["swept"][:k], d["standard"][:k])


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_swept_matches_reference(path):
    eqn, ic, g, its, ops, bs, d = _case(path)
    frames, _ = oracle.swept(eqn, ic, g, its, ops, bs)
    assert frames.shape == d["swept"].shape
    assert int(d["swept_array_shape0"]) == frames.shape[0]
    assert np.array_equal(frames, d["swept"])


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_standard_matches_reference(path):
    eqn, ic, g, its, ops, bs, d = _case(path)
    ref = d["standard"]
    frames, _, _ = oracle.standard(eqn, ic, g, its, (len(ref) - 1) * its)
    assert np.array_equal(frames[: len(ref)], ref)


def test_step_counts_follow_reference():
    # pysweep/core/solver.py:113-128 for the 384^2 heat case: 500 steps, bs 16 -> 497 steps
    dx = 1 / 384
    dt = 0.2 * dx * dx
    g = [0, 500 * dt, dt, dx, dx, 1, True]
    ts, mpss, mgss = oracle.step_data(g, 16, 1, 1)
    assert (ts, mpss, mgss) == (498, 7, 70)
    # Euler 1024^2, bs 32, ops 2, its 2, 2000 steps -> 1998 steps
    dx = 10 / 1024
    g = [0, 2000 * 0.1 * dx, 0.1 * dx, dx, dx, 1.4]
    assert oracle.step_data(g, 32, 2, 2) == (1999, 7, 570)


def test_known_answers_example_and_checker(golden_dir):
    # tests.py:282 data[i]==i, :314 data[i]==2i, :346-362 checker patterns
    d = np.load(os.path.join(golden_dir, "example_fe_n24_bs8.npz"))
    for i, fr in enumerate(d["swept"]):
        assert np.all(fr == i)
    d = np.load(os.path.join(golden_dir, "example_rk2_n24_bs8.npz"))
    for i, fr in enumerate(d["swept"]):
        assert np.all(fr == 2 * i)
    d = np.load(os.path.join(golden_dir, "checker_one_n24_bs8.npz"))
    n = d["ic"].shape[-1]
    p1 = np.zeros((n, n))
    p1[0::2, 0::2] = 1
    p1[1::2, 1::2] = 1
    p2 = 1 - p1
    for i, fr in enumerate(d["swept"]):
        assert np.array_equal(fr[0], p1 if i % 2 == 0 else p2)


def test_heat_matches_analytic_to_truncation_error():
    # heat.py:95-113: exp(-8 pi^2 alpha t) sin(2 pi x) sin(2 pi y) on x_i = i/n
    n = 64
    x = np.arange(n) / n
    ic = (np.sin(2 * np.pi * x)[:, None] * np.sin(2 * np.pi * x)[None, :])[None]
    dx = 1 / n
    dt = 0.2 * dx * dx
    steps = 200
    g = [0, steps * dt, dt, dx, dx, 1.0, True]
    _, u, _ = oracle.standard("heat", ic, g, 1, steps, frames=False)
    exact = np.exp(-8 * np.pi ** 2 * steps * dt) * ic
    assert np.abs(u - exact).max() < 5e-4


@pytest.mark.parametrize("path", GOLDEN_F32, ids=[os.path.basename(p)[:-4] for p in GOLDEN_F32])
def test_oracle_f32_matches_reference_standard(path):
    """Float32 storage, float64 arithmetic per level: every frame of the
    reference's float32 standard run, bitwise."""
    d = np.load(path)
    g = list(d["globals"])
    frames = d["standard"]
    u = d["ic"].astype(np.float32)
    assert np.array_equal(frames[0], u)
    for k in range(1, len(frames)):
        u = oracle.heat_f32(u, g, 1)
        assert np.array_equal(u.astype(np.float64), frames[k]), k


@pytest.mark.parametrize("path", GOLDEN_F32, ids=[os.path.basename(p)[:-4] for p in GOLDEN_F32])
def test_reference_f32_swept_within_ulps_of_standard(path):
    """The reference's float32 swept frames are not its float32 standard
    frames: from level 2 on some cells differ by a few float32 ulps of the
    field's scale (its swept CPU path rounds intermediate values
    differently), 1.2e-7 relative max-norm at most.  Recorded here; the
    float32 parity bar is the standard run, and the GPU swept and standard
    paths agree with each other bitwise."""
    d = np.load(path)
    sw, st = d["swept"], d["standard"]
    k = min(len(sw), len(st))
    assert np.array_equal(sw[:2], st[:2])
    rel = max(np.abs(sw[i] - st[i]).max() / np.abs(st[i]).max() for i in range(k))
    assert 0 < rel < 3e-7
