"""GPU parity: the CUDA swept and standard paths against the reference's own
frames (golden fixtures) and the CPU oracle.

Bar: heat, half, example and checker are bitwise equal to the reference's
numpy path.  Euler computes x**2 as x*x where numpy calls libm pow(), so the
Euler frames are bitwise equal to the oracle run with x*x and within a
relative max-norm of 1e-12 of the reference's own frames.  Swept and standard
GPU results are always bit-identical.
"""
import glob
import os

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if "_f32_" not in p)  # float32 runs: test_gpu_f32.py
EULER_RTOL = 1e-12


def _engine(eqn, shape, ops, its, bs, g):
    from pysweep_b200 import Engine, plugin_constants
    e = Engine(eqn, shape[1], shape[2], nv=shape[0], ops=ops, its=its, blocksize=bs)
    for k, v in plugin_constants(eqn, g).items():
        e.set_global(k, v)
    return e


def _gpu_frames(eqn, ic, g, ops, its, bs, nlevels, mode, **cfg):
    e = _engine(eqn, ic.shape, ops, its, bs, g)
    if cfg:
        e.configure(**cfg)
    e.set_state(ic)
    nfr = nlevels // its
    frames = np.zeros((nfr,) + ic.shape)
    e.run(nlevels, mode=mode, frames=frames)
    final = e.get_state()
    e.close()
    return np.concatenate([ic[None], frames]), final


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
@pytest.mark.parametrize("mode", ["swept", "standard"])
def test_golden_frames(path, mode):
    d = np.load(path)
    eqn, ic, g = str(d["eqn"]), d["ic"], list(d["globals"])
    ops, its, bs = int(d["ops"]), int(d["its"]), int(d["bs"])
    ref = d[mode]
    nlevels = (len(ref) - 1) * its
    got, _ = _gpu_frames(eqn, ic, g, ops, its, bs, nlevels, mode)
    assert got.shape == ref.shape
    if eqn == "euler":
        assert _rel(got, ref) < EULER_RTOL
        mul, _, _ = oracle.standard(eqn, ic, g, its, nlevels, euler_square="mul")
        assert np.array_equal(got, mul[: len(got)])
    else:
        assert np.array_equal(got, ref)


CONFIGS = [
    # eqn, n, bs, ops, its, steps, scheme, tiling
    ("heat", 64, 8, 1, 1, 40, True, {}),
    ("heat", 96, 16, 1, 1, 50, True, {"nseg": 3}),
    ("heat", 128, 32, 1, 1, 61, True, {}),
    ("heat", 128, 32, 1, 1, 61, True, {"h": 9, "nseg": 2}),
    ("heat", 128, 64, 1, 1, 70, True, {}),
    ("heat", 128, 16, 1, 2, 33, False, {"h": 4}),
    ("heat", 96, 24, 1, 2, 25, False, {"nseg": 2}),
    ("heat", 80, 8, 1, 1, 17, True, {"chunk": 64}),
    ("euler", 64, 16, 2, 2, 12, None, {}),
    ("euler", 64, 16, 2, 2, 11, None, {"nseg": 1}),
    ("euler", 64, 32, 2, 2, 10, None, {"nseg": 2}),
    ("euler", 96, 16, 2, 2, 9, None, {"h": 2, "nseg": 3}),
    ("euler", 128, 16, 2, 2, 9, None, {"chunk": 64}),
    ("half", 64, 16, 1, 2, 20, None, {}),
    ("checker", 48, 8, 2, 2, 12, False, {}),
    ("example", 48, 12, 1, 1, 21, True, {"nseg": 2}),
]


def _ic_and_globals(eqn, n, steps, scheme):
    rng = np.random.default_rng(n * 7 + steps)
    if eqn == "heat":
        dx = 1.0 / n
        dt = 0.2 * dx * dx
        return rng.standard_normal((1, n, n)), [0, steps * dt, dt, dx, dx, 1.0, scheme]
    if eqn == "euler":
        x = np.linspace(-5, 5, n, endpoint=False)
        X, Y = np.meshgrid(x, x, indexing="ij")
        r2 = X ** 2 + Y ** 2
        rho = 1 - 0.3 * np.exp(-r2)
        u = 1 + 0.2 * np.sin(2 * np.pi * Y / 10)
        v = 1 - 0.2 * np.cos(2 * np.pi * X / 10)
        p = 1 / 1.4 * (1 - 0.2 * np.exp(-r2))
        E = p / 0.4 + 0.5 * rho * (u * u + v * v)
        dx = 10.0 / n
        return np.stack([rho, rho * u, rho * v, E]), [0, steps * 0.1 * dx, 0.1 * dx, dx, dx, 1.4]
    if eqn == "half":
        return rng.standard_normal((1, n, n)), [0, 1, 0.1, 0.1, 0.1]
    return rng.integers(0, 2, (1, n, n)).astype(float), [0, 1, 0.1, 0.1, 0.1, scheme]


@pytest.mark.parametrize("cfg", CONFIGS, ids=[f"{c[0]}-n{c[1]}-bs{c[2]}-its{c[4]}-{c[7]}" for c in CONFIGS])
def test_swept_standard_oracle(cfg):
    eqn, n, bs, ops, its, steps, scheme, tiling = cfg
    ic, g = _ic_and_globals(eqn, n, steps, scheme)
    nlevels = steps * its
    sw, swf = _gpu_frames(eqn, ic, g, ops, its, bs, nlevels, "swept", **tiling)
    st, stf = _gpu_frames(eqn, ic, g, ops, its, bs, nlevels, "standard")
    assert np.array_equal(sw, st), "swept and standard differ"
    assert np.array_equal(swf, stf)
    ref, _, _ = oracle.standard(eqn, ic, g, its, nlevels,
                                euler_square="mul" if eqn == "euler" else "pow")
    assert np.array_equal(sw, ref[: len(sw)])


def test_heat_384_reference_step_count_and_analytic():
    """The 384^2 heat case: the reference's step rounding (497 steps for bs 16),
    bitwise against the oracle's reference swept decomposition, and the analytic
    decaying sine to truncation error."""
    n, bs = 384, 16
    dx = 1.0 / n
    dt = 0.2 * dx * dx
    g = [0, 500 * dt, dt, dx, dx, 1.0, True]
    ts, mpss, mgss = oracle.step_data(g, bs, 1, 1)
    nlevels = mpss * (mgss + 1)
    assert nlevels == 497
    x = np.arange(n) / n
    ic = (np.sin(2 * np.pi * x)[:, None] * np.sin(2 * np.pi * x)[None, :])[None]
    frames, final = _gpu_frames("heat", ic, g, 1, 1, bs, nlevels, "swept")
    ref, _ = oracle.swept("heat", ic, g, 1, 1, bs, nthreads=oracle.max_threads())
    assert np.array_equal(frames, ref)
    exact = np.exp(-8 * np.pi ** 2 * nlevels * dt) * ic
    assert np.abs(final - exact).max() < 1e-4


def test_euler_mass_conserved_and_decompositions_agree_at_256():
    n, steps = 256, 40
    ic, g = _ic_and_globals("euler", n, steps, None)
    sw, swf = _gpu_frames("euler", ic, g, 2, 2, 32, steps * 2, "swept", nseg=2)
    st, stf = _gpu_frames("euler", ic, g, 2, 2, 32, steps * 2, "standard")
    assert np.array_equal(swf, stf)
    m0, m1 = ic[0].sum(), swf[0].sum()
    assert abs(m1 - m0) / m0 < 1e-12


@pytest.mark.parametrize("bs,cfg", [(16, {}), (16, {"chunk": 32}), (16, {"chunk": 32, "nseg": 4}),
                                    (32, {}), (12, {"chunk": 32}), (8, {})])
def test_euler_shared_faces_match_per_cell_step(bs, cfg):
    """Euler's face-sharing kernels (standard tiles; stream levels where tile
    and scratch fit two CTAs per SM: 32-column chunks at bs 16 and 12, bs 8)
    against the per-cell step (threads = 256 selects the per-cell standard
    kernel; 64-column chunks and bs 32 use it in the streams), the swept
    decomposition and the oracle's x*x arithmetic, bitwise."""
    n = 96 if bs == 12 else (64 if bs == 8 else 128)
    steps = 7
    ic, g = _ic_and_globals("euler", n, steps, None)
    sw, swf = _gpu_frames("euler", ic, g, 2, 2, bs, steps * 2, "swept", **cfg)
    st, stf = _gpu_frames("euler", ic, g, 2, 2, bs, steps * 2, "standard")
    pc, pcf = _gpu_frames("euler", ic, g, 2, 2, bs, steps * 2, "standard", threads=256)
    assert np.array_equal(st, pc) and np.array_equal(sw, st)
    mul, _, _ = oracle.standard("euler", ic, g, 2, steps * 2, euler_square="mul")
    assert np.array_equal(st, mul[: len(st)])


FAST = [
    # n, bs, steps, tiling
    (128, 32, 45, {}),
    (128, 32, 40, {"nseg": 2}),
    (192, 16, 33, {}),
    (256, 16, 29, {"nseg": 4, "h": 5}),
    (128, 32, 20, {"h": 4}),
    (64, 32, 31, {}),
    (256, 32, 33, {"nseg": 3}),   # uneven segments: 1, 1 and 2 chunks
    (320, 16, 17, {"nseg": 4}),   # 5 chunks over 4 segments
    (384, 32, 40, {"nseg": 0}),   # automatic segment count
    (256, 32, 37, {"nseg": 1}),   # one segment: each seam joins a block to itself
    (384, 16, 20, {"nseg": 0}),   # automatic segment count at four CTAs per SM
    (1024, 16, 15, {}),           # 16 segments of one chunk per band
]


@pytest.mark.parametrize("cfg", FAST, ids=[f"n{c[0]}-bs{c[1]}-{c[3]}" for c in FAST])
def test_register_heat_streams_match_generic_and_oracle(cfg):
    """Heat with forward Euler takes the register-resident stream kernels;
    `threads=256` forces the shared-memory streams.  Both, and the standard
    path, are bitwise the oracle's, frames included."""
    n, bs, steps, tiling = cfg
    ic, g = _ic_and_globals("heat", n, steps, True)
    fast, fast_f = _gpu_frames("heat", ic, g, 1, 1, bs, steps, "swept", **tiling)
    # the shared-memory streams need equal segments; any tiling gives the same bits
    gtiling = {k: v for k, v in tiling.items() if k != "nseg" or (v and n % v == 0)}
    gen, gen_f = _gpu_frames("heat", ic, g, 1, 1, bs, steps, "swept", threads=256, **gtiling)
    ref, _, _ = oracle.standard("heat", ic, g, 1, steps)
    assert np.array_equal(fast, ref[: len(fast)])
    assert np.array_equal(gen, fast)
    assert np.array_equal(fast_f, gen_f)


@pytest.mark.parametrize("scheme,its", [(True, 1), (False, 2)])
@pytest.mark.parametrize("n", [64, 192, 320])
def test_streaming_standard_heat_matches_generic_and_oracle(scheme, its, n):
    """The streaming standard kernel (64-column strips) equals the per-cell
    generic kernel and the oracle bitwise, frames included."""
    steps = 23
    ic, g = _ic_and_globals("heat", n, steps, scheme)
    nl = steps * its
    fast, ff = _gpu_frames("heat", ic, g, 1, its, 16, nl, "standard")
    gen, gf = _gpu_frames("heat", ic, g, 1, its, 16, nl, "standard", threads=256)
    ref, _, _ = oracle.standard("heat", ic, g, its, nl)
    assert np.array_equal(fast, gen)
    assert np.array_equal(ff, gf)
    assert np.array_equal(fast, ref[: len(fast)])


def test_default_levels_per_half_cycle_and_tiling_query():
    """Heat with forward Euler at bs 32 runs 12 levels per half-cycle unless
    configured (every other shape MPSS); the tiling changes no bit."""
    from pysweep_b200 import Engine, plugin_constants
    n, steps = 256, 53
    ic, g = _ic_and_globals("heat", n, steps, True)
    out = {}
    for h in (0, 15, 9):
        e = Engine("heat", n, n, blocksize=32)
        for k, v in plugin_constants("heat", g).items():
            e.set_global(k, v)
        if h:
            e.configure(h=h)
        e.set_state(ic)
        e.run(steps)
        t = e.tiling()
        assert t["mpss"] == 15 and t["h"] == (h or 12) and t["nseg"] >= 1
        out[h] = e.get_state()
        e.close()
    ref, _, _ = oracle.standard("heat", ic, g, 1, steps)
    for h in out:
        assert np.array_equal(out[h], ref[-1])
    assert Engine("heat", 64, 64, blocksize=16).tiling()["h"] == 7
    assert Engine("euler", 64, 64, its=2, blocksize=32).tiling()["h"] == 7


def test_generic_streams_choose_segments_of_four_chunks():
    """The shared-memory streams cut each band into the most segments that
    divide the row and keep four chunks each (1024 columns in 32-column
    chunks, the widest whose bs-32 Euler tile fits: 8 segments), chosen at
    the first swept run."""
    from pysweep_b200 import Engine, plugin_constants
    from pysweep_b200.equations.euler import analytical_array
    n = 1024
    dx = 10.0 / n
    e = Engine("euler", n, n, its=2, blocksize=32)
    for k, v in plugin_constants("euler", [0.0, 1.0, 0.1 * dx, dx, dx, 1.4]).items():
        e.set_global(k, v)
    e.set_state(analytical_array(n, n, 0.0))
    e.run(2)
    t = e.tiling()
    assert t["chunk"] == 32 and t["nseg"] == n // (4 * t["chunk"])
    e.close()
