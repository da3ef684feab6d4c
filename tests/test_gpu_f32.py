"""float32 heat on the GPU (the reference's `dtype: float32`).

Bar: the GPU's float32 frames equal the reference's float32 standard frames
bitwise (every level evaluated in float64 and rounded to float32), the GPU's
swept and standard float32 paths agree bitwise, and both equal the oracle's
float32 stepper on larger grids and other tilings.
"""
import glob
import os

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

GOLDEN_F32 = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*_f32_*.npz")))


def _engine(n, bs, g, nx=None):
    from pysweep_b200 import Engine, plugin_constants
    e = Engine("heat", nx or n, n, blocksize=bs, dtype="float32")
    for k, v in plugin_constants("heat", g).items():
        e.set_global(k, v)
    return e


@pytest.mark.parametrize("path", GOLDEN_F32, ids=[os.path.basename(p)[:-4] for p in GOLDEN_F32])
@pytest.mark.parametrize("mode", ["swept", "standard"])
def test_golden_f32_frames(path, mode):
    d = np.load(path)
    g, bs, n = list(d["globals"]), int(d["bs"]), int(d["n"])
    ref = d["standard"]  # the reference's swept float32 frames are not its own standard ones
    ic = d["ic"].astype(np.float32)
    nl = len(ref) - 1
    e = _engine(n, bs, g)
    e.set_state(ic)
    frames = np.zeros((nl,) + ic.shape, dtype=np.float32)
    e.run(nl, mode=mode, frames=frames)
    got = np.concatenate([ic[None], frames]).astype(np.float64)
    assert np.array_equal(got, ref)
    assert np.array_equal(e.get_state(), frames[-1])
    e.close()


@pytest.mark.parametrize("n,bs,levels,cfg", [(256, 32, 100, {}), (256, 16, 45, {"nseg": 3}),
                                             (192, 32, 61, {"h": 9, "nseg": 2}),
                                             (320, 32, 31, {})])
def test_f32_swept_standard_and_oracle_agree(n, bs, levels, cfg):
    rng = np.random.default_rng(n + bs)
    ic = rng.standard_normal((1, n, n)).astype(np.float32)
    dx = 1.0 / n
    g = [0.0, 1.0, 0.2 * dx * dx, dx, dx, 1.0, True]
    out = {}
    for mode in ("swept", "standard"):
        e = _engine(n, bs, g)
        if cfg:
            e.configure(**cfg)
        e.set_state(ic)
        e.run(levels, mode=mode)
        out[mode] = e.get_state()
        e.close()
    assert out["swept"].dtype == np.float32
    assert np.array_equal(out["swept"], out["standard"])
    assert np.array_equal(out["swept"], oracle.heat_f32(ic, g, levels))


def test_f32_from_device_tensor_and_unsupported_configs():
    import torch
    from pysweep_b200 import Engine
    from pysweep_b200._lib import PySweepError
    n = 128
    dx = 1.0 / n
    g = [0.0, 1.0, 0.2 * dx * dx, dx, dx, 1.0, True]
    ic = np.random.default_rng(1).standard_normal((1, n, n)).astype(np.float32)
    e = _engine(n, 32, g)
    e.set_state(torch.from_numpy(ic).cuda())
    e.run(20)
    out = torch.empty((1, n, n), dtype=torch.float32, device="cuda")
    e.get_state(out=out)  # device copies are queued on the engine's stream
    e.synchronize()
    assert np.array_equal(out.cpu().numpy(), oracle.heat_f32(ic, g, 20))
    e.close()
    with pytest.raises(PySweepError):  # float32 is heat with forward Euler only
        Engine("euler", 64, 64, its=2, blocksize=16, dtype="float32")
