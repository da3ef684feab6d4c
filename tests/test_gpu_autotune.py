"""The autotuner picks a tiling that runs and gives the default tiling's field."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_tuned_tiling_runs_and_matches_default(tmp_path, monkeypatch):
    from pysweep_b200 import Engine, plugin_constants
    from pysweep_b200.autotune import tune
    monkeypatch.setenv("PYSWEEP_B200_CACHE", str(tmp_path / "tune.json"))
    n = 256
    best = tune("heat", n, n, levels=30, reps=1)
    assert best["candidates"] >= 2 and best["gcell_updates_s"] > 0
    assert tune("heat", n, n) == best  # second call: from the cache
    rng = np.random.default_rng(0)
    ic = rng.standard_normal((1, n, n))
    g = [0.0, 1.0, 0.2 / n / n, 1 / n, 1 / n, 1.0, True]
    out = []
    for bs, h, nseg in ((16, 0, 0), (best["blocksize"], best["h"], best["nseg"])):
        with Engine("heat", n, n, blocksize=bs) as e:
            for k, v in plugin_constants("heat", g).items():
                e.set_global(k, v)
            e.configure(h=h, nseg=nseg)
            e.set_state(ic)
            e.run(57)
            out.append(e.get_state())
    assert np.array_equal(out[0], out[1])
