"""Autotuner candidate sets and cache (no GPU needed)."""
import json

import pytest

from pysweep_b200 import autotune


@pytest.mark.parametrize("eq,n", [("heat", 4096), ("heat", 384), ("euler", 1024), ("half", 256)])
def test_candidates_are_valid_tilings(eq, n):
    c = autotune.candidates(eq, n, n)
    assert c
    ops = 2 if eq == "euler" else 1
    for bs, h, nseg in c:
        assert n % bs == 0 and bs % (2 * ops) == 0
        assert 1 <= h <= bs // (2 * ops) - 1
        assert nseg == 0 or 1 <= nseg <= n // 32
        if not autotune.register_streams(eq, n, 1, bs):
            assert nseg == 0 or n % nseg == 0
    assert len(set(c)) == len(c)


def test_cached_result_is_returned_without_timing(tmp_path, monkeypatch):
    cache = tmp_path / "tune.json"
    monkeypatch.setenv("PYSWEEP_B200_CACHE", str(cache))
    monkeypatch.setattr(autotune, "_gpu_name", lambda device: "test-gpu")
    best = {"blocksize": 32, "h": 15, "nseg": 6, "gcell_updates_s": 1.0, "candidates": 3}
    cache.write_text(json.dumps({"heat|512x512|nv1|its1|ops1|test-gpu": best}))

    def no_timing(*a, **k):
        raise AssertionError("timed a tiling although the cache had the shape")
    monkeypatch.setattr(autotune, "_time_config", no_timing)
    assert autotune.tune("heat", 512, 512) == best


def test_levels_candidates_include_four_fifths_of_mpss():
    """Heat at bs 32 (MPSS 15) is timed at 15, 12 and 10 levels per
    half-cycle; 12 is the library's own default for that shape."""
    hs = {h for bs, h, _ in autotune.candidates("heat", 512, 512) if bs == 32}
    assert hs == {15, 12, 10}
    hs16 = {h for bs, h, _ in autotune.candidates("heat", 512, 512) if bs == 16}
    assert hs16 == {7, 5, 4}
