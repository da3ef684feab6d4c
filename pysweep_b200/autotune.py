"""Autotuner for the swept decomposition's tiling.

For a given equation and grid shape it times candidate tilings -- blocksize
(8, 16, 32, 64: rows per band, which sets the maximum levels per half-cycle), levels per
half-cycle h, and column segments per band (how many units, i.e. warps or
CTAs, share the GPU) -- on the real shape with a short run, and keeps the
fastest.  Every tiling computes bit-identical results (the swept decomposition
is exact for any tiling), so the choice only affects speed.  Results are cached
per (equation, shape, its, GPU name) in a JSON file (``$PYSWEEP_B200_CACHE``
or ``~/.cache/pysweep_b200/autotune.json``).

    from pysweep_b200.autotune import tune
    best = tune("heat", 8192, 8192)      # {"blocksize": 32, "h": 15, "nseg": 6, ...}
    eng = Engine("heat", 8192, 8192, blocksize=best["blocksize"])
    eng.configure(h=best["h"], nseg=best["nseg"])
"""
import json
import os

import numpy as np

from .engine import Engine, plugin_constants

DEFAULT_BLOCKSIZES = {"heat": (8, 16, 32, 64), "euler": (8, 16, 32, 64), "half": (8, 16, 32),
                      "example": (8, 16, 32), "checker": (8, 16, 32)}


def _cache_path():
    p = os.environ.get("PYSWEEP_B200_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "pysweep_b200", "autotune.json")


def _gpu_name(device):
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:
        return "cuda"


def _load():
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save(d):
    p = _cache_path()
    os.makedirs(os.path.dirname(p), exist_ok=True)
    tmp = p + ".tmp"
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, p)


def _globals(equation, n):
    dx = 1.0 / n
    if equation == "heat":
        return [0.0, 1.0, 0.2 * dx * dx, dx, dx, 1.0, True]
    if equation == "euler":
        dx = 10.0 / n
        return [0.0, 1.0, 0.1 * dx, dx, dx, 1.4]
    if equation == "half":
        return [0.0, 1.0, 0.1, 0.1, 0.1]
    return [0.0, 1.0, 0.1, 0.1, 0.1, True]


def register_streams(equation, ny, its, bs):
    """Whether the library runs this shape on its register-resident heat
    streams (any segment count up to ny/32); the generic streams need ny to
    be a multiple of the segment count."""
    return equation == "heat" and its == 1 and bs in (16, 32) and ny % 32 == 0


def candidates(equation, nx, ny, its=1, ops=None, blocksizes=None):
    """(blocksize, h, nseg) tilings worth timing for this shape."""
    ops = ops or (2 if equation == "euler" else 1)
    out = []
    for bs in blocksizes or DEFAULT_BLOCKSIZES.get(equation, (16, 32)):
        if nx % bs or ny % bs or bs % (2 * ops):
            continue
        mpss = bs // (2 * ops) - 1
        if mpss < max(1, its):
            continue
        hs = sorted({mpss, max(its, (4 * mpss) // 5), max(its, (2 * mpss) // 3)})
        nb = nx // bs
        fast = register_streams(equation, ny, its, bs)
        segs = {0}  # 0 = the library's automatic choice
        for target in (4, 8, 12):
            n = max(1, (148 * target) // nb)
            if not fast:  # nearest divisor of ny at or below n
                while ny % n:
                    n -= 1
            if n <= ny // 32:
                segs.add(n)
        for h in hs:
            for s in sorted(segs):
                out.append((bs, h, s))
    return out


def _time_config(equation, nx, ny, nv, its, ops, bs, h, nseg, levels, reps, device, field):
    import torch
    with Engine(equation, nx, ny, nv=nv, ops=ops, its=its, blocksize=bs, device=device) as e:
        for k, v in plugin_constants(equation, _globals(equation, nx)).items():
            e.set_global(k, v)
        e.configure(h=h, nseg=nseg)
        e.set_state(field)
        e.run(levels)  # warm-up
        e.synchronize()
        best = float("inf")
        for _ in range(reps):
            e.set_state(field)
            e.profile(True)
            e.run(levels)
            prof = e.profile_read()
            ms = sum(v[0] for v in prof.values())
            best = min(best, ms)
    return nx * ny * levels / (best / 1000.0) / 1e9


def tune(equation, nx, ny, nv=None, its=1, ops=None, levels=None, reps=2, device=0,
         blocksizes=None, use_cache=True, verbose=False):
    """Time the candidate tilings and return the fastest (cached)."""
    import torch
    nv = nv or (4 if equation == "euler" else 1)
    ops = ops or (2 if equation == "euler" else 1)
    key = f"{equation}|{nx}x{ny}|nv{nv}|its{its}|ops{ops}|{_gpu_name(device)}"
    cache = _load() if use_cache else {}
    if key in cache:
        return cache[key]
    rng = np.random.default_rng(0)
    if equation == "euler":
        from .equations.euler import analytical_array
        field = analytical_array(nx, ny, 0.0)
    else:
        field = rng.standard_normal((nv, nx, ny))
    dfield = torch.from_numpy(field).cuda(device)
    levels = levels or 60 * its
    results = []
    for bs, h, nseg in candidates(equation, nx, ny, its, ops, blocksizes):
        try:
            g = _time_config(equation, nx, ny, nv, its, ops, bs, h, nseg, levels, reps, device,
                             dfield)
        except Exception as exc:  # a tiling this build rejects
            if verbose:
                print(f"  bs {bs} h {h} nseg {nseg}: {exc}")
            continue
        results.append({"blocksize": bs, "h": h, "nseg": nseg, "gcell_updates_s": g})
        if verbose:
            print(f"  bs {bs:3d} h {h:3d} nseg {nseg:4d}: {g:8.1f} Gcell-updates/s")
    if not results:
        raise RuntimeError(f"no tiling of {equation} {nx}x{ny} ran")
    best = max(results, key=lambda r: r["gcell_updates_s"])
    best = dict(best, candidates=len(results))
    if use_cache:
        cache = _load()
        cache[key] = best
        _save(cache)
    return best
