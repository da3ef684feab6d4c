"""ps_heat_swept_noalloc, the entry point for callers that cannot allocate.

Callers under a foreign memory pool that owns the device, or in loops that
must not touch the allocator, cannot cudaMalloc when they solve; this entry
point keeps its scratch in a static device array instead.  It must give exactly what the allocating path
(ps_run on a ps_solver) gives, on consecutive calls that share the array.
This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib, d_in, d_out, n, bs, steps, g, ny=None, stream=None):
    err = ctypes.create_string_buffer(256)
    rc = lib.ps_heat_swept_noalloc(ctypes.c_void_p(d_in.data_ptr()), ctypes.c_void_p(d_out.data_ptr()),
                                   n, ny or n, bs, steps, g[5], g[2], g[3], stream, err, 256)
    return rc, err.value.decode()


def _allocating(ic, bs, steps, g):
    from pysweep_b200 import Engine, plugin_constants
    with Engine("heat", ic.shape[1], ic.shape[2], its=1, blocksize=bs) as e:
        for k, v in plugin_constants("heat", g).items():
            e.set_global(k, v)
        e.set_state(ic)
        e.run(steps, mode="swept")
        return e.get_state()


@pytest.mark.parametrize("bs", [16, 32])
def test_noalloc_matches_allocating_path_on_consecutive_calls(bs):
    import torch
    from pysweep_b200 import _lib
    lib = _lib.lib()
    n = 512
    dx = 1.0 / n
    dt = 0.2 * dx * dx
    rng = np.random.default_rng(bs)
    results = []
    for call, steps in enumerate((47, 33)):  # two calls in a row share the scratch array
        g = [0.0, steps * dt, dt, dx, dx, 1.0, True]
        ic = rng.standard_normal((1, n, n))
        d_in = torch.from_numpy(ic).cuda()
        d_out = torch.full_like(d_in, float("nan"))
        rc, msg = _noalloc(lib, d_in, d_out, n, bs, steps, g)
        assert rc == 0, msg
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()
        ref = _allocating(ic, bs, steps, g)
        assert np.array_equal(got, ref), f"call {call}: differs by {np.abs(got - ref).max()}"
        assert np.array_equal(d_in.cpu().numpy(), ic), "input modified"
        results.append(got)
    assert not np.array_equal(results[0], results[1])


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    from pysweep_b200 import _lib
    lib = _lib.lib()
    n = 4096  # ~370 MB of scratch at blocksize 32
    d_in = torch.zeros((1, 64, 64), dtype=torch.float64, device="cuda")  # never read
    d_out = torch.zeros_like(d_in)
    err = ctypes.create_string_buffer(256)
    rc = lib.ps_heat_swept_noalloc(ctypes.c_void_p(d_in.data_ptr()), ctypes.c_void_p(d_out.data_ptr()),
                                   n, n, 32, 10, 1.0, 1e-8, 1.0 / n, None, err, 256)
    assert rc == -1
    assert b"scratch" in err.value


@pytest.mark.parametrize("nx,ny,bs,steps", [
    (2048, 2048, 32, 40),   # 27 segments over 64 column units: uneven segments
    (512, 256, 32, 29),     # rectangular: rows and columns tiled differently
    (256, 512, 16, 0),      # no steps: the output is a copy of the input
])
def test_noalloc_uneven_rectangular_and_empty_runs_on_a_side_stream(nx, ny, bs, steps):
    """The same bitwise bar on the sizes the first test does not reach: the
    segment rule's uneven segments, nx != ny, zero steps, and a call queued on
    a stream other than the default one."""
    import torch
    from pysweep_b200 import _lib
    lib = _lib.lib()
    dx = 1.0 / nx
    dt = 0.2 * dx * dx
    g = [0.0, steps * dt, dt, dx, dx, 1.0, True]
    ic = np.random.default_rng(nx + ny + bs).standard_normal((1, nx, ny))
    d_in = torch.from_numpy(ic).cuda()
    d_out = torch.full_like(d_in, float("nan"))
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    rc, msg = _noalloc(lib, d_in, d_out, nx, bs, steps, g, ny=ny, stream=side.cuda_stream)
    assert rc == 0, msg
    side.synchronize()
    got = d_out.cpu().numpy()
    ref = ic if steps == 0 else _allocating(ic, bs, steps, g)
    assert np.array_equal(got, ref), f"differs by {np.nanmax(np.abs(got - ref))}"


def test_noalloc_rejects_overlapping_fields():
    import torch
    from pysweep_b200 import _lib
    lib = _lib.lib()
    buf = torch.zeros((2, 128, 128), dtype=torch.float64, device="cuda")
    err = ctypes.create_string_buffer(256)
    half = ctypes.c_void_p(buf.data_ptr() + 64 * 128 * 8)  # starts inside the input field
    rc = lib.ps_heat_swept_noalloc(ctypes.c_void_p(buf.data_ptr()), half, 128, 128, 32, 3, 1.0,
                                   1e-6, 1.0 / 128, None, err, 256)
    assert rc == -1 and b"overlap" in err.value
