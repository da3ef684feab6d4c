#!/usr/bin/env python
"""Benchmark: FP64 swept heat on one B200 (row slabs over N GPUs under torchrun).

Workload (one "step" = one full solve): the 2-D heat equation u_t = u_xx + u_yy
on the periodic unit square, 8192 x 8192 FP64 cells, forward Euler with
dt = 0.2*dx^2, 5000 time steps, swept decomposition with blocksize 32
(12 levels per half-cycle, the library's default for this shape; at most
15 fit a 32-row band).  The initial field is a seeded sum of 8 periodic
Fourier modes (amplitudes U(0,1)).  The 537 MB field is larger than the
126 MB L2, so consecutive steps do not run from cache.

Reported on one JSON line (rank 0):
  value      Gcell-updates/s of the swept path with the field resident in HBM
  standard   the same workload through the standard (one step per launch) path
  e2e        the same metric through the public API with host buffers: pinned
             host -> device upload, the run, device -> host download
  swept_equals_standard  whether the two decompositions' 8192^2 results of
             the timed solves are bitwise equal
  roofline   the dominant kernel against its binding resource, the FP64 pipe
             (FP64 instructions/s against 64 lanes per SM at the maximum SM
             clock); its effective bandwidth (16 B per cell update: read and
             write of one FP64 value) against the measured HBM copy bandwidth,
             above 1.0 by the temporal reuse; and the DRAM bytes per launch
             that ncu measured at this size
  cpu_baseline  the reference's CPU swept algorithm (C restatement) on the
             host cores, on a bounded sample of the same workload
  secondary  the Euler, adjoint and batched targets (see secondary_lines)

Under torchrun with N > 1 ranks the grid is N*8192 x 8192, one 8192-row slab
per GPU (weak scaling), halo strips exchanged with NCCL after every swept
half-cycle; `value` counts the cell updates of all ranks over the slowest
rank's time.

`--impl reference` times that CPU algorithm alone as the reference arm.
`--batched`, `--adjoint` and `--euler` print the batched-instances, adjoint
and Euler lines instead.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gcell-updates/s FP64 swept vs standard (1 B200)"
UNIT = "Gcell-updates/s"
CELL_BYTES = 16  # one FP64 read + one FP64 write per cell update


def fourier_field(n, seed=0, modes=8):
    """Sum of `modes` periodic Fourier modes with U(0,1) amplitudes (seeded)."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(0, 1, modes)
    k = rng.integers(1, 9, modes)
    l = rng.integers(1, 9, modes)
    ph = rng.uniform(0, 2 * np.pi, modes)
    x = np.arange(n) / n
    f = np.zeros((n, n))
    for m in range(modes):
        # sin(2 pi (k x + l y) + phi) = sin(A)cos(B) + cos(A)sin(B)
        A = 2 * np.pi * k[m] * x[:, None] + ph[m]
        B = 2 * np.pi * l[m] * x[None, :]
        f += a[m] * (np.sin(A) * np.cos(B) + np.cos(A) * np.sin(B))
    return f[None]


def heat_globals(n, steps):
    dx = 1.0 / n
    dt = 0.2 * dx * dx
    return [0.0, steps * dt, dt, dx, dx, 1.0, True]


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": len(self.rows)}
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        if sm:
            out["sm_mhz"] = statistics.median(sm)
            out["sm_max_mhz"] = max(mx) if mx else None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        seen = set()
        for r in self.rows:
            if len(r) >= 9:
                for nm, v in zip(names, r[5:9]):
                    if v.lower().startswith("active"):
                        seen.add(nm)
        out["reasons"] = sorted(seen)
        pw = [float(r[3]) for r in self.rows if len(r) >= 9 and r[3].replace(".", "").isdigit()]
        if pw:
            out["power_w_max"] = max(pw)
        return out


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


SECONDARY_EULER_BATCH_STEPS = 100
FP64_OPS_PER_CELL = 8   # heat, forward Euler: 2 FMA, 4 add, 2 multiply (numpy's order)
FP64_LANES_PER_SM = 64  # B200: 148 SMs x 64 FP64 lanes x 1965 MHz = 18.6 T FP64 instructions/s


def max_sm_mhz(clk):
    """The GPU's maximum SM clock: sampled by nvidia-smi during the run, else
    the measured-peaks record, else B200's 1965 MHz."""
    mhz = (clk or {}).get("sm_max_mhz")
    if not mhz:
        try:
            mhz = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["sm_max_mhz"])
        except (OSError, KeyError, ValueError):
            mhz = 1965.0
    return float(mhz)


def fp64_roof(cells, ms, clk):
    """The swept streams are bound by FP64 issue, not HBM: FP64 instructions
    per second of a kernel against the FP64 pipe's rate (64 lanes per SM) at
    the GPU's maximum SM clock (an FMA counts as one instruction), in
    T instructions/s.  The rate at the sampled median clock is reported
    beside it."""
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    mhz = max_sm_mhz(clk)
    achieved = cells * FP64_OPS_PER_CELL / (ms / 1000) / 1e12
    peak = sms * FP64_LANES_PER_SM * mhz * 1e6 / 1e12
    med = (clk or {}).get("sm_mhz")
    out = {"ops_per_cell": FP64_OPS_PER_CELL, "achieved": achieved, "peak": peak,
           "frac": achieved / peak, "sm_max_mhz": mhz}
    if med:
        out["frac_at_median_clock"] = achieved / (peak * med / mhz)
        out["sm_median_mhz"] = med
    return out


def ncu_traffic(kind, n, bs, h):
    """DRAM bytes per launch of one kernel kind (h levels per half-cycle)
    from the committed ncu profile summary (measured at this grid size, or
    scaled from a smaller capture where its header says so); None where the
    summary has no line for this size."""
    p = os.path.join(ROOT, "profiles", f"heat2d_swept_{kind}_traffic.txt")
    try:
        for line in open(p):
            k, _, v = line.partition("=")
            if k.strip() == f"bytes_per_launch_n{n}_bs{bs}_h{h}":
                return float(v)
    except OSError:
        pass
    return None


def cpu_baseline(n_sample, bs, levels_cycles, threads):
    """The reference's CPU swept algorithm (C restatement) on a sample grid."""
    import oracle
    ic = fourier_field(n_sample)
    g = heat_globals(n_sample, 10)
    mpss = bs // 2 - 1
    t0 = time.perf_counter()
    _, fin = oracle.swept("heat", ic, g, 1, 1, bs, max_gss=levels_cycles - 1, nthreads=threads,
                          frames=False)
    dt = time.perf_counter() - t0
    cells = float(n_sample) ** 2 * mpss * levels_cycles
    return cells / dt / 1e9, dt, (ic, g, mpss * levels_cycles, fin)


def parity_check(sample, bs, device):
    """The GPU path on the CPU baseline's own sample, checked against the
    oracle's result of that run (max relative error, bitwise equality)."""
    from pysweep_b200 import Engine, plugin_constants
    ic, g, nlev, fin = sample
    n = ic.shape[-1]
    e = Engine("heat", n, n, blocksize=bs, device=device)
    for k, v in plugin_constants("heat", g).items():
        e.set_global(k, v)
    e.set_state(ic)
    e.run(nlev)
    got = e.get_state()
    e.close()
    err = float(np.max(np.abs(got - fin)) / max(np.max(np.abs(fin)), 1e-300))
    return {"sample": f"{n}x{n} heat, bs {bs}, {nlev} levels (the cpu_baseline run)",
            "max_rel_err_vs_oracle": err, "bitwise_equal": bool(np.array_equal(got, fin))}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    vals = []
    for i in range(args.warmup + args.steps):
        v, _, _ = cpu_baseline(args.ref_n, args.bs, args.ref_cycles, threads)
        if i >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    sample = (f"{args.ref_n}x{args.ref_n} heat, bs {args.bs}, {args.ref_cycles} swept "
              f"half-cycles ({(args.bs // 2 - 1) * args.ref_cycles} levels) per step")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(args):
    return {"workload": f"heat2d-fp64-periodic-{args.n}x{args.n}-{args.nsteps}steps-swept",
            "n": args.n, "time_steps": args.nsteps, "blocksize": args.bs,
            "l2": "inputs larger than L2 (field of n*n*8 bytes)"}


def roofline(prof, cell_bytes, clk, traffic_key=None):
    """Roofline of the dominant kernel of a run, from the per-launch CUDA-event
    profile {kind: (ms, launches, cell updates)}.

    The swept streams reuse every loaded value across the levels of a
    half-cycle, so their binding resource is the FP64 pipe, not HBM: `bound`,
    `achieved`, `peak` and `frac` are FP64 instructions per second against the
    pipe's rate at the maximum SM clock.  `effective_bytes` keeps the
    16-bytes-per-cell-update figure (a read and a write of each value) against
    the measured HBM copy bandwidth, which exceeds 1 by the temporal reuse, and
    `traffic` the DRAM bytes per launch that ncu measured at this size."""
    kinds = {k: v for k, v in prof.items() if v[1] > 0}
    dom = max(kinds, key=lambda k: kinds[k][0])
    dms, dn, dcells = kinds[dom]
    eff = dcells * cell_bytes / (dms / 1000) / 1e9
    peak_bw, peak_src = measured_peak()
    fp = fp64_roof(dcells, dms, clk)
    traffic = ncu_traffic(dom, *traffic_key) if traffic_key else None
    return {"bound": "fp64_pipe", "achieved": fp["achieved"], "peak": fp["peak"],
            "unit": "T FP64 instructions/s", "frac": fp["frac"], "traffic": traffic,
            "traffic_gbs": traffic / (dms / dn / 1000) / 1e9 if traffic else None,
            "kernel": dom, "launches": dn, "avg_launch_ms": dms / dn,
            "cell_updates_per_launch": dcells / dn, "fp64": fp,
            "effective_bytes": {"achieved": eff, "peak": peak_bw, "unit": "GB/s",
                                "frac": eff / peak_bw, "bytes_per_cell_update": cell_bytes,
                                "peak_source": peak_src,
                                "algorithmic_bytes_per_launch": dcells * cell_bytes / dn},
            "effective_bytes_frac": eff / peak_bw,
            "kernel_share": {k: v[0] / sum(x[0] for x in kinds.values()) for k, v in kinds.items()},
            "per_kernel": {k: dict(fp64_roof(v[2], v[0], clk), avg_launch_ms=v[0] / v[1],
                                   launches=v[1]) for k, v in kinds.items()}}


def run_b200(args):
    import torch
    import torch.distributed as dist

    from pysweep_b200 import Engine, plugin_constants

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    n, steps, bs = args.n, args.nsteps, args.bs
    f32 = args.f32
    metric = METRIC.replace("FP64", "FP32") if f32 else METRIC
    cell_bytes = CELL_BYTES // 2 if f32 else CELL_BYTES
    ic = fourier_field(n, seed=0).astype(np.float32 if f32 else np.float64)
    g = heat_globals(n, steps)
    eng = Engine("heat", n, n, its=1, blocksize=bs, device=local,
                 dtype="float32" if f32 else "float64")
    for k, v in plugin_constants("heat", g).items():
        eng.set_global(k, v)
    eng.configure(h=args.h, nseg=args.nseg)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)  # the solver and torch share one stream: no extra waits
    eng.set_stream(stream.cuda_stream)
    d_ic = torch.from_numpy(ic).cuda()
    cells_per_step = float(n) * n * steps

    def timed(mode, k):
        barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = eng.launches
        eng.profile(True)
        ev0.record(stream)
        for _ in range(k):
            eng.set_state(d_ic)
            eng.run(steps, mode=mode)
        ev1.record(stream)
        eng.synchronize()
        torch.cuda.synchronize()
        barrier()
        ms = ev0.elapsed_time(ev1) / k
        return max_over_ranks(ms), eng.launches - l0, eng.profile_read()

    # warm-up
    for _ in range(args.warmup):
        eng.set_state(d_ic)
        eng.run(steps, mode="swept")
    eng.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    ms_sw, launches, prof = timed("swept", args.steps)
    clk = clocks.stop()
    value = cells_per_step * world / (ms_sw / 1000) / 1e9
    # the swept result of the timed solves, kept on the device for the
    # bitwise comparison with the standard decomposition's
    swept_out = torch.empty_like(d_ic)
    eng.get_state(out=swept_out)

    std = None
    if args.standard_steps > 0:
        eng.set_state(d_ic)
        eng.run(steps, mode="standard")  # warm-up of the standard kernel
        ms_st, _, prof_st = timed("standard", args.standard_steps)
        std = {"value": cells_per_step * world / (ms_st / 1000) / 1e9, "ms_per_step": ms_st,
               "steps": args.standard_steps}
        pk = prof_st["standard"]
        if pk[1]:
            std["kernel_effective_gbs"] = pk[2] * cell_bytes / (pk[0] / 1000) / 1e9
        std_out = torch.empty_like(d_ic)
        eng.get_state(out=std_out)
        torch.cuda.synchronize()
        std["swept_equals_standard"] = bool(torch.equal(swept_out, std_out))
        del std_out

    # end to end through the public API with pinned host buffers
    h_in = torch.from_numpy(ic).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    h_in_np, h_out_np = h_in.numpy(), h_out.numpy()
    for _ in range(1):
        eng.set_state(h_in_np)
        eng.run(steps)
        eng.get_state(out=h_out_np)
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.e2e_steps):
        eng.set_state(h_in_np)
        eng.run(steps)
        eng.get_state(out=h_out_np)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(ev0.elapsed_time(ev1) / args.e2e_steps)
    e2e = {"value": cells_per_step * world / (ms_e2e / 1000) / 1e9, "unit": UNIT,
           "h2d_bytes_per_step": int(h_in.numel() * 8), "d2h_bytes_per_step": int(h_out.numel() * 8),
           "ms_per_step": ms_e2e, "steps": args.e2e_steps}

    roof = roofline(prof, cell_bytes, clk, None if f32 else (n, bs, eng.tiling()["h"]))

    cfg = workload_config(args)
    if f32:
        cfg["workload"] = cfg["workload"].replace("fp64", "fp32")
    line = {"metric": metric, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_sw,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 storage, f64 arithmetic" if f32 else "f64",
            "data": "synthetic", "config": cfg, "standard": std,
            "swept_vs_standard": (value / std["value"]) if std else None,
            "swept_equals_standard": std["swept_equals_standard"] if std else None,
            "roofline": roof, "e2e": e2e, "clocks": clk, "gpu_launches": launches,
            "tiling": dict(eng.tiling(), nseg_auto=not args.nseg)}
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not f32:
        threads = os.cpu_count() or 1
        v, secs, sample = cpu_baseline(args.ref_n, bs, args.ref_cycles, threads)
        line["cpu_baseline"] = {
            "value": v, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{args.ref_n}x{args.ref_n} heat, bs {bs}, {args.ref_cycles} swept "
                      f"half-cycles, {secs:.1f} s"}
        line["parity"] = parity_check(sample, bs, local)
    eng.close()
    del d_ic, swept_out
    if rank == 0 and world == 1 and not args.no_secondary and not f32:
        torch.cuda.empty_cache()
        line["secondary"] = secondary_lines(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def hook_line(args, n=4096, steps=600):
    """A user step hook (tests/hooks/heat_numpy_order.cu: the heat plugin's
    arithmetic in the reference's plugin format, compiled at run time) through
    the swept and the standard decomposition, against the built-in heat
    kernels on the same field."""
    import torch

    from pysweep_b200 import Engine, plugin_constants
    hook = os.path.join(ROOT, "tests", "hooks", "heat_numpy_order.cu")
    ic = fourier_field(n)
    g = heat_globals(n, steps)
    d_ic = torch.from_numpy(ic).cuda()
    out, res = {}, {}
    for label, eq, bs in (("hook", hook, 32), ("builtin", "heat", 32)):
        e = Engine(eq, n, n, blocksize=bs)
        for k, v in plugin_constants("heat", g).items():
            e.set_global(k, v)
        st = torch.cuda.Stream()
        e.set_stream(st.cuda_stream)
        for mode in ("swept", "standard"):
            e.set_state(d_ic)
            e.run(steps, mode=mode)
            e.synchronize()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(st)
            e.set_state(d_ic)
            e.run(steps, mode=mode)
            ev1.record(st)
            e.synchronize()
            res[(label, mode)] = float(n) * n * steps / (ev0.elapsed_time(ev1) / 1000) / 1e9
            out[(label, mode)] = e.get_state()
        e.close()
    return {"metric": "step hook Gcell-updates/s FP64 (heat in the plugin format, NVRTC)",
            "unit": "Gcell-updates/s", "n": n, "time_steps": steps,
            "hook_blocksize": 32, "builtin_blocksize": 32,
            "hook_swept": res[("hook", "swept")], "hook_standard": res[("hook", "standard")],
            "builtin_swept": res[("builtin", "swept")],
            "builtin_standard": res[("builtin", "standard")],
            "hook_equals_builtin": bool(np.array_equal(out[("hook", "swept")],
                                                       out[("builtin", "swept")])),
            "hook_swept_equals_standard": bool(np.array_equal(out[("hook", "swept")],
                                                              out[("hook", "standard")]))}


def secondary_lines(args):
    """The other targets of the metric, on the same GPU after the headline:
    Euler swept vs standard (4096^2, blocksize 16, 1000 steps), a user step
    hook compiled at run time against the built-in heat kernels, the adjoint's
    cost against its forward pass (2048^2, 2000 steps, 32 finite-difference
    directions) and the batched instances against one solver per instance
    (256 heat instances for 1000 steps; the 64 Euler instances for
    SECONDARY_EULER_BATCH_STEPS steps; one timed run of each side, to keep the
    default run within a few minutes)."""
    import copy

    import torch
    out = {}
    # the batched comparison builds 320 solvers per timing: one warm-up and
    # one timed run of each side
    quick = copy.copy(args)
    quick.steps, quick.warmup = 1, 1
    for name, fn in (("euler", lambda: euler_line(args)),
                     ("hook", lambda: hook_line(args)),
                     ("adjoint", lambda: adjoint_line(args)),
                     ("batched", lambda: batched_line(quick, SECONDARY_EULER_BATCH_STEPS))):
        t0 = time.perf_counter()
        out[name] = fn()
        out[name]["wall_s"] = time.perf_counter() - t0
        torch.cuda.empty_cache()
    return out


def run_b200_slabs(args):
    """N > 1 GPUs: one periodic (N*n) x n grid in row slabs of n rows per GPU
    (weak scaling), each slab with its own seeded Fourier field, solved with
    the swept kernels inside each GPU's window and the bs/2-row halo strips
    exchanged with NCCL point-to-point sends after every half-cycle."""
    import datetime

    import torch
    import torch.distributed as dist

    from pysweep_b200 import plugin_constants
    from pysweep_b200.distributed import SlabSolver

    world = int(os.environ["WORLD_SIZE"])
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device("cuda", local))
    n, steps, bs = args.n, args.nsteps, args.bs
    sol = SlabSolver("heat", n * world, n, its=1, blocksize=bs, h=args.h, nseg=args.nseg,
                     device=local)
    for k, v in plugin_constants("heat", heat_globals(n, steps)).items():
        sol.set_global(k, v)
    eng = sol.win.eng
    slab = fourier_field(n, seed=rank)
    d_slab = torch.from_numpy(slab).cuda()
    cells_per_step = float(n) * n * steps  # per rank

    def timed(k, fn):
        dist.barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(k):
            fn()
        ev1.record()
        torch.cuda.synchronize()
        dist.barrier()
        t = torch.tensor([ev0.elapsed_time(ev1) / k], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def device_pass():
        sol.set_slab(d_slab)
        sol.run(steps)

    for _ in range(args.warmup):
        device_pass()
    sol.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = eng.launches
    eng.profile(True)
    ms_sw = timed(args.steps, device_pass)
    prof = eng.profile_read()
    launches = eng.launches - l0
    clk = clocks.stop()
    value = cells_per_step * world / (ms_sw / 1000) / 1e9

    h_in = torch.from_numpy(slab).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()

    def host_pass():
        sol.set_slab(h_in.cuda(non_blocking=True))
        sol.run(steps)
        h_out.copy_(sol.win.get_rows(sol.halo, sol.rows, 0))

    host_pass()
    ms_e2e = timed(args.e2e_steps, host_pass)
    e2e = {"value": cells_per_step * world / (ms_e2e / 1000) / 1e9, "unit": UNIT,
           "h2d_bytes_per_step": int(h_in.numel() * 8), "d2h_bytes_per_step": int(h_out.numel() * 8),
           "ms_per_step": ms_e2e, "steps": args.e2e_steps}
    roof = roofline(prof, CELL_BYTES, clk)
    cfg = workload_config(args)
    cfg.update({"workload": f"heat2d-fp64-periodic-{n * world}x{n}-{steps}steps-swept-slabs",
                "global_rows": n * world, "rows_per_gpu": n, "halo_rows": bs // 2,
                "parallelism": f"row slabs x{world}, NCCL halo exchange per half-cycle"})
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_sw,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": cfg, "standard": None, "swept_vs_standard": None,
            "roofline": roof, "e2e": e2e, "clocks": clk, "gpu_launches": launches,
            "tiling": dict(eng.tiling(), nseg_auto=not args.nseg)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    sol.close()
    dist.destroy_process_group()
    return 0


def euler_field(n, seed=0, modes=8, gamma=1.4):
    """Uniform state (rho = 1, u = v = 1, p = 1) plus 8 seeded periodic Fourier
    modes on rho and p, scaled so that the perturbation's maximum is 0.1;
    conserved variables (rho, rho u, rho v, E)."""
    f = fourier_field(n, seed=seed, modes=modes)[0]
    f *= 0.1 / np.abs(f).max()
    rho, p = 1.0 + f, 1.0 + f
    out = np.empty((4, n, n))
    out[0] = rho
    out[1] = rho
    out[2] = rho
    out[3] = p / (gamma - 1) + 0.5 * rho * 2.0
    return out


def run_euler(args):
    print(json.dumps(euler_line(args)), flush=True)
    return 0


def euler_line(args):
    """Euler swept vs standard on one GPU (vortex-free periodic field of Fourier
    modes, CFL 0.1, two RK stages per step)."""
    import torch

    from pysweep_b200 import Engine, plugin_constants

    n, steps, bs = args.euler_n, args.euler_steps, args.euler_bs
    dx = 10.0 / n
    g = [0.0, steps * 0.1 * dx, 0.1 * dx, dx, dx, 1.4]
    d_ic = torch.from_numpy(euler_field(n)).cuda()
    eng = Engine("euler", n, n, its=2, blocksize=bs)
    for k, v in plugin_constants("euler", g).items():
        eng.set_global(k, v)
    if args.euler_chunk:
        eng.configure(chunk=args.euler_chunk)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    eng.set_stream(stream.cuda_stream)
    nl = 2 * steps
    cells = float(n) * n * nl

    def timed(mode, k):
        for _ in range(3):  # warm-up on a short run
            eng.set_state(d_ic)
            eng.run(40, mode=mode)
        eng.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        eng.profile(True)
        ev0.record(stream)
        for _ in range(k):
            eng.set_state(d_ic)
            eng.run(nl, mode=mode)
        ev1.record(stream)
        eng.synchronize()
        return ev0.elapsed_time(ev1) / k, eng.profile_read()

    ms_sw, prof = timed("swept", args.steps)
    out_sw = eng.get_state()
    ms_st, _ = timed("standard", args.steps)
    out_st = eng.get_state()
    kinds = {k: v[0] for k, v in prof.items() if v[1] > 0}
    line = {"metric": "Euler Gcell-stage-updates/s FP64 swept vs standard (1 B200)",
            "value": cells / (ms_sw / 1000) / 1e9, "unit": "Gcell-stage-updates/s",
            "standard": cells / (ms_st / 1000) / 1e9, "swept_ms": ms_sw, "standard_ms": ms_st,
            "swept_equals_standard": bool(np.array_equal(out_sw, out_st)),
            "kernel_share": {k: v / sum(kinds.values()) for k, v in kinds.items()},
            "n": n, "time_steps": steps, "blocksize": bs, "chunk": args.euler_chunk or "default",
            "stages_per_step": 2,
            "dtype": "f64", "data": "synthetic", "steps": args.steps}
    eng.close()
    return line


def batched_instances(seed=1, n_heat=256, n_euler=64):
    """Sizes (multiples of 32 in [128, 2048]), heat diffusivities U(0.5, 2) and
    vortex strengths U(1, 5), seeded."""
    rng = np.random.default_rng(seed)
    choices = np.arange(128, 2049, 32)
    heat = [(int(rng.choice(choices)), float(rng.uniform(0.5, 2.0))) for _ in range(n_heat)]
    euler = [(int(rng.choice(choices)), float(rng.uniform(1.0, 5.0))) for _ in range(n_euler)]
    return heat, euler


def run_batched(args):
    print(json.dumps(batched_line(args)), flush=True)
    return 0


def batched_line(args, euler_steps=None):
    """Batched persistent launches (one CUDA graph) vs one solver per instance.
    euler_steps: time steps of the Euler group (default: the heat group's)."""
    import torch

    from pysweep_b200 import Engine, plugin_constants
    from pysweep_b200.batch import Batch
    from pysweep_b200.equations.euler import analytical_array

    heat, euler = batched_instances(n_heat=args.batch_heat, n_euler=args.batch_euler)
    out = {"metric": "batched speedup (per-instance time / batched time)", "unit": "x",
           "higher_is_better": True, "dtype": "f64", "data": "synthetic",
           "steps": args.steps, "warmup": args.warmup, "time_steps": args.batched_steps}
    groups = []
    for eqn, inst in (("heat", heat), ("euler", euler)):
        if not inst:
            continue
        its = 1 if eqn == "heat" else 2
        bs = 32 if eqn == "heat" else 16
        tsteps = args.batched_steps if (eqn == "heat" or not euler_steps) else euler_steps
        nl = tsteps * its
        fields, consts = [], []
        for n, par in inst:
            if eqn == "heat":
                dx = 1.0 / n
                dt = 0.2 * dx * dx / par
                g = [0.0, 1.0, dt, dx, dx, par, True]
                fields.append(fourier_field(n, seed=n)[0][None])
            else:
                dx = 10.0 / n
                g = [0.0, 1.0, 0.1 * dx, dx, dx, 1.4]
                fields.append(analytical_array(n, n, 0.0, strength=par))
            consts.append(plugin_constants(eqn, g))
        dev = [torch.from_numpy(np.ascontiguousarray(f)).cuda() for f in fields]
        cells = float(sum(n * n for n, _ in inst)) * nl
        # batched
        b = Batch(eqn, [(n, n) for n, _ in inst], its=its, blocksize=bs)
        for i in range(len(inst)):
            b.set_constants(i, consts[i])
        for _ in range(args.warmup):
            for i in range(len(inst)):
                b.set_state(i, dev[i])
            b.run(nl, graph=True)
        b.synchronize()
        t = []
        for _ in range(args.steps):
            for i in range(len(inst)):
                b.set_state(i, dev[i])
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            b.run(nl, graph=True)
            b.synchronize()
            t.append(time.perf_counter() - t0)
        t_batch = statistics.median(t)
        batch_out = [b.get_state(i) for i in range(min(3, len(inst)))]
        b.close()
        # one solver per instance: all on one stream, then each on its own
        engines = []
        for i, (n, _) in enumerate(inst):
            e = Engine(eqn, n, n, its=its, blocksize=bs)
            for k, v in consts[i].items():
                e.set_global(k, v)
            engines.append(e)
        res = {}
        shared = torch.cuda.Stream()
        for label in ("one_stream", "own_streams"):
            if label == "one_stream":
                for e in engines:
                    e.set_stream(shared.cuda_stream)
            else:
                for e in engines:
                    e.set_stream(0)  # back to a stream of its own
            for _ in range(max(1, args.warmup - 2)):
                for i, e in enumerate(engines):
                    e.set_state(dev[i])
                    e.run(nl)
                torch.cuda.synchronize()
            t = []
            for _ in range(args.steps):
                for i, e in enumerate(engines):
                    e.set_state(dev[i])
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                for e in engines:
                    e.run(nl)
                torch.cuda.synchronize()
                t.append(time.perf_counter() - t0)
            res[label] = statistics.median(t)
        for i in range(len(batch_out)):
            if not np.array_equal(engines[i].get_state(), batch_out[i]):
                raise AssertionError(f"batched {eqn} instance {i} differs from its single run")
        for e in engines:
            e.close()
        best = min(res.values())
        groups.append({"equation": eqn, "instances": len(inst), "time_steps": tsteps,
                       "blocksize": bs, "batched_s": t_batch, "per_instance_one_stream_s": res["one_stream"],
                       "per_instance_own_streams_s": res["own_streams"],
                       "speedup_vs_best_per_instance": best / t_batch,
                       "batched_gcell_updates_s": cells / t_batch / 1e9})
    out["groups"] = groups
    out["value"] = (sum(g["per_instance_one_stream_s"] for g in groups) /
                    sum(g["batched_s"] for g in groups))
    out["value_vs_own_streams"] = (sum(g["per_instance_own_streams_s"] for g in groups) /
                                   sum(g["batched_s"] for g in groups))
    out["timing"] = "wall clock around the run with device synchronisation on both sides"
    return out


def run_adjoint(args):
    print(json.dumps(adjoint_line(args)), flush=True)
    return 0


def heatvar_line(args):
    """The swept kernels of the differentiable solve alone: one segment of
    `--adj-steps` levels at `--adj-n`^2 through Engine("heatvar") (the
    recompute: courant numbers 0.1, every level's Laplacian stored) or
    Engine("heatvar_adjoint_mu") (the adjoint: courant numbers, the
    Laplacians and the sum set), from a seeded random field; one step = one
    run of the segment.  Throughput and the per-kernel device time."""
    import torch

    from pysweep_b200 import Engine
    n, nl = args.adj_n, args.adj_steps
    rng = np.random.default_rng(0)
    u0 = torch.tensor(rng.standard_normal((n, n)), device="cuda")
    C = torch.full((n, n), 0.1, dtype=torch.float64, device="cuda")
    lap = torch.zeros((nl, n, n), dtype=torch.float64, device="cuda")
    acc = torch.zeros_like(u0)
    eq = "heatvar" if args.heatvar == "fwd" else "heatvar_adjoint_mu"
    e = Engine(eq, n, n, blocksize=32)
    e.set_field(0, C)
    e.set_field(1, lap)
    e.set_global("LEN", nl)
    if args.heatvar == "adj":
        e.set_field(2, acc)
    st = torch.cuda.Stream()
    e.set_stream(st.cuda_stream)
    for _ in range(args.warmup):
        e.set_state(u0)
        e.run(nl)
    e.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(st)
    for _ in range(args.steps):
        e.set_state(u0)
        e.run(nl)
    ev1.record(st)
    e.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    e.profile(True)
    e.set_state(u0)
    e.run(nl)
    e.synchronize()
    prof = {k: {"ms": v[0], "launches": v[1]} for k, v in e.profile_read().items() if v[1]}
    tiling = e.tiling()
    e.close()
    return {"metric": f"{eq} swept Gcell-updates/s FP64", "value": n * n * nl / ms / 1e6,
            "unit": "Gcell-updates/s", "ms_per_step": ms, "n": n, "levels": nl,
            "tiling": tiling, "profile": prof, "dtype": "f64", "data": "synthetic",
            "steps": args.steps, "warmup": args.warmup}


def adjoint_line(args):
    """Inverse heat problem: forward vs adjoint cost, gradients vs central differences."""
    import torch

    from pysweep_b200.adjoint import heat_solve

    n, steps, every = args.adj_n, args.adj_steps, 64
    rng = np.random.default_rng(2)
    x = np.arange(n) / n

    def fourier(modes=8):
        f = np.zeros((n, n))
        for _ in range(modes):
            k, l = rng.integers(1, 9, 2)
            f += rng.uniform(0, 1) * np.sin(2 * np.pi * (k * x[:, None] + l * x[None, :]) +
                                            rng.uniform(0, 2 * np.pi))
        return f / modes

    dev = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda")  # noqa: E731
    alpha_star = dev(1.0 + 0.5 * fourier())
    alpha0 = dev(1.0 + 0.5 * fourier())
    u0 = dev(fourier())
    dx = 1.0 / n
    dt = 0.2 * dx * dx / 1.5  # stable for alpha <= 1.5
    target = heat_solve(u0, alpha_star, steps, dt, dx, every)

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), r

    for _ in range(args.warmup):  # both passes, so the timed ones reuse cached buffers
        xu = u0.clone().requires_grad_(True)
        xa = alpha0.clone().requires_grad_(True)
        (0.5 * ((heat_solve(xu, xa, steps, dt, dx, every) - target) ** 2).sum()).backward()
    fwd, bwd = [], []
    for _ in range(args.steps):
        xu = u0.clone().requires_grad_(True)
        xa = alpha0.clone().requires_grad_(True)
        t_f, uT = timed(lambda: heat_solve(xu, xa, steps, dt, dx, every))
        loss = 0.5 * ((uT - target) ** 2).sum()
        t_b, _ = timed(lambda: loss.backward())
        fwd.append(t_f)
        bwd.append(t_b)
    gu, ga = xu.grad, xa.grad

    def J(a, b):
        return 0.5 * ((heat_solve(a, b, steps, dt, dx, every) - target) ** 2).sum().item()

    # central differences with h = 1e-6 along unit directions (roundoff-limited,
    # about eps*J/h), and Richardson-extrapolated ones, (4 D(h/2) - D(h)) / 3
    # with h = 1e-3 (truncation O(h^4))
    h, hr = 1e-6, 1e-3
    gen = torch.Generator(device="cuda").manual_seed(0)
    worst = worst_r = 0.0
    for _ in range(args.adj_dirs):
        du = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=gen)
        da = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=gen)
        du /= du.norm()
        da /= da.norm()
        d = lambda e: (J(u0 + e * du, alpha0 + e * da) - J(u0 - e * du, alpha0 - e * da)) / (2 * e)  # noqa: E731
        an = (gu * du).sum().item() + (ga * da).sum().item()
        worst = max(worst, abs(d(h) - an) / max(abs(an), 1e-300))
        worst_r = max(worst_r, abs((4 * d(hr / 2) - d(hr)) / 3 - an) / max(abs(an), 1e-300))
    t_f, t_b = statistics.median(fwd), statistics.median(bwd)
    # the same solve through the swept decomposition (SweptHeatVar): forward,
    # and backward with each segment recomputed by the swept forward kernels
    # and walked back by the swept adjoint kernels
    for _ in range(args.warmup):
        xu = u0.clone().requires_grad_(True)
        xa = alpha0.clone().requires_grad_(True)
        (0.5 * ((heat_solve(xu, xa, steps, dt, dx, every, swept=True) - target) ** 2).sum()).backward()
    sfwd, sbwd = [], []
    for _ in range(args.steps):
        su = u0.clone().requires_grad_(True)
        sa = alpha0.clone().requires_grad_(True)
        t_sf, suT = timed(lambda: heat_solve(su, sa, steps, dt, dx, every, swept=True))
        sloss = 0.5 * ((suT - target) ** 2).sum()
        t_sb, _ = timed(lambda: sloss.backward())
        sfwd.append(t_sf)
        sbwd.append(t_sb)
    t_sf, t_sb = statistics.median(sfwd), statistics.median(sbwd)
    rel = lambda x, y: ((x - y).abs().max() / y.abs().max()).item()  # noqa: E731
    # the lambda-form swept adjoint (generic kernels) once, untimed: bitwise
    lu = u0.clone().requires_grad_(True)
    la = alpha0.clone().requires_grad_(True)
    (0.5 * ((heat_solve(lu, la, steps, dt, dx, every, swept="lambda") - target) ** 2).sum()).backward()
    same = bool((lu.grad == gu).all()) and bool((la.grad == ga).all())
    return {
        "metric": "adjoint/forward cost", "value": t_b / t_f, "unit": "x", "higher_is_better": False,
        "forward_ms": t_f, "backward_ms": t_b, "n": n, "time_steps": steps, "checkpoint_every": every,
        "swept": {"form": "mu", "forward_ms": t_sf, "backward_ms": t_sb,
                  "backward_over_swept_forward": t_sb / t_sf,
                  "backward_over_fastest_forward": t_sb / min(t_f, t_sf),
                  "forward_equal_standard": bool((suT.detach() == uT.detach()).all()),
                  "grad_u0_max_rel_diff": rel(su.grad, gu), "grad_alpha_max_rel_diff": rel(sa.grad, ga),
                  "lambda_form_gradients_equal_standard": same},
        "fd_directions": args.adj_dirs, "fd_h": h, "fd_max_rel_err": worst,
        "fd_richardson_h": hr, "fd_richardson_max_rel_err": worst_r, "dtype": "f64",
        "data": "synthetic", "steps": args.steps, "warmup": args.warmup}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=8192)
    ap.add_argument("--nsteps", type=int, default=5000)
    ap.add_argument("--bs", type=int, default=32)
    ap.add_argument("--h", type=int, default=0)
    ap.add_argument("--nseg", type=int, default=0, help="column segments per band (0: automatic)")
    ap.add_argument("--standard-steps", type=int, default=2)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--ref-n", type=int, default=2048)
    ap.add_argument("--ref-cycles", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the Euler, adjoint and batched lines of the default run")
    ap.add_argument("--f32", action="store_true",
                    help="float32 fields (the reference's dtype: float32) on one GPU")
    ap.add_argument("--batched", action="store_true",
                    help="batched instances vs one solver per instance (separate JSON line)")
    ap.add_argument("--batched-steps", type=int, default=1000)
    ap.add_argument("--batch-heat", type=int, default=256)
    ap.add_argument("--batch-euler", type=int, default=64)
    ap.add_argument("--euler", action="store_true",
                    help="Euler swept vs standard (separate JSON line)")
    ap.add_argument("--euler-n", type=int, default=4096)
    ap.add_argument("--euler-steps", type=int, default=1000)
    ap.add_argument("--euler-bs", type=int, default=16)
    ap.add_argument("--euler-chunk", type=int, default=0, help="32 or 64 (0: the default)")
    ap.add_argument("--adjoint", action="store_true",
                    help="inverse heat problem: adjoint vs forward cost (separate JSON line)")
    ap.add_argument("--adj-n", type=int, default=2048)
    ap.add_argument("--adj-steps", type=int, default=2000)
    ap.add_argument("--adj-dirs", type=int, default=32)
    ap.add_argument("--heatvar", choices=["fwd", "adj"], default=None,
                    help="the differentiable solve's swept kernels alone: the recompute (fwd) or "
                         "the adjoint (adj), one --adj-steps segment at --adj-n (separate JSON line)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    if args.impl == "reference":
        return run_reference(args)
    if args.batched:
        return run_batched(args)
    if args.adjoint:
        return run_adjoint(args)
    if args.heatvar:
        print(json.dumps(heatvar_line(args)), flush=True)
        return 0
    if args.euler:
        return run_euler(args)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        return run_b200_slabs(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
