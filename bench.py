#!/usr/bin/env python
"""Benchmark: converged T-matrices per second for a batch of 4096 spheroids.

Workload (the batched-forward configuration): 4096 independent spheroids from
a seeded generator -- size parameter x = 2 pi r_ev / lambda uniform in
[0.1, 10], axis ratio log-uniform in [0.5, 2], Re m uniform in [1.3, 2.0],
Im m log-uniform in [1e-3, 1], lambda = 1 um -- run through the task-based
schedule (min_order 10, max_order 100, ngauss = 2 * order, tolerance 1e-4):
the m = 0 convergence loop, every m block at the converged order, and the
full Qsca/Qext sums. One step = one batch. Data are synthetic.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank runs its own batch (weak scaling, no
data-path collective: the grains are independent); the time is the maximum
over ranks.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_GRAINS = 4096
SCHEDULE = dict(min_order=10, max_order=100, gauss_legendre_factor=2,
                tolerance=1e-4)
# grains per reference-CPU step: a bounded sample of the 4096-grain
# workload (step s takes slice s mod 4 of the same seeded grains), so that a
# 25-step reference run ends within a few minutes on 16 host cores
CPU_SAMPLE = 1024
# contexts (host threads) of the end-to-end measurement
E2E_CONTEXTS = 3
MODE_NAMES = {0: "host", 1: "graph"}


def grains(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.1, 10.0, n)
    d = np.exp(rng.uniform(np.log(0.5), np.log(2.0), n))
    mr = rng.uniform(1.3, 2.0, n)
    mi = np.exp(rng.uniform(np.log(1e-3), np.log(1.0), n))
    lam = 1e-6
    r = x * lam / (2 * np.pi)
    return r, np.full(n, lam), mr + 1j * mi, d


def rank_seed(rank):
    """Each rank computes its own independent grains (weak scaling)."""
    return 1 + rank


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Dist:
    """Barrier and max-reduction across ranks (NCCL when world > 1; gloo on
    CPU for the multi-process tests)."""

    def __init__(self, world, local, backend="nccl"):
        self.world = world
        self.pg = None
        self.device = "cuda" if backend == "nccl" else "cpu"
        if world > 1:
            import datetime

            import torch
            import torch.distributed as td
            if backend == "nccl":
                torch.cuda.set_device(local)
            td.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.td = td
            self.torch = torch

    def barrier(self):
        if self.world > 1:
            self.td.barrier()

    def max(self, v):
        if self.world == 1:
            return v
        t = self.torch.tensor([v], dtype=self.torch.float64, device=self.device)
        self.td.all_reduce(t, op=self.td.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.td.destroy_process_group()


class ClockSampler:
    """SM clock and throttle-reason samples during the timed region: NVML
    polled every few milliseconds from a thread (a timed region of a few
    steps lasts tens of ms), else nvidia-smi at its 200 ms minimum."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
             "sw_power_cap"]

    def __init__(self, device, period_s=0.002):
        self.device = device
        self.period = period_s
        self.proc = None
        self.nvml = None
        self.lines = []
        self.samples = []  # (sm MHz, reason bits)
        self.smax = None
        self.bits = {}
        self.done = threading.Event()

    def _nvml_start(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        idx = self.device
        if hasattr(torch.cuda, "_get_nvml_device_index"):
            idx = torch.cuda._get_nvml_device_index(self.device)
        h = pynvml.nvmlDeviceGetHandleByIndex(idx)
        get_reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons",
                              None) or pynvml.nvmlDeviceGetCurrentClocksThrottleReasons

        def bit(name, default):
            for pre in ("nvmlClocksEventReason", "nvmlClocksThrottleReason"):
                if hasattr(pynvml, pre + name):
                    return getattr(pynvml, pre + name)
            return default
        self.bits = {"hw_slowdown": bit("HwSlowdown", 0x8),
                     "hw_thermal_slowdown": bit("HwThermalSlowdown", 0x40),
                     "sw_thermal_slowdown": bit("SwThermalSlowdown", 0x20),
                     "sw_power_cap": bit("SwPowerCap", 0x4)}
        self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))

        def poll():
            while not self.done.is_set():
                try:
                    self.samples.append(
                        (float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)),
                         int(get_reasons(h))))
                except pynvml.NVMLError:
                    pass
                time.sleep(self.period)
        self.nvml = pynvml
        self.th = threading.Thread(target=poll, daemon=True)
        self.th.start()

    def start(self):
        try:
            self._nvml_start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self.done.set()
            self.th.join(timeout=5)
            sm = [c for c, _ in self.samples]
            reasons = sorted({nm for _, b in self.samples
                              for nm, v in self.bits.items() if b & v})
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
            return {"sm_mhz": float(np.median(sm)) if sm else None,
                    "sm_max_mhz": self.smax, "samples": len(sm),
                    "source": "NVML every %g ms" % (1e3 * self.period),
                    "reasons": reasons}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 8:
                continue
            try:
                sm.append(float(p[0]))
                smax = float(p[1])
            except ValueError:
                continue
            for nm, v in zip(self.NAMES, p[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": smax, "samples": len(sm),
                "source": "nvidia-smi every 200 ms", "reasons": sorted(reasons)}


def flush_l2(buf):
    # write a buffer larger than the 126 MB L2 between timed steps
    buf.zero_()


BUCKETS = ["nb<=8", "9..16", "17..32", "33..64", "65..128"]


def class_size(N, m, cls):
    """Members of parity class `cls` of block m at order N (the work items of
    the block kernels)."""
    if m == 0:
        n0 = 1 if cls & 1 else 2
        return (N - n0) // 2 + 1 if N >= n0 else 0
    na0 = m if (m & 1) == cls else m + 1
    nb0 = m if (m & 1) == (cls ^ 1) else m + 1
    r0 = (N - na0) // 2 + 1 if N >= na0 else 0
    r1 = (N - nb0) // 2 + 1 if N >= nb0 else 0
    return r0 + r1


def bucket_flops(nmax, ngauss):
    """Executed-flop model of the block kernels per class-size bucket for
    every (m, class) item of the grains at their orders: assembly
    8 t nb^2 ng (t = 2 terms for m = 0, 4 otherwise), LU 8/3 nb^3, the two
    triangular solves 8 nb^3; and the items per bucket."""
    fl = np.zeros(5)
    cnt = np.zeros(5, np.int64)
    orders, counts = np.unique(np.stack([nmax, ngauss], 1), axis=0, return_counts=True)
    for (N, ng), c in zip(orders, counts):
        if N <= 0:
            continue
        for m in range(N + 1):
            for cls in range(4 if m == 0 else 2):
                nb = class_size(int(N), m, cls)
                if nb <= 0:
                    continue
                b = 0 if nb <= 8 else 1 if nb <= 16 else 2 if nb <= 32 else 3 if nb <= 64 else 4
                t = 2.0 if m == 0 else 4.0
                fl[b] += c * (8 * t * nb * nb * ng + (8.0 / 3.0) * nb ** 3 + 8.0 * nb ** 3)
                cnt[b] += c
    return fl, cnt


def workload_config():
    """The workload both arms name in their JSON line."""
    return {"workload": "batched T-matrices, config-2 distribution "
                        "(4096 spheroids, x in [0.1,10])",
            "grains_per_gpu": N_GRAINS, **SCHEDULE,
            "l2": "flushed between steps (256 MB write); working set > L2"}


def reference_sample(nthreads, step):
    """One bounded sample of the workload through the reference's own task
    objects under QuickSched (oracle/_ref, built from the reference): slice
    step mod (N_GRAINS / CPU_SAMPLE) of the seeded grains the GPU arm times
    on rank 0."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    r, lam, m, d = grains(N_GRAINS, rank_seed(0))
    nsl = max(1, N_GRAINS // CPU_SAMPLE)
    lo = (step % nsl) * CPU_SAMPLE
    sl = slice(lo, min(N_GRAINS, lo + CPU_SAMPLE))
    r, lam, m, d = r[sl], lam[sl], m[sl], d[sl]
    t = time.perf_counter()
    out = O.ref_batch(r, lam, m, d, nthreads=nthreads, want_t=False, **{
        "min_order": SCHEDULE["min_order"], "max_order": SCHEDULE["max_order"],
        "glfac": SCHEDULE["gauss_legendre_factor"],
        "tolerance": SCHEDULE["tolerance"]})
    dt = time.perf_counter() - t
    return len(out), dt


def cpu_baseline_block(nthreads, steps=3, warmup=1):
    """The reference arm's measurement on a bounded sample: warm-up slices,
    then the median rate of `steps` slices of the same workload."""
    vals = []
    for s in range(warmup + steps):
        n, dt = reference_sample(nthreads, s)
        if s >= warmup:
            vals.append(n / dt)
    v = float(np.median(vals))
    return {"value": v, "unit": "T-matrices/s", "cores": nthreads,
            "kind": "reference",
            "sample": "%d-grain slices of the same 4096 seeded grains, reference "
                      "task objects (InteractionTask/TMatrixM0Task chain + "
                      "TMatrixMAllTask) under QuickSched, maximum_order 100, "
                      "%d threads, %d warm-up slice(s), median of %d slices"
                      % (CPU_SAMPLE, nthreads, warmup, steps)}


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    nthreads = os.cpu_count() or 1
    times, done = [], 0
    for s in range(args.warmup + args.steps):
        n, dt = reference_sample(nthreads, s)
        if s >= args.warmup:
            times.append(dt)
            done += n
    value = done / sum(times)
    line = {
        "impl": "reference", "metric": "T-matrices/s (converged, batched)",
        "value": value, "unit": "T-matrices/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": workload_config(),
        "cpu_baseline": {"value": value, "unit": "T-matrices/s",
                         "cores": nthreads, "kind": "reference",
                         "sample": "each step a %d-grain slice of the same 4096 "
                                   "seeded grains (4 slices in turn), reference "
                                   "task objects under QuickSched, %d threads"
                                   % (CPU_SAMPLE, nthreads)},
        "e2e": {"value": value, "unit": "T-matrices/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_ours(args):
    import torch

    from costuum_b200 import _lib
    from costuum_b200.tmatrix import Context

    rank, world, local = dist_env()
    dist = Dist(world, local)
    ctx = Context(local)
    lib = _lib.load()
    h = ctx._h
    dfma = ctx.probe_fp64(0)
    dmma = ctx.probe_fp64(1)

    r, lam, m, d = grains(N_GRAINS, rank_seed(rank))
    mr = np.ascontiguousarray(m.real)
    mi = np.ascontiguousarray(m.imag)
    sched = _lib.TmxSchedule(SCHEDULE["min_order"], SCHEDULE["max_order"],
                             SCHEDULE["gauss_legendre_factor"], 0,
                             SCHEDULE["tolerance"])
    P = _lib.ptr
    # untimed: the block-kernel dispatch table tuned on these grains at their
    # converged orders (every family in every size bucket it can run)
    conv = ctx.tmatrix_batch(r, lam, m, d, **SCHEDULE)
    autotune = None
    if not args.skip_tune:
        table, tune_ms = ctx.autotune(r, lam, m, d, conv.nmax.copy(),
                                      conv.ngauss.copy(), reps=3)
        autotune = {"table": [Context.FAMILIES[f] for f in table],
                    "buckets": ["nb<=8", "9..16", "17..32", "33..64", "65..128"],
                    "median_ms": [[round(float(x), 4) for x in row] for row in tune_ms],
                    "what": "per size bucket, median ms per batch of each kernel "
                            "family (columns: %s; -1 not run), buckets serialised"
                            % ", ".join(Context.FAMILIES)}
    _lib.check(h, lib.tmx_batch_upload(h, N_GRAINS, P(r), P(lam), P(mr), P(mi),
                                       P(d), sched), "upload")
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda:%d" % local)

    def step_device():
        flush_l2(flush)
        torch.cuda.synchronize()
        _lib.check(h, lib.tmx_timer_start(h), "timer")
        _lib.check(h, lib.tmx_batch_compute(h), "compute")
        ms = np.zeros(1)
        _lib.check(h, lib.tmx_timer_stop(h, P(ms)), "timer")
        return float(ms[0])

    # batch mode: the host-driven loop or the device-driven graph, whichever
    # runs this workload faster on this box (measured on untimed steps; the
    # host-driven mode depends on the host thread's speed, the graph not)
    mode_ms = {}
    for mode in (Context.BATCH_HOST, Context.BATCH_GRAPH):
        ctx.set_batch_mode(mode)
        for _ in range(2):
            step_device()
        mode_ms[mode] = float(np.median([step_device() for _ in range(3)]))
    chosen = min(mode_ms, key=mode_ms.get)
    other = Context.BATCH_GRAPH if chosen == Context.BATCH_HOST else Context.BATCH_HOST
    ctx.set_batch_mode(chosen)
    for _ in range(args.warmup):
        step_device()
    # ---- device-resident timed region (no per-launch events in it: the
    # kernel profile below runs on separate, untimed steps)
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = ctx.kernel_launches
    dist.barrier()
    torch.cuda.synchronize()
    total = 0.0
    host_t = []
    step_ms = []
    for _ in range(args.steps):
        t = step_device()
        step_ms.append(t)
        total += t
        ht = np.zeros(4)
        lib.tmx_batch_host_times(h, P(ht))
        host_t.append(ht)
    torch.cuda.synchronize()
    dist.barrier()
    launches = ctx.kernel_launches - launches0
    clocks = sampler.stop()
    chosen_ok = ctx.last_batch_mode == chosen
    # ---- the same batch in the other mode, timed the same way
    ctx.set_batch_mode(other)
    for _ in range(max(2, args.warmup)):
        step_device()
    other_ms = [step_device() for _ in range(args.steps)]
    other_ok = ctx.last_batch_mode == other
    ctx.set_batch_mode(Context.BATCH_HOST)
    # ---- kernel profile: the same steps again with CUDA events around every
    # block and table launch and the launch timeline (untimed)
    lib.tmx_profile_enable(h, 1)
    prof_total = 0.0
    for _ in range(args.steps):
        prof_total += step_device()
    bk_ms = np.zeros(1)
    bk_n = ctypes.c_int64()
    bk_fl = np.zeros(1)
    lib.tmx_profile_read(h, 0, P(bk_ms), ctypes.byref(bk_n), P(bk_fl))
    tb_ms = np.zeros(1)
    tb_n = ctypes.c_int64()
    lib.tmx_profile_read(h, 1, P(tb_ms), ctypes.byref(tb_n), P(np.zeros(1)))
    # per timed batch, from the launch timeline: when the order loop's last
    # launch and the batch's last launch finished after its first launch
    tl = ctx.timeline()
    marks = tl[tl["kind"] < 0]
    loop_ms, gpu_ms = [], []
    t_start = None
    for rec in marks:
        if rec["kind"] == -1:
            t_start = rec["start_ms"]
        elif t_start is not None and rec["kind"] == -2:
            loop_ms.append(rec["start_ms"] - t_start)
        elif t_start is not None and rec["kind"] == -3:
            gpu_ms.append(rec["start_ms"] - t_start)
    lib.tmx_profile_enable(h, 0)
    flops_survey = lib.tmx_batch_flops_survey(h)
    total_max = dist.max(total)
    ms_step = total_max / args.steps
    value = world * N_GRAINS / (ms_step * 1e-3)

    # per-grain outcome of the last step
    nmax = np.zeros(N_GRAINS, np.int32)
    status = np.zeros(N_GRAINS, np.int32)
    q = np.zeros((N_GRAINS, 6))
    lib.tmx_batch_results(h, _lib.iptr(nmax), None, _lib.iptr(status), P(q))

    # ---- end to end through the public API with host buffers: the inputs
    # from host arrays, and every converged T-matrix back in page-locked host
    # memory (each block round streams its range while the batch runs; the
    # rest follows in tmatrices()) together with the per-grain results
    flat, _ = ctx.tmatrices()
    ctx.stream_tmatrices(int(flat.size * 1.25) + 4096)
    ctx.tmatrix_batch(r, lam, m, d, **SCHEDULE)
    ctx.tmatrices()
    e2e_ms, t_bytes = 0.0, 0
    for s in range(max(1, args.steps)):
        flush_l2(flush)
        torch.cuda.synchronize()
        dist.barrier()
        t0 = time.perf_counter()
        res = ctx.tmatrix_batch(r, lam, m, d, **SCHEDULE)
        flat, off = ctx.tmatrices()
        e2e_ms += (time.perf_counter() - t0) * 1e3
        t_bytes = flat.nbytes
    e2e_max = dist.max(e2e_ms) / max(1, args.steps)
    # ---- the same end to end with batches in flight on several contexts:
    # E2E_CONTEXTS contexts on as many host threads, in the device-driven
    # mode (no per-order device-to-host reads that would queue behind the
    # other batches' T-matrix downloads), so that the downloads (PCIe,
    # ~57 GB/s: 6.7 ms for the 382 MB of a step) overlap the other batches'
    # compute, as a serving loop would run them. Every step still uploads
    # its inputs and downloads all its T-matrices and results inside the
    # timed region (no L2 flush between steps: the 0.4 GB of T-matrices and
    # tables per step exceed the 126 MB L2)
    pipe_ctx = [ctx] + [Context(local) for _ in range(E2E_CONTEXTS - 1)]
    for c in pipe_ctx:
        if c is not ctx:
            # page-locked destination of the download, as on the first one;
            # a first batch in the host-driven mode gives the graph its
            # extent (the largest converged order) and its storage sizes
            c.stream_tmatrices(int(flat.size * 1.25) + 4096)
            c.tmatrix_batch(r, lam, m, d, **SCHEDULE)
        c.set_batch_mode(Context.BATCH_GRAPH)
        for _ in range(2):
            c.tmatrix_batch(r, lam, m, d, **SCHEDULE)
            c.tmatrices()
    pipe_steps = max(2, args.steps)
    pipe_err = []

    def pipe_worker(c):
        try:
            for _ in range(pipe_steps):
                c.tmatrix_batch(r, lam, m, d, **SCHEDULE)
                c.tmatrices()
        except Exception as e:  # noqa: BLE001
            pipe_err.append(e)

    torch.cuda.synchronize()
    dist.barrier()
    t0 = time.perf_counter()
    workers = [threading.Thread(target=pipe_worker, args=(c,)) for c in pipe_ctx]
    for w in workers:
        w.start()
    for w in workers:
        w.join()
    pipe_ms = (time.perf_counter() - t0) * 1e3 / (len(pipe_ctx) * pipe_steps)
    if pipe_err:
        raise pipe_err[0]
    pipe_mode_ok = all(c.last_batch_mode == Context.BATCH_GRAPH for c in pipe_ctx)
    pipe_max = dist.max(pipe_ms)
    for c in pipe_ctx[1:]:
        c.stream_tmatrices(0)
        c.close()
    ctx.stream_tmatrices(0)
    ctx.set_batch_mode(Context.BATCH_HOST)
    # host -> device: five input arrays; device -> host: the T-matrices, the
    # chain states (64 B), done list (8 B), Q sums (16 B) and status (4 B)
    # per grain
    h2d = N_GRAINS * 5 * 8
    d2h = t_bytes + N_GRAINS * (64 + 8 + 16 + 4)

    # ---- plain path: the same kernels, one grain per call (no batching)
    plain = None
    grad = None
    if rank == 0 and world == 1 and not args.skip_extras:
        ev = lambda: np.zeros(1)  # noqa: E731
        nplain = 64
        t_ms = 0.0
        for i in range(nplain):
            lib.tmx_timer_start(h)
            rr, ll, mm_, dd = grains(1, 5000 + i)
            ctx.tmatrix_batch(rr, ll, mm_, dd, **SCHEDULE)
            ms = ev()
            lib.tmx_timer_stop(h, P(ms))
            t_ms += float(ms[0])
        plain = {"value": nplain / (t_ms * 1e-3), "unit": "T-matrices/s",
                 "grains": nplain,
                 "what": "one grain per library call (same kernels, no batching)"}
        # the same calls in the device-driven mode (after two untimed calls
        # that build the one-grain graph)
        ctx.set_batch_mode(Context.BATCH_GRAPH)
        t_ms = 0.0
        graph_calls = 0
        for i in range(-2, nplain):
            rr, ll, mm_, dd = grains(1, 5000 + max(i, 0))
            lib.tmx_timer_start(h)
            ctx.tmatrix_batch(rr, ll, mm_, dd, **SCHEDULE)
            ms = ev()
            lib.tmx_timer_stop(h, P(ms))
            if i >= 0:
                t_ms += float(ms[0])
                graph_calls += int(ctx.last_batch_mode == Context.BATCH_GRAPH)
        ctx.set_batch_mode(Context.BATCH_HOST)
        plain["device_driven"] = {"value": nplain / (t_ms * 1e-3),
                                  "calls_in_graph_mode": graph_calls}
        # ---- gradient pass vs forward pass on the same batch
        th = np.arccos(np.linspace(-1, 1, 32))
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from costuum_b200.CosTuuM import RandomOrientationDistribution
        co = RandomOrientationDistribution(2 * SCHEDULE["max_order"]).coefficients
        fwd, bwd = [], []
        # one untimed pass (buffers and table caches of the observable and
        # gradient paths), then the best of three; each gradient follows its
        # forward batch, whose block rounds keep their LU factors
        ctx.tmatrix_batch(r, lam, m, d, **SCHEDULE)
        ctx.observables(th, co)
        ctx.gradients(th, co)
        for _ in range(3):
            flush_l2(flush)
            torch.cuda.synchronize()
            lib.tmx_timer_start(h)
            ctx.tmatrix_batch(r, lam, m, d, **SCHEDULE)
            ctx.observables(th, co)
            ms = ev()
            lib.tmx_timer_stop(h, P(ms))
            fwd.append(float(ms[0]))
            flush_l2(flush)
            torch.cuda.synchronize()
            lib.tmx_timer_start(h)
            ctx.gradients(th, co)
            ms = ev()
            lib.tmx_timer_stop(h, P(ms))
            bwd.append(float(ms[0]))
        grad = {"forward_ms": min(fwd), "gradient_ms": min(bwd),
                "ratio": min(bwd) / min(fwd),
                "what": "forward = convergence loop + blocks + orientation-"
                        "averaged Qext/Qpol at 32 angles; gradient (after the "
                        "forward) = tangents for (Re m, Im m, r_ev, d) on the "
                        "LU factors the forward's block rounds kept + their "
                        "observables"}
        # the same through torch.autograd (costuum_b200.autograd.extinction):
        # forward, then backward of a weighted sum of the coefficients
        from costuum_b200 import autograd as AG
        params = np.stack([m.real, m.imag, r, d], axis=1)
        wts = torch.tensor(np.random.default_rng(7).standard_normal((N_GRAINS, len(th), 3)))
        tf, tb = [], []
        for it in range(4):  # the first pass is untimed
            pt = torch.tensor(params, dtype=torch.float64, requires_grad=True)
            flush_l2(flush)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            qt = AG.extinction(pt, 1e-6, th, co, **SCHEDULE)
            t1 = time.perf_counter()
            (qt * wts).sum().backward()
            t2 = time.perf_counter()
            if it:
                tf.append(t1 - t0)
                tb.append(t2 - t1)
        grad["torch_autograd"] = {
            "forward_ms": 1e3 * min(tf), "backward_ms": 1e3 * min(tb),
            "ratio": min(tb) / min(tf),
            "what": "Extinction.apply (convergence loop + blocks + averaged "
                    "Qext at 32 angles) and .backward() of a weighted sum, "
                    "host wall time; backward runs the tangent kernels on the "
                    "forward's kept LU factors"}

    # ---- plain-path workload: 256 grains, x in [10, 30], d log-uniform in
    # [0.33, 3], calculator schedule, random-orientation average, Z at 181
    # scattering angles (0..180 deg) for incidence along the axis
    c5 = None
    if rank == 0 and world == 1 and not args.skip_extras:
        from costuum_b200.CosTuuM import RandomOrientationDistribution
        rng = np.random.default_rng(55)
        n5 = 256
        x5 = rng.uniform(10.0, 30.0, n5)
        d5 = np.exp(rng.uniform(np.log(0.33), np.log(3.0), n5))
        m5 = rng.uniform(1.3, 2.0, n5) + 1j * np.exp(rng.uniform(np.log(1e-3), 0.0, n5))
        lam5 = 1e-6
        r5 = x5 * lam5 / (2 * np.pi)
        tout = np.radians(np.arange(181.0))
        times = []
        for _ in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res5 = ctx.tmatrix_batch_calculator(r5, lam5, m5, d5)
            t1 = time.perf_counter()
            nm5 = res5.nmax.copy()
            co = RandomOrientationDistribution(2 * int(nm5.max())).coefficients
            ctx.orientation_average(co, np.where(nm5 > 0, 0, -1).astype(np.int32))
            g = np.repeat(np.arange(n5), 181)
            Z5 = ctx.scattering_matrix(g, 0.0, 0.0, np.tile(tout, n5), 0.0)
            t2 = time.perf_counter()
            times.append((t1 - t0, t2 - t0))
        tm, tz = min(t[0] for t in times), min(t[1] for t in times)
        # forward Q_ext and its adjoint (derivatives in Re m, Im m, r_ev, d) at
        # 32 zenith angles for random orientation, on the same grains
        th32 = np.arccos(np.linspace(-1, 1, 32))
        co5 = RandomOrientationDistribution(2 * int(nm5.max())).coefficients
        fa = []
        for _ in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ctx.tmatrix_batch_calculator(r5, lam5, m5, d5)
            ctx.observables(th32, co5)
            t1 = time.perf_counter()
            _, dq5 = ctx.gradients(th32, co5)
            t2 = time.perf_counter()
            fa.append((t1 - t0, t2 - t1))
        tf5, ta5 = min(t[0] for t in fa), min(t[1] for t in fa)
        c5 = {"what": "256 grains x~U[10,30], d log-U[0.33,3], calculator "
                      "schedule (maximum_order 200, ngauss loop to 500), "
                      "random-orientation average, Z at 181 angles; host wall "
                      "time through the public API",
              "tmatrices_per_s": n5 / tm,
              "with_orientation_and_z_per_s": n5 / tz,
              "nmax_max": int(nm5.max()), "nmax_mean": float(nm5[nm5 > 0].mean()),
              "converged": int((res5.status == 0).sum()),
              "status_nonzero": int((res5.status != 0).sum()),
              "status_note": "grains the reference's calculator cannot converge "
                             "either (it aborts); flagged, not aborted",
              "z_finite": bool(np.isfinite(Z5).all()),
              "forward_q_ms": tf5 * 1e3,
              "adjoint_ms": ta5 * 1e3,
              "adjoint_over_forward": ta5 / tf5,
              "adjoint_what": "forward = calculator schedule + Q_ext/Q_abs at 32 "
                              "angles (random orientation); adjoint = their "
                              "derivatives in (Re m, Im m, r_ev, d) with the kept "
                              "LU factors",
              "adjoint_finite": bool(np.isfinite(dq5[res5.status == 0]).all())}

    avg = None
    if rank == 0 and world == 1 and not args.skip_extras:
        avg = averaging_leg(ctx, lib, dmma)

    # Roofline of the dominant kernel. The block launches of a live step
    # overlap on several streams, so their event times are not kernel
    # durations; the tuning pass above times each size bucket's launch alone
    # (all of the bucket's items of the 4096 grains at their converged
    # orders, one launch, CUDA events, serialised). The dominant kernel is
    # the bucket launch with the longest time under the tuned table;
    # achieved = its executed-flop model (bucket_flops) / that time. The step
    # figure (model flops of the whole step over the step time) is beside it.
    # DRAM bytes per item of the dominant kernel from one ncu capture of that
    # launch on a 1024-grain case (profiles/k_blocks_warp_dmma_fixed_1024.md),
    # scaled by its item count (traffic grows with the items: every item
    # reads its own table rows and writes its own T block).
    DMMA_BYTES_PER_ITEM = 10.29e3
    bk_s = bk_ms[0] * 1e-3
    executed = bk_fl[0] / bk_s / 1e12 if bk_s > 0 else 0.0
    dominant, buckets_roof = None, []
    if autotune is not None:
        bfl, bcnt = bucket_flops(conv.nmax, conv.ngauss)
        for b in range(5):
            fam = table[b]
            ms = float(tune_ms[b][fam])
            if bcnt[b] == 0 or ms <= 0:
                continue
            row = {"bucket": BUCKETS[b], "family": Context.FAMILIES[fam],
                   "items": int(bcnt[b]), "ms": ms, "gflop": bfl[b] / 1e9,
                   "tflops": bfl[b] / (ms * 1e-3) / 1e12}
            buckets_roof.append(row)
            if dominant is None or ms > dominant["ms"]:
                dominant = row
    out = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.skip_cpu:
            cpu = cpu_baseline_block(os.cpu_count() or 1)
        out = {
            "metric": "T-matrices/s (converged, batched)",
            "value": value, "unit": "T-matrices/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": workload_config(),
            "batch": {"nmax_mean": float(nmax[nmax > 0].mean()),
                      "nmax_max": int(nmax.max()),
                      "status_nonzero": int((status != 0).sum())},
            "e2e": {"value": world * N_GRAINS / (pipe_max * 1e-3),
                    "unit": "T-matrices/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "ms_per_step": pipe_max,
                    "what": "tmatrix_batch from host arrays + every converged "
                            "T-matrix in host memory (tmatrices()) + per-grain "
                            "results; %d contexts on as many host threads in the "
                            "device-driven mode, so that one batch's download "
                            "overlaps the others' compute (%d steps each, wall "
                            "time)" % (E2E_CONTEXTS, pipe_steps),
                    "mode_ok": bool(pipe_mode_ok),
                    "sequential": {
                        "value": world * N_GRAINS / (e2e_max * 1e-3),
                        "ms_per_step": e2e_max,
                        "what": "the same calls one batch at a time on one "
                                "context in the host-driven mode, T-matrices "
                                "streamed by the block rounds (L2 flushed "
                                "before each step)"}},
            "roofline": {"bound": "tensor",
                         "kernel": ("k_blocks_warp %s, classes %s: assembly + LU "
                                    "+ solve" % (dominant["family"], dominant["bucket"])
                                    if dominant else "block kernels"),
                         "achieved": dominant["tflops"] if dominant else None,
                         "peak": dmma, "unit": "TFLOP/s",
                         "frac": dominant["tflops"] / dmma if dominant else None,
                         "peak_kind": "measured FP64 DMMA (mma.sync m8n8k4 f64) this run "
                                      "(of measured); DFMA peak %.1f" % dfma,
                         "launch_ms": dominant["ms"] if dominant else None,
                         "what": "one launch of the bucket's items of the 4096 grains "
                                 "at their converged orders, timed alone with CUDA "
                                 "events (tuning pass); executed-flop model",
                         "buckets": buckets_roof,
                         "traffic": (DMMA_BYTES_PER_ITEM * dominant["items"]
                                     if dominant and dominant["family"] == "warp_dmma"
                                     else None),
                         "traffic_unit": "DRAM bytes per launch (ncu per-item figure "
                                         "of a 1024-grain capture x items)",
                         "flops_model_step": "per-grain model: chain orders "
                                             "F_asm(k,2k,4)+F_lu(2k)+F_solve(2k), m "
                                             "blocks F_asm(N+1-m,2N,10)+F_lu+F_solve",
                         "flops_per_step": flops_survey,
                         "step_tflops": flops_survey / (ms_step * 1e-3) / 1e12,
                         "step_frac": flops_survey / (ms_step * 1e-3) / 1e12 / dmma},
            "batch_mode": {
                "timed": MODE_NAMES[chosen], "ran_as_timed": bool(chosen_ok),
                "untimed_median_ms": {MODE_NAMES[k]: v for k, v in mode_ms.items()},
                "other": {"mode": MODE_NAMES[other],
                          "ms_per_step": float(np.median(other_ms)),
                          "value": world * N_GRAINS / (float(np.median(other_ms)) * 1e-3),
                          "ran_as_asked": bool(other_ok)},
                "what": "host: the order loop driven by the host thread one group "
                        "of orders ahead, block rounds formed on the host; graph: "
                        "one CUDA graph of conditional nodes, every decision on "
                        "the device, one host synchronisation per batch. The "
                        "timed steps use the mode that was faster on 3 untimed "
                        "steps; the other is timed after them the same way"},
            "profiled_pass": {
                "ms_per_step": prof_total / args.steps,
                "block_launches": int(bk_n.value),
                "block_event_ms_per_step": bk_ms[0] / args.steps,
                "executed_tflops_over_event_time": executed,
                "what": "the same steps again with CUDA events around every "
                        "block and table launch (untimed); block launches "
                        "overlap, so their summed event time exceeds the step"},
            "phases_ms_per_step": {"tables": tb_ms[0] / args.steps},
            # host side of the timed steps (medians): the batch call's wall
            # time, the time it blocked on the order loop's events and the
            # final synchronisation, and its host set-up of block rounds
            "timeline_ms_per_step": {
                "order_loop": float(np.median(loop_ms)) if loop_ms else None,
                "first_to_last_launch": float(np.median(gpu_ms)) if gpu_ms else None},
            "host_ms_per_step": {
                "wall": float(np.median([x[0] for x in host_t])),
                "blocked": float(np.median([x[1] for x in host_t])),
                "round_setup": float(np.median([x[2] for x in host_t])),
                "order_groups": float(np.median([x[3] for x in host_t]))},
            "gpu_launches": int(launches),
            "autotune": autotune,
            "plain_gpu": plain,
            "batched_vs_plain": (value / plain["value"]) if plain else None,
            "gradient": grad,
            "plain_path_config5": c5,
            "averaging": avg,
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        print(json.dumps(out))
    ctx.close()
    dist.close()
    return 0


def hbm_peak():
    """Measured HBM copy bandwidth of this pool's B200s (GB/s) and its
    source: MEASURED_PEAKS.json beside this file, else the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            v = json.load(f).get("hbm_gbs")
        if v:
            return float(v), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, ValueError):
        pass
    return 6650.0, "fallback (no MEASURED_PEAKS.json)"


def averaging_leg(ctx, lib, fp64_peak):
    """The averaging kernels on a sub-grid of the averaged-coefficients
    workload: 16 of the 64 radii (0.01-2 um) x every 8th wavelength of
    logspace(0.1, 100 um, 200) with x <= 50 x the 20-node Draine-Hensley
    shape distribution, Davis-Greenstein alignment above 0.1 um, Qabs and
    Qext at 32 zenith angles, through get_table. Per kernel: device time
    (CUDA events), algorithmic bytes and flops over that time, against the
    measured HBM and FP64 peaks."""
    from costuum_b200 import CosTuuM as C
    P = ctypes.c_double
    sizes = np.logspace(np.log10(0.01e-6), np.log10(2e-6), 64)[::4]
    lams = np.logspace(-7, -4, 200)
    lams = lams[2 * np.pi * sizes[-1] / lams <= 50.0][::8]
    th = np.arccos(np.linspace(-1, 1, 32))

    def run():
        return C.get_table(
            types=np.array([0]), sizes=sizes, wavelengths=lams, thetas=th,
            shape_distribution=C.DraineHensleyShapeDistribution(20),
            alignment_distribution=C.SizeBasedAlignmentDistribution(
                1e-7, C.DAVIS_GREENSTEIN_ALIGNMENT, maximum_order=100),
            dust_properties=C.CustomDustProperties(lambda w, s, t: dielectric_m(w)),
            maximum_order=100, do_absorption=True, do_extinction=True,
            context=ctx)

    run()  # tables, plans and buffers of this grid
    h = ctx._h
    lib.tmx_profile_enable(h, 1)
    t0 = time.perf_counter()
    out = run()
    wall = time.perf_counter() - t0
    peak_gbs, peak_src = hbm_peak()
    kernels = {}
    for k, name in ((2, "k_orient_pairs"), (3, "k_amp"), (4, "k_shape_avg")):
        ms = np.zeros(1)
        n = ctypes.c_int64()
        fl = np.zeros(1)
        by = P()
        lib.tmx_profile_read(h, k, _ptr(ms), ctypes.byref(n), _ptr(fl))
        lib.tmx_profile_bytes(h, k, ctypes.byref(by))
        s = max(ms[0] * 1e-3, 1e-12)
        kernels[name] = {"ms": ms[0], "launches": n.value,
                         "bytes": by.value, "gbs": by.value / s / 1e9,
                         "hbm_frac": by.value / s / 1e9 / peak_gbs,
                         "flops": fl[0], "tflops": fl[0] / s / 1e12,
                         "fp64_frac": fl[0] / s / 1e12 / fp64_peak}
    lib.tmx_profile_enable(h, 0)
    return {"what": "averaging kernels on a 16-radius x %d-wavelength x 20-shape "
                    "sub-grid of the averaged-coefficients workload (%d grains; "
                    "Draine-Hensley shapes, Davis-Greenstein alignment above "
                    "0.1 um, Qabs and Qext at 32 angles)"
                    % (len(lams), len(sizes) * len(lams) * 20),
            "grains": len(sizes) * len(lams) * 20, "get_table_s": wall,
            "hbm_peak_gbs": peak_gbs, "hbm_peak": peak_src,
            "fp64_peak_tflops": fp64_peak,
            "bytes_model": "orientation average: T in + averaged T out; "
                           "amplitudes: averaged T in + 4 complex per job and "
                           "azimuth out; shape average: 8 (n_shape + 1) n_theta "
                           "n_coef per (size, wavelength) + weights",
            "kernels": kernels, "finite": bool(np.isfinite(out).all())}


def _ptr(a):
    from costuum_b200 import _lib
    return _lib.ptr(a)


def _lib_load():
    from costuum_b200 import _lib
    return _lib.load()


def dielectric_m(lam):
    """Seeded-style refractive index model of the averaged-grid workload:
    eps = eps_inf + sum_j f_j w_j^2 / (w_j^2 - w^2 - i g_j w) - wp^2 / (w^2 +
    i gD w) with resonances at 9.7, 18 and 25 um (w = 1 / lambda[um]),
    m = sqrt(eps) on the branch with Im m >= 0."""
    w = 1.0 / (lam * 1e6)
    eps = 2.5 + 0j
    for lj, f in ((9.7, 0.8), (18.0, 0.4), (25.0, 0.2)):
        wj = 1.0 / lj
        eps += f * wj * wj / (wj * wj - w * w - 1j * 0.1 * wj * w)
    eps -= 0.05 ** 2 / (w * w + 1j * 0.01 * w)
    m = np.sqrt(eps)
    return complex(m if m.imag >= 0 else -m)


def run_config3(args):
    """The averaged-grid workload: 64 radii (0.01-2 um) x wavelengths
    logspace(0.1, 100 um, 200) with x = 2 pi r / lambda <= 50 at the largest
    radius (the 27 shortest wavelengths dropped, maximum_order 100) x the
    20-node Draine-Hensley shape distribution, Davis-Greenstein alignment
    above 0.1 um, Qabs and Qext at 32 zenith angles, through get_table. CPU:
    the reference module's get_table on a 2 x 2-cell sub-grid of small size
    parameters (cells with larger ones take the reference minutes each)."""
    from costuum_b200 import CosTuuM as C
    sizes = np.logspace(np.log10(0.01e-6), np.log10(2e-6), 64)
    lams = np.logspace(-7, -4, 200)
    lams = lams[2 * np.pi * sizes[-1] / lams <= 50.0]
    th = np.arccos(np.linspace(-1, 1, 32))
    kw = dict(thetas=th, do_absorption=True, do_extinction=True)

    def run(mod, sz, lm, nthreads):
        return mod.get_table(
            types=np.array([0]), sizes=sz, wavelengths=lm,
            shape_distribution=mod.DraineHensleyShapeDistribution(20),
            alignment_distribution=mod.SizeBasedAlignmentDistribution(
                1e-7, mod.DAVIS_GREENSTEIN_ALIGNMENT, maximum_order=100),
            dust_properties=mod.CustomDustProperties(
                lambda w, s, t: dielectric_m(w)),
            maximum_order=100, number_of_threads=nthreads, **kw)

    run(C, sizes[:4], lams[:4], 1)  # warm-up (tables, contexts)
    t0 = time.perf_counter()
    out = run(C, sizes, lams, 1)
    gpu_s = time.perf_counter() - t0
    ncell = len(sizes) * len(lams)
    line = {"metric": "grains/s (averaged get_table grid)",
            "value": ncell * 20 / gpu_s, "unit": "grains/s",
            "cells": ncell, "grains": ncell * 20, "seconds": gpu_s,
            "finite": bool(np.isfinite(out).all())}
    if not args.skip_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        R = O.ref_module()
        sub_s = sizes[[10, 30]]
        sub_l = lams[[100, 150]]
        t0 = time.perf_counter()
        run(R, sub_s, sub_l, os.cpu_count() or 1)
        cpu_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        run(C, sub_s, sub_l, 1)
        gpu_sub = time.perf_counter() - t0
        line["cpu_reference"] = {"value": 4 * 20 / cpu_s, "unit": "grains/s",
                                 "cores": os.cpu_count(),
                                 "sample": "2 sizes x 2 wavelengths x 20 shapes "
                                           "(small-x cells) of the same grid, "
                                           "reference get_table",
                                 "gpu_same_sample": 4 * 20 / gpu_sub}
    print(json.dumps(line))
    return 0


def main():
    global N_GRAINS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--skip-cpu", action="store_true",
                    help="omit the CPU-baseline leg")
    ap.add_argument("--skip-extras", action="store_true",
                    help="omit the plain-path and gradient measurements")
    ap.add_argument("--grains", type=int, default=N_GRAINS,
                    help="grains per GPU (smaller cases for profiling)")
    ap.add_argument("--config3", action="store_true",
                    help="measure the averaged get_table grid instead")
    ap.add_argument("--averaging", action="store_true",
                    help="only the averaging kernels' sub-grid leg (for profiling)")
    ap.add_argument("--skip-tune", action="store_true",
                    help="keep the default dispatch table (for profiling)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    N_GRAINS = args.grains
    if args.config3:
        return run_config3(args)
    if args.averaging:
        from costuum_b200.tmatrix import Context
        ctx = Context(0)
        print(json.dumps(averaging_leg(ctx, _lib_load(), ctx.probe_fp64(1))))
        ctx.close()
        return 0
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
