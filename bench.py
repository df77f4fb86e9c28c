"""Benchmark: SOCS-24 aerial images/s at 1024x1024 (configuration 3), one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

A step is one batch of 64 binary Manhattan clips (1024x1024, 2 nm/pixel) imaged with the 24 SOCS kernels of
the vector TCC of an annular 0.7/0.95 source (PntNum 41).  Kernels are built once per optics key (TCC + FP64
eigendecomposition, reported as `setup_s`) and stay resident, as they do in serving.

  value  images/s with the masks already in HBM (256 MB of float32 masks per step: larger than L2)
  e2e    images/s through the public host-buffer API (SocsKernels.image_host) from pinned host uint8 masks to
         pinned host float32 images,
         host<->device copies inside the timed region
  serving  the same clips as requests through the continuous-batching server, against the plain FP32 path
         (one request at a time), with p50/p99 latency
  forms  the precision study: images/s and max / RMS error vs the FP64 oracle of the FP32 FFT form, the FP32
         DFT form and the split-BF16x3 tensor-core form
--form picks the form of the timed path (default bf16x3, the split-precision form).
The path shards by clip with no exchange, so N GPUs run N independent replicas ("scaling": "weak").
--impl reference times the reference's SOCS algorithm (full-grid FFTs, complex64) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "aerial images/s + p99 ms (1024², SOCS-24), served vs plain, err≤1e-4 vs FP64"
UNIT = "images/s"
N_PIX, PERIOD, ORDER = 1024, 2048.0, 24
BATCH = 64
WORKLOAD = ("config 3: SOCS-24 from the vector TCC of an annular 0.7/0.95 source (PntNum 41, 2048 nm period, "
            "immersion-mapped optics), batches of 64 binary Manhattan clips 1024x1024 at 2 nm/pixel (~35% fill)")


def peaks():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as fh:
            p = json.load(fh)
        return float(p['hbm_gbs']), float(p['bf16_tflops']), 'measured'
    except (OSError, KeyError, ValueError):
        return 6650.0, 1590.0, 'fallback'


class ClockSampler:
    """nvidia-smi clock/throttle samples (200 ms) while the timed region runs."""
    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index, self.proc, self.lines = index, None, []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', f'--id={self.index}', f'--query-gpu={self.FIELDS}',
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_samples(self, n, timeout=3.0):
        """Block until at least n samples have arrived (or the timeout passes)."""
        t0 = time.perf_counter()
        while self.proc is not None and len(self.lines) < n and time.perf_counter() - t0 < timeout:
            time.sleep(0.02)

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ('hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap')
        for ln in self.lines:
            f = [x.strip() for x in ln.split(',')]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == 'active':
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        torch.distributed.init_process_group('nccl', timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device('cuda', local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return world, rank, local


def barrier(world):
    if world > 1:
        torch.distributed.barrier()


def max_over_ranks(x, world):
    """The largest x over the ranks (NCCL reduces a device tensor, gloo a host one)."""
    if world == 1:
        return x
    dev = 'cuda' if torch.distributed.get_backend() == 'nccl' else 'cpu'
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, ms, world):
    """Whole-job throughput of `world` replicas that each processed `units_per_rank` units, `ms` being this
    rank's device time: every rank's units over the slowest rank's time.  Returns (units per second, max ms)."""
    m = max_over_ranks(ms, world)
    return world * units_per_rank / (m / 1000.0), m


def build_kernels():
    from opticalimaging_b200 import imaging, workloads as W
    sr, po, nm = W.config3_optics(order=ORDER)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    T, fg = imaging.CalculateTCCMatrix(sr, [PERIOD, PERIOD], po, 0.0, nm)
    sk = imaging.socs_kernels_from_tcc(T, fg, [N_PIX, N_PIX], nm)
    torch.cuda.synchronize()
    return sk, time.perf_counter() - t0, (sr, po, nm, T, fg)


def stage_times(sk, masks, out, form, reps=5):
    """Average device time of each native stage over `reps` batches (CUDA events on the launching stream).

    The output buffer is reused and the first batch is not counted, so no allocation sits between events."""
    acc = {}
    sk.image(masks, out=out, form=form)
    for _ in range(reps):
        marks = []
        sk.image(masks, out=out, marks=marks, form=form)
        torch.cuda.synchronize()
        for (_, a), (name, b) in zip(marks[:-1], marks[1:]):
            acc[name] = acc.get(name, 0.0) + a.elapsed_time(b) / reps
    return acc


def wait_until(t):
    """Wait for perf_counter() to reach t without holding the GIL (the server's scheduler thread shares it):
    sleeps while more than 0.2 ms remain, then yields with sleep(0)."""
    while True:
        d = t - time.perf_counter()
        if d <= 0:
            return
        time.sleep(d - 1e-4 if d > 2e-4 else 0)


def poisson_run(srv, stream, rate, seed, submit):
    """Open-loop arrivals: request i of `stream` is submitted at the i-th arrival of a Poisson process of
    `rate` per second (the schedule runs from the start time, so late submissions do not lower the rate).
    Returns (requests per second achieved, latency statistics)."""
    import random
    srv.completed.clear()
    rng = random.Random(seed)
    futs = []
    t_next = t0 = time.perf_counter()
    for item in stream:
        t_next += rng.expovariate(rate)
        wait_until(t_next)
        futs.append(submit(item))
    for f in futs:
        f.result()
    return len(stream) / (time.perf_counter() - t0), srv.latency_ms()


def serve_measure(sk, info, masks_np, dev, args, latency_budget_ms=None):
    """Served throughput and latency of config-3 requests, against the plain path on the same requests.

    The client keeps a ring of pinned result buffers and passes one with each request (the server copies the
    image into it).  Saturated: a closed loop keeping `window` requests outstanding (throughput).  Poisson:
    open-loop arrivals at 70 % of the saturated rate (latency under load), result buffers recycled as each
    request completes.  Plain: one request at a time.  `latency_budget_ms` turns on the server's latency-aware
    batch cap (both the saturated and the Poisson measurements run under it)."""
    import collections
    from opticalimaging_b200 import serve
    spec = serve.ModelSpec(('socs24', N_PIX, PERIOD, args.form), N_PIX, N_PIX, 1,
                           build=lambda: serve_model_from(sk, args.form))
    plain_spec = serve.ModelSpec(('socs24', N_PIX, PERIOD, 'fft'), N_PIX, N_PIX, 1,
                                 build=lambda: serve_model_from(sk, 'fft'))
    # masks and result buffers as views of one pinned slab each: consecutive requests' buffers are adjacent, so
    # the executor moves a batch's runs with one copy each
    pinned = list(torch.from_numpy(np.stack([m.astype(np.uint8) for m in masks_np])).pin_memory())
    nreq = max(4 * BATCH, args.serve_requests)
    window = 4 * BATCH
    ring = list(torch.empty((nreq, 1, N_PIX, N_PIX), dtype=torch.float32).pin_memory())
    ex = serve.CudaExecutor(device=dev, nslots=3)
    srv = serve.Server(ex, hbm_budget=150e9, max_batch=BATCH, latency_budget_ms=latency_budget_ms)
    ex.prepare(spec, torch.uint8, srv.batch_ceiling(spec))   # every bucket's graph before any timing

    def closed_loop(n):
        q = collections.deque()
        for i in range(n):
            if len(q) >= window:
                q.popleft().result()
            q.append(srv.submit(spec, pinned[i % len(pinned)], out=ring[i % window]))
        while q:
            q.popleft().result()

    closed_loop(2 * window)                                       # warm-up: model, buffers, graphs
    srv.completed.clear()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    closed_loop(nreq)
    dt = time.perf_counter() - t0
    sat = srv.latency_ms()
    served = nreq / dt
    rate = 0.7 * served
    free = collections.deque(ring)
    lock = threading.Lock()

    def submit(i):
        with lock:
            buf = free.popleft() if free else None
        if buf is None:
            buf = torch.empty((1, N_PIX, N_PIX), dtype=torch.float32).pin_memory()
        f = srv.submit(spec, pinned[i % len(pinned)], out=buf)

        def recycle(_f, buf=buf):
            with lock:
                free.append(buf)
        f.add_done_callback(recycle)
        return f

    batches0 = srv.batches
    npois = max(nreq, args.poisson_requests)
    _, poisson = poisson_run(srv, range(npois), rate, 5, submit)
    batches = srv.batches - batches0
    srv.close()
    nplain = min(32, nreq)
    serve.plain_run([(plain_spec, pinned[0])], device=dev)       # build the plain model outside the timing
    _, tp = serve.plain_run([(plain_spec, pinned[i % len(pinned)]) for i in range(nplain)], device=dev)
    plain = nplain / tp
    return {"images_per_s": served, "p50_ms": poisson.get("p50_ms"), "p99_ms": poisson.get("p99_ms"),
            "latency_at": f"Poisson arrivals at {rate:.0f} requests/s (70 % of the saturated rate)",
            "latency_budget_ms": latency_budget_ms, "batch_limit": srv.batch_limit(spec),
            "saturated_p50_ms": sat.get("p50_ms"), "saturated_p99_ms": sat.get("p99_ms"),
            "requests": nreq, "poisson_requests": npois, "window": window, "poisson_batches": batches,
            "form": args.form, "plain_images_per_s": plain,
            "served_over_plain": served / plain,
            "plain": "one request at a time: H2D, image (batch 1, FP32 FFT form, no graph), D2H, synchronise",
            "h2d_bytes_per_image": N_PIX * N_PIX, "d2h_bytes_per_image": 4 * N_PIX * N_PIX}


def serve_mix(dev, args, state):
    """Configuration 5: a Poisson stream of mixed requests (clip sizes 256..2048, SOCS-24 / vector Abbe /
    three-plane SOCS) through the server with a 150 GB HBM budget, against the plain FP32 path on a sample of the
    same requests, with the served form's error against the FP32 form (every model) and the FP64 oracle."""
    import collections
    from opticalimaging_b200 import serve, workloads as W
    from tests.fixtures import rel_err
    t_setup = time.perf_counter()
    specs = W.config5_specs('bf16x3')
    plain_specs = W.config5_specs(None)
    stream = W.config5_stream(args.mix_requests)
    pool = {n: [torch.from_numpy(m.astype(np.uint8)).pin_memory()
                for m in W.manhattan_masks(4, n, 2.0 * n, seed=50 + n)] for n in W.CONFIG5_SIZES}
    ex = serve.CudaExecutor(device=dev, nslots=3, max_batch=BATCH)
    srv = serve.Server(ex, hbm_budget=150e9, max_batch=BATCH)

    # caller-provided pinned result buffers, recycled when their request completes (as a client that consumes
    # each image would): no pinned allocation per batch, bounded host memory
    free = collections.defaultdict(list)
    lock = threading.Lock()

    def submit(k, n, i):
        sp = specs[(k, n)]
        shape = (sp.planes, sp.ny, sp.nx)
        with lock:
            buf = free[shape].pop() if free[shape] else None
        if buf is None:
            buf = torch.empty(shape, dtype=torch.float32).pin_memory()
        f = srv.submit(sp, pool[n][i % len(pool[n])], out=buf)

        def recycle(_f, buf=buf, shape=shape):
            with lock:
                free[shape].append(buf)
        f.add_done_callback(recycle)
        return f

    # every model built and the graph of every batch bucket captured before any timing; then a short warm-up
    for sp in specs.values():
        ex.prepare(sp, torch.uint8, srv.batch_ceiling(sp))
    futs = [submit(k, n, i) for k, n, i in stream[:min(len(stream), 300)]]
    for f in futs:
        f.result()
    del futs
    setup_s = time.perf_counter() - t_setup
    # saturated throughput: a closed loop keeping 256 requests outstanding
    srv.completed.clear()
    q = collections.deque()
    t0 = time.perf_counter()
    for k, n, i in stream:
        if len(q) >= 256:
            q.popleft().result()
        q.append(submit(k, n, i))
    while q:
        q.popleft().result()
    sat_rate = len(stream) / (time.perf_counter() - t0)
    # Poisson arrivals at 70 % of the saturated rate: latency under load
    rate = 0.7 * sat_rate
    batches0 = srv.batches
    served_rate, lat = poisson_run(srv, stream, rate, 11, lambda item: submit(*item))
    batches = srv.batches - batches0
    resident = ex.resident_bytes()
    srv.close()
    # plain FP32 path, one request at a time, on a sample with the same mix (models built outside the timing)
    sample = stream[:min(len(stream), 60)]
    serve.plain_run([(plain_specs[(k, n)], pool[n][0]) for k, n in {(k, n) for k, n, _ in sample}], device=dev)
    _, tp = serve.plain_run([(plain_specs[(k, n)], pool[n][i % len(pool[n])]) for k, n, i in sample], device=dev)
    plain_rate = len(sample) / tp
    # accuracy of the served form: against the FP32 form on every model, against the FP64 oracle on two
    worst = 0.0
    for key, sp in specs.items():
        m = ex.models.get(sp.key) or sp.build()
        mask = pool[key[1]][0].to(dev).unsqueeze(0)
        a = m.image(mask).cpu().numpy()
        b = m.image(mask, form='fft' if m.plan.fft else 'dft').cpu().numpy()
        worst = max(worst, rel_err(a, b))
    state["specs"], state["ex"], state["pool"] = specs, ex, pool
    return {"requests": len(stream), "mix": "50 % SOCS-24, 30 % vector Abbe (quasar PntNum 31), 20 % SOCS-24 x 3 "
            "focus planes; clip sizes uniform over 256, 512, 1024, 2048 (2 nm/pixel); binary Manhattan masks "
            "(~35 % fill) as uint8; float32 images returned to the host",
            "images_per_s": served_rate, "saturated_images_per_s": sat_rate,
            "latency_at": f"Poisson arrivals at {rate:.0f} requests/s (70 % of the saturated rate)",
            "p50_ms": lat.get("p50_ms"), "p99_ms": lat.get("p99_ms"), "batches": batches,
            "plain_images_per_s": plain_rate, "served_over_plain": served_rate / plain_rate,
            "plain": f"{len(sample)} requests of the same stream one at a time, FP32 form, no batching or graphs",
            "hbm_budget_gb": 150, "resident_gb": resident / 1e9, "setup_s": setup_s,
            "max_err_vs_fp32_form": worst}


def mix_fp64_check(specs, ex, pool, dev):
    """Served-form images of the 256 x 256 SOCS-24 and Abbe models against the FP64 oracle (relative to peak)."""
    from oracle import optics64 as O
    from opticalimaging_b200 import imaging, workloads as W
    from opticalimaging_b200.params import Scatter
    from tests.fixtures import rel_err
    out = {}
    mask = pool[256][0].float().numpy()
    sc = Scatter()
    sc.Period_X = sc.Period_Y = 512.0
    sc.ScatterField = W.thin_field(mask)
    md = torch.from_numpy(mask).to(dev).unsqueeze(0)
    sr, po, nm = W.config3_optics(order=24)
    T, fg = imaging.CalculateTCCMatrix(sr, [512.0, 512.0], po, 0.0, nm)
    K = imaging.DecomposeTCC_SOCS(T, fg, [256, 256], nm).cpu().numpy().astype(np.complex128)
    m = ex.models.get(specs[('socs24', 256)].key) or specs[('socs24', 256)].build()
    out["socs24_256"] = rel_err(m.image(md)[0, 0].cpu().numpy(), O.socs(sc, K, sr, po))
    q = specs[('abbe', 256)]
    m = ex.models.get(q.key) or q.build()
    import math
    from opticalimaging_b200.params import Numerics, Projection, Source
    s2, p2, n2 = Source(), Projection(), Numerics()
    s2.Shape, s2.PntNum, s2.SigmaIn, s2.SigmaOut, s2.OpenAngle = 'quasar', 31, 0.5, 0.85, math.pi / 6
    s2.PolarizationVector = [1.0, 0.0]
    W.mapped_optics(p2, s2)
    n2.ImageCalculationMode = 'vector'
    p2.FocusRange = torch.tensor([0.0])
    out["abbe_256"] = rel_err(m.image(md)[0, 0].cpu().numpy(), O.abbe(s2, sc, p2, n2)[0])
    return out


def compact(x, digits=4):
    """Floats rounded to `digits` significant digits, recursively (keeps the one JSON line short)."""
    if isinstance(x, float):
        return float(f'{x:.{digits}g}')
    if isinstance(x, dict):
        return {k: compact(v, digits) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [compact(v, digits) for v in x]
    return x


def reference_torch_socs(h, kernels, npx, npy):
    """The reference's SOCS image as its own torch code, on whatever device its tensors live on: the spectrum of
    Scatter.CalculateSpectrum (Scatter.py:10-21) and CalculateAerialImage_SOCS.py:3-11 -- a full-grid ifft2 per
    channel, a full-grid fft2 per (kernel, channel), |.|^2 summed and fftshifted.  With CUDA tensors this is the
    reference run with torch's default device set to the GPU: the plain GPU path it would give a user."""
    hk = (npx * npy) * torch.fft.fftshift(torch.fft.ifft2(torch.fft.ifftshift(h, dim=(0, 1)), dim=(0, 1)),
                                          dim=(0, 1))
    sp = hk.unsqueeze(3).permute(0, 1, 3, 2)
    es = kernels.unsqueeze(3) * torch.fft.ifftshift(sp, dim=(0, 1))
    e = ((1.0 / npx) * (1.0 / npy)) * torch.fft.fft2(es, dim=(0, 1))
    return torch.fft.fftshift(torch.sum(torch.abs(e) ** 2, dim=(2, 3)), dim=(0, 1))


def plain_reference_cuda(sk_info, masks_np, dev, count=16):
    """The reference's torch code on the GPU, one request at a time: the host [N, N, 3] complex64 field copied
    in, the image computed by reference_torch_socs with the reference-layout kernels resident on the device,
    the image copied back.  Returns images/s over `count` clips (after one warm-up clip)."""
    from opticalimaging_b200 import imaging
    sr, po, nm, T, fg = sk_info
    kern = imaging.DecomposeTCC_SOCS(T, fg, [N_PIX, N_PIX], nm)            # [N, N, K] complex64 on the device
    npx = PERIOD / (sr.Wavelength / po.NA)
    fields = []
    for m in masks_np[:count + 1]:
        f = np.zeros((N_PIX, N_PIX, 3), np.complex64)
        f[:, :, 0] = m
        fields.append(torch.from_numpy(f))
    reference_torch_socs(fields[0].to(dev), kern, npx, npx).cpu()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for f in fields[1:]:
        reference_torch_socs(f.to(dev), kern, npx, npx).cpu()
    return count / (time.perf_counter() - t0)


def e2e_dropin(sk_info, masks_np, dev, count=16):
    """Images/s of the drop-in call as a reference user makes it: CalculateAerialImage_SOCS per clip with a host
    complex64 [N, N, 3] ScatterField and the reference-layout kernels DecomposeTCC_SOCS returned; the image comes
    back on the host.  Host-to-device bytes per clip: the 24 MiB field (the reference's format)."""
    from opticalimaging_b200 import imaging
    from opticalimaging_b200.params import Scatter
    sr, po, nm, T, fg = sk_info
    kern = imaging.DecomposeTCC_SOCS(T, fg, [N_PIX, N_PIX], nm)
    scs = []
    for m in masks_np[:count + 1]:
        f = np.zeros((N_PIX, N_PIX, 3), np.complex64)
        f[:, :, 0] = m
        sc = Scatter()
        sc.Period_X = sc.Period_Y = PERIOD
        sc.ScatterField = torch.from_numpy(f)
        scs.append(sc)
    imaging.CalculateAerialImage_SOCS(scs[0], kern, sr, po)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for sc in scs[1:]:
        img, _ = imaging.CalculateAerialImage_SOCS(sc, kern, sr, po)
    dt = time.perf_counter() - t0
    t1 = time.perf_counter()   # the field's copy alone (pageable host memory, as the caller holds it)
    for sc in scs[1:]:
        sc.ScatterField.to(dev)
    torch.cuda.synchronize(dev)
    h2d = (time.perf_counter() - t1) / count
    return {"images_per_s": count / dt, "h2d_ms_per_image": 1e3 * h2d, "h2d_bytes_per_image": N_PIX * N_PIX * 3 * 8,
            "d2h_bytes_per_image": N_PIX * N_PIX * 4,
            "call": "CalculateAerialImage_SOCS(scatter, kernels, source, projector) per clip, host complex64 "
                    "[1024, 1024, 3] ScatterField in, host float32 image out"}


def time_device(fn, steps):
    """Average device time (ms) of fn() over `steps` calls, CUDA events on the current stream, after two warm-up
    calls."""
    fn()
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / steps


def configs_measure(dev, steps=5):
    """Configurations 1, 2 and 4 at their own sizes: images/s through the resident models (masks in HBM) per form,
    error of one image against the FP64 oracle (max and RMS, relative to the FP64 peak; every plane for
    configuration 2), and the configuration-4 adjoint step (forward + resist loss + backward) in ms."""
    from oracle import optics64 as O
    from opticalimaging_b200 import imaging, workloads as W
    from opticalimaging_b200.autograd import aerial_image
    from opticalimaging_b200.params import Scatter
    out = {}

    def errs(got, ref):
        d = np.asarray(got, np.float64) - ref
        pk = float(np.max(np.abs(ref)))
        return float(np.max(np.abs(d)) / pk), float(np.sqrt(np.mean(d * d)) / pk)

    # configuration 1: scalar Abbe 256^2, annular 0.6/0.9 PntNum 21, 12 rectangles; batches of 64 masks
    sr, sc, po, nm = W.config1()
    model = imaging.abbe_model(sr, po, nm, 1024.0, 1024.0, 256, 256)
    masks = np.stack([W.rect_mask(256, 256, 1024, 1024, 12, 40.0, 300.0, np.random.default_rng(100 + i))
                      for i in range(64)])
    md = torch.from_numpy(masks).to(dev)
    sc.ScatterField = W.thin_field(masks[0])
    ref = O.abbe(sr, sc, po, nm)[0]
    c1 = {"fields": model.count, "band": [model.band.br, model.band.bc], "batch": 64,
          "packed_fields": None if model.packed is None else model.packed[0].shape[1]}
    for form in ('fft', 'bf16x3'):
        o = torch.empty((64, 1, 256, 256), device=dev)
        ms = time_device(lambda: model.image(md, out=o, form=form), steps)
        mx, rms = errs(o[0, 0].cpu().numpy(), ref)
        c1[form] = {"images_per_s": 64 / (ms / 1e3), "max": mx, "rms": rms}
    out["config1"] = c1
    # configuration 2: vector Abbe 512^2, quasar PntNum 31, 5 planes, Zernike; batches of 16 line/space clips
    sr, sc, po, nm = W.config2()
    model = imaging.abbe_model(sr, po, nm, 2048.0, 2048.0, 512, 512)
    masks = np.stack([W.line_space_mask(512, 2048, np.random.default_rng(2 if i == 0 else 200 + i))
                      for i in range(16)])
    md = torch.from_numpy(masks).to(dev)
    ref = O.abbe(sr, sc, po, nm)                   # clip 0 is the configuration's own (seed 2)
    c2 = {"fields": model.count, "planes": model.planes, "band": [model.band.br, model.band.bc], "batch": 16,
          "packed_fields": None if model.packed is None else model.packed[0].shape[1]}
    for form in ('fft', 'bf16x3'):
        o = torch.empty((16, 5, 512, 512), device=dev)
        ms = time_device(lambda: model.image(md, out=o, form=form), steps)
        got = o[0].cpu().numpy()
        per = [errs(got[z], ref[z]) for z in range(5)]
        c2[form] = {"images_per_s": 16 / (ms / 1e3), "max_per_plane": [p[0] for p in per],
                    "rms_per_plane": [p[1] for p in per]}
    out["config2"] = c2
    # configuration 4: the adjoint step at 1024^2 with the engine's SOCS-16 kernels
    sr, po, nm, logits, target = W.config4()
    T, fg = imaging.CalculateTCCMatrix(sr, [2048.0, 2048.0], po, 0.0, nm)
    sk = imaging.socs_kernels_from_tcc(T, fg, [1024, 1024], nm)
    lt = torch.from_numpy(logits).to(dev)
    tg = torch.from_numpy(target).to(dev)
    box = {}

    def step(batch=1):
        x = lt.expand(batch, -1, -1).clone().requires_grad_(True)
        I = aerial_image(sk, torch.sigmoid(x))
        loss = torch.sum((torch.sigmoid(50.0 * (I - 0.25)) - tg) ** 2)
        loss.backward()
        box['grad'], box['I'], box['loss'] = x.grad, I, loss
    ms1 = time_device(lambda: step(1), steps)
    g1 = box['grad'][0].cpu().numpy()
    ms8 = time_device(lambda: step(8), steps)
    K = imaging.DecomposeTCC_SOCS(T, fg, [1024, 1024], nm).cpu().numpy().astype(np.complex128)
    I64, L64, G64 = O.socs_resist(logits, target, K, 50.0, 0.25)
    mx, rms = errs(g1, G64)
    out["config4"] = {"kernels": sk.count, "adjoint_ms_per_step": ms1, "adjoint_ms_per_step_batch8": ms8,
                      "adjoint_clips_per_s_batch8": 8 / (ms8 / 1e3), "grad_max_vs_fp64": mx, "grad_rms_vs_fp64": rms,
                      "step": "forward (recomputed in the backward), sigmoid resist loss, backward through the "
                              "adjoint kernel; 1024^2 continuous mask"}
    return out


def serve_model_from(sk, form):
    from opticalimaging_b200.engine import CoherentModel
    return CoherentModel(sk.pupils, sk.weights, sk.band, sk.ny, sk.nx, form=form)


def cpu_reference_sample(sk_info, masks_np, budget_s, threads):
    """Time the reference's algorithm (oracle/cpu_reference.py) on host cores for a bounded sample of clips."""
    from oracle import cpu_reference as R
    from opticalimaging_b200 import imaging
    sr, po, nm, T, fg = sk_info
    kern = imaging.DecomposeTCC_SOCS(T, fg, [N_PIX, N_PIX], nm).cpu().numpy()
    npx = PERIOD / (sr.Wavelength / po.NA)
    times, n = [], 0
    t_start = time.perf_counter()
    while n < len(masks_np) and (time.perf_counter() - t_start) < budget_s:
        field = np.zeros((N_PIX, N_PIX, 3), np.complex64)
        field[:, :, 0] = masks_np[n]
        t0 = time.perf_counter()
        R.socs_clip(field, kern, npx, npx, threads)
        times.append(time.perf_counter() - t0)
        n += 1
    med = statistics.median(times[1:] if len(times) > 2 else times)
    return 1.0 / med, n


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the three largest kernels at this
# workload, measured by ncu on a B200 for the kernels as they are built now; a constant, re-measured whenever
# those kernels change (the date and the capture command travel with the numbers: NCU_TRAFFIC_SOURCE).
NCU_TRAFFIC = {"rows_fwd_tc": 278.7e6, "rows_inv_tc": 249.3e6, "coherent_tc": 2.3e6, "synth_tc": 17.4e6}
NCU_TRAFFIC_SOURCE = ("ncu --set full --clock-control none -k regex:<kernel> -s 1 -c 1 on bench.py --steps 2 "
                      "--warmup 3 --no-cpu --no-serve --no-configs: dram__bytes_read.sum + dram__bytes_write.sum of "
                      "one 64-clip launch of each kernel, measured 2026-12-04")


def kernel_rooflines(sk, masks, reps=10):
    """Device time of the three largest kernels of the split form, each launched alone through its ABI entry
    (CUDA events on the launching stream, after warm-up), against the measured peaks."""
    from opticalimaging_b200 import _native as N
    from opticalimaging_b200.engine import Plan, TC_COARSE, band_spectrum
    hbm, bf16, src = peaks()
    dev = masks.device
    b, B = sk.band, masks.shape[0]
    plan = sk.plan
    tplan = Plan.get(sk.ny, sk.nx, b, dev, coarse=TC_COARSE)
    s = N.stream_handle(dev)
    t = torch.empty(B * sk.ny * b.bc, dtype=torch.complex64, device=dev)
    band = band_spectrum(masks, N.FIELD_REAL_F32, plan, form='bf16x3')
    pupils, weights = sk.fields_for(N.FIELD_REAL_F32)   # the fields the image path runs for real masks
    nf = pupils.shape[1]
    ctas, nparts = N.tc_layout(B, nf)   # nparts also sizes the synthesis kernel's partial sums
    coarse = torch.empty((nparts, B, 1, 128, 128), device=dev)
    v = torch.zeros(B * b.bc * sk.ny, dtype=torch.complex64, device=dev)
    tiles = torch.empty(B * sk.ny * 512, dtype=torch.uint8, device=dev)
    out = torch.empty((B, sk.ny, sk.nx), device=dev)
    # the forward row pass as the image path runs it: the Hermitian half for a symmetric band
    if plan.symmetric_band():
        fwd = lambda: N.call('oi_rows_fwd_tc_half', N.ptr(masks), N.FIELD_REAL_F32, B, sk.ny, sk.nx,  # noqa: E731
                             (b.bc + 1) // 2, N.ptr(plan.rows_consts(2)), N.ptr(t), s)
    else:
        fwd = lambda: N.call('oi_rows_fwd_tc', N.ptr(masks), N.FIELD_REAL_F32, B, sk.ny, sk.nx, b.m0c,  # noqa: E731
                             b.bc, N.ptr(plan.rows_consts(0)), N.ptr(t), s)
    scoarse = torch.rand((nparts, B, 128, 128), device=dev)
    stiles = torch.empty(B * sk.ny * 512, dtype=torch.uint8, device=dev)
    calls = {
        "rows_fwd_tc": fwd,
        "synth_tc": lambda: N.call('oi_synth_tiles_tc', N.ptr(scoarse), nparts, B, b.br, b.bc,    # noqa: E731
                                   N.ptr(tplan.synth_consts()), sk.ny, N.ptr(stiles), s),
        "coherent_tc": lambda: N.call('oi_coherent_coarse_tc', N.ptr(band), B, 1, b.m0r, b.br, b.m0c, b.bc,
                                      N.ptr(pupils), 0, N.ptr(weights), 1, nf,
                                      N.ptr(tplan.tc_constants()), ctas, nparts, N.ptr(coarse), s),
        "rows_inv_tc": lambda: N.call('oi_rows_inv_tc_tiles', N.ptr(tiles), B, sk.ny, sk.nx,
                                      N.ptr(tplan.rows_consts(1)), N.ptr(out), s),
    }
    # operand tiles for the synthesis row pass (the image path writes them in its column pass)
    N.call('oi_rows_inv_tc', N.ptr(v), B, sk.ny, sk.nx, b.bc, N.ptr(tplan.rows_consts(1)), N.ptr(tiles), N.ptr(out), s)
    px = B * sk.ny * sk.nx
    res = {}
    for name, fn in calls.items():
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) / 1e3 / reps
        if name == "coherent_tc":
            flops = 8.0 * B * nf * (128 * b.br * b.bc + 128 * 128 * b.br)
            ach = flops / sec / 1e12
            res[name] = {"bound": "tensor", "achieved": ach, "peak": bf16, "unit": "TFLOP/s", "frac": ach / bf16,
                         "traffic": NCU_TRAFFIC.get(name), "us": sec * 1e6, "peak_source": src,
                         "algorithmic": f"8 (M B^2 + M^2 B) flops per field, M = {128}, B = {b.br}, {nf} fields per "
                                        f"image (the {sk.count} SOCS kernels of a real mask as packed real fields)",
                         "executed_tflops": 3 * 8.0 * B * nf * (128 * 64 * 64 + 128 * 128 * 64) / sec / 1e12}
        elif name == "synth_tc":   # two real GEMMs per image: U = c G (128 x 2bc x 128), v = A U (ny x 2bc x 128)
            flops = 2.0 * B * (128 * 2 * b.bc * 128 + sk.ny * 2 * b.bc * 128)
            ach = flops / sec / 1e12
            res[name] = {"bound": "tensor", "achieved": ach, "peak": bf16, "unit": "TFLOP/s", "frac": ach / bf16,
                         "traffic": NCU_TRAFFIC.get(name), "us": sec * 1e6, "peak_source": src,
                         "algorithmic": "2 (M 2bc M + ny 2bc M) flops per image, M = 128, bc = 59",
                         "executed_tflops": 3 * 2.0 * B * (128 * 128 * 128 + sk.ny * 128 * 128) / sec / 1e12}
        else:
            ach = 4.0 * px / sec / 1e9
            res[name] = {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                         "traffic": NCU_TRAFFIC.get(name), "us": sec * 1e6, "peak_source": src,
                         "algorithmic": "4 bytes per pixel: the float32 mask read" if name == "rows_fwd_tc"
                         else "4 bytes per pixel: the float32 image written"}
    res["traffic_source"] = NCU_TRAFFIC_SOURCE
    return res


def fp64_image(sk_info, mask):
    """FP64 oracle SOCS image of one clip with the engine's K kernels (the precision reference)."""
    from oracle import optics64 as O
    from opticalimaging_b200 import imaging, workloads as W
    from opticalimaging_b200.params import Scatter
    sr, po, nm, T, fg = sk_info
    kern = imaging.DecomposeTCC_SOCS(T, fg, [N_PIX, N_PIX], nm).cpu().numpy().astype(np.complex128)
    sc = Scatter()
    sc.Period_X = sc.Period_Y = PERIOD
    sc.ScatterField = W.thin_field(mask)
    return O.socs(sc, kern, sr, po)


def precision_study(sk, masks, ref, steps=5):
    """Per form: images/s on the HBM-resident batch and max / RMS error of clip 0 vs the FP64 image, both
    relative to the FP64 image's peak."""
    from opticalimaging_b200.engine import FORMS
    out = torch.empty((masks.shape[0], N_PIX, N_PIX), dtype=torch.float32, device=masks.device)
    peak = float(np.max(np.abs(ref)))
    res = {}
    for form in FORMS:
        for _ in range(2):
            sk.image(masks, out=out, form=form)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(steps):
            sk.image(masks, out=out, form=form)
        b.record()
        torch.cuda.synchronize()
        d = out[0].cpu().numpy().astype(np.float64) - ref
        res[form] = {"images_per_s": masks.shape[0] * steps / (a.elapsed_time(b) / 1e3),
                     "max": float(np.max(np.abs(d)) / peak), "rms": float(np.sqrt(np.mean(d ** 2)) / peak)}
    res["relative_to"] = "peak of the FP64 SOCS-24 image of clip 0 (same kernels, FP64 transforms)"
    return res


def run_reference(args, world, rank):
    if rank != 0:
        return
    from opticalimaging_b200 import workloads as W
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    masks = W.config3_masks(count=args.steps + args.warmup, n=N_PIX, seed=3)
    from oracle import cpu_reference as R
    sr, po, nm = W.config3_optics(order=ORDER)
    t0 = time.perf_counter()
    kern = R.socs_kernels(sr, po, nm, [PERIOD, PERIOD], [N_PIX, N_PIX])
    setup_s = time.perf_counter() - t0
    npx = PERIOD / (sr.Wavelength / po.NA)
    fields = []
    for m in masks:
        f = np.zeros((N_PIX, N_PIX, 3), np.complex64)
        f[:, :, 0] = m
        fields.append(f)
    for i in range(args.warmup):
        R.socs_clip(fields[i], kern, npx, npx, threads)
    t0 = time.perf_counter()
    for i in range(args.steps):
        R.socs_clip(fields[args.warmup + i], kern, npx, npx, threads)
    dt = time.perf_counter() - t0
    v = args.steps / dt
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "step": "one clip per step on the host cores"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{args.steps} clips of 1024x1024, 72 full-grid complex64 FFTs each "
                                       "(torch CPU FFT, all host threads)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "setup_s": setup_s}
    print(json.dumps(line), flush=True)


def run_engine(args, world, rank, local):
    from opticalimaging_b200 import workloads as W, _native as N
    dev = torch.device('cuda', local)
    sk, setup_s, info = build_kernels()
    masks_np = W.config3_masks(count=BATCH, n=N_PIX, seed=3 + 1000 * rank)
    masks = torch.from_numpy(masks_np).to(dev)
    out = torch.empty((BATCH, N_PIX, N_PIX), dtype=torch.float32, device=dev)
    # ---- device-resident throughput; clocks sampled from the warm-up through the timed region
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        clk.wait_samples(1)
        for _ in range(max(args.warmup, 3)):
            sk.image(masks, out=out, form=args.form)
        torch.cuda.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        n0 = N.launch_count()
        start.record()
        for _ in range(args.steps):
            sk.image(masks, out=out, form=args.form)
        end.record()
        launches = N.launch_count() - n0
        torch.cuda.synchronize()
        barrier(world)
        clk.wait_samples(len(clk.lines) + 1, timeout=0.5)
    status = N.device_status(reset=True)      # a kernel whose bounded wait expired invalidates the run
    value, ms = job_rate(BATCH * args.steps, start.elapsed_time(end), world)
    # the same clips held as uint8 (binary masks are exact in one byte): 1 byte per pixel read instead of 4
    masks_u8 = masks.to(torch.uint8)
    for _ in range(3):
        sk.image(masks_u8, out=out, form=args.form)
    torch.cuda.synchronize()
    barrier(world)
    su, eu = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    su.record()
    for _ in range(args.steps):
        sk.image(masks_u8, out=out, form=args.form)
    eu.record()
    torch.cuda.synchronize()
    barrier(world)
    value_u8, ms_u8 = job_rate(BATCH * args.steps, su.elapsed_time(eu), world)
    del masks_u8
    # ---- end to end through the public API: pinned uint8 masks in, float32 images out
    host_in = torch.from_numpy(masks_np.astype(np.uint8)).pin_memory()
    host_out = torch.empty((BATCH, N_PIX, N_PIX), dtype=torch.float32).pin_memory()

    def e2e_step():   # host masks in, host images out: copies of neighbouring chunks overlap the compute
        sk.image_host(host_in, host_out, form=args.form)

    for _ in range(max(args.warmup, 3)):
        e2e_step()
    torch.cuda.synchronize()
    barrier(world)
    s2, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s2.record()
    for _ in range(args.steps):
        e2e_step()
    e2.record()
    torch.cuda.synchronize()
    barrier(world)
    status |= N.device_status(reset=True)
    e2e_value, _ = job_rate(BATCH * args.steps, s2.elapsed_time(e2), world)
    if rank != 0:   # the last collective is behind us; what follows is reported by rank 0 alone
        return
    # ---- served: the same clips as requests through the continuous-batching server (pinned uint8 in,
    # host float32 images out), saturated arrival; and the plain one-request-at-a-time path
    serving, unbounded = None, None
    if not args.no_serve:   # latency-aware batching (the reported figures), and unbounded batches beside it
        serving = serve_measure(sk, info, masks_np, dev, args, latency_budget_ms=args.latency_budget_ms)
        unbounded = serve_measure(sk, info, masks_np, dev, args, latency_budget_ms=None)
        serving["unbounded_batches"] = {k: unbounded[k] for k in ("images_per_s", "p50_ms", "p99_ms", "batch_limit")}
    mix, mix_state = None, {}
    if not args.no_serve and args.mix_requests > 0:
        try:
            mix = serve_mix(dev, args, mix_state)
        except Exception as e:  # the configuration-3 line must still print
            mix = {"error": f"{type(e).__name__}: {e}"}
    # ---- per-stage device times (outside the timed region) and the roofline of the dominant stage
    st = stage_times(sk, masks, out, args.form)
    hbm, bf16, src = peaks()
    if args.form == 'bf16x3':
        kern = kernel_rooflines(sk, masks)
        dominant = max((k for k in kern if k != "traffic_source"), key=lambda k: kern[k]["us"])
        roof = dict(kern[dominant], kernel=dominant)
    else:
        kern = None
        dominant = max(st, key=st.get)
        px = BATCH * N_PIX * N_PIX
        ach = 4 * px / (st[dominant] / 1e3) / 1e9
        roof = {"kernel": dominant, "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
                "frac": ach / hbm, "traffic": None, "peak_source": src,
                "algorithmic": "4 bytes per pixel (float32 mask read / image written), per stage"}
    # ---- the drop-in call as a reference user makes it, and the reference's own torch code on the GPU
    dropin = e2e_dropin(info, masks_np, dev) if not args.no_serve else None
    plain_ref = plain_reference_cuda(info, masks_np, dev) if not args.no_serve else None
    if serving is not None and plain_ref:
        serving["plain_reference_torch_cuda_images_per_s"] = plain_ref
        serving["served_over_plain_reference_torch_cuda"] = serving["images_per_s"] / plain_ref
    status |= N.device_status(reset=True)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16x3" if args.form == 'bf16x3' else "fp32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "batch_per_gpu": BATCH, "kernels": sk.count,
                       "coherent_fields": int(sk.fields_for(N.FIELD_REAL_F32)[0].shape[1]),
                       "band": [sk.band.br, sk.band.bc], "form": args.form,
                       "coarse": [128, 128] if args.form == 'bf16x3' else [sk.plan.mr, sk.plan.mc],
                       "l2": "inputs larger than L2 (256 MB float32 masks + 256 MB images per step)",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(host_in.numel()),
                    "d2h_bytes_per_step": int(host_out.numel() * 4)},
            "gpu_launches": launches, "setup_s": setup_s, "device_status": status,
            "uint8_masks": {"value": value_u8, "ms_per_step": ms_u8 / args.steps,
                            "note": "the same clips held in HBM as uint8 (1 byte per pixel read instead of 4)"},
            "stage_ms": {k: round(v, 4) for k, v in st.items()}, "roofline": roof, "roofline_kernels": kern,
            "clocks": clk.summary(), "e2e_dropin": dropin}
    if status:
        line["invalid"] = "a kernel's bounded wait expired during the run (device status %d)" % status
    if rank == 0 and not args.no_cpu and not args.no_configs:
        try:
            line["configs"] = configs_measure(dev)
        except Exception as e:  # the configuration-3 line must still print
            line["configs"] = {"error": f"{type(e).__name__}: {e}"}
    if rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        torch.set_num_threads(threads)
        ref = fp64_image(info, masks_np[0])
        forms = precision_study(sk, masks, ref)
        line["forms"] = forms
        line["accuracy_vs_fp64"] = dict(forms[args.form], relative_to=forms["relative_to"])
        if mix is not None and "error" not in mix:
            mix["err_vs_fp64"] = mix_fp64_check(mix_state["specs"], mix_state["ex"], mix_state["pool"], dev)
        v, n = cpu_reference_sample(info, masks_np, args.cpu_budget, threads)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{n} clips of 1024x1024 through the reference's SOCS algorithm "
                                          "(72 full-grid complex64 FFTs per clip, torch CPU FFT)"}
    line["serving_mix"] = mix
    line["serving"] = serving            # last: the end of the line is what a log tail keeps
    if rank == 0:
        print(json.dumps(compact(line)), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='engine', choices=['engine', 'reference'])
    ap.add_argument('--cpu-budget', type=float, default=15.0)
    ap.add_argument('--no-cpu', action='store_true', help='skip the CPU baseline and the precision study')
    ap.add_argument('--no-serve', action='store_true', help='skip the served measurements (profiling runs)')
    ap.add_argument('--no-configs', action='store_true', help='skip configurations 1, 2 and 4')
    ap.add_argument('--latency-budget-ms', type=float, default=4.0,
                    help='latency budget of the served measurement\'s batch cap (see serve.Server)')
    ap.add_argument('--mix-requests', type=int, default=2000,
                    help='requests of the mixed serving stream (configuration 5); 0 skips it')
    ap.add_argument('--batch', type=int, default=64, help='clips per step (64 in the benchmark configuration)')
    ap.add_argument('--serve-requests', type=int, default=512, help='requests in the saturated served measurement')
    ap.add_argument('--poisson-requests', type=int, default=2048,
                    help='requests of the served measurement under Poisson arrivals')
    ap.add_argument('--form', default='bf16x3', choices=['fft', 'dft', 'bf16x3'],
                    help='transform form of the timed path (bf16x3: split-BF16x3 contraction on tensor cores)')
    args = ap.parse_args()
    global BATCH
    BATCH = args.batch
    world, rank, local = dist_setup()
    try:
        if args.impl == 'reference':
            run_reference(args, world, rank)
        else:
            run_engine(args, world, rank, local)
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()


if __name__ == '__main__':
    main()
