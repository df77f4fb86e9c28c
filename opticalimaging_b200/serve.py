"""Continuous-batching aerial-image server.

Requests -- one mask each, for any optics key and grid -- arrive from any thread through ``Server.submit`` and
get a ``concurrent.futures.Future``.  A scheduler thread groups waiting requests that share a resident model
(same optics key, grid and mask dtype), and whenever an execution slot is free it admits the oldest group's
next batch, provided the device memory it needs fits the HBM budget (idle models and buffers are evicted,
least recently used first, to make room).  The executor runs the batch on the slot's own CUDA stream: one
host->device copy per mask, the replay of the CUDA graph captured for that (model, batch size, slot), one
device->host copy of the images.  Batches on different slots overlap on the device, so copies of one batch run
under the kernels of another, and requests that arrive while batches are in flight join the next batch formed
-- continuous batching rather than a queue.

The scheduler only talks to an executor interface (``launch`` / ``poll`` / ``collect`` / memory accounting), so
its batching, admission and failure handling are exercised on the CPU with a fake executor in the tests; the
device executor is ``CudaExecutor``.  Masks and caller-provided result buffers that are consecutive views of one
(pinned) slab are moved with one copy per run rather than one per request (``adjacent_runs``).

Failure behaviour: a malformed request (wrong shape or dtype) fails at submit; a request whose batch can never
fit the budget fails with MemoryError; a cancelled future is dropped before launch; an executor error fails
the futures of its batch and the server keeps serving; a batch collected while the device status word shows an
expired kernel wait fails with DeviceWaitError, and so do the batches in flight beside it (``StatusGuard``).
An error that escapes the scheduler thread itself (for
instance the executor's thread set-up) closes the server and fails every request it holds; later submits fail
at once.
"""
from __future__ import annotations

import collections
import concurrent.futures as cf
import math
import threading
import time
from dataclasses import dataclass, field

import torch


# ------------------------------------------------------------------------------------------- requests
@dataclass(frozen=True)
class ModelSpec:
    """A resident imaging model: `key` identifies it, `build()` creates it on the device (CoherentModel)."""
    key: tuple
    ny: int
    nx: int
    planes: int
    build: object = field(compare=False, hash=False, repr=False)

    @property
    def pixels(self):
        return self.ny * self.nx


@dataclass
class Request:
    spec: ModelSpec
    mask: torch.Tensor
    future: cf.Future
    t_submit: float
    t_done: float = 0.0
    rid: int = 0
    out: torch.Tensor | None = None   # caller-provided result storage [planes, ny, nx] float32


def adjacent_runs(tensors) -> list:
    """Split a batch's host tensors into runs [i, j) that lie back to back in one storage: same shape, dtype and
    device, contiguous, tensors[k + 1] starting where tensors[k] ends (views of one slab, in order).  A run moves
    between host and device as one copy instead of j - i."""
    runs, i, n = [], 0, len(tensors)
    while i < n:
        j, t0 = i + 1, tensors[i]
        if t0.is_contiguous():
            base = t0.untyped_storage().data_ptr()
            while j < n:
                a, b = tensors[j - 1], tensors[j]
                if not (b.is_contiguous() and b.shape == t0.shape and b.dtype == t0.dtype and b.device == t0.device
                        and b.untyped_storage().data_ptr() == base
                        and b.storage_offset() == a.storage_offset() + a.numel()):
                    break
                j += 1
        runs.append((i, j))
        i = j
    return runs


def run_view(tensors, i: int, j: int) -> torch.Tensor:
    """The run [i, j) of adjacent_runs as one tensor [j - i, *shape] over the same memory."""
    t0 = tensors[i]
    if j - i == 1:
        return t0.unsqueeze(0)
    return torch.empty(0, dtype=t0.dtype, device=t0.device).set_(t0.untyped_storage(), t0.storage_offset(),
                                                                  (j - i,) + tuple(t0.shape))


def bucket(n: int) -> int:
    """Batch sizes are rounded up to powers of two, so one captured graph serves a range of batch sizes."""
    return 1 << max(0, math.ceil(math.log2(max(1, n))))


# ------------------------------------------------------------------------------------------ scheduler
class Server:
    """Continuous-batching scheduler over an executor (see module docstring)."""

    def __init__(self, executor, hbm_budget: float = 150e9, max_batch_pixels: int = 64 * 1024 * 1024,
                 max_batch: int = 256, idle_wait: float = 0.0002, latency_budget_ms: float | None = None):
        self.ex = executor
        self.budget = float(hbm_budget)
        self.max_batch_pixels = max_batch_pixels
        self.max_batch = max_batch
        self.idle_wait = idle_wait
        # Latency-aware batching: a request's batch waits behind at most (slots - 1) other batches on the slowest
        # pipeline stage (for the CUDA executor the device-to-host copy of the images), then takes its own turn;
        # batches are capped so that slots x batch x (time per image on that stage) stays within the budget.
        self.latency_budget = None if latency_budget_ms is None else latency_budget_ms / 1e3
        self._inbox = collections.deque()
        self._cv = threading.Condition()
        self._pending: dict = collections.OrderedDict()   # group key -> deque of requests
        self._slots = [None] * executor.nslots            # slot -> (spec, [requests])
        self._delivered = [0] * executor.nslots           # slot -> requests of its batch already completed
        self._last_used: dict = {}
        self._closed = False
        self.error = None            # the exception that ended the scheduler thread, if one did
        self._rid = 0
        self.completed = []          # (submit, done) times of finished requests, for latency statistics
        self.batches = 0
        self.rejected = 0
        self._thread = threading.Thread(target=self._run, name='oi-serve', daemon=True)
        self._thread.start()

    # ---- public
    def submit(self, spec: ModelSpec, mask: torch.Tensor, out: torch.Tensor | None = None) -> cf.Future:
        """Queue one mask [ny, nx] (uint8 or float32, host or device) for imaging with `spec`'s model.

        The future's result is the image [planes, ny, nx] float32: written into `out` when given (pinned host
        or device memory the caller owns and reuses -- the high-throughput form), else a new tensor on the
        executor's result device."""
        fut = cf.Future()
        if out is not None and (tuple(out.shape) != (spec.planes, spec.ny, spec.nx) or out.dtype != torch.float32):
            fut.set_exception(ValueError(f'out must be a float32 [{spec.planes}, {spec.ny}, {spec.nx}] tensor'))
            return fut
        if not isinstance(mask, torch.Tensor) or mask.dim() != 2 or tuple(mask.shape) != (spec.ny, spec.nx):
            fut.set_exception(ValueError(f'mask must be a [{spec.ny}, {spec.nx}] tensor, got '
                                         f'{tuple(mask.shape) if isinstance(mask, torch.Tensor) else type(mask)}'))
            return fut
        if mask.dtype not in (torch.uint8, torch.float32):
            fut.set_exception(ValueError(f'mask dtype must be uint8 or float32, got {mask.dtype}'))
            return fut
        with self._cv:
            if self._closed:
                fut.set_exception(RuntimeError('server is closed' if self.error is None else
                                               f'server is closed: its scheduler thread failed ({self.error!r})'))
                return fut
            self._rid += 1
            self._inbox.append(Request(spec, mask, fut, time.perf_counter(), rid=self._rid, out=out))
            self._cv.notify()
        return fut

    def close(self, wait: bool = True):
        with self._cv:
            self._closed = True
            self._cv.notify()
        if wait:
            self._thread.join()

    def drain(self, timeout: float = 600.0):
        """Block until every submitted request has completed."""
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < timeout:
            with self._cv:
                busy = self._inbox or any(self._pending.values()) or any(s is not None for s in self._slots)
            if not busy:
                return
            time.sleep(0.0005)
        raise TimeoutError('requests still pending')

    def latency_ms(self):
        lat = sorted((done - sub) * 1e3 for sub, done in self.completed)
        if not lat:
            return {}
        pick = lambda q: lat[min(len(lat) - 1, int(math.ceil(q * len(lat))) - 1)]  # noqa: E731
        return {"p50_ms": pick(0.50), "p99_ms": pick(0.99), "max_ms": lat[-1], "count": len(lat)}

    # ---- scheduler thread
    def _group_key(self, r: Request):
        return (r.spec.key, r.mask.dtype)

    def _max_batch(self, spec: ModelSpec, backlog: int = 0) -> int:
        b = max(1, min(self.max_batch, self.max_batch_pixels // spec.pixels, self.ex.max_batch(spec)))
        if self.latency_budget is not None:
            per = getattr(self.ex, 'time_per_image', None)
            t = per(spec) if per is not None else None
            if t:
                cap = max(1, min(b, int(self.latency_budget / (self.ex.nslots * t))))
                # A backlog that the slots cannot clear at the capped size within the budget is late already:
                # it is shared out over the slots (larger batches spread the per-batch costs), so overload is
                # absorbed at close to full throughput while light load keeps the capped latency.  Taking the whole
                # backlog instead made a burst at 70 % load cascade: each long batch let a longer queue build.
                if backlog > cap * self.ex.nslots:
                    return max(cap, min(b, -(-backlog // self.ex.nslots)))
                return cap
        return b

    def batch_limit(self, spec: ModelSpec) -> int:
        """The largest batch this server forms for `spec` under light load (by max_batch, max_batch_pixels and
        the latency budget); a backlog beyond what the slots clear within the budget is taken in larger batches."""
        return self._max_batch(spec)

    def batch_ceiling(self, spec: ModelSpec) -> int:
        """The largest batch this server ever forms for `spec` (under any backlog): the size up to which an
        executor's graphs should be prepared."""
        return self._max_batch(spec, backlog=1 << 30)

    def _run(self):
        try:
            self._loop()
        except BaseException as e:  # noqa: BLE001 -- the scheduler must not die silently with requests waiting
            self._fail_all(e)

    def _fail_all(self, err: BaseException):
        """The scheduler thread is ending on an unexpected error: close the server and fail every request it
        holds -- queued, pending and in flight -- with that error, so no caller waits forever."""
        with self._cv:
            self._closed = True
            self.error = err
            reqs = list(self._inbox)
            self._inbox.clear()
            for q in self._pending.values():
                reqs.extend(q)
            self._pending.clear()
            for i, s in enumerate(self._slots):
                if s is not None:
                    reqs.extend(s[1])
                    self._slots[i] = None
        failure = RuntimeError(f'the server\'s scheduler thread failed: {type(err).__name__}: {err}')
        failure.__cause__ = err
        for r in reqs:
            if not r.future.done():
                try:
                    r.future.set_exception(failure)
                except cf.InvalidStateError:   # completed or cancelled meanwhile
                    pass

    def _loop(self):
        init = getattr(self.ex, 'thread_init', None)
        if init is not None:
            init()
        while True:
            with self._cv:
                while self._inbox:
                    r = self._inbox.popleft()
                    self._pending.setdefault(self._group_key(r), collections.deque()).append(r)
                closing = self._closed
            progressed = self._complete() | self._launch()
            with self._cv:
                idle = not self._inbox and not any(self._pending.values()) and all(s is None for s in self._slots)
                if closing and idle:
                    self.ex.shutdown()
                    return
                if not progressed and not self._inbox:
                    self._cv.wait(self.idle_wait)

    def _deliver(self, reqs, results, err, now):
        for j, r in enumerate(reqs):
            r.t_done = now
            if err is not None:
                r.future.set_exception(err)
            else:
                r.future.set_result(results[j])
                self.completed.append((r.t_submit, now))   # not the request: it holds the result

    def _complete(self) -> bool:
        """Hand finished results to their futures.  An executor with ``ready`` / ``collect_range`` / ``release``
        reports results in order as their copies land (requests of a batch complete progressively); the slot is
        freed once the whole batch has finished.  Otherwise a batch completes as one (``poll`` / ``collect``)."""
        if getattr(self.ex, 'ready', None) is not None:
            return self._complete_progressive()
        done = False
        for i, s in enumerate(self._slots):
            if s is None or not self.ex.poll(i):
                continue
            spec, reqs = s
            try:
                results = self.ex.collect(i)
                err = None
            except Exception as e:  # noqa: BLE001 -- an executor failure fails this batch only
                results, err = None, e
            self._deliver(reqs, results, err, time.perf_counter())
            self._slots[i] = None
            done = True
        return done

    def _complete_progressive(self) -> bool:
        done = False
        for i, s in enumerate(self._slots):
            if s is None:
                continue
            spec, reqs = s
            d = self._delivered[i]
            if d < len(reqs):
                k = self.ex.ready(i)
                if k > d:
                    try:
                        results = self.ex.collect_range(i, d, k)
                        err = None
                    except Exception as e:  # noqa: BLE001 -- an executor failure fails this batch only
                        results, err = None, e
                    if err is not None:   # the rest of the batch cannot be trusted either
                        self._deliver(reqs[d:], None, err, time.perf_counter())
                        self._delivered[i] = len(reqs)
                    else:
                        self._deliver(reqs[d:k], results, None, time.perf_counter())
                        self._delivered[i] = k
                    done = True
            if self._delivered[i] == len(reqs) and self.ex.poll(i):   # every copy of the batch is done
                self.ex.release(i)
                self._slots[i] = None
                self._delivered[i] = 0
                done = True
        return done

    def _take(self, key, limit):
        q = self._pending[key]
        batch = []
        while q and len(batch) < limit:
            r = q.popleft()
            if r.future.set_running_or_notify_cancel():
                batch.append(r)
        if not q:
            del self._pending[key]
        return batch

    def _fits(self, spec, n) -> bool:
        need = self.ex.bytes_needed(spec, n)
        if self.ex.resident_bytes() + need <= self.budget:
            return True
        busy = {s[0].key for s in self._slots if s is not None}
        for key in sorted(self._last_used, key=self._last_used.get):   # least recently used first
            if key in busy or key == spec.key:
                continue
            self.ex.evict(key)
            self._last_used.pop(key, None)
            if self.ex.resident_bytes() + need <= self.budget:
                return True
        return False

    def _launch(self) -> bool:
        launched = False
        while self._pending:
            free = [i for i, s in enumerate(self._slots) if s is None]
            if not free:
                break
            # the group whose oldest request has waited longest
            key = min(self._pending, key=lambda k: self._pending[k][0].t_submit if self._pending[k] else math.inf)
            if not self._pending[key]:
                del self._pending[key]
                continue
            spec = self._pending[key][0].spec
            limit = self._max_batch(spec, len(self._pending[key]))
            n = min(len(self._pending[key]), limit)
            if not self._fits(spec, n):
                if all(s is None for s in self._slots):     # nothing will free memory: refuse the group
                    err = MemoryError(f'model {spec.key!r} with a batch of {n} needs '
                                      f'{self.ex.bytes_needed(spec, n) / 1e9:.2f} GB, over the '
                                      f'{self.budget / 1e9:.2f} GB budget')
                    for r in self._pending.pop(key):
                        if r.future.set_running_or_notify_cancel():
                            r.future.set_exception(err)
                            self.rejected += 1
                    continue
                break                                          # wait for an in-flight batch to free memory
            batch = self._take(key, limit)
            if not batch:
                continue
            slot = free[0]
            try:
                self.ex.launch(slot, spec, batch)
            except Exception as e:  # noqa: BLE001
                for r in batch:
                    r.future.set_exception(e)
                continue
            self._slots[slot] = (spec, batch)
            self._last_used[spec.key] = time.perf_counter()
            self.batches += 1
            launched = True
        return launched


# ------------------------------------------------------------------------------------------- executor
class StatusGuard:
    """Attributes expired kernel waits to batches.  A tensor-core kernel whose bounded wait runs out sets the
    device's status word and returns early with a partial result; the word is one per device, so when it is
    found set at the collection of one batch it may come from any batch that ran alongside: the collected batch
    fails, and so does every batch in flight at that moment (each when it is collected).  `reader(reset)` reads
    the word (default: the library's oi_device_status)."""

    def __init__(self, reader=None):
        self.reader = reader
        self.suspect = set()

    def check(self, slot: int, in_flight) -> None:
        """Raise DeviceWaitError if the batch just collected from `slot` cannot be trusted."""
        from . import _native as N
        suspect = slot in self.suspect
        self.suspect.discard(slot)
        try:
            N.check_device_status(f'batch on slot {slot}', self.reader)
        except N.DeviceWaitError:
            self.suspect.update(s for s in in_flight if s != slot)
            raise
        if suspect:
            raise N.DeviceWaitError(f'batch on slot {slot} ran alongside a batch whose kernel wait expired; its '
                                    'results are invalid')


class CudaExecutor:
    """Runs batches on `nslots` CUDA streams of one device, with CUDA graphs per (model, batch bucket, slot).

    Device memory it holds (and reports to the scheduler): resident models, and per (model, slot) an input and
    an output buffer for the largest batch plus the graph pools.  Results are host float32 tensors (views of a
    pinned batch buffer) or, with result_device='cuda', device tensors.
    """

    def __init__(self, device=None, nslots: int = 3, use_graphs: bool = True, result_device: str = 'cpu',
                 max_batch: int = 256, status_reader=None, result_chunk: int = 8):
        from .engine import require_cuda
        self.device = require_cuda(device)
        self.guard = StatusGuard(status_reader)   # every collected batch is checked against expired kernel waits
        self.nslots = nslots
        self.use_graphs = use_graphs
        self.result_device = result_device
        self._max_batch = max_batch
        self.streams = [torch.cuda.Stream(self.device) for _ in range(nslots)]
        self.result_chunk = max(1, int(result_chunk))     # requests per device-to-host copy (and completion mark)
        self.marks = [[] for _ in range(nslots)]          # slot -> [(requests complete, event)], in order
        self.events = [None] * nslots
        self.pending = [None] * nslots
        self.batch = [None] * nslots
        self.models: dict = {}        # key -> CoherentModel
        self.buffers: dict = {}       # (key, slot, dtype) -> (d_in, d_out)
        self.graphs: dict = {}        # (key, slot, dtype, bucket) -> (graph, bytes)
        self._bytes: dict = {}        # key -> device bytes attributed to it
        self._link = None             # measured (h2d, d2h) bytes per second
        self._device_tpi: dict = {}   # key -> device seconds per image (timed graph replay)

    def thread_init(self):
        torch.cuda.set_device(self.device)

    def max_batch(self, spec):
        return self._max_batch

    def time_per_image(self, spec) -> float:
        """Seconds per image on the slowest stage of a batch: the host<->device copies at the link rates measured
        once (pinned memory; float32 images out, masks in at up to 4 bytes per pixel) or the device time of the
        image itself when a graph of the spec has been timed (``prepare``)."""
        if self._link is None:
            self._link = measure_link(self.device)
        h2d, d2h = self._link
        t = max(4.0 * spec.pixels / h2d, 4.0 * spec.planes * spec.pixels / d2h)
        return max(t, self._device_tpi.get(spec.key, 0.0))

    def resident_bytes(self):
        return sum(self._bytes.values())

    def bytes_needed(self, spec, n):
        """Device bytes a batch of n would add: the model if absent, plus one slot's buffers and graph pool
        for the batch bucket (an upper bound: buffers already allocated are counted again)."""
        b = bucket(n)
        model = self.models.get(spec.key)
        need = 0 if model is not None else self._model_bytes(spec)
        per = spec.pixels * (4 + 4 * spec.planes)
        ws = model.workspace_bytes(b) if model is not None else 16 * b * spec.pixels // 4
        return need + b * per + ws

    def _model_bytes(self, spec):
        return 64 << 20

    def _model(self, spec):
        m = self.models.get(spec.key)
        if m is None:
            with torch.cuda.device(self.device):
                m = spec.build()
            torch.cuda.synchronize(self.device)   # built on the default stream; the slot streams read it
            self.models[spec.key] = m
            self._bytes[spec.key] = self._bytes.get(spec.key, 0) + m.nbytes
        return m

    def _buffers(self, spec, slot, dtype, n):
        key = (spec.key, slot, dtype)
        buf = self.buffers.get(key)
        if buf is None or buf[0].shape[0] < n:
            cap = bucket(max(n, 1))
            if buf is not None:
                self._bytes[spec.key] -= buf[0].numel() * buf[0].element_size() + buf[1].numel() * 4
                for gk in [g for g in self.graphs if g[:3] == key]:
                    self._bytes[spec.key] -= self.graphs.pop(gk)[1]
            d_in = torch.empty((cap, spec.ny, spec.nx), dtype=dtype, device=self.device)
            d_out = torch.empty((cap, spec.planes, spec.ny, spec.nx), dtype=torch.float32, device=self.device)
            buf = self.buffers[key] = (d_in, d_out)
            self._bytes[spec.key] = self._bytes.get(spec.key, 0) + d_in.numel() * d_in.element_size() + \
                d_out.numel() * 4
        return buf

    def _graph(self, spec, model, slot, dtype, b, d_in, d_out):
        gk = (spec.key, slot, dtype, b)
        g = self.graphs.get(gk)
        if g is None:
            s = self.streams[slot]
            s.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.stream(s):
                model.image(d_in[:b], out=d_out[:b])            # warm-up: plans, attributes, allocator
            torch.cuda.current_stream(self.device).wait_stream(s)
            torch.cuda.synchronize(self.device)
            free0 = torch.cuda.mem_get_info(self.device)[0]
            graph = torch.cuda.CUDAGraph()
            # thread-local capture: client threads may allocate pinned memory or copy while a bucket is captured
            with torch.cuda.graph(graph, stream=s, capture_error_mode='thread_local'):
                model.image(d_in[:b], out=d_out[:b])
            used = max(0, free0 - torch.cuda.mem_get_info(self.device)[0])
            g = self.graphs[gk] = (graph, used)
            self._bytes[spec.key] = self._bytes.get(spec.key, 0) + used
            if b >= 8:   # device time per image of this spec, from a warm replay (the copies are timed apart)
                graph.replay()                                     # the first replay uploads the graph
                a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(s)
                graph.replay()
                z.record(s)
                z.synchronize()
                # the steady per-image cost: the least over the timed buckets (a small batch's time is mostly
                # the step's fixed part)
                t = a.elapsed_time(z) / 1e3 / b
                self._device_tpi[spec.key] = min(self._device_tpi.get(spec.key, t), t)
        return g[0]

    def prepare(self, spec, dtype=torch.uint8, max_batch: int | None = None):
        """Build `spec`'s model, the slot buffers and the CUDA graph of every batch bucket up to `max_batch` on
        every slot, so that no capture -- and no device-wide synchronisation -- happens while serving.  Call it
        before the first request of a model (not while batches run)."""
        model = self._model(spec)
        top = bucket(max_batch or self._max_batch)
        for slot in range(self.nslots):
            d_in, d_out = self._buffers(spec, slot, dtype, top)
            b = 1
            while self.use_graphs and b <= top:
                self._graph(spec, model, slot, dtype, b, d_in, d_out)
                b *= 2

    def launch(self, slot, spec, reqs):
        model = self._model(spec)
        n = len(reqs)
        b = bucket(n)
        dtype = reqs[0].mask.dtype
        d_in, d_out = self._buffers(spec, slot, dtype, b)
        graph = self._graph(spec, model, slot, dtype, b, d_in, d_out) if self.use_graphs else None
        s = self.streams[slot]
        with torch.cuda.device(self.device), torch.cuda.stream(s):
            masks = [r.mask for r in reqs]
            for i, j in adjacent_runs(masks):             # masks that are adjacent views of one slab: one copy
                d_in[i:j].copy_(run_view(masks, i, j), non_blocking=True)
            if graph is not None:
                graph.replay()
            else:
                model.image(d_in[:n], out=d_out[:n])
            marks, c = [], self.result_chunk

            def mark(end):   # requests [0, end) have their images where they are going once this event completes
                ev = torch.cuda.Event()
                ev.record(s)
                marks.append((end, ev))
            if all(r.out is not None for r in reqs):      # caller-provided storage: copy each image there
                outs = [r.out for r in reqs]
                for i, j in adjacent_runs(outs):          # runs of adjacent views, cut into chunks of c requests
                    for a in range(i, j, c):
                        e = min(j, a + c)
                        run_view(outs, a, e).copy_(d_out[a:e], non_blocking=True)
                        mark(e)
                out = outs
            elif self.result_device == 'cpu':
                # bucket-sized pinned buffer: sizes repeat, so the host caching allocator recycles them
                host = torch.empty((b, spec.planes, spec.ny, spec.nx), dtype=torch.float32, pin_memory=True)
                mixed = any(r.out is not None for r in reqs)
                for a in range(0, n, c):
                    e = min(n, a + c)
                    host[a:e].copy_(d_out[a:e], non_blocking=True)
                    if not mixed:
                        mark(e)
                out = host
            else:
                out = d_out[:n].clone()
            for i, r in enumerate(reqs):
                if r.out is not None and not isinstance(out, list):
                    r.out.copy_(d_out[i], non_blocking=True)
            if not marks or marks[-1][0] != n:
                mark(n)
            ev = marks[-1][1]
        self.marks[slot] = marks
        self.events[slot] = ev
        self.pending[slot] = out
        self.batch[slot] = reqs

    def poll(self, slot):
        ev = self.events[slot]
        return ev is not None and ev.query()

    def ready(self, slot) -> int:
        """How many leading requests of the slot's batch have their images in place (their copy has finished)."""
        n = 0
        for end, ev in self.marks[slot]:
            if not ev.query():
                break
            n = end
        return n

    def collect_range(self, slot, a: int, b: int):
        """Results of requests [a, b) of the slot's batch (b <= ready(slot)).  The first call of a batch checks the
        device status: its kernels have all finished once its first copy has."""
        out, reqs = self.pending[slot], self.batch[slot]
        if a == 0:
            self.guard.check(slot, [i for i, e in enumerate(self.events) if e is not None and i != slot])
        if isinstance(out, list):
            return out[a:b]
        return [r.out if r.out is not None else out[i] for i, r in enumerate(reqs) if a <= i < b]

    def release(self, slot):
        """The slot's batch has finished (poll): its buffers may take the next batch.  A suspicion the status
        guard attached to the slot belonged to this batch (it was checked, or found clean before)."""
        self.guard.suspect.discard(slot)
        self.events[slot] = None
        self.pending[slot] = None
        self.batch[slot] = None
        self.marks[slot] = []

    def collect(self, slot):
        out, reqs = self.pending[slot], self.batch[slot]
        self.events[slot] = None
        self.pending[slot] = None
        self.batch[slot] = None
        self.guard.check(slot, [i for i, e in enumerate(self.events) if e is not None])
        if isinstance(out, list):
            return out
        return [r.out if r.out is not None else out[i] for i, r in enumerate(reqs)]

    def evict(self, key):
        self.models.pop(key, None)
        for k in [k for k in self.buffers if k[0] == key]:
            del self.buffers[k]
        for k in [k for k in self.graphs if k[0] == key]:
            del self.graphs[k]
        self._bytes.pop(key, None)

    def shutdown(self):
        for s in self.streams:
            s.synchronize()


def measure_link(device, nbytes: int = 32 << 20, reps: int = 3):
    """(host-to-device, device-to-host) bytes per second of pinned copies of `nbytes`, best of `reps`."""
    dev = torch.device(device)
    host = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    d = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    s = torch.cuda.Stream(dev)
    rates = []
    for src, dst in ((host, d), (d, host)):
        best = None
        for _ in range(reps):
            a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(s):
                a.record(s)
                dst.copy_(src, non_blocking=True)
                z.record(s)
            z.synchronize()
            t = a.elapsed_time(z) / 1e3
            best = t if best is None else min(best, t)
        rates.append(nbytes / best)
    return rates[0], rates[1]


def plain_run(spec_masks, device=None):
    """The plain path: one request at a time, no batching, no graphs, no overlap -- copy in, image, copy out,
    synchronise.  Returns (results, seconds)."""
    dev = torch.device('cuda', torch.cuda.current_device()) if device is None else torch.device(device)
    models = {}
    out = []
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for spec, mask in spec_masks:
        m = models.get(spec.key)
        if m is None:
            m = models[spec.key] = spec.build()
        d = mask.to(dev).unsqueeze(0)
        img = m.image(d)
        out.append(img[0].cpu())
    torch.cuda.synchronize(dev)
    return out, time.perf_counter() - t0


# ------------------------------------------------------------------------------------------- specs
def _with_form(model, form):
    """Give a built model its serving form: 'bf16x3' where the band allows it (<= 64 x 64), else the FP32 FFT
    form; None keeps the model's default."""
    from .engine import tc_supported
    if model is not None and form is not None:
        model.form = form if form != 'bf16x3' or tc_supported(model.band) else 'fft'
    return model


def socs_spec(source, projector, numerics, period, n, focus=(0.0,), name='socs', form=None):
    """SOCS model of an n x n clip of `period` nm with the kernels of every focus plane; `form` as in
    _with_form."""
    from .imaging import socs_model
    key = (name, n, float(period), tuple(float(z) for z in focus), form)
    return ModelSpec(key, n, n, len(focus),
                     lambda: _with_form(socs_model(source, projector, numerics, period, period, n, n,
                                                   focus=list(focus)), form))


def abbe_spec(source, projector, numerics, period, n, focus=(0.0,), name='abbe', form=None):
    """Abbe model (resident pupils of every source point) of an n x n clip of `period` nm; `form` as in
    _with_form."""
    from .imaging import abbe_model
    key = (name, n, float(period), tuple(float(z) for z in focus), form)
    return ModelSpec(key, n, n, len(focus),
                     lambda: _with_form(abbe_model(source, projector, numerics, period, period, n, n,
                                                   focus=list(focus)), form))
