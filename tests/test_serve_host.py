"""Scheduler of the continuous-batching server on the CPU, with a fake executor: batching, admission by the
memory budget, eviction, cancellation, malformed requests and executor failures.  No GPU involved."""
import threading
import time

import pytest
import torch

from opticalimaging_b200.serve import ModelSpec, Server, bucket


class FakeExecutor:
    """Completes a batch `delay` seconds after launch; the 'image' of a mask is 2 * mask as one plane."""

    def __init__(self, nslots=2, delay=0.002, model_bytes=100, per_image=10, fail_keys=()):
        self.nslots, self.delay = nslots, delay
        self.model_bytes, self.per_image = model_bytes, per_image
        self.fail_keys = set(fail_keys)
        self.models, self.evicted, self.launched = {}, [], []
        self.slot = [None] * nslots
        self.lock = threading.Lock()

    def max_batch(self, spec):
        return 8

    def resident_bytes(self):
        return sum(self.models.values())

    def bytes_needed(self, spec, n):
        return (0 if spec.key in self.models else self.model_bytes) + self.per_image * bucket(n)

    def launch(self, slot, spec, reqs):
        if spec.key in self.fail_keys:
            raise RuntimeError('device failure injected on the host')
        self.models[spec.key] = self.model_bytes + self.per_image * bucket(len(reqs))
        self.launched.append((spec.key, len(reqs)))
        self.slot[slot] = (time.perf_counter() + self.delay, [2 * r.mask.float().unsqueeze(0) for r in reqs])

    def poll(self, slot):
        return self.slot[slot] is not None and time.perf_counter() >= self.slot[slot][0]

    def collect(self, slot):
        out = self.slot[slot][1]
        self.slot[slot] = None
        return out

    def evict(self, key):
        self.evicted.append(key)
        self.models.pop(key, None)

    def shutdown(self):
        pass


def spec(name, n=4):
    return ModelSpec((name, n), n, n, 1, build=None)


def test_every_request_completes_and_batches_form():
    ex = FakeExecutor()
    srv = Server(ex, hbm_budget=1e9)
    a, b = spec('a'), spec('b')
    futs = [(m, srv.submit(a if i % 3 else b, m)) for i, m in enumerate(torch.randint(0, 2, (50, 4, 4)).float())]
    for m, f in futs:
        torch.testing.assert_close(f.result(timeout=10), 2 * m.unsqueeze(0))
    srv.drain()
    srv.close()
    assert srv.batches < 50                        # requests were batched
    assert all(n <= 8 for _, n in ex.launched)
    lat = srv.latency_ms()
    assert lat['count'] == 50 and lat['p50_ms'] <= lat['p99_ms']


def test_requests_arriving_during_flight_join_later_batches():
    ex = FakeExecutor(nslots=1, delay=0.02)
    srv = Server(ex, hbm_budget=1e9)
    a = spec('a')
    first = [srv.submit(a, torch.ones(4, 4)) for _ in range(3)]
    time.sleep(0.005)                               # the first batch is in flight
    later = [srv.submit(a, torch.zeros(4, 4)) for _ in range(5)]
    for f in first + later:
        f.result(timeout=10)
    srv.close()
    # the first batch launched before the later requests existed; they joined later batches
    assert ex.launched[0][1] <= 3 and sum(n for _, n in ex.launched) == 8 and len(ex.launched) >= 2


def test_malformed_and_cancelled_requests():
    ex = FakeExecutor(nslots=1, delay=0.05)
    srv = Server(ex, hbm_budget=1e9)
    a = spec('a')
    with pytest.raises(ValueError):
        srv.submit(a, torch.zeros(3, 4)).result(timeout=1)
    with pytest.raises(ValueError):
        srv.submit(a, torch.zeros(4, 4, dtype=torch.float64)).result(timeout=1)
    busy = srv.submit(a, torch.ones(4, 4))          # occupies the only slot
    time.sleep(0.01)
    victim = srv.submit(a, torch.ones(4, 4))
    assert victim.cancel()                          # cancelled while waiting: dropped before launch
    ok = srv.submit(a, torch.ones(4, 4))
    assert busy.result(timeout=10) is not None and ok.result(timeout=10) is not None
    srv.close()
    assert victim.cancelled()


def test_budget_refusal_and_eviction():
    ex = FakeExecutor(nslots=1, delay=0.001, model_bytes=100, per_image=10)
    srv = Server(ex, hbm_budget=150)
    a, b, huge = spec('a'), spec('b'), spec('huge', n=4)
    assert srv.submit(a, torch.ones(4, 4)).result(timeout=10) is not None
    # b does not fit next to a: a is idle, so it is evicted to make room
    assert srv.submit(b, torch.ones(4, 4)).result(timeout=10) is not None
    assert ('a', 4) in ex.evicted
    # a batch that can never fit is refused with MemoryError
    ex.model_bytes = 10 ** 6
    with pytest.raises(MemoryError):
        srv.submit(huge, torch.ones(4, 4)).result(timeout=10)
    srv.close()
    assert srv.rejected == 1


def test_executor_failure_fails_only_its_batch():
    ex = FakeExecutor(fail_keys={('bad', 4)})
    srv = Server(ex, hbm_budget=1e9)
    bad = srv.submit(spec('bad'), torch.ones(4, 4))
    good = srv.submit(spec('good'), torch.ones(4, 4))
    with pytest.raises(RuntimeError, match='injected'):
        bad.result(timeout=10)
    assert good.result(timeout=10) is not None
    srv.close()


def test_submit_after_close_is_refused():
    srv = Server(FakeExecutor(), hbm_budget=1e9)
    srv.close()
    with pytest.raises(RuntimeError):
        srv.submit(spec('a'), torch.ones(4, 4)).result(timeout=1)


def test_adjacent_runs_groups_slab_views_only():
    from opticalimaging_b200.serve import adjacent_runs, run_view
    slab = torch.arange(6 * 2 * 3, dtype=torch.float32).reshape(6, 2, 3)
    views = list(slab)
    assert adjacent_runs(views) == [(0, 6)]
    r = run_view(views, 1, 4)
    assert r.shape == (3, 2, 3) and r.data_ptr() == views[1].data_ptr() and torch.equal(r, slab[1:4])
    r.fill_(-1.0)                                  # the view writes the slab itself
    assert torch.equal(slab[2], torch.full((2, 3), -1.0))
    # out of order, a gap, another storage, another dtype or shape, a non-contiguous view: runs break there
    other = torch.zeros(2, 3)
    mixed = [views[0], views[1], views[3], other, views[4], views[5].to(torch.float64), slab[:, 0][0:2].t()[0]]
    assert adjacent_runs(mixed) == [(0, 2), (2, 3), (3, 4), (4, 5), (5, 6), (6, 7)]
    assert adjacent_runs([views[2], views[1]]) == [(0, 1), (1, 2)]
    assert adjacent_runs([]) == []
    single = run_view([other], 0, 1)
    assert single.shape == (1, 2, 3) and single.data_ptr() == other.data_ptr()


class SetupFailsExecutor(FakeExecutor):
    def thread_init(self):
        raise ValueError('thread set-up failed (injected on the host)')


class PollFailsExecutor(FakeExecutor):
    """Fails inside the scheduler loop once a batch is in flight (an error outside launch/collect)."""

    def poll(self, slot):
        if self.slot[slot] is not None:
            raise KeyError('poll failed (injected on the host)')
        return False


def test_scheduler_setup_failure_fails_requests_instead_of_hanging():
    srv = Server(SetupFailsExecutor(), hbm_budget=1e9)
    srv._thread.join(timeout=10)
    assert not srv._thread.is_alive()
    f = srv.submit(spec('a'), torch.ones(4, 4))
    with pytest.raises(RuntimeError, match='scheduler thread failed'):
        f.result(timeout=5)
    assert isinstance(srv.error, ValueError)
    srv.close()


def test_scheduler_failure_in_flight_fails_queued_and_running_requests():
    ex = PollFailsExecutor(nslots=1, delay=0.5)
    srv = Server(ex, hbm_budget=1e9)
    futs = [srv.submit(spec('a'), torch.full((4, 4), float(i))) for i in range(20)]   # more than one batch
    for f in futs:
        with pytest.raises(RuntimeError, match='scheduler thread failed'):
            f.result(timeout=10)
    assert isinstance(srv.error, KeyError)
    late = srv.submit(spec('a'), torch.ones(4, 4))
    with pytest.raises(RuntimeError, match='scheduler thread failed'):
        late.result(timeout=1)
    srv.drain(timeout=5)
    srv.close()


class StatusExecutor(FakeExecutor):
    """FakeExecutor whose collect() checks a fake device status word through serve.StatusGuard, as
    CudaExecutor checks the library's: the word is set by the test, as a kernel whose wait expired would."""

    def __init__(self, **kw):
        super().__init__(**kw)
        from opticalimaging_b200.serve import StatusGuard
        self.word = 0
        self.guard = StatusGuard(self.read)

    def read(self, reset):
        v = self.word
        if reset:
            self.word = 0
        return v

    def collect(self, slot):
        out = super().collect(slot)
        self.guard.check(slot, [i for i, s in enumerate(self.slot) if s is not None])
        return out


def test_expired_device_wait_fails_the_batch_and_its_neighbours():
    from opticalimaging_b200._native import DeviceWaitError
    ex = StatusExecutor(nslots=2, delay=0.05)
    srv = Server(ex, hbm_budget=1e9)
    a, b = spec('a'), spec('b')
    fa = srv.submit(a, torch.ones(4, 4))
    time.sleep(0.01)
    fb = srv.submit(b, torch.ones(4, 4))          # in flight beside the first batch
    time.sleep(0.01)
    ex.word = 1                                   # a kernel's bounded wait ran out
    with pytest.raises(DeviceWaitError):
        fa.result(timeout=10)
    with pytest.raises(DeviceWaitError):          # it ran alongside: suspect too
        fb.result(timeout=10)
    assert ex.word == 0                           # the word was cleared after the failure was reported
    ok = srv.submit(a, torch.ones(4, 4))          # later batches are served normally
    torch.testing.assert_close(ok.result(timeout=10), 2 * torch.ones(1, 4, 4))
    srv.close()


def test_check_device_status_raises_and_clears():
    from opticalimaging_b200._native import DeviceWaitError, check_device_status
    word = [3]

    def read(reset):
        v = word[0]
        if reset:
            word[0] = 0
        return v
    with pytest.raises(DeviceWaitError, match='device status 3'):
        check_device_status('test', read)
    check_device_status('test', read)             # cleared: no error the second time


class TimedExecutor(FakeExecutor):
    """FakeExecutor that reports a time per image on its slowest stage."""

    def __init__(self, tpi, **kw):
        super().__init__(**kw)
        self.tpi = tpi

    def time_per_image(self, spec):
        return self.tpi

    def max_batch(self, spec):
        return 64


def test_latency_budget_caps_batches():
    """With a latency budget, batches are capped at budget / (slots x time per image) while the backlog is within
    what the slots clear at that size; a larger backlog is shared out over the slots (up to the executor's limit);
    without a budget batches fill."""
    a = spec('a')
    ex = TimedExecutor(tpi=1e-4, nslots=2, delay=0.02)
    srv = Server(ex, hbm_budget=1e9, max_batch=64, latency_budget_ms=2.0)
    assert srv.batch_limit(a) == 10                       # 2 ms / (2 slots x 0.1 ms)
    assert srv._max_batch(a, backlog=20) == 10            # the slots clear 2 x 10 within the budget
    assert srv._max_batch(a, backlog=60) == 30            # 60 queued: late already, shared over the two slots
    assert srv._max_batch(a, backlog=500) == 64           # the executor's limit
    assert srv.batch_ceiling(a) == 64                     # what an executor prepares graphs up to
    for _ in range(12):                                   # light load: one request at a time
        srv.submit(a, torch.ones(4, 4)).result(timeout=10)
    assert max(n for _, n in ex.launched) == 1
    futs = [srv.submit(a, torch.ones(4, 4)) for _ in range(60)]   # a burst: batches grow above the cap
    for f in futs:
        f.result(timeout=10)
    srv.close()
    burst = [n for _, n in ex.launched[12:]]
    assert sum(burst) == 60 and max(burst) > 10 and max(burst) <= 64
    ex2 = TimedExecutor(tpi=1e-4, nslots=2, delay=0.02)
    srv2 = Server(ex2, hbm_budget=1e9, max_batch=64)
    assert srv2.batch_limit(a) == 64
    srv2.close()
    ex3 = TimedExecutor(tpi=1.0, nslots=2)                 # a budget below one image still admits one
    srv3 = Server(ex3, hbm_budget=1e9, latency_budget_ms=1.0)
    assert srv3.batch_limit(a) == 1
    srv3.close()


class ProgressiveExecutor(FakeExecutor):
    """FakeExecutor whose batch results land one request every `step` seconds after `delay` (as chunked
    device-to-host copies do), reported through ready / collect_range / release."""

    def __init__(self, step=0.004, fail_at=None, **kw):
        super().__init__(**kw)
        self.step, self.fail_at, self.released = step, fail_at, 0

    def ready(self, slot):
        t0, out = self.slot[slot]
        return max(0, min(len(out), int((time.perf_counter() - t0) / self.step) + 1))

    def poll(self, slot):
        t0, out = self.slot[slot]
        return time.perf_counter() >= t0 + self.step * len(out)

    def collect_range(self, slot, a, b):
        if self.fail_at is not None and a <= self.fail_at < b:
            raise RuntimeError('copy failure injected on the host')
        return self.slot[slot][1][a:b]

    def release(self, slot):
        self.released += 1
        self.slot[slot] = None


def test_results_of_a_batch_complete_progressively():
    ex = ProgressiveExecutor(nslots=1, delay=0.0, step=0.01)
    srv = Server(ex, hbm_budget=1e9)
    a = spec('a')
    futs = [srv.submit(a, torch.full((4, 4), float(i))) for i in range(6)]
    for i, f in enumerate(futs):
        torch.testing.assert_close(f.result(timeout=10), torch.full((1, 4, 4), 2.0 * i))
    srv.drain()
    done = sorted(t for _, t in srv.completed)
    assert done[-1] - done[0] > 0.02                  # the batch's requests did not all complete at once
    assert ex.released == srv.batches
    srv.close()


def test_progressive_failure_fails_the_rest_and_frees_the_slot():
    """A batch whose fourth result fails to arrive: its first three requests complete, the rest fail with the
    error, and the slot comes free for later batches."""
    ex = ProgressiveExecutor(nslots=1, delay=0.05, step=0.005, fail_at=3)
    srv = Server(ex, hbm_budget=1e9)
    a = spec('a')
    first = srv.submit(a, torch.ones(4, 4))          # occupies the only slot while the six below queue up
    time.sleep(0.01)
    futs = [srv.submit(a, torch.ones(4, 4)) for _ in range(6)]
    first.result(timeout=10)
    outcomes = []
    for f in futs:
        try:
            f.result(timeout=10)
            outcomes.append('ok')
        except RuntimeError:
            outcomes.append('failed')
    assert outcomes == ['ok'] * 3 + ['failed'] * 3
    ex.fail_at = None
    later = srv.submit(a, torch.ones(4, 4))           # the slot came free: later batches are served
    torch.testing.assert_close(later.result(timeout=10), 2 * torch.ones(1, 4, 4))
    srv.close()
