"""Host logic of the continuous-batching server (pdynamo3_b200.serving) with stand-in engines:
admission by free device memory, routing of follow-ups to the slot that holds the system,
warm starts, eviction of resident systems, error isolation and the latency summary."""
import threading
import time

import numpy as np
import pytest

from pdynamo3_b200.serving import GPUServer, Request, latency_summary


class FakeResult:
    def __init__(self, energy):
        self.energy = energy
        self.converged = True


class FakeEngine:
    """Deterministic 'energy' of the coordinates; counts concurrent calls across engines."""
    lock = threading.Lock()
    active = 0
    peak = 0
    closed = 0

    def __init__(self, request, fail=False, delay=0.01):
        self.atomic_numbers = request.atomic_numbers
        self.fail = fail
        self.delay = delay
        self.calls = 0

    def energy(self, coordinates_bohr, do_gradients=True):
        with FakeEngine.lock:
            FakeEngine.active += 1
            FakeEngine.peak = max(FakeEngine.peak, FakeEngine.active)
        time.sleep(self.delay)
        with FakeEngine.lock:
            FakeEngine.active -= 1
        self.calls += 1
        if self.fail:
            raise RuntimeError("engine failure")
        return FakeResult(float(np.sum(coordinates_bohr ** 2)))

    def close(self):
        with FakeEngine.lock:
            FakeEngine.closed += 1


@pytest.fixture(autouse=True)
def reset():
    FakeEngine.active = FakeEngine.peak = FakeEngine.closed = 0


def _requests(n_systems, follow_ups, rng):
    out = []
    for s in range(n_systems):
        z = [8, 1, 1] * (1 + s % 3)
        x = rng.normal(size=(len(z), 3))
        for k in range(follow_ups + 1):
            out.append(Request(len(out), "sys%d" % s, z, x + 0.01 * k))
    return out


def test_every_request_completes_with_its_own_result():
    rng = np.random.default_rng(0)
    srv = GPUServer(n_slots=3, engine_factory=lambda r: FakeEngine(r), free_memory=lambda: None)
    reqs = _requests(5, 3, rng)
    for r in reqs:
        srv.submit(r)
    assert srv.drain(timeout=30)
    srv.close()
    for r in reqs:
        assert r.error is None
        assert r.result.energy == pytest.approx(float(np.sum(r.coordinates_bohr ** 2)), rel=0, abs=0)
    assert FakeEngine.peak > 1          # slots really overlap
    s = latency_summary(reqs)
    assert s["completed"] == len(reqs) and s["p99_s"] >= s["p50_s"] > 0


def test_follow_ups_go_to_the_resident_slot_and_start_warm():
    rng = np.random.default_rng(1)
    srv = GPUServer(n_slots=4, engine_factory=lambda r: FakeEngine(r), free_memory=lambda: None)
    reqs = _requests(3, 4, rng)
    for r in reqs:              # follow-ups submitted one by one after their predecessor finished
        srv.submit(r)
        r.done.wait(10)
    srv.close()
    by_system = {}
    for r in reqs:
        by_system.setdefault(r.system, []).append(r)
    for rs in by_system.values():
        assert len({r.slot for r in rs}) == 1
        assert not rs[0].warm and all(r.warm for r in rs[1:])


def test_admission_waits_for_device_memory():
    rng = np.random.default_rng(2)
    # free memory only ever fits one request beyond the reserve: at most one in flight
    srv = GPUServer(n_slots=4, engine_factory=lambda r: FakeEngine(r), free_memory=lambda: 3 << 30,
                    memory_reserve=3 << 30)
    reqs = _requests(6, 0, rng)
    for r in reqs:
        srv.submit(r)
    assert srv.drain(timeout=30)
    srv.close()
    assert all(r.error is None for r in reqs)
    assert FakeEngine.peak == 1


def test_resident_systems_are_evicted_beyond_the_limit():
    rng = np.random.default_rng(3)
    srv = GPUServer(n_slots=1, resident_per_slot=2, engine_factory=lambda r: FakeEngine(r), free_memory=lambda: None)
    reqs = _requests(4, 0, rng)
    for r in reqs:
        srv.submit(r)
    assert srv.drain(timeout=30)
    assert FakeEngine.closed == 2
    srv.close()
    assert FakeEngine.closed == 4


def test_a_failing_request_does_not_stop_the_server():
    rng = np.random.default_rng(4)
    srv = GPUServer(n_slots=2, engine_factory=lambda r: FakeEngine(r, fail=(r.system == "sys1")),
                    free_memory=lambda: None)
    reqs = _requests(3, 1, rng)
    for r in reqs:
        srv.submit(r)
    assert srv.drain(timeout=30)
    srv.close()
    for r in reqs:
        if r.system == "sys1":
            assert isinstance(r.error, RuntimeError)
        else:
            assert r.error is None and r.result is not None


def test_eviction_keeps_systems_with_queued_requests_and_reregisters_owner():
    """A slot never evicts a system whose requests wait in its private queue, and a system whose
    engine is (re)built on a slot is owned by that slot, so its follow-ups go there."""
    from pdynamo3_b200.serving import GPUServer, Request

    class Eng:
        def __init__(self, r):
            self.atomic_numbers = r.atomic_numbers
            self.closed = False

        def energy(self, x, do_gradients=True):
            return type("R", (), {"energy": 0.0, "gradients": None, "converged": True})()

        def close(self):
            self.closed = True

    srv = GPUServer(n_slots=1, resident_per_slot=1, engine_factory=Eng, free_memory=lambda: None)
    try:
        z = np.array([1, 1])
        x = np.zeros((2, 3))
        srv._private[0].append(Request(9, "a", z, x))           # a request of "a" waiting on slot 0
        e_a, warm = srv._engine_for(0, Request(1, "a", z, x))
        assert not warm and srv._owner["a"] == 0
        e_b, _ = srv._engine_for(0, Request(2, "b", z, x))      # over the limit, but "a" is queued: kept
        assert "a" in srv._resident[0] and not e_a.closed
        srv._private[0].clear()
        e_c, _ = srv._engine_for(0, Request(3, "c", z, x))      # now the least recently used goes
        assert srv._owner["c"] == 0 and len(srv._resident[0]) == 1 and e_a.closed and e_b.closed
    finally:
        srv.close()


class FakeProfileContext:
    """Per-engine region records: each energy adds one eri_jk call of 2 ms."""
    def __init__(self):
        self.calls = 0

    def profile(self, enable):
        self.calls = 0

    def profile_region(self, name):
        return (self.calls, 2.0 * self.calls) if name == "eri_jk" else (0, 0.0)


class ProfiledEngine(FakeEngine):
    def __init__(self, request):
        super().__init__(request)
        self.ctx = FakeProfileContext()

    def energy(self, coordinates_bohr, do_gradients=True):
        self.ctx.calls += 1
        return super().energy(coordinates_bohr, do_gradients)


def test_profile_totals_count_resident_engines_once_and_reset_drops_earlier_work():
    rng = np.random.default_rng(5)
    srv = GPUServer(n_slots=2, engine_factory=lambda r: ProfiledEngine(r), free_memory=lambda: None, profile=True)
    try:
        for r in _requests(3, 1, rng):     # warm-up traffic, some of it left resident
            srv.submit(r)
        assert srv.drain(timeout=30)
        srv.reset_profile()
        assert srv.profile_totals()["eri_jk"] == [0, 0.0]
        reqs = [Request(100 + k, "new%d" % k, [8, 1, 1], rng.normal(size=(3, 3))) for k in range(5)]
        for r in reqs:
            srv.submit(r)
        assert srv.drain(timeout=30)
        assert all(r.error is None for r in reqs)
        assert srv.profile_totals()["eri_jk"] == [5, 10.0]
    finally:
        srv.close()
