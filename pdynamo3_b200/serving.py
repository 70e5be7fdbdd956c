"""Continuous-batching energy+gradient server on one GPU.

Requests (an atomic-number/coordinate pair plus a system key) arrive at any time.  The server
keeps ``n_slots`` worker slots, each a host thread driving its own library context, so its own
CUDA stream: while one request is in its SCF on the device another slot's request is in its grid
build or its gradient, and the device overlaps them.  A request is admitted to a slot when the
slot is free and the device has room for it (``memory_need`` against the free device memory less
a reserve); otherwise it waits in the queue.  Each slot keeps the engines of the systems it has
served resident (basis, grid buffers, last converged density) up to ``resident_per_slot``, and a
follow-up request of a resident system is routed to that slot, where its SCF starts from the
previous density (MD steps, optimisation steps, chain-of-states images).

This is the serving form of the callers pDynamo3 drives through ``SGOFProcessPool``
(pSimulation/SGOFProcessPool.py:20-230): many independent energy+gradient evaluations.  Results
do not depend on what else runs: each request's arithmetic is the same alone and in the mix.
"""
import collections
import threading
import time

import numpy as np

from .qcmodel import GPUQCEngine


class Request:
    """One energy+gradient request.  ``system`` keys the resident state (same atoms, new geometry)."""

    __slots__ = ("id", "system", "atomic_numbers", "coordinates_bohr", "do_gradients", "arrival", "start", "end",
                 "slot", "result", "error", "done", "warm")

    def __init__(self, rid, system, atomic_numbers, coordinates_bohr, do_gradients=True):
        self.id = rid
        self.system = system
        self.atomic_numbers = np.asarray(atomic_numbers, dtype=np.int32)
        self.coordinates_bohr = np.ascontiguousarray(coordinates_bohr, dtype=np.float64)
        self.do_gradients = do_gradients
        self.arrival = self.start = self.end = None
        self.slot = None
        self.result = None
        self.error = None
        self.warm = False
        self.done = threading.Event()

    @property
    def latency(self):
        return None if self.end is None else self.end - self.arrival


def _device_free_bytes(device):
    """Free device memory from the CUDA runtime (cudaMemGetInfo)."""
    try:
        import torch
        free, _ = torch.cuda.mem_get_info(device)
        return int(free)
    except Exception:
        return None


def memory_need(n_atoms, n_functions, grid_points_per_atom=75 * 302, significant_fraction=0.35):
    """Rough device bytes one request needs: n^2 work matrices and DIIS history, the grid, and the
    resident basis values (4 values per significant function and point)."""
    n2 = 8.0 * n_functions * n_functions
    points = n_atoms * grid_points_per_atom
    values = 4 * 8.0 * points * max(1.0, significant_fraction * n_functions)
    return int(30 * n2 + 48.0 * points + values + (64 << 20))


class GPUServer:
    """Continuous-batching server.  ``engine_options`` go to GPUQCEngine (basis, functional, grid,
    converger tolerances); ``precision_mode``/``mixed_cut`` to the ERI options of every engine."""

    def __init__(self, n_slots=4, device=0, resident_per_slot=4, memory_reserve=2 << 30, precision_mode=0,
                 mixed_cut=1.0e-6, engine_factory=None, free_memory=None, **engine_options):
        self.n_slots = n_slots
        self.device = device
        self.resident_per_slot = resident_per_slot
        self.memory_reserve = memory_reserve
        self.precision_mode = precision_mode
        self.mixed_cut = mixed_cut
        self.engine_options = engine_options
        self.engine_factory = engine_factory or self._make_engine
        self.free_memory = free_memory or (lambda: _device_free_bytes(device))
        self._lock = threading.Condition()
        self._shared = collections.deque()                  # requests of systems resident nowhere
        self._private = [collections.deque() for _ in range(n_slots)]
        self._owner = {}                                    # system key -> slot holding its engine
        self._resident = [collections.OrderedDict() for _ in range(n_slots)]
        self._busy = [False] * n_slots
        self._inflight_bytes = 0
        self._stop = False
        self._threads = [threading.Thread(target=self._worker, args=(k,), daemon=True) for k in range(n_slots)]
        for t in self._threads:
            t.start()

    # ---- engines ----
    def _make_engine(self, request):
        e = GPUQCEngine(request.atomic_numbers, device=self.device, **self.engine_options)
        if self.precision_mode:
            e.ctx.set_eri_options(precision_mode=self.precision_mode, mixed_cut=self.mixed_cut)
        return e

    def _engine_for(self, slot, request):
        res = self._resident[slot]
        e = res.get(request.system)
        if e is not None and np.array_equal(e.atomic_numbers, request.atomic_numbers):
            res.move_to_end(request.system)
            return e, True
        if e is not None:
            e.close()
            del res[request.system]
        e = self.engine_factory(request)
        res[request.system] = e
        while len(res) > self.resident_per_slot:
            key, old = res.popitem(last=False)
            old.close()
            with self._lock:
                if self._owner.get(key) == slot:
                    del self._owner[key]
        return e, False

    # ---- admission ----
    def submit(self, request):
        request.arrival = time.perf_counter()
        with self._lock:
            owner = self._owner.get(request.system)
            if owner is not None:
                self._private[owner].append(request)
            else:
                self._shared.append(request)
            self._lock.notify_all()
        return request

    def _fits(self, request):
        free = self.free_memory()
        if free is None:
            return True
        need = memory_need(len(request.atomic_numbers), 15 * len(request.atomic_numbers))
        return free - self._inflight_bytes - need >= self.memory_reserve or self._inflight_bytes == 0

    def _take(self, slot):
        """Next request for this slot: its own resident systems first, then the shared queue."""
        if self._private[slot]:
            return self._private[slot].popleft()
        for _ in range(len(self._shared)):
            r = self._shared[0]
            owner = self._owner.get(r.system)
            if owner is not None and owner != slot:
                self._shared.popleft()
                self._private[owner].append(r)
                continue
            if not self._fits(r):
                return None
            self._shared.popleft()
            self._owner[r.system] = slot
            return r
        return None

    def _worker(self, slot):
        while True:
            with self._lock:
                while True:
                    if self._stop:
                        return
                    r = self._take(slot)
                    if r is not None:
                        break
                    self._lock.wait(0.05)
                self._busy[slot] = True
                need = memory_need(len(r.atomic_numbers), 15 * len(r.atomic_numbers))
                self._inflight_bytes += need
            r.slot = slot
            r.start = time.perf_counter()
            try:
                engine, r.warm = self._engine_for(slot, r)
                r.result = engine.energy(r.coordinates_bohr, do_gradients=r.do_gradients)
            except Exception as exc:  # reported on the request, the slot carries on
                r.error = exc
            r.end = time.perf_counter()
            with self._lock:
                self._busy[slot] = False
                self._inflight_bytes -= need
                self._lock.notify_all()
            r.done.set()

    def drain(self, timeout=None):
        """Wait until every submitted request has finished."""
        t0 = time.perf_counter()
        while True:
            with self._lock:
                idle = not any(self._busy) and not self._shared and not any(self._private)
            if idle:
                return True
            if timeout is not None and time.perf_counter() - t0 > timeout:
                return False
            time.sleep(0.002)

    def close(self):
        with self._lock:
            self._stop = True
            self._lock.notify_all()
        for t in self._threads:
            t.join()
        for res in self._resident:
            for e in res.values():
                e.close()
            res.clear()


def latency_summary(requests):
    """p50 / p99 latency (s) and throughput (requests/s) of finished requests."""
    lat = np.array([r.latency for r in requests if r.latency is not None])
    if lat.size == 0:
        return {"p50_s": None, "p99_s": None, "throughput": 0.0, "completed": 0}
    t0 = min(r.arrival for r in requests)
    t1 = max(r.end for r in requests if r.end is not None)
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "throughput": float(lat.size / max(t1 - t0, 1e-12)), "completed": int(lat.size)}


__all__ = ["GPUServer", "Request", "latency_summary", "memory_need"]
