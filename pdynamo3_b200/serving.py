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


def _out_of_memory(exc):
    """A library allocation failure (PDG_ERR_ALLOC) or a CUDA out-of-memory report."""
    status = getattr(exc, "status", None)
    return status == 3 or "out of memory" in str(exc) or "allocation" in str(exc)


class RequestCancelled(Exception):
    """The request was withdrawn with GPUServer.cancel before it started."""


def _device_free_bytes(device):
    """Free device memory from the CUDA runtime (cudaMemGetInfo)."""
    try:
        import torch
        free, _ = torch.cuda.mem_get_info(device)
        return int(free)
    except Exception:
        return None


def memory_need(n_atoms, n_functions, grid_points_per_atom=75 * 302, significant_per_block=120):
    """Rough device bytes one request needs: n^2 work matrices and DIIS history, the grid, and the
    resident basis values (4 values per point for each function significant on its 128-point
    block, at most significant_per_block of them)."""
    n2 = 8.0 * n_functions * n_functions
    points = n_atoms * grid_points_per_atom
    values = 4 * 8.0 * points * max(1.0, min(float(n_functions), significant_per_block))
    return int(30 * n2 + 48.0 * points + values + (64 << 20))


def _functions_estimate(atomic_numbers):
    """Cartesian 6-31G*-size basis: 15 functions per first-row atom, 2 per hydrogen."""
    z = np.asarray(atomic_numbers)
    return int(15 * np.count_nonzero(z > 2) + 2 * np.count_nonzero(z <= 2))


class GPUServer:
    """Continuous-batching server.  ``engine_options`` go to GPUQCEngine (basis, functional, grid,
    converger tolerances); ``precision_mode``/``mixed_cut`` to the ERI options of every engine."""

    REGIONS = ("eri_jk", "eri_grad", "oneint", "oneint_grad", "xc_rho", "xc_vxc", "xc_grad", "xc_weight_grad",
               "pairs", "grid_build", "scf_diag")

    def __init__(self, n_slots=4, device=0, resident_per_slot=4, memory_reserve=2 << 30, precision_mode=0,
                 mixed_cut=1.0e-6, engine_factory=None, free_memory=None, profile=False, **engine_options):
        self.n_slots = n_slots
        self.device = device
        self.resident_per_slot = resident_per_slot
        self.memory_reserve = memory_reserve
        self.precision_mode = precision_mode
        self.mixed_cut = mixed_cut
        self.engine_options = engine_options
        self._custom_factory = engine_factory is not None
        self.engine_factory = engine_factory or self._make_engine
        self.free_memory = free_memory or (lambda: _device_free_bytes(device))
        # library contexts owned by the server, reused by the engines of one slot after another:
        # their device buffers and cached atomic guesses carry over, and no context is created or
        # destroyed (cudaFree synchronises every stream) while other slots run
        self._spare = [[] for _ in range(n_slots)]
        self._contexts = []
        self._ctx_slot = {}
        # profile: per-region device times of every engine, summed when the engine is released
        self.profile = profile
        self.regions = {name: [0, 0.0] for name in self.REGIONS}
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
    def _make_engine(self, request, context=None):
        e = GPUQCEngine(request.atomic_numbers, device=self.device, context=context, **self.engine_options)
        if self.precision_mode:
            e.ctx.set_eri_options(precision_mode=self.precision_mode, mixed_cut=self.mixed_cut)
        if self.profile:
            e.ctx.profile(True)
        return e

    def _release(self, engine):
        """Close an engine, first adding its region times when profiling."""
        if self.profile and getattr(engine, "ctx", None) is not None:
            try:
                add = {name: engine.ctx.profile_region(name) for name in self.REGIONS}
                with self._lock:
                    for name, (c, t) in add.items():
                        self.regions[name][0] += c
                        self.regions[name][1] += t
            except Exception:  # instrumentation never fails a request
                pass
        ctx = getattr(engine, "ctx", None)
        reuse = ctx is not None and not getattr(engine, "_owns_ctx", True)
        engine.close()
        if reuse:
            with self._lock:
                self._spare[self._ctx_slot.get(id(ctx), 0)].append(ctx)

    def _engine_for(self, slot, request):
        res = self._resident[slot]
        e = res.get(request.system)
        if e is not None and np.array_equal(e.atomic_numbers, request.atomic_numbers):
            res.move_to_end(request.system)
            return e, True
        if e is not None:
            self._release(e)
            del res[request.system]
        free = self.free_memory()
        if free is not None and not self._custom_factory:
            need = memory_need(len(request.atomic_numbers), _functions_estimate(request.atomic_numbers))
            if free - need < self.memory_reserve:
                # the device is short of memory for a new system: this slot gives back what it
                # keeps resident (other systems, spare contexts) before building one
                self._shrink_slot(slot, keep=None)
        e = self._new_engine(slot, request)
        res[request.system] = e
        with self._lock:
            # the slot now holds this system's engine: its follow-ups come here
            self._owner[request.system] = slot
        while len(res) > self.resident_per_slot:
            with self._lock:
                # least recently used first; a system with requests still queued on this slot stays
                queued = {r.system for r in self._private[slot]}
                key = next((k for k in res if k != request.system and k not in queued), None)
                if key is None:
                    break
                if self._owner.get(key) == slot:
                    del self._owner[key]
            self._release(res.pop(key))
        return e, False

    def _new_engine(self, slot, request):
        if self._custom_factory:
            return self.engine_factory(request)
        with self._lock:
            ctx = self._spare[slot].pop() if self._spare[slot] else None
        if ctx is None:
            from .lib import Context
            ctx = Context(self.device)
            with self._lock:
                self._contexts.append(ctx)
                self._ctx_slot[id(ctx)] = slot
        return self._make_engine(request, context=ctx)

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

    def cancel(self, request):
        """Withdraw a request that has not started: it leaves the queue with error
        RequestCancelled and its done event set.  A request already on the GPU runs to its end (a
        kernel is never interrupted); returns False then."""
        with self._lock:
            for q in [self._shared] + self._private:
                try:
                    q.remove(request)
                except ValueError:
                    continue
                request.error = RequestCancelled("request %r cancelled before it started" % (request.id,))
                request.end = time.perf_counter()
                request.done.set()
                self._lock.notify_all()
                return True
        return False

    def _fits(self, request):
        free = self.free_memory()
        if free is None:
            return True
        need = memory_need(len(request.atomic_numbers), _functions_estimate(request.atomic_numbers))
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
                need = memory_need(len(r.atomic_numbers), _functions_estimate(r.atomic_numbers))
                self._inflight_bytes += need
            r.slot = slot
            r.start = time.perf_counter()
            try:
                try:
                    engine, r.warm = self._engine_for(slot, r)
                    r.result = engine.energy(r.coordinates_bohr, do_gradients=r.do_gradients)
                except Exception as exc:
                    if not _out_of_memory(exc):
                        raise
                    # device memory ran out: give back this slot's other resident systems and
                    # spare contexts, then run the request once more from a cold start
                    self._shrink_slot(slot, keep=r.system)
                    engine, r.warm = self._engine_for(slot, r)
                    getattr(engine, "forget_density", lambda: None)()
                    r.result = engine.energy(r.coordinates_bohr, do_gradients=r.do_gradients)
            except Exception as exc:  # reported on the request, the slot carries on
                r.error = exc
            r.end = time.perf_counter()
            with self._lock:
                self._busy[slot] = False
                self._inflight_bytes -= need
                self._lock.notify_all()
            r.done.set()

    def _shrink_slot(self, slot, keep=None):
        """Release every resident engine of the slot except `keep`, and destroy its spare contexts."""
        res = self._resident[slot]
        for key in [k for k in res if k != keep]:
            with self._lock:
                if self._owner.get(key) == slot:
                    del self._owner[key]
            self._release(res.pop(key))
        with self._lock:
            spare, self._spare[slot] = self._spare[slot], []
            for ctx in spare:
                self._contexts.remove(ctx)
        for ctx in spare:
            ctx.close()

    def reset_profile(self):
        """Zero the region sums and restart the records of the resident engines (call while idle)."""
        with self._lock:
            for name in self.regions:
                self.regions[name] = [0, 0.0]
            engines = [e for res in self._resident for e in res.values()]
        if self.profile:
            for e in engines:
                try:
                    if getattr(e, "ctx", None) is not None:
                        e.ctx.profile(True)
                except Exception:  # instrumentation never fails the server
                    pass

    def profile_totals(self):
        """Region (calls, total ms) over released and resident engines since the last reset (call
        while idle)."""
        with self._lock:
            out = {name: list(v) for name, v in self.regions.items()}
            engines = [e for res in self._resident for e in res.values()]
        if self.profile:
            for e in engines:
                if getattr(e, "ctx", None) is None:
                    continue
                try:
                    add = {name: e.ctx.profile_region(name) for name in self.REGIONS}
                except Exception:  # instrumentation never fails the server
                    continue
                for name, (c, t) in add.items():
                    out[name][0] += c
                    out[name][1] += t
        return out

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
                self._release(e)
            res.clear()
        for ctx in self._contexts:
            ctx.close()
        self._contexts = []
        self._spare = [[] for _ in range(self.n_slots)]


def latency_summary(requests):
    """p50 / p99 latency (s) and throughput (requests/s) of finished requests."""
    lat = np.array([r.latency for r in requests if r.latency is not None])
    if lat.size == 0:
        return {"p50_s": None, "p99_s": None, "throughput": 0.0, "completed": 0}
    t0 = min(r.arrival for r in requests)
    t1 = max(r.end for r in requests if r.end is not None)
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "throughput": float(lat.size / max(t1 - t0, 1e-12)), "completed": int(lat.size)}


__all__ = ["GPUServer", "Request", "RequestCancelled", "latency_summary", "memory_need"]
