"""Failure handling of the continuous-batching server on the host, with stand-in engines (no GPU):
a request whose engine fails (device allocation failure, after the one retry the server makes with
the slot's other resident systems released; a non-finite value; an SCF that reaches its iteration
limit) reports the failure on that request alone and the slot carries on with the
rest of the batch, whose results are unchanged; queued requests can be cancelled mid-batch.  These
mirror the reference's behaviour of raising on a non-OK Status (GaussianBasisIntegralEvaluator.pyx:
418,458) and on SCF failure (QCModelBase.py:184) for the one energy call concerned."""
import threading
import time

import numpy as np
import pytest

from pdynamo3_b200.lib import PDG_ERR_ALLOC, PDG_ERR_NAN, PDGError
from pdynamo3_b200.serving import GPUServer, Request, RequestCancelled


class Result:
    def __init__(self, x, converged=True):
        self.energy = float(np.sum(x))
        self.gradients = np.ones_like(x)
        self.converged = converged


class Engine:
    """Fails by system key: 'alloc' raises the allocation status, 'nan' the non-finite status,
    'noconv' returns an unconverged result; others return sum(x).  gate: an event the engine waits
    on before its first request (to hold a slot busy)."""
    gate = None

    def __init__(self, request):
        self.atomic_numbers = request.atomic_numbers
        self.key = request.system

    def energy(self, x, do_gradients=True):
        if Engine.gate is not None:
            Engine.gate.wait(10)
        time.sleep(0.001)
        if self.key.startswith("alloc"):
            raise PDGError(PDG_ERR_ALLOC, "device allocation of 1 bytes failed")
        if self.key.startswith("nan"):
            raise PDGError(PDG_ERR_NAN, "pdg_scf_run: non-finite energy")
        return Result(np.asarray(x), converged=not self.key.startswith("noconv"))

    def close(self):
        pass


def _server(n=2):
    return GPUServer(n_slots=n, resident_per_slot=2, engine_factory=Engine, free_memory=lambda: None)


def test_failing_requests_are_isolated_and_the_batch_is_unchanged():
    Engine.gate = None
    z = np.array([1, 1])
    keys = ["m0", "alloc1", "m2", "nan3", "m4", "noconv5", "m6", "m7"]
    xs = [np.full((2, 3), 0.1 * (i + 1)) for i in range(len(keys))]
    srv = _server(3)
    try:
        reqs = [srv.submit(Request(i, k, z, x)) for i, (k, x) in enumerate(zip(keys, xs))]
        assert srv.drain(timeout=30)
    finally:
        srv.close()
    alone = {}
    for i, k in enumerate(keys):
        if k.startswith("m"):
            alone[i] = Engine(Request(i, k, z, xs[i])).energy(xs[i]).energy
    for i, r in enumerate(reqs):
        assert r.done.is_set()
        if keys[i].startswith("alloc"):
            assert isinstance(r.error, PDGError) and r.error.status == PDG_ERR_ALLOC
        elif keys[i].startswith("nan"):
            assert isinstance(r.error, PDGError) and r.error.status == PDG_ERR_NAN
        elif keys[i].startswith("noconv"):
            assert r.error is None and not r.result.converged
        else:
            assert r.error is None and r.result.converged and r.result.energy == alone[i]


def test_cancellation_mid_batch_leaves_the_rest_unchanged():
    z = np.array([1, 1])
    Engine.gate = threading.Event()          # hold the single slot on its first request
    srv = _server(1)
    try:
        reqs = [srv.submit(Request(i, "m%d" % i, z, np.full((2, 3), float(i)))) for i in range(6)]
        time.sleep(0.05)
        assert not srv.cancel(reqs[0]) or reqs[0].error is not None    # the first may already run
        assert srv.cancel(reqs[2]) and srv.cancel(reqs[4])
        Engine.gate.set()
        assert srv.drain(timeout=30)
    finally:
        Engine.gate = None
        srv.close()
    for i, r in enumerate(reqs):
        assert r.done.is_set()
        if i in (2, 4):
            assert isinstance(r.error, RequestCancelled) and r.result is None
        else:
            assert r.error is None and r.result.energy == pytest.approx(6.0 * i)


def test_out_of_memory_releases_the_slot_and_retries_once():
    """A request that runs out of device memory gets the slot's other resident systems released
    and runs once more; it succeeds when the memory they held was what it lacked."""
    z = np.array([1, 1])
    state = {"resident_released": False}

    class Tight(Engine):
        def energy(self, x, do_gradients=True):
            if self.key == "big" and not state["resident_released"]:
                raise PDGError(PDG_ERR_ALLOC, "device allocation of 8 GB failed")
            return Result(np.asarray(x))

        def close(self):
            if self.key != "big":
                state["resident_released"] = True

    srv = GPUServer(n_slots=1, resident_per_slot=4, engine_factory=Tight, free_memory=lambda: None)
    try:
        small = [srv.submit(Request(i, "s%d" % i, z, np.full((2, 3), 1.0))) for i in range(3)]
        assert srv.drain(timeout=30)
        big = srv.submit(Request(9, "big", z, np.full((2, 3), 2.0)))
        assert srv.drain(timeout=30)
    finally:
        srv.close()
    assert all(r.error is None for r in small)
    assert big.error is None and big.result.energy == pytest.approx(12.0)
    assert state["resident_released"]
