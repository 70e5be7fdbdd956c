"""The continuous-batching server on the GPU: every request's result is the same alone (one slot,
one request at a time, cold start) and in the mix (three slots running concurrently on separate
streams, follow-ups routed to their resident system and warm-started), to 1e-8 hartree in energy
and 1e-6 hartree/bohr in gradient (FP64, SCF converged to 1e-10 in the density)."""
import numpy as np
import pytest

from conftest import ANGSTROM_TO_BOHR
from pdynamo3_b200 import geometry
from pdynamo3_b200.serving import GPUServer, Request, latency_summary

pytestmark = pytest.mark.gpu

OPTIONS = dict(orbital_basis="6-31g_st_cart", functional="b3lyp", grid_accuracy=2, density_tolerance=1e-10,
               energy_tolerance=1e-9)


def _workload():
    systems = []
    for k, nh in enumerate((3, 4, 5)):
        z, x = geometry.organic_molecule(nh, 100 + k)
        systems.append(("mol%d" % k, z, x * ANGSTROM_TO_BOHR))
    z, x = geometry.water_cluster(3, 4.5, 7)
    systems.append(("water3", z, x * ANGSTROM_TO_BOHR))
    rng = np.random.default_rng(5)
    reqs = []
    for name, z, x in systems:
        for f in range(3):  # a request and two follow-ups at displaced geometries
            reqs.append((name, z, x + (0.01 * ANGSTROM_TO_BOHR) * f * rng.normal(size=x.shape)))
    return reqs


def _run(n_slots, work, one_at_a_time):
    srv = GPUServer(n_slots=n_slots, **OPTIONS)
    out = []
    try:
        for i, (name, z, x) in enumerate(work):
            r = srv.submit(Request(i, name if not one_at_a_time else "%s/%d" % (name, i), z, x))
            if one_at_a_time:
                r.done.wait(300)
            out.append(r)
        assert srv.drain(timeout=600)
    finally:
        srv.close()
    for r in out:
        assert r.error is None, r.error
        assert r.result.converged
    return out


def test_results_are_the_same_alone_and_in_the_mix(cuda_device):
    work = _workload()
    alone = _run(1, work, one_at_a_time=True)
    mixed = _run(3, work, one_at_a_time=False)
    assert len({r.slot for r in mixed}) > 1
    assert any(r.warm for r in mixed)
    for a, m in zip(alone, mixed):
        assert abs(a.result.energy - m.result.energy) < 1e-8
        assert np.abs(a.result.gradients - m.result.gradients).max() < 1e-6
    s = latency_summary(mixed)
    assert s["completed"] == len(work) and s["p99_s"] >= s["p50_s"] > 0.0
