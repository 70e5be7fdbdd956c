"""Many-molecule workloads: a batch of uneven organic molecules and a served request stream.

* ``batch_molecules(n, seed)``: closed-shell neutral saturated trees of 4-24 heavy atoms (C/N/O
  70/15/15, geometry.organic_molecule), the batch shape of pDynamo3 users who screen many
  molecules.
* ``run_batch``: every molecule's B3LYP/6-31G* energy+gradient through the continuous-batching
  server, FP64 and mixed precision side by side, with per-molecule energy and gradient error of the
  mixed form against FP64.
* ``run_stream``: Poisson arrivals of requests drawn from organic molecules and water clusters,
  each followed by a chain of follow-ups at geometries displaced by 0.01 A Gaussian noise that are
  submitted when their predecessor returns (MD steps, path images); p50/p99 latency and throughput.
"""
import threading
import time

import numpy as np

from . import geometry
from .qcmodel import ANGSTROM_TO_BOHR
from .serving import GPUServer, Request, latency_summary


def batch_molecules(n, seed=0, heavy=(4, 24)):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nh = int(rng.integers(heavy[0], heavy[1] + 1))
        z, x = geometry.organic_molecule(nh, seed * 100003 + i)
        out.append(("mol%d" % i, z, x * ANGSTROM_TO_BOHR))
    return out


def _serve_all(molecules, n_slots, precision_mode, options):
    srv = GPUServer(n_slots=n_slots, precision_mode=precision_mode, **options)
    reqs = []
    try:
        t0 = time.perf_counter()
        for i, (name, z, x) in enumerate(molecules):
            reqs.append(srv.submit(Request(i, name, z, x)))
        srv.drain()
        wall = time.perf_counter() - t0
    finally:
        srv.close()
    return reqs, wall


def run_batch(molecules, n_slots=4, warmup=2, options=None):
    """Returns a dict with FP64 and mixed throughput, latencies and the mixed-vs-FP64 errors."""
    import torch
    options = dict(orbital_basis="6-31g_st_cart", functional="b3lyp", grid_accuracy=3, density_tolerance=1e-8,
                   **(options or {}))
    out = {}
    results = {}
    for mode, label in ((0, "fp64"), (1, "mixed")):
        if warmup:
            _serve_all(molecules[:warmup], min(n_slots, warmup), mode, options)
        torch.cuda.synchronize()
        reqs, wall = _serve_all(molecules, n_slots, mode, options)
        torch.cuda.synchronize()
        errors = [r.error for r in reqs if r.error is not None]
        summ = latency_summary(reqs)
        out[label] = {"wall_s": wall, "energy_grad_per_s": len(reqs) / wall, "p50_s": summ["p50_s"],
                      "p99_s": summ["p99_s"], "failed": len(errors),
                      "not_converged": sum(1 for r in reqs if r.result is not None and not r.result.converged)}
        results[label] = reqs
    de, dg = [], []
    for a, b in zip(results["fp64"], results["mixed"]):
        if (a.result is not None and b.result is not None and a.result.converged and b.result.converged
                and a.result.gradients is not None and b.result.gradients is not None):
            de.append(abs(a.result.energy - b.result.energy))
            dg.append(float(np.abs(a.result.gradients - b.result.gradients).max()) * ANGSTROM_TO_BOHR)
    out["mixed_vs_fp64"] = {"max_abs_dE_hartree": max(de) if de else None,
                            "max_abs_dgrad_hartree_per_A": max(dg) if dg else None,
                            "speedup": out["fp64"]["wall_s"] / out["mixed"]["wall_s"]}
    return out


def run_stream(n_requests, rate_per_s, n_slots=4, precision_mode=1, seed=0, max_follow_ups=20, heavy=(4, 12),
               waters=(4, 12), options=None, resident_per_slot=2):
    """Poisson arrivals at ``rate_per_s``; each arrival starts a chain of 1..max_follow_ups
    follow-ups (submitted when the previous link returns).  ``n_requests`` counts every link."""
    options = dict(orbital_basis="6-31g_st_cart", functional="b3lyp", grid_accuracy=3, density_tolerance=1e-8,
                   **(options or {}))
    rng = np.random.default_rng(seed)
    srv = GPUServer(n_slots=n_slots, precision_mode=precision_mode, resident_per_slot=resident_per_slot, **options)
    done_reqs, lock = [], threading.Lock()
    remaining = [n_requests]
    chains = []

    def chain(cid, z, x, links):
        # one MD-like trajectory: each link waits for its predecessor
        crng = np.random.default_rng(seed * 1000003 + cid)
        for k in range(links):
            with lock:
                if remaining[0] <= 0:
                    return
                remaining[0] -= 1
            xr = x + (0.01 * ANGSTROM_TO_BOHR) * crng.normal(size=x.shape) * (k > 0)
            r = srv.submit(Request(len(done_reqs), "chain%d" % cid, z, xr))
            r.done.wait()
            with lock:
                done_reqs.append(r)
            x = xr

    t0 = time.perf_counter()
    cid = 0
    try:
        while True:
            with lock:
                if remaining[0] <= 0:
                    break
            if rng.random() < 0.5:
                z, x = geometry.organic_molecule(int(rng.integers(heavy[0], heavy[1] + 1)), seed * 7919 + cid)
            else:
                nw = int(rng.integers(waters[0], waters[1] + 1))
                z, x = geometry.water_cluster(nw, 3.2 * nw ** (1.0 / 3.0), seed * 7919 + cid)
            links = 1 + int(rng.integers(1, max_follow_ups + 1))
            t = threading.Thread(target=chain, args=(cid, z, x * ANGSTROM_TO_BOHR, links), daemon=True)
            t.start()
            chains.append(t)
            cid += 1
            time.sleep(rng.exponential(1.0 / rate_per_s))
        for t in chains:
            t.join()
        wall = time.perf_counter() - t0
    finally:
        srv.close()
    summ = latency_summary(done_reqs)
    errors = sorted({str(r.error)[:160] for r in done_reqs if r.error is not None})
    summ.update({"wall_s": wall, "requests": len(done_reqs), "chains": cid,
                 "failed": sum(1 for r in done_reqs if r.error is not None), "errors": errors[:5],
                 "warm_fraction": float(np.mean([r.warm for r in done_reqs])) if done_reqs else 0.0})
    return summ
