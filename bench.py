#!/usr/bin/env python
"""Benchmark: PBE/6-31G* (Cartesian) energy + analytic gradient of a 16-water cluster on one B200.

Workload (the configuration the headline metric is quoted on): 16 rigid waters placed by seeded
rejection sampling in an 8 A cube (48 atoms, 304 Cartesian basis functions), PBE with a
75 radial x 302 Lebedev grid per atom (Becke-partitioned, ~1.1M points before weight screening),
SCF from the core-Hamiltonian guess to 1e-8 RMS density change, then the full analytic gradient
(one-electron, two-electron, XC and grid-weight terms).  All arithmetic is FP64.  One step is one
complete energy+gradient of a fresh geometry (seed = step index), so nothing is reused between
steps except the basis definition.

Arms:
  default            the pdgpu C-ABI library (pdynamo3_b200/lib/libpdgpu.so) on cuda:LOCAL_RANK.
  --impl reference   the CPU path: the oracle's restatement of the reference's FP64 two-electron
                     code (oracle/oracle.c) on all host cores, on a bounded sample of shell quartets
                     of the same workload, extrapolated to one energy+gradient (see cpu_sample()).
Under torchrun every rank runs its own replica (independent molecules, no collective); the
job value is the sum over ranks, the time the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

ANG = 1.0e-10 / 5.291772083e-11
N_WATERS, BOX, FUNCTIONAL, GRID = 16, 8.0, "pbe", (3, 75, 29)
METRIC = "SCF energy+gradient/s (PBE/6-31G*, 16 H2O, FP64)"
UNIT = "energy+grad/s"


def workload_config(extra=None):
    cfg = {"workload": "PBE/6-31G*(6d) energy+gradient, 16-water cluster in 8 A cube, 75x302 grid, SCF to 1e-8",
           "n_atoms": 3 * N_WATERS, "basis_functions": 304, "grid": "75 radial x 302 Lebedev (Becke)",
           "l2": "working set larger than L2 (resident basis values ~GBs); no flush needed"}
    if extra:
        cfg.update(extra)
    return cfg


def dist_info():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        # the raw samples go to a scratch file (its summary goes into the JSON line); PDG_CLOCKS_DIR
        # keeps them somewhere else
        self.path = os.path.join(os.environ.get("PDG_CLOCKS_DIR", tempfile.gettempdir()), "pdgpu_bench_clocks_%d.csv" % index)

    def start(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap,utilization.gpu")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons, util = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
            if len(parts) > 9:
                try:
                    util.append(float(parts[9]))
                except ValueError:
                    pass
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "gpu_busy_pct_median": float(np.median(util)) if util else None}


def max_over_ranks(values, world, device):
    """Element-wise maximum over the ranks of the job (each rank times its own replica)."""
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.barrier()
    return [float(v) for v in t]


def job_throughput(steps_per_rank, world, max_seconds):
    """Whole-job units per second: every rank's steps over the slowest rank's time."""
    return steps_per_rank * world / max_seconds


def make_context(device, precision="fp64"):
    from pdynamo3_b200 import geometry
    from pdynamo3_b200.basis import ShellTable
    from pdynamo3_b200.lib import Context
    z, _ = geometry.water_cluster(N_WATERS, BOX, 0)
    ctx = Context(device)
    ctx.set_basis(ShellTable("6-31g_st_cart", z))
    ctx.set_functional(FUNCTIONAL)
    if precision == "mixed":
        ctx.set_eri_options(precision_mode=1, mixed_cut=1e-6)
    return ctx


def geometry_for(step):
    from pdynamo3_b200 import geometry
    z, xyz = geometry.water_cluster(N_WATERS, BOX, 1000 + step)
    return xyz * ANG


def energy_gradient(ctx, coords):
    """One complete energy + gradient through the C-ABI with host buffers (coordinates in,
    density, energies and gradients out)."""
    ctx.set_geometry(coords)
    ctx.grid_build(*GRID)
    P, res = ctx.scf(density_tolerance=1e-8, maximum_iterations=100)
    g = ctx.scf_gradients()
    return P, res, g


def run_gpu(args):
    import torch
    world, rank, local = dist_info()
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    from pdynamo3_b200 import lib
    ctx = make_context(local, args.precision)
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=local)
    # warm-up (untimed)
    res = None
    for w in range(args.warmup):
        P, res, g = energy_gradient(ctx, geometry_for(-1 - w))
    # timed region
    geoms = [geometry_for(k + rank * 1000) for k in range(args.steps)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local) if rank == 0 else None
    if clocks:
        clocks.start()
    ctx.profile(True)
    l0 = lib.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    iters, energies, h2d, d2h = [], [], 0, 0
    t0 = time.perf_counter()
    ev0.record(stream)
    for k in range(args.steps):
        P, res, g = energy_gradient(ctx, geoms[k])
        iters.append(res.iterations)
        energies.append(res.energy_total)
        h2d += geoms[k].nbytes
        d2h += P.nbytes + g.nbytes + 8 * 6
    ev1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    dev_ms = ev0.elapsed_time(ev1)
    launches = lib.launch_count() - l0
    regions = {}
    for name in ("eri_jk", "eri_grad", "oneint", "oneint_grad", "xc_rho", "xc_vxc", "xc_grad", "xc_weight_grad",
                 "pairs", "grid_build", "scf_diis", "scf_diag"):
        c, t = ctx.profile_region(name)
        regions[name] = {"calls": c, "total_ms": t}
    ctx.profile(False)
    clk = clocks.stop() if clocks else None
    dev_ms, wall = max_over_ranks([dev_ms, wall], world, "cuda")
    if rank == 0:
        value = job_throughput(args.steps, world, dev_ms / 1e3)
        e2e = job_throughput(args.steps, world, wall)
        # roofline of the dominant kernel region
        dom = max(regions, key=lambda n: regions[n]["total_ms"])
        flops, bytes_, quartets = ctx.work_estimate(dom) if dom in ("eri_jk", "eri_grad", "xc_rho", "xc_vxc") else (0, 0, 0)
        calls = max(1, regions[dom]["calls"])
        avg_s = regions[dom]["total_ms"] / calls / 1e3
        full_note = None
        if dom == "eri_jk":
            # The SCF's Coulomb builds are density-screened (difference builds skip most quartets),
            # so their average time does not belong to the full-build FLOP count: time three full,
            # unscreened builds of the last converged density instead (outside the timed region).
            ctx.profile(True)
            for _ in range(3):
                ctx.fock_two_electron(P, 0.0)
            c, t = ctx.profile_region("eri_jk")
            ctx.profile(False)
            calls, avg_s = c, t / max(1, c) / 1e3
            full_note = "full unscreened Coulomb builds of the last converged density (3, after the timed region)"
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
            os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
        # FP64 kernels: the denominator is the FP64 FMA pipe measured on this device (of measured), the
        # measured dense bf16 GEMM rate beside it; HBM-bound kernels use the measured copy bandwidth.
        if dom in ("xc_rho", "xc_vxc") and args.xc_bound == "hbm":
            achieved = bytes_ / avg_s / 1e9
            peak = peaks.get("hbm_gbs", 6650.0)
            roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": None, "peak_source": "MEASURED_PEAKS.json (of measured)" if peaks else "fallback"}
        else:
            achieved = flops / avg_s / 1e12
            peak = lib.measure_fp64_peak(local, 0)
            roof = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                    "traffic": None, "peak_source": "FP64 FMA pipe measured on this device by pdg_measure_fp64_peak "
                                                    "(of measured); DMMA path %.1f TFLOP/s" % lib.measure_fp64_peak(local, 1)}
            if peaks.get("bf16_tflops"):
                roof["bf16_tensor_frac"] = achieved / peaks["bf16_tflops"]
        roof.update({"kernel": dom, "calls": calls, "avg_ms": avg_s * 1e3, "algorithmic_flops_per_call": flops})
        if full_note:
            roof["timed_on"] = full_note
        traffic_file = os.path.join(ROOT, "profiles", "roofline_traffic.json")
        if os.path.exists(traffic_file):
            t = json.load(open(traffic_file)).get(dom)
            if t:
                roof["traffic"] = t["dram_bytes_per_call"]
                roof["traffic_source"] = t["source"]
        # achieved algorithmic FP64 rate of the unscreened regions (the last step's geometry)
        for name in ("eri_grad", "xc_rho", "xc_vxc"):
            r = regions[name]
            if r["calls"]:
                f, b, _ = ctx.work_estimate(name)
                avg = r["total_ms"] / r["calls"] / 1e3
                r["tflops"] = f / avg / 1e12
                if b:
                    r["gbs"] = b / avg / 1e9
        cpu = cpu_sample(ctx, P, res, args) if args.cpu_baseline else None
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f64+f32",
                "data": "synthetic (seeded water clusters)",
                "config": workload_config({"parallelism": "replicas" if world > 1 else "single", "precision": args.precision,
                                           "mean_scf_iterations":
                                           float(np.mean(iters))}),
                "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d // args.steps,
                        "d2h_bytes_per_step": d2h // args.steps},
                "gpu_launches": launches, "roofline": roof, "regions_ms": regions,
                "clocks": clk, "cpu_baseline": cpu}
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def _cpu_worker(job):
    """Time the oracle's two-electron Coulomb Fock build and gradient on one hash slice."""
    import oracle
    from pdynamo3_b200 import geometry
    from pdynamo3_b200.basis import ShellTable
    coords, P, mod, lo, hi = job
    z, _ = geometry.water_cluster(N_WATERS, BOX, 0)
    o = oracle.Oracle(ShellTable("6-31g_st_cart", z), coords)
    L = oracle.lib()
    # the reference's own libcint root routine when it was built (its fitted formulas cost what the
    # reference pays per primitive quartet; the restated Stieltjes rule costs several times more)
    oracle.use_reference_roots(True)
    L.orc_set_sample(mod, lo, hi)
    t0 = time.perf_counter()
    o.fock(P, 0.0, True)
    t1 = time.perf_counter()
    g = np.zeros(3 * o.natom)
    L.orc_eri_gradient(np.ascontiguousarray(P), 0.0, 1, g)
    t2 = time.perf_counter()
    L.orc_set_sample(0, 0, 0)
    return t1 - t0, t2 - t1


def _roots_note():
    import oracle
    return ("Rys roots from the reference's libcint routine built from its sources" if oracle.reference_roots_available()
            else "restated Stieltjes Rys roots (reference libcint build absent; slower than the reference's)")


def cpu_estimate(coords, P, iterations, fraction_slices, cores):
    """Extrapolated CPU seconds for one energy+gradient: iterations x (two-electron Coulomb Fock
    build) + two-electron gradient, from the oracle timed on `fraction_slices` of a 1/MOD hash
    sample of the shell quartets.  XC quadrature, one-electron terms and linear algebra are left
    out, and every cycle's Fock build recomputes its integrals (integral-direct, where the reference's
    conventional path stores them once per geometry), so the figure is an estimate of the two-electron
    CPU time, not a bound on the reference's."""
    mod = 1000
    jobs = [(coords, P, mod, s, s + 1) for s in range(fraction_slices)]
    if cores > 1:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(cores) as pool:
            t0 = time.perf_counter()
            res = pool.map(_cpu_worker, jobs)
            wall = time.perf_counter() - t0
        # parallel wall time of the sample; scale the per-slice work to the full quartet set
        tf = sum(r[0] for r in res) / len(res) * mod
        tg = sum(r[1] for r in res) / len(res) * mod
        serial = iterations * tf + tg
        return serial / cores, wall, serial
    res = [_cpu_worker(j) for j in jobs]
    tf = sum(r[0] for r in res) / len(res) * mod
    tg = sum(r[1] for r in res) / len(res) * mod
    serial = iterations * tf + tg
    return serial, sum(r[0] + r[1] for r in res), serial


def cpu_sample(ctx, P, res, args):
    from oracle import build as ob
    ob.build()
    coords = geometry_for(args.steps - 1 + 0)
    # the density of the last timed step belongs to that geometry
    coords = geometry_for(args.steps - 1)
    est, sample_s, serial = cpu_estimate(coords, P, res.iterations, args.cpu_slices, 1)
    return {"value": 1.0 / est, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": ("oracle two-electron Coulomb Fock build + two-electron gradient on %d/1000 of the shell "
                       "quartets of the last timed geometry (%.1f s of CPU work), extrapolated to %d SCF cycles + 1 "
                       "gradient, integrals recomputed each cycle; XC, one-electron and linear algebra excluded "
                       "(an estimate of the two-electron CPU time, not a bound); %s")
            % (args.cpu_slices, sample_s, res.iterations, _roots_note())}


def run_reference(args):
    world, rank, local = dist_info()
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    # The timed sample needs a density of the right sparsity, not a converged one: the
    # core-Hamiltonian density (an SCF on the CPU would take hours).  The cycle count is the
    # reference DIIS converger's on the fixture molecules (11-15 cycles to 1e-10), taken at the
    # low end so that the extrapolation favours the CPU.
    import oracle
    from pdynamo3_b200 import geometry
    from pdynamo3_b200.basis import ShellTable
    from oracle import build as ob
    ob.build()
    z, xyz = geometry.water_cluster(N_WATERS, BOX, 1000)
    coords = xyz * ANG
    o = oracle.Oracle(ShellTable("6-31g_st_cart", z), coords)
    S, H, _ = o.one_electron()
    Sm, Hm = oracle.unpack(S, o.n), oracle.unpack(H, o.n)
    s, U = np.linalg.eigh(Sm)
    X = U @ np.diag(s ** -0.5) @ U.T
    e, C = np.linalg.eigh(X.T @ Hm @ X)
    C = X @ C
    P = oracle.pack(2 * C[:, :5 * N_WATERS] @ C[:, :5 * N_WATERS].T)
    iterations = 12
    times = []
    for k in range(args.warmup + args.steps):
        est, wall, serial = cpu_estimate(coords, P, iterations, max(cores, args.cpu_slices), cores)
        if k >= args.warmup:
            times.append(est)
    t = float(np.mean(times))
    value = 1.0 / t
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded water clusters)",
            "config": workload_config({"parallelism": "host cores"}),
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": ("oracle (C restatement of the reference's FP64 two-electron code) on %d/1000 of "
                                        "the shell quartets per step across %d processes, extrapolated to %d SCF "
                                        "Coulomb Fock builds + the two-electron gradient, integrals recomputed each "
                                        "cycle; XC, one-electron and linear algebra excluded (an estimate of the "
                                        "two-electron CPU time, not a bound); %s") % (
                                 max(cores, args.cpu_slices), cores, iterations, _roots_note())}}
    print(json.dumps(line), flush=True)


def run_kernel_case(args):
    """Fixed case for kernel profiles: PBE/6-31G* on `--kernel-case` waters (seed 0, in a cube of
    5 A for 4 waters grown with the cube root of the count, 7.9 A at 16)
    with the 75x302 grid; one Coulomb Fock build, one quadrature Fock build and both gradient passes
    from the core-Hamiltonian density (no SCF, so every hot kernel launches a known number of times:
    each ERI class once, rho_xc_kernel twice, vxc_kernel once).  Prints one status line."""
    from pdynamo3_b200 import geometry, workloads
    from pdynamo3_b200.basis import ShellTable
    from pdynamo3_b200.lib import Context
    functional, cx = (FUNCTIONAL if args.kernel_xc else "hf"), 0.0
    if args.kernel_molecule >= 0:
        # molecule `kernel_molecule` of the organic batch, B3LYP: the builds carry exchange
        _, z, coords = workloads.batch_molecules(args.kernel_molecule + 1, seed=1)[args.kernel_molecule]
        functional, cx = ("b3lyp" if args.kernel_xc else "hf"), 0.2
        grid = (3, 0, 0)
    else:
        z, xyz = geometry.water_cluster(args.kernel_case, 5.0 * max(1.0, args.kernel_case / 4.0) ** (1.0 / 3.0), 0)
        coords = xyz * ANG
        grid = GRID
    ctx = Context(0)
    ctx.set_basis(ShellTable("6-31g_st_cart", z))
    ctx.set_geometry(coords)
    if args.precision == "mixed":
        ctx.set_eri_options(precision_mode=1, mixed_cut=1e-6)
    ctx.set_functional(functional)
    npts = ctx.grid_build(*grid) if args.kernel_xc else 0
    S, H, _ = ctx.one_electron()
    n = int((np.sqrt(8 * len(S) + 1) - 1) / 2)

    def unpack(p):
        a = np.zeros((n, n))
        a[np.tril_indices(n)] = p
        return a + np.tril(a, -1).T
    s, U = np.linalg.eigh(unpack(S))
    X = U @ np.diag(s ** -0.5) @ U.T
    e, C = np.linalg.eigh(X @ unpack(H) @ X)
    C = X @ C
    nocc = int(z.sum()) // 2
    P = (2.0 * C[:, :nocc] @ C[:, :nocc].T)[np.tril_indices(n)]
    W = (-2.0 * (C[:, :nocc] * e[:nocc]) @ C[:, :nocc].T)[np.tril_indices(n)]
    F2, E2 = ctx.fock_two_electron(P, cx)
    exc, rho, g2 = 0.0, 0.0, np.zeros(1)
    if args.kernel_xc:
        F, exc, rho = ctx.fock_quadrature(P)
    g1 = ctx.gradients(P, W, cx)
    if args.kernel_xc:
        g2 = ctx.gradients_quadrature(P)
    print("kernel case: %s, %d basis functions, %d grid points, E2 %.10f Exc %.10f rho %.8f |g| %.3e %.3e"
          % ("organic molecule %d (%d atoms)" % (args.kernel_molecule, len(z)) if args.kernel_molecule >= 0
             else "%d waters" % args.kernel_case, n, npts, E2, exc, rho, np.abs(g1).max(), np.abs(g2).max()),
          flush=True)
    ctx.close()



# ---------------------------------------------------------------------------------------------
# The headline workload: the 256-molecule organic batch, the served mixed-precision form against
# the plain FP64 path.
# ---------------------------------------------------------------------------------------------
BATCH_N, BATCH_SEED = 256, 1
BATCH_OPTS = dict(orbital_basis="6-31g_st_cart", functional="b3lyp", grid_accuracy=3, density_tolerance=1e-8)
BATCH_METRIC = ("SCF energy+grad/s, served mixed precision vs plain FP64 (B3LYP/6-31G*, 256 organic molecules of "
                "4-24 heavy atoms, |dE|<=1e-5 Eh); p50/p99 latency")
BATCH_REF_CYCLES = 20   # the reference converger's B3LYP cycle count on the batch fixtures (17 and 20)


def batch_config(extra=None):
    cfg = {"workload": "256 closed-shell organic molecules (seeded saturated C/N/O trees, 4-24 heavy atoms, H-filled), "
                       "B3LYP/6-31G* (Cartesian d), Medium grid, SCF to 1e-8 in the density, energy + analytic gradient",
           "molecules": BATCH_N, "seed": BATCH_SEED,
           "step": "one sub-batch of the 256 molecules, submitted together; the timed steps cover the batch once",
           "l2": "working set larger than L2 (resident basis values of several molecules); no flush needed"}
    if extra:
        cfg.update(extra)
    return cfg


def batch_parts(n_steps, rank):
    from pdynamo3_b200 import workloads
    mols = workloads.batch_molecules(BATCH_N, seed=BATCH_SEED + 1000 * rank)
    parts = [list(map(int, p)) for p in np.array_split(np.arange(len(mols)), max(1, n_steps))]
    return mols, parts


def warm_molecules(rank, count=4):
    """Small molecules of another seed for the untimed warm-up steps."""
    from pdynamo3_b200 import workloads
    out = [m for m in workloads.batch_molecules(48, seed=BATCH_SEED + 1 + 1000 * rank) if int((m[1] > 1).sum()) <= 6]
    return out[:count]


def run_batch_metric(args):
    """Default workload.  Timed: the served mixed-precision form (the value: continuous-batching
    server, args.slots slots on their own streams, FP32 quartets below the Schwarz x density bound
    1e-6) and then the plain FP64 path (one molecule at a time through the drop-in engine), each over
    the same K sub-batches that together are the 256-molecule batch.  Per molecule, the mixed
    result is checked against the FP64 one (|dE| <= 1e-5 Eh, |dg| <= 1e-4 Eh/A)."""
    import torch
    world, rank, local = dist_info()
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=1800))
    torch.cuda.set_device(local)
    from pdynamo3_b200 import lib
    from pdynamo3_b200.qcmodel import GPUQCEngine
    from pdynamo3_b200.serving import GPUServer, Request, latency_summary
    mols, parts = batch_parts(args.steps, rank)
    warm = warm_molecules(rank)
    srv = GPUServer(n_slots=args.slots, device=local, resident_per_slot=1, precision_mode=1, profile=True,
                    **BATCH_OPTS)

    def served(items, tag):
        reqs = [srv.submit(Request(k, "%s%d" % (tag, k), z, x)) for k, (name, z, x) in items]
        srv.drain()
        for r in reqs:
            if r.error is not None:
                raise RuntimeError("request %s failed: %s" % (r.system, r.error))
        return reqs

    def plain(items):
        out = []
        for k, (name, z, x) in items:
            e = GPUQCEngine(z, device=local, **BATCH_OPTS)
            try:
                out.append(e.energy(x))
            finally:
                e.close()
        return out

    try:
        for w in range(args.warmup):
            items = list(enumerate(warm))
            served(items, "w%d_" % w)
            plain(items)
        srv.reset_profile()
        tuned = tune_eri_lanes(local, rank) if args.autotune else {}

        def timed(fn):
            if world > 1:
                torch.distributed.barrier()
            torch.cuda.synchronize()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            l0 = lib.launch_count()
            ev0.record()
            t0 = time.perf_counter()
            out = fn()
            torch.cuda.synchronize()
            ev1.record()
            ev1.synchronize()
            return out, ev0.elapsed_time(ev1), time.perf_counter() - t0, lib.launch_count() - l0

        clocks = Clocks(local) if rank == 0 else None
        if clocks:
            clocks.start()
        reqs, dev_ms, wall, launches = timed(lambda: [r for p in parts for r in served([(k, mols[k]) for k in p], "m")])
        clk = clocks.stop() if clocks else None
        regions = {n: {"calls": c, "total_ms": t} for n, (c, t) in srv.profile_totals().items()}
        plain_res, dev_ms64, wall64, launches64 = timed(lambda: plain([(k, mols[k]) for k in range(len(mols))]))
    finally:
        srv.close()
    # per-molecule errors of the mixed form against FP64
    byid = {r.id: r for r in reqs}
    de, dg, nconv, unconverged = [], [], 0, []
    h2d = d2h = 0
    for k, rp in enumerate(plain_res):
        rm = byid[k].result
        h2d += mols[k][2].nbytes
        d2h += rm.density.nbytes + (rm.gradients.nbytes if rm.gradients is not None else 0) + 8 * 8
        if not (rm.converged and rp.converged):
            # reported, not compared: an SCF that reached its iteration limit has no gradient
            unconverged.append({"molecule": k, "atoms": len(mols[k][1]), "mixed_converged": bool(rm.converged),
                                "fp64_converged": bool(rp.converged), "mixed_iterations": int(rm.iterations),
                                "fp64_iterations": int(rp.iterations)})
            continue
        nconv += 1
        de.append(abs(rm.energy - rp.energy))
        dg.append(float(np.abs(rm.gradients - rp.gradients).max()) * ANG)
    lat = latency_summary(reqs)
    dev_ms, wall, dev_ms64, wall64 = max_over_ranks([dev_ms, wall, dev_ms64, wall64], world, "cuda")
    if rank == 0:
        n = len(mols)
        value = n * world / (dev_ms / 1e3)
        fp64_value = n * world / (dev_ms64 / 1e3)
        roof = batch_roofline(mols, local)
        line = {"metric": BATCH_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": len(parts),
                "warmup": args.warmup, "ms_per_step": dev_ms / len(parts), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic (seeded organic molecules)",
                "config": batch_config({"parallelism": "replicas" if world > 1 else "single",
                                        "server_slots": args.slots, "precision": "mixed (FP32 quartets below 1e-6)",
                                        "autotuned_lanes": {"%d,%d" % k: v for k, v in tuned.items()},
                                        "mean_scf_iterations": float(np.mean([r.result.iterations for r in reqs]))}),
                "e2e": {"value": n * world / wall, "unit": UNIT, "h2d_bytes_per_step": h2d // len(parts),
                        "d2h_bytes_per_step": d2h // len(parts)},
                "gpu_launches": int(launches),
                "fp64_plain": {"value": fp64_value, "unit": UNIT, "wall_s": wall64, "device_s": dev_ms64 / 1e3,
                               "gpu_launches": int(launches64),
                               "form": "one molecule at a time through the drop-in engine (GPUQCEngine), FP64"},
                "mixed_vs_fp64": {"speedup": fp64_value and value / fp64_value,
                                  "max_abs_dE_hartree": max(de) if de else None,
                                  "max_abs_dgrad_hartree_per_A": max(dg) if dg else None,
                                  "within_1e-5_Eh_and_1e-4_Eh_per_A": bool(de and max(de) <= 1e-5 and max(dg) <= 1e-4),
                                  "both_converged": nconv, "molecules": n, "not_converged": unconverged},
                "latency": {"p50_s": lat["p50_s"], "p99_s": lat["p99_s"],
                            "definition": "submission to result of each request of the served form"},
                "roofline": roof, "regions_ms": regions, "clocks": clk,
                "cpu_baseline": cpu_batch_sample(mols, args) if args.cpu_baseline else None}
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def tune_eri_lanes(device, rank):
    """The library's tile autotuner (pdg_autotune_eri) run once, untimed, on a mid-size molecule of
    another seed; its choice of lanes per quartet holds for both timed forms."""
    from pdynamo3_b200 import workloads
    from pdynamo3_b200.qcmodel import GPUQCEngine
    cands = workloads.batch_molecules(40, seed=BATCH_SEED + 2 + 1000 * rank)
    name, z, x = min(cands, key=lambda m: abs(int((m[1] > 1).sum()) - 14))
    e = GPUQCEngine(z, device=device, **BATCH_OPTS)
    try:
        e.energy(x, do_gradients=False)
        return e.ctx.autotune_eri()
    finally:
        e.close()


def batch_roofline(mols, device):
    """The dominant kernel region of the batch, the two-electron J+K build: algorithmic FLOPs per
    build (pdg_work_estimate) over the CUDA-event time of three full, unscreened FP64 builds of the
    converged density of the batch's median-size molecule, against the FP64 pipe's throughput measured
    on this device (pdg_measure_fp64_peak, DFMA; the bf16 tensor figure is given beside it)."""
    from pdynamo3_b200 import lib
    from pdynamo3_b200.qcmodel import GPUQCEngine
    order = sorted(range(len(mols)), key=lambda k: len(mols[k][1]))
    k = order[len(order) // 2]
    name, z, x = mols[k]
    e = GPUQCEngine(z, device=device, **BATCH_OPTS)
    try:
        r = e.energy(x)
        ctx = e.ctx
        ctx.fock_two_electron(r.density, e.exchange_scaling)
        ctx.profile(True)
        for _ in range(3):
            ctx.fock_two_electron(r.density, e.exchange_scaling)
        calls, t = ctx.profile_region("eri_jk")
        ctx.profile(False)
        flops, _, quartets = ctx.work_estimate("eri_jk")
    finally:
        e.close()
    avg_s = t / max(1, calls) / 1e3
    peak = lib.measure_fp64_peak(device, 0)
    peak_dmma = lib.measure_fp64_peak(device, 1)
    achieved = flops / avg_s / 1e12
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    roof = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "traffic": None, "kernel": "eri_jk (two-electron J+K build, all classes)", "calls": calls,
            "avg_ms": avg_s * 1e3, "algorithmic_flops_per_call": flops, "quartets_per_call": quartets,
            "timed_on": "3 full unscreened FP64 J+K builds of the converged density of batch molecule %d "
                        "(%d atoms), after the timed region" % (k, len(z)),
            "peak_source": "FP64 FMA pipe measured on this device by pdg_measure_fp64_peak (of measured); "
                           "DMMA path %.1f TFLOP/s" % peak_dmma}
    if peaks.get("bf16_tflops"):
        roof["bf16_tensor_frac"] = achieved / peaks["bf16_tflops"]
    traffic_file = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(traffic_file):
        t = json.load(open(traffic_file)).get("eri_jk_batch")
        if t:
            roof["traffic"] = t["dram_bytes_per_call"]
            roof["traffic_source"] = t["source"]
    return roof


def _cpu_batch_worker(job):
    """The reference's conventional two-electron path (oracle restatement) on one molecule, on a
    1/mod hash sample of its shell quartets: unique integrals computed and stored once, one digest of
    the stored integrals (per SCF cycle), the two-electron gradient.  Returns the three times scaled
    to the whole quartet set."""
    import oracle
    from pdynamo3_b200.basis import ShellTable
    z, x, mod, lo, hi = job
    o = oracle.Oracle(ShellTable("6-31g_st_cart", z), x)
    L = oracle.lib()
    oracle.use_reference_roots(True)
    L.orc_set_sample(mod, lo, hi)
    rng = np.random.default_rng(5)
    a = rng.normal(size=(o.n, o.n)) * 0.05
    P = (a + a.T)[np.tril_indices(o.n)]
    t0 = time.perf_counter()
    o.store_integrals()
    t1 = time.perf_counter()
    o.fock_stored(P, 0.2)
    t2 = time.perf_counter()
    g = np.zeros(3 * o.natom)
    L.orc_eri_gradient(np.ascontiguousarray(P), 0.2, 1, g)
    t3 = time.perf_counter()
    o.free_stored()
    L.orc_set_sample(0, 0, 0)
    scale = mod / float(hi - lo)
    return (t1 - t0) * scale, (t2 - t1) * scale, (t3 - t2) * scale


def batch_cpu_jobs(mols, per_molecule_fraction=None):
    """A size-stratified sample of the batch (8 molecules, every 32nd in size order), each on a hash
    sample of its shell quartets small enough for a few seconds of one core."""
    order = sorted(range(len(mols)), key=lambda k: len(mols[k][1]))
    pick = order[16::32]
    jobs = []
    for k in pick:
        name, z, x = mols[k]
        heavy = int((z > 1).sum())
        mod = 2000
        width = max(1, int(round(2000 * min(1.0, (4.0 / heavy) ** 4))))
        jobs.append((z, x, mod, 0, width))
    return pick, jobs


def cpu_batch_estimate(mols, cores):
    """CPU seconds per energy+gradient of the batch's sample on one core and the sample's wall time
    on `cores` processes."""
    pick, jobs = batch_cpu_jobs(mols)
    t0 = time.perf_counter()
    if cores > 1:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(min(cores, len(jobs))) as pool:
            res = pool.map(_cpu_batch_worker, jobs)
    else:
        res = [_cpu_batch_worker(j) for j in jobs]
    wall = time.perf_counter() - t0
    per_mol = [ti + BATCH_REF_CYCLES * td + tg for ti, td, tg in res]
    return float(np.mean(per_mol)), wall, pick


def cpu_batch_sample(mols, args):
    from oracle import build as ob
    ob.build()
    mean_s, wall, pick = cpu_batch_estimate(mols, 1)
    return {"value": 1.0 / mean_s, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": ("oracle restatement of the reference's conventional two-electron path (unique integrals "
                       "stored once, %d digests of the stored integrals, the two-electron gradient) on 8 molecules "
                       "of the batch spread over its sizes (indices %s in size order), each on a hash sample of "
                       "its shell quartets scaled to the whole; XC quadrature, one-electron terms and linear "
                       "algebra excluded, so the CPU time is understated (%.1f s of CPU work)")
            % (BATCH_REF_CYCLES, pick, wall)}


def run_reference_batch(args):
    """--impl reference for the default workload: the CPU reference path (the oracle's restatement
    of the reference's stored-integral two-electron code) on the host cores.  Step k times one
    molecule of the batch's size-stratified sample (molecule k mod 8, on its hash sample of shell
    quartets, scaled to the whole); all W + K steps run at once, one process per core, and the W
    warm-up steps are dropped.  Value: cores / mean CPU seconds per molecule (one molecule per core,
    as the reference's SGOFProcessPool runs independent systems)."""
    world, rank, local = dist_info()
    if rank != 0:
        return
    from oracle import build as ob
    ob.build()
    cores = os.cpu_count() or 1
    mols, _ = batch_parts(1, 0)
    pick, jobs = batch_cpu_jobs(mols)
    steps = [jobs[k % len(jobs)] for k in range(args.warmup + args.steps)]
    t0 = time.perf_counter()
    if cores > 1:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(min(cores, len(steps))) as pool:
            res = pool.map(_cpu_batch_worker, steps)
    else:
        res = [_cpu_batch_worker(j) for j in steps]
    wall = time.perf_counter() - t0
    # CPU seconds per molecule, averaged first over the repeats of each sampled molecule so that every
    # size of the sample weighs the same
    byk = {}
    for k, (ti, td, tg) in enumerate(res):
        if k >= args.warmup:
            byk.setdefault(k % len(jobs), []).append(ti + BATCH_REF_CYCLES * td + tg)
    t = float(np.mean([np.mean(v) for v in byk.values()]))
    value = cores / t     # one molecule per process, every core busy
    line = {"impl": "reference", "metric": BATCH_METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3 / cores, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded organic molecules)",
            "config": batch_config({"parallelism": "host cores, one process per molecule",
                                    "sample_wall_s": wall}),
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": ("oracle restatement of the reference's conventional two-electron path "
                                        "(integrals stored once per geometry, %d digests, two-electron gradient), one "
                                        "molecule per step from 8 size-stratified molecules of the batch (indices %s in "
                                        "size order), each on a hash sample of its shell quartets scaled to the whole; "
                                        "XC, one-electron terms and linear algebra excluded (CPU time understated); %s")
                             % (BATCH_REF_CYCLES, pick, _roots_note())}}
    print(json.dumps(line), flush=True)


def run_water64(args):
    """Config 4: B3LYP/6-31G* (Cartesian, 1216 functions; the reference ships no 6-31G**) energy +
    gradient of a 64-water cluster in a 12 A cube, Medium grid, FP64 and the mixed mode (FP32
    quartets below the Schwarz x density bound 1e-6) on the same geometry; the mixed form's energy
    and largest gradient error against FP64 are stated.  The reference cannot run this system (it
    stores every integral, about 13 TB, and its memory guard refuses), so the FP64 GPU path is the
    comparison.  CUDA events on the context stream around each energy+gradient."""
    import torch
    torch.cuda.set_device(0)
    from pdynamo3_b200 import geometry, lib
    from pdynamo3_b200.qcmodel import GPUQCEngine
    z, xyz = geometry.water_cluster(64, 12.0, 64)
    x = xyz * ANG
    out = {}
    for mode, label in ((0, "fp64"), (1, "mixed")):
        e = GPUQCEngine(z, orbital_basis="6-31g_st_cart", functional="b3lyp", grid_accuracy=3, density_tolerance=1e-8)
        try:
            if mode:
                e.ctx.set_eri_options(precision_mode=1, mixed_cut=1e-6)
            stream = torch.cuda.ExternalStream(e.ctx.stream_handle(), device=0)
            e.ctx.profile(True)
            torch.cuda.synchronize()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            ev0.record(stream)
            r = e.energy(x)
            ev1.record(stream)
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
            regions = {n: e.ctx.profile_region(n) for n in ("eri_jk", "eri_grad", "xc_rho", "xc_vxc", "xc_grad",
                                                             "xc_weight_grad", "grid_build", "scf_diag")}
            out[label] = {"device_s": ev0.elapsed_time(ev1) / 1e3, "wall_s": wall, "energy_hartree": r.energy,
                          "converged": r.converged, "iterations": r.iterations,
                          "grid_points": r.report.get("Quadrature Points"), "gradients": r.gradients,
                          "regions_ms": {k: {"calls": c, "total_ms": t} for k, (c, t) in regions.items()}}
        finally:
            e.close()
    de = abs(out["mixed"]["energy_hartree"] - out["fp64"]["energy_hartree"])
    dg = float(np.abs(out["mixed"]["gradients"] - out["fp64"]["gradients"]).max()) * ANG
    for k in out:
        out[k].pop("gradients")
    line = {"metric": "energy+gradient/s, B3LYP/6-31G* 64-water cluster (1216 Cartesian functions), mixed vs FP64",
            "value": 1.0 / out["mixed"]["device_s"], "unit": UNIT, "n_gpus": 1, "steps": 1, "warmup": 0,
            "higher_is_better": True, "dtype": "f64+f32", "data": "synthetic (seeded 64-water cluster, 12 A cube)",
            "config": {"workload": "64 rigid waters in a 12 A cube (seed 64), B3LYP/6-31G* Cartesian (6-31G** is not "
                                   "among the reference's basis sets), Medium grid, SCF to 1e-8, energy + gradient",
                       "basis_functions": 1216, "atoms": 192},
            "fp64": out["fp64"], "mixed": out["mixed"],
            "mixed_vs_fp64": {"speedup": out["fp64"]["device_s"] / out["mixed"]["device_s"], "abs_dE_hartree": de,
                              "max_abs_dgrad_hartree_per_A": dg}}
    print(json.dumps(line), flush=True)

def run_many(args):
    """Many-molecule forms: ``batch`` (uneven organic molecules, FP64 and mixed precision side by
    side through the continuous-batching server) and ``stream`` (Poisson arrivals with follow-up
    chains, p50/p99 latency).  Wall-clock timing around a device synchronize on both sides: the
    slots run on separate streams.  One JSON line on stdout."""
    import torch
    from pdynamo3_b200 import workloads
    torch.cuda.set_device(0)
    if args.workload == "batch32":
        mols = workloads.batch_molecules(args.molecules, seed=1)
        r = workloads.run_batch(mols, n_slots=args.slots, warmup=min(2, args.molecules))
        line = {"metric": "energy+gradient/s, %d organic molecules (4-24 heavy atoms), B3LYP/6-31G*, mixed" % len(mols),
                "value": r["mixed"]["energy_grad_per_s"], "unit": UNIT, "n_gpus": 1, "higher_is_better": True,
                "dtype": "f64+f32", "data": "synthetic (seeded saturated C/N/O trees)",
                "config": {"workload": "batch of %d molecules, %d server slots" % (len(mols), args.slots)},
                "fp64": r["fp64"], "mixed": r["mixed"], "mixed_vs_fp64": r["mixed_vs_fp64"]}
    else:
        # swept arrival rates, the served mixed form and the served FP64 form at each; molecules of
        # 4-40 heavy atoms and water clusters of 4-48 waters, each followed by 1-20 displaced steps
        rates = [float(v) for v in args.rates.split(",")] if args.rates else [args.rate]
        sweep = []
        for rate in rates:
            row = {"rate_per_s": rate}
            for mode, label in ((1, "mixed"), (0, "fp64")):
                r = workloads.run_stream(args.requests, rate, n_slots=args.slots, precision_mode=mode, seed=1,
                                         heavy=(4, 40), waters=(4, 48))
                row[label] = {k: r[k] for k in ("throughput", "p50_s", "p99_s", "requests", "failed", "errors",
                                                "warm_fraction", "wall_s")}
            row["mixed_vs_fp64_throughput"] = row["mixed"]["throughput"] / max(row["fp64"]["throughput"], 1e-12)
            sweep.append(row)
            print(json.dumps(row), flush=True)
        line = {"metric": "served energy+gradient requests/s with p50/p99 latency, B3LYP/6-31G*, mixed vs FP64",
                "value": sweep[-1]["mixed"]["throughput"], "unit": "requests/s", "n_gpus": 1, "higher_is_better": True,
                "dtype": "f64+f32", "data": "synthetic (organic molecules and water clusters, follow-up chains)",
                "config": {"workload": "Poisson arrivals at %s /s, %d requests per run, %d slots; organic molecules of "
                                       "4-40 heavy atoms and water clusters of 4-48 waters, each followed by 1-20 "
                                       "requests at 0.01 A Gaussian displacements (warm starts)"
                                       % (",".join("%g" % r for r in rates), args.requests, args.slots)},
                "sweep": sweep}
    print(json.dumps(line), flush=True)


def mm_waters(n, seed, r_in=10.0, r_out=22.0):
    """n rigid point-charge waters (TIP3P charges O -0.834, H +0.417; O-H 0.9572 A, 104.52 deg) with
    seeded random centres in a spherical shell r_in..r_out A around the QC cluster and random
    orientations.  Returns charges (3n) and coordinates (3n x 3, bohr)."""
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    r = (r_in ** 3 + rng.uniform(size=n) * (r_out ** 3 - r_in ** 3)) ** (1.0 / 3.0)
    centre = d * r[:, None] + 0.5 * BOX
    a = np.deg2rad(104.52) / 2.0
    local = np.array([[0.0, 0.0, 0.0], [0.9572 * np.sin(a), 0.0, 0.9572 * np.cos(a)],
                      [-0.9572 * np.sin(a), 0.0, 0.9572 * np.cos(a)]])
    xyz = np.empty((3 * n, 3))
    for i in range(n):
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        xyz[3 * i:3 * i + 3] = centre[i] + local @ q.T
    charges = np.tile([-0.834, 0.417, 0.417], n)
    return charges, xyz * ANG


def run_qcmm(args):
    """QC/MM: the 16-water PBE/6-31G* energy+gradient in the field of --mm-waters point-charge
    waters; each step also returns the charges' gradients (electronic and nucleus-charge terms).
    Same timing as the default workload (CUDA events on the library stream, host copies inside)."""
    import torch
    torch.cuda.set_device(0)
    from pdynamo3_b200 import lib
    ctx = make_context(0)
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=0)
    q, xmm = mm_waters(args.mm_waters, 7)

    def step(coords):
        ctx.set_geometry(coords)
        ctx.grid_build(*GRID)
        ctx.set_point_charges(q, xmm)
        P, res = ctx.scf(density_tolerance=1e-8, maximum_iterations=100)
        g = ctx.scf_gradients()
        gq, gm = ctx.qcmm_gradients()
        ec, cq, cm = ctx.qcmm_core()
        return P, res, g + gq + cq, gm + cm
    for w in range(args.warmup):
        step(geometry_for(-1 - w))
    geoms = [geometry_for(k) for k in range(args.steps)]
    torch.cuda.synchronize()
    clocks = Clocks(0)
    clocks.start()
    ctx.profile(True)
    l0 = lib.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    iters, h2d, d2h = [], 0, 0
    t0 = time.perf_counter()
    ev0.record(stream)
    for k in range(args.steps):
        P, res, g, gm = step(geoms[k])
        iters.append(res.iterations)
        h2d += geoms[k].nbytes + q.nbytes + xmm.nbytes
        d2h += P.nbytes + g.nbytes + gm.nbytes + 8 * 7
    ev1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    dev_ms = ev0.elapsed_time(ev1)
    launches = lib.launch_count() - l0
    regions = {}
    for name in ("eri_jk", "eri_grad", "xc_rho", "xc_vxc", "xc_grad", "xc_weight_grad", "qcmm_potentials", "qcmm_grad",
                 "oneint", "oneint_grad", "grid_build", "scf_diag"):
        c, t = ctx.profile_region(name)
        regions[name] = {"calls": c, "total_ms": t}
    ctx.profile(False)
    clk = clocks.stop()
    line = {"metric": "QC/MM SCF energy+gradient/s (PBE/6-31G*, 16 H2O + %d MM point charges, FP64)" % len(q),
            "value": args.steps / (dev_ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded water cluster, seeded point-charge waters)",
            "config": workload_config({"workload": "PBE/6-31G* 16-water energy+gradient in the field of %d TIP3P-charge "
                                                   "waters (shell 10-22 A), charges' gradients included" % args.mm_waters,
                                       "mm_charges": int(len(q)), "mean_scf_iterations": float(np.mean(iters))}),
            "e2e": {"value": args.steps / wall, "unit": UNIT, "h2d_bytes_per_step": h2d // args.steps,
                    "d2h_bytes_per_step": d2h // args.steps},
            "gpu_launches": int(launches), "regions_ms": regions, "clocks": clk}
    print(json.dumps(line), flush=True)
    ctx.close()


def run_uhf(args):
    """Spin-unrestricted HF/6-31G* energy+gradient of the 16-water cluster cation (doublet, 80 alpha
    and 79 beta electrons), a fresh seeded geometry per step, atomic-density start; same timing as
    the default workload (CUDA events on the library stream, host copies inside)."""
    import torch
    torch.cuda.set_device(0)
    from pdynamo3_b200 import geometry, lib
    from pdynamo3_b200.basis import ShellTable
    from pdynamo3_b200.lib import Context
    z, _ = geometry.water_cluster(N_WATERS, BOX, 0)
    ctx = Context(0)
    ctx.set_basis(ShellTable("6-31g_st_cart", z))
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=0)
    na, nb = 80, 79

    def step(coords):
        ctx.set_geometry(coords)
        Pa, Pb, res = ctx.uscf(na, nb, density_tolerance=1e-8, total_charge=1.0, maximum_iterations=150)
        return Pa, Pb, res, ctx.scf_gradients()
    for w in range(args.warmup):
        step(geometry_for(-1 - w))
    geoms = [geometry_for(k) for k in range(args.steps)]
    torch.cuda.synchronize()
    clocks = Clocks(0)
    clocks.start()
    ctx.profile(True)
    l0 = lib.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    iters, s2, h2d, d2h = [], [], 0, 0
    t0 = time.perf_counter()
    ev0.record(stream)
    for k in range(args.steps):
        Pa, Pb, res, g = step(geoms[k])
        iters.append(res.iterations)
        s2.append(res.s2)
        h2d += geoms[k].nbytes
        d2h += Pa.nbytes + Pb.nbytes + g.nbytes + 8 * 8
    ev1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    dev_ms = ev0.elapsed_time(ev1)
    regions = {}
    for name in ("eri_jk", "eri_grad", "oneint", "oneint_grad", "pairs", "scf_diag"):
        c, t = ctx.profile_region(name)
        regions[name] = {"calls": c, "total_ms": t}
    ctx.profile(False)
    line = {"metric": "UHF energy+gradient/s (HF/6-31G*, (H2O)16+ doublet, FP64)", "value": args.steps / (dev_ms / 1e3),
            "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded water clusters)",
            "config": {"workload": "spin-unrestricted HF/6-31G* energy+gradient of the 16-water cluster cation, doublet",
                       "n_atoms": 48, "basis_functions": 304, "n_alpha": na, "n_beta": nb,
                       "mean_scf_iterations": float(np.mean(iters)), "mean_s2": float(np.mean(s2))},
            "e2e": {"value": args.steps / wall, "unit": UNIT, "h2d_bytes_per_step": h2d // args.steps,
                    "d2h_bytes_per_step": d2h // args.steps},
            "gpu_launches": int(lib.launch_count() - l0), "regions_ms": regions, "clocks": clocks.stop()}
    print(json.dumps(line), flush=True)
    ctx.close()


def run_chain(args):
    """Chain-of-states traffic through the GPU process-pool backend (the reference's SGOFProcessPool
    interface): --images images of the 16-water PBE/6-31G* cluster (seeded 0.05 A displacements of
    one geometry), --steps pool calls in which every image moves by 0.01 A (an optimiser step), after
    one cold call.  Wall time around each FunctionGradients call (its slots run on separate
    streams), device synchronised on both sides; value = image energy+gradients per second over the
    timed calls."""
    import torch
    from pdynamo3_b200 import geometry
    from pdynamo3_b200.pool import ArrayObjective, SGOFProcessPoolGPU
    torch.cuda.set_device(0)
    z, xyz = geometry.water_cluster(N_WATERS, BOX, 1000)
    obj = ArrayObjective(z, xyz, orbital_basis="6-31g_st_cart", functional=FUNCTIONAL, grid=GRID[1:],
                         grid_accuracy=GRID[0], density_tolerance=1e-8)
    rng = np.random.default_rng(3)
    x = [(xyz + rng.normal(scale=0.05, size=xyz.shape)).reshape(-1) for _ in range(args.images)]
    pool = SGOFProcessPoolGPU.FromObjectiveFunction(obj, maximumProcesses=args.slots)
    try:
        g = [np.zeros(obj.numberOfVariables) for _ in x]
        t0 = time.perf_counter()
        pool.FunctionGradients(x, g)
        cold_s = time.perf_counter() - t0
        cold_it = [r.result.iterations for r in pool.last_requests]
        torch.cuda.synchronize()
        times, its = [], []
        for k in range(args.steps):
            x = [xi + rng.normal(scale=0.01, size=xi.shape) for xi in x]
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            pool.FunctionGradients(x, g)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
            its.append(float(np.mean([r.result.iterations for r in pool.last_requests])))
    finally:
        pool.Finalize()
    total = float(np.sum(times))
    line = {"metric": "chain-of-states image energy+gradient/s through the process-pool backend (PBE/6-31G*, 16 H2O)",
            "value": args.images * args.steps / total, "unit": "images/s", "n_gpus": 1, "steps": args.steps,
            "warmup": 1, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded water cluster images)",
            "config": workload_config({"workload": "%d images, %d server slots, pool calls after a cold one" % (
                args.images, args.slots), "mean_scf_iterations_warm": float(np.mean(its)),
                "mean_scf_iterations_cold": float(np.mean(cold_it)), "cold_call_s": cold_s})}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="pdgpu", choices=["pdgpu", "reference"])
    ap.add_argument("--cpu-slices", type=int, default=8, help="1/1000 hash slices timed for the CPU baseline")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--xc-bound", default="hbm", choices=["hbm", "fp64"],
                    help="single: roofline of an XC region as HBM-bound (resident basis values read) or against "
                         "the measured FP64 pipe")
    ap.add_argument("--kernel-case", type=int, default=0,
                    help="run only the small kernel-profiling case with this many waters and exit")
    ap.add_argument("--kernel-xc", type=int, default=1, help="kernel case: 0 skips the grid and the XC passes")
    ap.add_argument("--kernel-molecule", type=int, default=-1,
                    help="kernel case: molecule of the organic batch (B3LYP, Medium grid) instead of waters")
    ap.add_argument("--workload", default="batch", choices=["batch", "single", "batch32", "stream", "qcmm", "chain", "uhf", "water64"],
                    help="batch (default): the 256-molecule organic batch, served mixed vs plain FP64; single: the "
                         "16-water PBE energy+gradient")
    ap.add_argument("--images", type=int, default=8, help="chain: images per pool call")
    ap.add_argument("--mm-waters", type=int, default=1000, help="qcmm: point-charge waters around the cluster")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="single workload: FP64 (default) or the mixed-precision mode")
    ap.add_argument("--molecules", type=int, default=32, help="batch: number of molecules")
    ap.add_argument("--slots", type=int, default=8, help="batch/stream: server slots")
    ap.add_argument("--requests", type=int, default=64, help="stream: requests in total")
    ap.add_argument("--rate", type=float, default=4.0, help="stream: arrivals per second")
    ap.add_argument("--rates", default="", help="stream: comma-separated arrival rates to sweep")
    ap.add_argument("--autotune", action="store_true",
                    help="batch: run the library's ERI lanes autotuner before the timed steps (off: the "
                         "built-in lanes tables, its choice on a 14-heavy-atom batch molecule)")
    args = ap.parse_args()
    if args.kernel_case > 0 or args.kernel_molecule >= 0:
        run_kernel_case(args)
    elif args.workload == "qcmm":
        run_qcmm(args)
    elif args.workload == "chain":
        run_chain(args)
    elif args.workload == "uhf":
        run_uhf(args)
    elif args.workload == "water64":
        run_water64(args)
    elif args.workload == "batch":
        if args.impl == "reference":
            run_reference_batch(args)
        else:
            run_batch_metric(args)
    elif args.workload != "single":
        run_many(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
