"""The drop-in engine's SCF retries, with a stand-in for the library context (no GPU): a cold SCF
that does not converge is repeated with complete Fock builds, and in the mixed mode in FP64, after
which the context's options are restored."""
import types

import numpy as np

from pdynamo3_b200.qcmodel import GPUQCEngine


class FakeContext:
    def __init__(self, failures):
        self.failures = failures
        self.eri_options = dict(schwarz_cut=1e-13, tei_underflow=1e-12, precision_mode=0, mixed_cut=1e-6)
        self.incremental = True
        self.calls = []
        self.n = 0

    def set_eri_options(self, schwarz_cut=1e-13, tei_underflow=1e-12, precision_mode=0, mixed_cut=1e-6):
        self.eri_options = dict(schwarz_cut=schwarz_cut, tei_underflow=tei_underflow, precision_mode=precision_mode,
                                mixed_cut=mixed_cut)

    def set_incremental(self, enable=True, density_cut=1e-13, rebuild_period=16):
        self.incremental = bool(enable)

    def set_basis(self, shells):
        self.n = shells.n_functions()

    def set_functional(self, name):
        return 1.0

    def set_geometry(self, xyz):
        pass

    def scf(self, guess=None, total_charge=0.0, raise_on_noconv=True, **opts):
        self.calls.append({"precision_mode": self.eri_options["precision_mode"], "incremental": self.incremental,
                           "history": opts.get("maximum_history")})
        ok = len(self.calls) > self.failures
        res = types.SimpleNamespace(energy_total=-76.0, energy_nuclear=9.0, energy_one=-120.0, energy_two=35.0,
                                    energy_xc=0.0, rho_integral=0.0, converged=ok, iterations=7)
        return np.zeros(self.n * (self.n + 1) // 2), res

    def scf_gradients(self):
        return np.zeros((3, 3))

    def close(self):
        pass


WATER = np.array([[0.0, 0.0, 0.0], [1.8, 0.0, 0.0], [-0.45, 1.75, 0.0]])


def engine(ctx, mixed):
    e = GPUQCEngine([8, 1, 1], orbital_basis="6-31g_st_cart", functional="hf", context=ctx)
    if mixed:
        ctx.set_eri_options(precision_mode=1, mixed_cut=1e-6)
    return e


def test_mixed_mode_retry_runs_in_fp64_with_complete_builds_and_restores_the_options():
    ctx = FakeContext(failures=1)
    r = engine(ctx, mixed=True).energy(WATER)
    assert r.converged and r.iterations == 14
    assert ctx.calls[0] == {"precision_mode": 1, "incremental": True, "history": 10}
    assert ctx.calls[1] == {"precision_mode": 0, "incremental": False, "history": 16}
    assert ctx.eri_options["precision_mode"] == 1 and ctx.incremental


def test_fp64_retry_keeps_fp64_and_a_failed_retry_reports_no_convergence():
    ctx = FakeContext(failures=2)
    r = engine(ctx, mixed=False).energy(WATER)
    assert not r.converged and r.gradients is None
    assert [c["precision_mode"] for c in ctx.calls] == [0, 0]
    assert ctx.calls[1]["incremental"] is False and ctx.incremental
