"""The allocation-free XC entry point (pdg_xc_evaluate_static) through the C-ABI.

It serves callers that must not allocate device memory while they run (fixed memory budgets, no
cudaMalloc/cudaFree synchronisation against other streams): its device staging is a fixed array
inside the library.  Two calls in a row with different inputs must each reproduce the allocating
entry point pdg_xc_evaluate to the tolerance of the other functional tests (relative 1e-12), so a
call never sees stale data from the one before; oversized requests are refused.
This file is collected last on purpose.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(seed, n):
    rng = np.random.default_rng(seed)
    rho = np.exp(rng.uniform(np.log(1e-8), np.log(1e2), n))
    sigma = rho ** (8.0 / 3.0) * np.exp(rng.uniform(np.log(1e-4), np.log(1e2), n))
    return rho, sigma


def _close(a, b):
    for x, y in zip(a, b):
        scale = np.maximum(np.abs(x), 1e-300)
        assert np.max(np.abs(x - y) / scale) <= 1e-12


def test_static_entry_matches_allocating_entry_twice(cuda_device):
    from pdynamo3_b200.lib import xc_evaluate, xc_evaluate_static
    # first call: many points; second call: fewer points, different values and functional, so a
    # leftover from the first call would show up in the comparison
    rho1, sig1 = _inputs(1, 50000)
    rho2, sig2 = _inputs(2, 3000)
    _close(xc_evaluate_static("pbe", rho1, sig1), xc_evaluate("pbe", rho1, sig1))
    _close(xc_evaluate_static("b3lyp", rho2, sig2), xc_evaluate("b3lyp", rho2, sig2))


def test_static_entry_refuses_oversized_requests(cuda_device):
    from pdynamo3_b200.lib import PDGError, xc_evaluate_static
    rho, sig = _inputs(3, 65537)
    with pytest.raises(PDGError) as err:
        xc_evaluate_static("pbe", rho, sig)
    assert "maximum" in str(err.value)


def test_static_entry_allocates_no_device_memory_and_takes_the_maximum(cuda_device):
    """The entry point's purpose: no device allocation per call (the free device memory is the
    same before and after a warm call), and exactly the stated maximum of points is accepted."""
    import torch
    from pdynamo3_b200.lib import xc_evaluate, xc_evaluate_static
    rho, sig = _inputs(4, 65536)
    xc_evaluate_static("blyp", rho[:10], sig[:10])      # the first call on the device sets up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    got = xc_evaluate_static("blyp", rho, sig)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0
    _close(got, xc_evaluate("blyp", rho, sig))
    # the names of the allocating entry point, "hf" (zero) included
    z = xc_evaluate_static("hf", rho[:100], sig[:100])
    assert all(np.all(a == 0.0) for a in z)
