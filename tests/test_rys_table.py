"""The device Rys table (Chebyshev fits + Hermite limit) against the oracle's independent rule."""
import os
import re

import numpy as np
import pytest

import oracle
from conftest import ROOT

INC = os.path.join(ROOT, "pdynamo3_b200", "csrc", "rys_table.inc")


def load_table():
    text = open(INC).read()
    nmax = int(re.search(r"#define RYS_NMAX (\d+)", text).group(1))
    H = [float(v) for v in re.search(r"RYS_HN\[RYS_NMAX\] = \{([^}]*)\}", text).group(1).split(",")]
    ncoef = [int(v) for v in re.search(r"RYS_NCOEFN\[RYS_NMAX\] = \{([^}]*)\}", text).group(1).split(",")]
    nint = [int(v) for v in re.search(r"rys_nint\[RYS_NMAX\] = \{([^}]*)\}", text).group(1).split(",")]
    offs = [int(v) for v in re.search(r"rys_offset\[RYS_NMAX\] = \{([^}]*)\}", text).group(1).split(",")]

    def arr(name):
        body = re.search(name + r"\[[^\]]*\] = \{(.*?)\};", text, re.S).group(1)
        return np.array([float(v) for v in body.replace("\n", " ").split(",") if v.strip()])
    return nmax, H, ncoef, nint, offs, arr("rys_cheb"), arr("rys_herm_u"), arr("rys_herm_w")


def table_roots(tab, n, x):
    nmax, Hs, ncoefs, nint, offs, cheb, hu, hw = tab
    H, ncoef = Hs[n - 1], ncoefs[n - 1]
    if x >= nint[n - 1] * H:
        return hu[(n - 1) * nmax:(n - 1) * nmax + n] / x, hw[(n - 1) * nmax:(n - 1) * nmax + n] / np.sqrt(x)
    it = min(int(x / H), nint[n - 1] - 1)
    t = (x - it * H) * 2.0 / H - 1.0
    c = cheb[offs[n - 1] + it * ncoef * 2 * n: offs[n - 1] + (it + 1) * ncoef * 2 * n].reshape(ncoef, 2 * n)
    vals = np.polynomial.chebyshev.chebval(t, c)
    return vals[:n], vals[n:]


@pytest.mark.parametrize("n", range(1, 8))
def test_table_matches_independent_rule(n):
    tab = load_table()
    rng = np.random.default_rng(n)
    xs = np.concatenate([[0.0, 1e-9, 2.0, 39.999, 40.0, 77.9, 78.0, 250.0, 1e4], rng.uniform(0, 90, 40),
                         np.exp(rng.uniform(-10, 8, 20))])
    worst = 0.0
    for x in xs:
        u, w = table_roots(tab, n, x)
        uo, wo = oracle.rys_roots(n, x)
        worst = max(worst, np.max(np.abs(u - uo) / uo), np.max(np.abs(w - wo) / wo))
    assert worst < 5e-14, worst
