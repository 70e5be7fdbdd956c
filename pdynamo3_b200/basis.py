"""Gaussian basis sets for the Fock-build engine.

Mirrors what ``GaussianBasisContainer.FromParameterDirectory`` hands to the reference's C layer
(pMolecule/QCModel/GaussianBases/__extensions__/pyrex/pMolecule.QCModel.GaussianBases.GaussianBasisContainer.pyx:122-152):
one basis per atom, shells in file order, exponents and contraction coefficients of normalised
primitives.  The tables are the package's JSON copies (data/make_basis_data.py).  The name
"6-31g_st_cart" selects the 6-31G* tables with Cartesian d functions.
"""
import json
import os

import numpy as np

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
_CACHE = {}
_TYPES = {"S": (0, 0), "P": (1, 1), "SP": (0, 1), "D": (2, 2), "F": (3, 3)}


def _table(name):
    if name not in _CACHE:
        with open(os.path.join(_DATA, "basis_%s.json" % name)) as f:
            _CACHE[name] = json.load(f)
    return _CACHE[name]


class ShellTable:
    """Flat shell arrays in the layout of pdg_basis_upload."""

    def __init__(self, name, atomic_numbers):
        cart = name.endswith("_cart")
        table = _table(name[:-5] if cart else name)
        atom, llo, lhi, nprim, ex, co = [], [], [], [], [], []
        spherical = None
        normalized = None
        for a, z in enumerate(atomic_numbers):
            el = table["elements"].get(str(int(z)))
            if el is None:
                raise KeyError("basis %s has no entry for Z=%d" % (name, z))
            sph = False if cart else el["spherical"]
            if spherical is None:
                spherical, normalized = sph, el["normalized_primitives"]
            for sh in el["shells"]:
                lo, hi = _TYPES[sh["type"]]
                atom.append(a)
                llo.append(lo)
                lhi.append(hi)
                nprim.append(len(sh["exponents"]))
                ex.extend(sh["exponents"])
                for c in sh["coefficients"]:
                    co.extend(c)
        self.name = name
        self.atomic_numbers = np.asarray(atomic_numbers, dtype=np.int32)
        self.nuclear_charges = self.atomic_numbers.astype(np.float64)
        self.shell_atom = np.asarray(atom, dtype=np.int32)
        self.shell_l_low = np.asarray(llo, dtype=np.int32)
        self.shell_l_high = np.asarray(lhi, dtype=np.int32)
        self.shell_nprim = np.asarray(nprim, dtype=np.int32)
        self.exponents = np.asarray(ex, dtype=np.float64)
        self.coefficients = np.asarray(co, dtype=np.float64)
        self.spherical = bool(spherical)
        self.normalized_primitives = bool(normalized)

    @property
    def n_shells(self):
        return len(self.shell_atom)

    def n_functions(self):
        n = 0
        for lo, hi in zip(self.shell_l_low, self.shell_l_high):
            for l in range(lo, hi + 1):
                n += (2 * l + 1) if (self.spherical and l > 1) or (self.spherical and l == 1) else (l + 1) * (l + 2) // 2
        return n

    def upload_args(self):
        return (len(self.atomic_numbers), self.nuclear_charges, self.n_shells, self.shell_atom, self.shell_l_low,
                self.shell_l_high, self.shell_nprim, self.exponents, self.coefficients,
                int(self.normalized_primitives))
