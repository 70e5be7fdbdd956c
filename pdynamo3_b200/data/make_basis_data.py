"""Extract Gaussian basis-set tables into this package's JSON format.

Reads the YAML basis-set parameter files of a pDynamo3 source tree
(``parameters/gaussianBasisSets/<name>/<Element>.yaml``, the format read by
``pMolecule/QCModel/GaussianBases/__extensions__/pyrex/pMolecule.QCModel.GaussianBases.GaussianBasis.pyx:110-137``)
and writes ``basis_<name>.json`` beside this script.  The tables are published
basis-set data (exponents and contraction coefficients of normalised
primitives); the JSON keeps them verbatim, keyed by atomic number.

Usage:  python make_basis_data.py <pDynamo3 root> [basis names ...]
"""
import json
import os
import sys

import yaml


def convert(root, name):
    d = os.path.join(root, "parameters", "gaussianBasisSets", name)
    out = {"name": name, "elements": {}}
    for fn in sorted(os.listdir(d)):
        if not fn.endswith(".yaml"):
            continue
        with open(os.path.join(d, fn)) as f:
            y = yaml.safe_load(f)
        shells = []
        for sh in y["Shells"]:
            exps = [float(p[0]) for p in sh["Primitives"]]
            ncoef = len(sh["Primitives"][0][1])
            coefs = [[float(p[1][c]) for p in sh["Primitives"]] for c in range(ncoef)]
            shells.append({"type": sh["Type"], "exponents": exps, "coefficients": coefs})
        out["elements"][str(int(y["Atomic Number"]))] = {
            "symbol": fn[:-5],
            "spherical": bool(y["Is Spherical"]),
            "normalized_primitives": bool(y["Normalized Primitives"]),
            "shells": shells,
        }
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "basis_%s.json" % name)
    with open(path, "w") as f:
        json.dump(out, f, indent=0, sort_keys=True)
    print("wrote", path, len(out["elements"]), "elements")


if __name__ == "__main__":
    root = sys.argv[1]
    for name in (sys.argv[2:] or ["6-31g_st", "sto-3g"]):
        convert(root, name)
