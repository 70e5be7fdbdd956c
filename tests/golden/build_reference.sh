#!/bin/sh
# Build the pDynamo3 reference for generating the golden fixtures in this directory (test
# infrastructure only; nothing in the library uses it).
#
#   tests/golden/build_reference.sh <pDynamo3 source tree> [build directory, default /tmp/pdref]
#
# Steps, all inside the build directory (the source tree is only read):
#  1. copy the source tree (without examples/ and structures/);
#  2. add to the copy a Cartesian variant of the 6-31G* parameters, parameters/gaussianBasisSets/
#     6-31g_st_cart, identical to 6-31g_st except "Is Spherical: false" (the shipped files are
#     spherical);
#  3. patch the copy's DFTGrid_Atom_Parameters (pMolecule/QCModel/__extensions__/csource/DFTGrid.c)
#     so that the environment variable PDYNAMO3_GRID_OVERRIDE="nR,l" replaces the per-element number
#     of radial shells and the Lebedev order of the chosen accuracy (the maximum radius stays that
#     of the accuracy), which is how the library's pdg_grid_build(accuracy, n_radial, angular_l)
#     defines an override; unset, the reference is unchanged;
#  4. run the reference's own installer (installation/Install.py -f).
# Afterwards source <build>/env.sh to import it.
set -e
SRC=${1:?usage: build_reference.sh <pDynamo3 source tree> [build dir]}
DST=${2:-/tmp/pdref}
rm -rf "$DST"
mkdir -p "$DST"
(cd "$SRC" && tar --exclude=./examples --exclude=./structures -cf - .) | (cd "$DST" && tar xf -)
chmod -R u+w "$DST"
P=$DST/parameters/gaussianBasisSets
mkdir -p "$P/6-31g_st_cart"
for f in "$P"/6-31g_st/*; do
    sed 's/Is Spherical: *true/Is Spherical: false/' "$f" > "$P/6-31g_st_cart/$(basename "$f")"
done
python3 - "$DST/pMolecule/QCModel/__extensions__/csource/DFTGrid.c" <<'EOF'
import sys
path = sys.argv[1]
src = open(path).read()
head = "static void DFTGrid_Atom_Parameters ( const DFTGridAccuracy accuracy, const Integer ni, Integer *nR, Integer *lValue, Real *maximumRadius )"
i = src.index(head)
j = src.index("\n}\n", i)
patch = ("\n    { const char *ov = getenv ( \"PDYNAMO3_GRID_OVERRIDE\" ) ; int a, b ;\n"
         "      if ( ( ov != NULL ) && ( sscanf ( ov, \"%d,%d\", &a, &b ) == 2 ) ) { (*nR) = a ; (*lValue) = b ; } }")
src = src[:j] + patch + src[j:]
src = src.replace("# include <stdio.h>", "# include <stdio.h>\n# include <stdlib.h>", 1)
open(path, "w").write(src)
EOF
cd "$DST/installation"
PDYNAMO3_HOME=$DST PDYNAMO3_PYTHONCOMMAND=python3 python3 Install.py -f
cat > "$DST/env.sh" <<EOF
export PDYNAMO3_HOME=$DST
export PYTHONPATH=$DST:\$PYTHONPATH
export PDYNAMO3_PARAMETERS=$DST/parameters
export PDYNAMO3_SCRATCH=/tmp/pdscratch
export PDYNAMO3_PYTHONCOMMAND=python3
export PDYNAMO3_STYLE=$DST/parameters/cssStyleSheets/defaultStyle.css
mkdir -p /tmp/pdscratch
EOF
echo "reference built in $DST; source $DST/env.sh"
