#!/bin/sh
# Build two pieces of the reference from the sources where they lie in a pDynamo3 tree, for test
# infrastructure only:
#  - its vendored libxc 1.2 (pMolecule/QCModel/__extensions__/cxc) -> oracle/_ref/libxc_ref.so;
#    the XC functional tests compare the device functionals against it;
#  - its vendored libcint Rys-root routines (pMolecule/QCModel/GaussianBases/__extensions__/csource/
#    libcint_*.c) -> oracle/_ref/librys_ref.so; the oracle's roots are checked against it and the
#    CPU timing runs use it as the oracle's root rule.
# Usage: oracle/build_ref.sh [pDynamo3 root, default /root/reference]
set -e
ROOT=${1:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
if [ ! -d "$ROOT/pMolecule" ]; then
    echo "build_ref.sh: no pDynamo3 tree at $ROOT; reference checkers not built"
    exit 0
fi
EXT=$ROOT/pMolecule/QCModel/__extensions__
mkdir -p "$HERE/_ref"
gcc -O2 -fPIC -shared -w -I"$EXT/cxc" -I"$EXT/cinclude" "$EXT"/cxc/*.c -o "$HERE/_ref/libxc_ref.so" -lm
GB=$ROOT/pMolecule/QCModel/GaussianBases/__extensions__
gcc -O2 -fPIC -shared -w -I"$GB/cinclude" "$GB/csource/libcint_rys_roots.c" "$GB/csource/libcint_rys_wheeler.c" \
    "$GB/csource/libcint_fmt.c" "$GB/csource/libcint_eigh.c" -o "$HERE/_ref/librys_ref.so" -lm
echo "$HERE/_ref/libxc_ref.so $HERE/_ref/librys_ref.so"
