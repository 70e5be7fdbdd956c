#!/bin/sh
# Build the reference's vendored libxc 1.2 (pMolecule/QCModel/__extensions__/cxc) from the sources
# where they lie in a pDynamo3 tree into oracle/_ref/libxc_ref.so.  Test infrastructure only: the
# XC functional tests compare the device functionals against it.
# Usage: oracle/build_ref.sh [pDynamo3 root, default /root/reference]
set -e
ROOT=${1:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
EXT=$ROOT/pMolecule/QCModel/__extensions__
mkdir -p "$HERE/_ref"
gcc -O2 -fPIC -shared -w -I"$EXT/cxc" -I"$EXT/cinclude" "$EXT"/cxc/*.c -o "$HERE/_ref/libxc_ref.so" -lm
echo "$HERE/_ref/libxc_ref.so"
