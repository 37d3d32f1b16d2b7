#!/bin/sh
# TEST INFRASTRUCTURE: build oracle/_ref/ref_tables from the reference's own
# sources (read where they lie under the reference tree; nothing is copied)
# with the Eigen/boost stand-ins in oracle/refshim.  Run in the development
# container only; the GPU box never needs the reference tree.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${SPHERAL_REFERENCE:-/root/reference}/src
mkdir -p "$HERE/_ref"
${CXX:-g++} -std=c++11 -O2 -ffp-contract=off -fno-fast-math -w \
  -I"$HERE/refshim" -I"$REF" \
  "$HERE/refshim/ref_tables.cc" \
  "$REF/Geometry/Dimension.cc" "$REF/Geometry/GeomVector.cc" \
  "$REF/Geometry/GeomTensor.cc" "$REF/Geometry/GeomSymmetricTensor.cc" \
  -o "$HERE/_ref/ref_tables"
echo "$HERE/_ref/ref_tables"
