#!/bin/sh
# ORACLE test infrastructure: compiles the reference program (main.cpp and
# src/*.cpp of ESDGSEM_MPIOCCA, read where they lie, unmodified) against the
# OCCA-v0 shim and the single-rank MPI stub in oracle/ref_shim/.  Output only
# under oracle/_ref/.  The reference tree defaults to /root/reference.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${ESDG_REFERENCE:-/root/reference}
OUT="$HERE/_ref"
mkdir -p "$OUT/obj"
FLAGS="-O2 -ffp-contract=off -w -std=gnu++14 -I$HERE/ref_shim -I$REF/include"
for f in "$REF"/src/*.cpp "$REF"/main.cpp "$HERE"/ref_shim/occa_shim.cpp; do
  o="$OUT/obj/$(basename "$f" .cpp).o"
  if [ ! -f "$o" ] || [ "$f" -nt "$o" ]; then
    g++ $FLAGS -Ddfloat=double -Ddfloat4=double4 -DMPI_DFLOAT=MPI_DOUBLE '-DdfloatString="double"' \
        '-Ddfloat4String="double4"' -c "$f" -o "$o"
  fi
done
g++ -o "$OUT/esdg_ref" "$OUT"/obj/*.o -ldl
echo "$OUT/esdg_ref"
