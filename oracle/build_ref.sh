#!/bin/sh
# ORACLE test infrastructure: compiles the reference program (main.cpp and
# src/*.cpp of ESDGSEM_MPIOCCA, read where they lie, unmodified) against the
# OCCA-v0 shim and the single-rank MPI stub in oracle/ref_shim/.  Output only
# under oracle/_ref/.  The reference tree is $ESDG_REFERENCE, else a checkout
# named `reference` beside this repository.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${ESDG_REFERENCE:-$(cd "$HERE/../.." && pwd)/reference}
OUT="$HERE/_ref"
mkdir -p "$OUT/obj"
FLAGS="-O2 -ffp-contract=off -w -std=gnu++14 -I$HERE/ref_shim -I$REF/include"
for f in "$REF"/src/*.cpp "$REF"/main.cpp "$HERE"/ref_shim/occa_shim.cpp "$HERE"/ref_shim/bench_case.cpp; do
  o="$OUT/obj/$(basename "$f" .cpp).o"
  if [ ! -f "$o" ] || [ "$f" -nt "$o" ] || [ "$HERE/ref_shim/occa.hpp" -nt "$o" ] || [ "$HERE/ref_shim/mpi.h" -nt "$o" ]; then
    g++ $FLAGS -Ddfloat=double -Ddfloat4=double4 -DMPI_DFLOAT=MPI_DOUBLE '-DdfloatString="double"' \
        '-Ddfloat4String="double4"' -c "$f" -o "$o"
  fi
done
# SW2D::InitB / SW2D::InitQ calls from main.cpp go through the case hook
# (oracle/ref_shim/bench_case.cpp), which forwards them unless ESDG_REF_CASE is set
WRAP="-Wl,--wrap=_ZN4SW2D5InitBEi16MeshPartitioningiiiPKdS2_Pd -Wl,--wrap=_ZN4SW2D5InitQEi16MeshPartitioningiiiPKdS2_PddS2_dd"
g++ -o "$OUT/esdg_ref" "$OUT"/obj/*.o -ldl $WRAP
echo "$OUT/esdg_ref"
# the reference's Okada routine alone, on points from a file
g++ $FLAGS -Ddfloat=double -Ddfloat4=double4 -DMPI_DFLOAT=MPI_DOUBLE '-DdfloatString="double"' \
    '-Ddfloat4String="double4"' -o "$OUT/okada_driver" "$HERE/ref_shim/okada_driver.cpp" "$OUT/obj/okada.o"

# The reference's main.cpp and host sources (everything but its deviceclass)
# linked against the B200 engine through include/dropin/deviceclass.h: the
# drop-in boundary exercised by the reference's own driver.
if [ "$1" = "dropin" ]; then
  REPO=$(cd "$HERE/.." && pwd)
  LIB="$REPO/esdgsem_mpiocca_b200"
  mkdir -p "$OUT/dropin_obj"
  DFLAGS="-O2 -ffp-contract=off -w -std=gnu++14 -I$REPO/include/dropin -I$REPO/include -I$HERE/ref_shim -I$REF/include"
  for f in "$REF"/src/*.cpp "$REF"/main.cpp; do
    case "$f" in *deviceclass.cpp) continue;; esac
    o="$OUT/dropin_obj/$(basename "$f" .cpp).o"
    g++ $DFLAGS -Ddfloat=double -Ddfloat4=double4 -DMPI_DFLOAT=MPI_DOUBLE '-DdfloatString="double"' \
        '-Ddfloat4String="double4"' -c "$f" -o "$o"
  done
  g++ -o "$OUT/esdg_dropin" "$OUT"/dropin_obj/*.o -L"$LIB" -lesdg_b200 -Wl,-rpath,'$ORIGIN/../../esdgsem_mpiocca_b200'
  echo "$OUT/esdg_dropin"
fi
