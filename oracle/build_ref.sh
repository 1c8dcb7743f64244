#!/usr/bin/env bash
# Builds the unmodified reference (FAME-Isotropic-GPU) from its sources where they
# lie, for sm_100a, into oracle/_ref/.  Test infrastructure only: the product
# never links or runs anything built here.
#
#   oracle/build_ref.sh REFERENCE_ROOT      (the reference project's root directory)
#
# Outputs (git-ignored):
#   oracle/_ref/fame_ref_main     the reference's own Main.cpp program
#   oracle/_ref/fame_ref_harness  oracle/ref_harness.cu linked with every reference
#                                 object except Main.o
#   oracle/_ref/fame_ref_evwriter oracle/ref_evwriter.cpp with the reference's
#                                 FAME_Save_Eigenvector
# Only header shims are added (oracle/ref_shims/); no reference source is edited or
# copied.  LAPACKE_zpteqr is bound to scipy's bundled OpenBLAS (LP64 LAPACKE).
set -euo pipefail
REF=${1:?"usage: $0 REFERENCE_ROOT"}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
OBJ="$OUT/obj"
SHIM="$HERE/ref_shims"
if [ ! -d "$REF/FAME_Main" ]; then
  echo "reference sources not found at $REF" >&2
  exit 1
fi
mkdir -p "$OBJ"
NVCC=${NVCC:-nvcc}
ARCH="-gencode arch=compute_100a,code=sm_100a"
OPENBLAS=$(python3 -c "import glob,os,scipy;d=os.path.join(os.path.dirname(scipy.__file__),'..','scipy.libs');print(os.path.realpath(sorted(glob.glob(os.path.join(d,'libscipy_openblas*.so')))[0]))")
CXXFLAGS="-O3 -m64 -w -I$REF/include -I$SHIM"

pids=()
for src in "$REF"/FAME_Main/*.cpp "$REF"/FAME_Preprocessing/*.cpp "$REF"/FAME_Tools/*.cpp "$REF"/Main.cpp; do
  o="$OBJ/$(basename "${src%.cpp}").o"
  extra="-include time.h"
  case "$(basename "$src")" in
    vec_norm.cpp|vec_inner_prod.cpp) extra="$extra -std=gnu++11 -fext-numeric-literals" ;;
  esac
  g++ -c "$src" -o "$o" $CXXFLAGS $extra &
  pids+=($!)
done
for src in "$REF"/FAME_Main/*.cu "$REF"/FAME_Tools/*.cu; do
  o="$OBJ/$(basename "${src%.cu}").o"
  $NVCC -c "$src" -o "$o" -O3 -m64 $ARCH -w -I"$REF/include" -I"$SHIM" -include fame_ref_prelude.h &
  pids+=($!)
done
$NVCC -c "$HERE/ref_harness.cu" -o "$OBJ/ref_harness.o" -O2 $ARCH -w -I"$REF/include" -I"$SHIM" \
  -include fame_ref_prelude.h &
pids+=($!)
for p in "${pids[@]}"; do wait "$p"; done

LIBS="-L/usr/local/cuda/lib64 -lcudart -lcublas -lcufft -lpthread -ldl $OPENBLAS -Wl,-rpath,$(dirname "$OPENBLAS") -Wl,-rpath,/usr/local/cuda/lib64"
REFOBJS=$(ls "$OBJ"/*.o | grep -v -e '/Main.o$' -e '/ref_harness.o$')
g++ -o "$OUT/fame_ref_main" "$OBJ/Main.o" $REFOBJS $LIBS
g++ -o "$OUT/fame_ref_harness" "$OBJ/ref_harness.o" $REFOBJS $LIBS
# the reference's eigenvector writer alone, for the byte-for-byte writer test
g++ -O2 -w -o "$OUT/fame_ref_evwriter" "$HERE/ref_evwriter.cpp" "$OBJ/FAME_Save_Eigenvector.o"
echo "built $OUT/fame_ref_main, $OUT/fame_ref_harness and $OUT/fame_ref_evwriter"
