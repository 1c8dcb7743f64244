#!/usr/bin/env bash
# Links the reference's own Main.cpp, preprocessing and host tools with
# FAME_Main_Code_b200.cpp and libfame_b200.so: the drop-in program that reads
# Popt.txt and the material description and writes Data_Omega_array.txt exactly as
# the reference's Main.out does, with the band-structure solve on this library.
#
#   fame-isotropic-gpu_b200/shim/build_main.sh REFERENCE_ROOT   (the reference project's root directory)
#
# The reference sources are compiled where they lie (none is copied or edited);
# objects and the program go to fame-isotropic-gpu_b200/shim/_build/.  Run
# `make -C fame-isotropic-gpu_b200` first.
set -euo pipefail
REF=${1:?"usage: $0 REFERENCE_ROOT"}
HERE=$(cd "$(dirname "$0")" && pwd)
PKG=$(dirname "$HERE")
OUT="$HERE/_build"
if [ ! -f "$REF/Main.cpp" ]; then
  echo "reference sources not found at $REF" >&2
  exit 1
fi
if [ ! -f "$PKG/libfame_b200.so" ]; then
  echo "build libfame_b200.so first (make -C $PKG)" >&2
  exit 1
fi
mkdir -p "$OUT/obj"
CXXFLAGS="-O2 -m64 -w -I$REF/include -I$PKG/../include"
pids=()
for src in "$REF"/Main.cpp "$REF"/FAME_Preprocessing/*.cpp "$REF"/FAME_Tools/*.cpp; do
  extra="-include time.h"
  case "$(basename "$src")" in
    vec_norm.cpp|vec_inner_prod.cpp) extra="$extra -std=gnu++11 -fext-numeric-literals" ;;
  esac
  g++ -c "$src" -o "$OUT/obj/$(basename "${src%.cpp}").o" $CXXFLAGS $extra &
  pids+=($!)
done
g++ -c "$HERE/FAME_Main_Code_b200.cpp" -o "$OUT/obj/FAME_Main_Code_b200.o" $CXXFLAGS -include time.h &
pids+=($!)
for p in "${pids[@]}"; do wait "$p"; done
g++ -pthread -o "$OUT/fame_b200_main" "$OUT"/obj/*.o -L"$PKG" -lfame_b200 -Wl,-rpath,"\$ORIGIN/../.." \
  -L/usr/local/cuda/lib64 -lcudart -Wl,-rpath,/usr/local/cuda/lib64
echo "built $OUT/fame_b200_main"
