#!/bin/sh
# Builds oracle A: the unmodified feMorph reference sources, compiled where
# they lie (read-only) with the project-written Boost/Armadillo shim in
# oracle/shim, linked with oracle/refdrv.cpp (driver + full-precision state
# hooks).  Outputs go to oracle/_ref/ only.  Needs the reference tree; the GPU
# host only runs the prebuilt oracle/_ref/fm_refdrv.
#   FEMORPH_REFERENCE=<path to the reference project>  (default /root/reference)
# Exit status 2: the reference sources are not there (nothing is built).
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
SRC=${FEMORPH_REFERENCE:-/root/reference}/src
OUT=$HERE/_ref
OBJ=$OUT/obj
[ -d "$SRC" ] || { echo "reference sources not found at $SRC" >&2; exit 2; }
mkdir -p "$OBJ"
CXXFLAGS="-std=c++11 -O2 -w -DUSE_ARMADILLO -include unistd.h -I$HERE/shim -I$SRC"
pids=""
for f in "$SRC"/*.cpp; do
  b=$(basename "$f" .cpp)
  [ "$b" = main ] && continue
  if [ ! -f "$OBJ/$b.o" ] || [ "$f" -nt "$OBJ/$b.o" ]; then
    g++ $CXXFLAGS -c "$f" -o "$OBJ/$b.o" &
    pids="$pids $!"
  fi
done
for p in $pids; do wait $p; done
# Hooked members: every call from the solvers to these two femModel members is
# redirected (GNU ld --wrap) to oracle/refdrv.cpp, which forwards to the real one.
EXPORT_SYM=$(nm "$OBJ/femVMSExplicitFluidSolver.o" | awk '/ U .*femModel.*ExportToVTKLegacy/ {print $2}')
SETVEL_SYM=$(nm "$OBJ/femVMSExplicitFluidSolver.o" | awk '/ U .*femModel.*setNodeVelocity/ {print $2}')
[ -n "$EXPORT_SYM" ] && [ -n "$SETVEL_SYM" ] || { echo "hook symbols not found" >&2; exit 3; }
g++ $CXXFLAGS -DFM_EXPORT_SYM="\"$EXPORT_SYM\"" -DFM_SETVEL_SYM="\"$SETVEL_SYM\"" \
  "$HERE/refdrv.cpp" "$OBJ"/*.o -o "$OUT/fm_refdrv" \
  -Wl,--wrap="$EXPORT_SYM" -Wl,--wrap="$SETVEL_SYM"
echo "built $OUT/fm_refdrv"
# Drop-in check binary: the same driver linked with femorph_b200's femSolver
# adapters (femorph_b200/adapter) and libfemorph_b200.so.
LIBDIR=$HERE/../femorph_b200
if [ -f "$LIBDIR/libfemorph_b200.so" ]; then
  g++ $CXXFLAGS -DFM_WITH_GPU_ADAPTER -I"$LIBDIR/adapter" -I"$HERE/../include" \
    -DFM_EXPORT_SYM="\"$EXPORT_SYM\"" -DFM_SETVEL_SYM="\"$SETVEL_SYM\"" \
    "$HERE/refdrv.cpp" "$LIBDIR/adapter/femExplicitFluidSolverGPU.cpp" "$LIBDIR/adapter/femPoissonSolverGPU.cpp" \
    "$OBJ"/*.o -o "$OUT/fm_gpudrv" \
    -L"$LIBDIR" -lfemorph_b200 -Wl,-rpath,'$ORIGIN/../../femorph_b200' \
    -Wl,--wrap="$EXPORT_SYM" -Wl,--wrap="$SETVEL_SYM"
  echo "built $OUT/fm_gpudrv"
fi
