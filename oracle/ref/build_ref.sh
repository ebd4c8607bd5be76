#!/usr/bin/env bash
# oracle/ref/build_ref.sh -- TEST INFRASTRUCTURE.
#
# Builds the reference's own transport/grid/opacity/utils sources, unchanged
# and where they lie under the reference checkout, into the oracle harness
# binary oracle/_ref/sedona_ref.  MPI, GSL and HDF5 are replaced by the
# stand-ins in oracle/ref (one rank, Philox RNG, in-memory HDF5 store); Lua
# 5.2.1 is built from the reference's vendored tarball in a temporary
# directory and only its static library is kept (oracle/_ref/liblua.a).
#
# usage: oracle/ref/build_ref.sh [reference_root]
#   reference_root: the argument, else $SEDONA_REFERENCE, else /root/reference.
#   Exits 3 (nothing built) when no reference sources are there.
set -euo pipefail
REF=${1:-${SEDONA_REFERENCE:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=$(cd "$HERE/.." && pwd)/_ref
if [ ! -d "$REF/src" ]; then
  echo "reference sources not found at $REF (pass the reference root or set SEDONA_REFERENCE); nothing built" >&2
  exit 3
fi
mkdir -p "$OUT"
JOBS=${JOBS:-8}
# pick a C++ driver that can link OpenMP (the plain g++ wrapper on this image
# cannot find libgomp.spec; the triplet-named driver can)
PROBE=$(mktemp -d)
echo 'int main(){return 0;}' > "$PROBE/t.cpp"
PICK=""
for c in ${CXX:-} x86_64-linux-gnu-g++-13 x86_64-linux-gnu-g++ g++; do
  if command -v "$c" >/dev/null && "$c" -fopenmp "$PROBE/t.cpp" -o "$PROBE/t" 2>/dev/null; then PICK=$c; break; fi
done
rm -rf "$PROBE"
CXX=${PICK:-g++}

# --- Lua 5.2.1 from the vendored tarball (static library only) -------------
if [ ! -f "$OUT/liblua.a" ]; then
  TMP=$(mktemp -d)
  tar -xzf "$REF/src/external/lua-5.2.1.tar.gz" -C "$TMP"
  make -C "$TMP/lua-5.2.1/src" -s liblua.a SYSCFLAGS="-DLUA_USE_POSIX" MYCFLAGS="-fPIC -O2" >/dev/null
  cp "$TMP/lua-5.2.1/src/liblua.a" "$OUT/liblua.a"
  mkdir -p "$OUT/lua_include"
  for h in lua.h luaconf.h lualib.h lauxlib.h; do cp "$TMP/lua-5.2.1/src/$h" "$OUT/lua_include/"; done
  rm -rf "$TMP"
fi

# --- reference translation units on the transport path -----------------------
SRCS=(
  transport/transport.cpp transport/transport_init.cpp transport/transport_opacity.cpp
  transport/transport_mpi.cpp transport/transport_output.cpp transport/emission.cpp
  transport/scatter.cpp transport/relativity.cpp transport/radioactive.cpp
  transport/spectrum_array.cpp transport/thread_RNG.cpp transport/discrete_diffusion.cpp
  transport/solve_equilibrium.cpp transport/VoigtProfile.cpp
  opacity/AtomicData.cpp opacity/AtomicSpecies_init.cpp opacity/AtomicSpecies_opacities.cpp
  opacity/AtomicSpecies_state.cpp opacity/GasState.cpp opacity/GasState_opacities.cpp
  opacity/user_defined_opacity.cpp
  grid/grid_general.cpp grid/grid_1D_sphere.cpp grid/grid_3D_cart.cpp
  grid/grid_test.cpp grid/grid_1D_sphere_test.cpp transport/transport_test.cpp
  utils/locate_array.cpp utils/xy_array.cpp utils/h5utils.cpp utils/LuaInterface.cpp
  hydro/hydro_homologous.cpp
)
INC=(-I"$HERE/include" -I"$OUT/lua_include")
for d in main transport opacity grid utils hydro; do INC+=(-I"$REF/src/$d"); done
# -ffp-contract=off: no fused multiply-add, so the reference rounds every
# product and sum exactly as written (the GPU parity build does the same).
FLAGS=(-std=c++17 -O3 -march=native -ffp-contract=off -fopenmp -w -fPIC)

OBJ="$OUT/obj"
mkdir -p "$OBJ"
pids=()
for s in "${SRCS[@]}"; do
  o="$OBJ/$(echo "$s" | tr '/' '_').o"
  if [ ! -f "$o" ] || [ "$REF/src/$s" -nt "$o" ]; then
    $CXX "${FLAGS[@]}" "${INC[@]}" -c "$REF/src/$s" -o "$o" &
    pids+=($!)
    if [ ${#pids[@]} -ge $JOBS ]; then wait "${pids[0]}"; pids=("${pids[@]:1}"); fi
  fi
done
for p in "${pids[@]}"; do wait "$p"; done

$CXX "${FLAGS[@]}" "${INC[@]}" -c "$HERE/shims.cpp" -o "$OBJ/shims.o"
$CXX "${FLAGS[@]}" "${INC[@]}" -c "$HERE/ref_harness.cpp" -o "$OBJ/ref_harness.o"
$CXX "${FLAGS[@]}" -o "$OUT/sedona_ref" "$OBJ"/*.o "$OUT/liblua.a" -ldl -lm
# the reference's own locate_array test program (prints value/index pairs)
$CXX "${FLAGS[@]}" "${INC[@]}" -o "$OUT/locate_array_test" "$REF/src/utils/locate_array_test.cpp" \
  "$OBJ/utils_locate_array.cpp.o" "$OBJ/utils_h5utils.cpp.o" "$OBJ/shims.o" -lm
echo "built $OUT/sedona_ref"

# --- the compiled C++ binding of the B200 library -----------------------------
# sedona_ref_gpu: the same harness with its "gpu" mode, linking the binding
# (pubsed_b200/binding/transport_gpu.cpp, compiled here against the
# reference's own headers) and pubsed_b200/libsedona_gpu.so, found at run time
# next to the repository's oracle/_ref through $ORIGIN
ROOT=$(cd "$HERE/../.." && pwd)
if [ -f "$ROOT/pubsed_b200/libsedona_gpu.so" ]; then
  OBJG="$OUT/obj_gpu"
  mkdir -p "$OBJG"
  GINC=("${INC[@]}" -I"$ROOT/include" -I"$ROOT/pubsed_b200/binding")
  $CXX "${FLAGS[@]}" "${GINC[@]}" -c "$ROOT/pubsed_b200/binding/transport_gpu.cpp" -o "$OBJG/transport_gpu.o"
  $CXX "${FLAGS[@]}" "${GINC[@]}" -DSED_GPU_BINDING -c "$HERE/ref_harness.cpp" -o "$OBJG/ref_harness_gpu.o"
  REFOBJ=()
  for o in "$OBJ"/*.o; do [ "$(basename "$o")" = "ref_harness.o" ] || REFOBJ+=("$o"); done
  $CXX "${FLAGS[@]}" -o "$OUT/sedona_ref_gpu" "${REFOBJ[@]}" "$OBJG/ref_harness_gpu.o" "$OBJG/transport_gpu.o" \
    "$OUT/liblua.a" -L"$ROOT/pubsed_b200" -lsedona_gpu -Wl,-rpath,'$ORIGIN/../../pubsed_b200' -ldl -lm
  echo "built $OUT/sedona_ref_gpu"
fi
