#!/usr/bin/env bash
# Builds the reference-source oracle: SAMoS's own hot-path sources, compiled
# unmodified from the reference tree, plus oracle/ref_driver.cpp, into the
# git-ignored oracle/_ref/.  Test infrastructure: tests/ and bench.py's
# reference arm load the result; the product never does.
#
#   oracle/_ref/libsamos_ref.so       parity build: -O2, no fast-math, no FMA
#                                     contraction (the oracle's arithmetic rules)
#   oracle/_ref/libsamos_ref_fast.so  timing build: the reference's Release flags
#                                     (CMakeCFlagsSetup.txt: -O3 -funroll-loops
#                                     -ffast-math -DNDEBUG; -march=x86-64-v3 in
#                                     place of -march=native, because the library
#                                     is built here and run on another host)
#
# What stands in for the reference's dependencies (none is installed here):
#   oracle/ref_shim/boost/...  the Boost subset the sources include (format,
#                              lexical_cast, regex, string algorithms,
#                              property_tree writers, posix_time)
#   oracle/ref_shim/gsl/...    GSL's generator API over the project's counter
#                              noise stream (oracle/samos_oracle.c), so the
#                              reference consumes the oracle's and the GPU's noise
#   oracle/ref_shim/cgal_stub.hpp  compile-only CGAL names for the triangulation
#                              helpers neighbour_list.cpp defines outside its
#                              HAS_CGAL guard (they are never called)
#   oracle/ref_shim/parse_parameters.hpp  the parameter-map typedef without the
#                              Spirit grammar (the driver builds the maps)
#
# Usage: oracle/build_ref.sh [reference-src-dir]   (default /root/reference/src)
set -euo pipefail
here="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
src="${1:-/root/reference/src}"
out="$here/_ref"
if [ ! -d "$src/system" ]; then
  echo "build_ref.sh: reference sources not found at $src" >&2
  exit 2
fi
mkdir -p "$out/strict" "$out/fast"

files=(
  system/system.cpp system/particle.cpp system/cell_list.cpp system/neighbour_list.cpp
  system/mesh.cpp system/vertex.cpp system/edge.cpp system/face.cpp system/vector3d.cpp
  system/matrix3d.cpp messenger/messenger.cpp utils/rng.cpp potentials/potential.cpp
  potentials/pair/pair_soft_potential.cpp potentials/pair/pair_lj_potential.cpp
  potentials/pair/pair_morse_potential.cpp potentials/pair/pair_gaussian_potential.cpp
  potentials/external/external_self_propulsion.cpp aligner/aligner.cpp
  aligner/pair/pair_polar_aligner.cpp aligner/pair/pair_nematic_aligner.cpp
  aligner/pair/pair_vicsek_aligner.cpp constraints/constraint.cpp
  constraints/constraint_sphere.cpp constraints/constraint_plane.cpp
  constraints/constraint_cylinder.cpp constraints/constraint_torus.cpp
  constraints/constraint_ellipsoid.cpp constraints/constraint_peanut.cpp
  constraints/constraint_gyroid.cpp constraints/constraint_hourglass.cpp
  constraints/constraint_gaussian_bump.cpp constraints/constraint_tetrahedron.cpp
  constraints/constraint_slab.cpp constraints/constraint_plane_walls.cpp
  integrators/integrator_brownian.cpp integrators/integrator_brownian_pos.cpp
  integrators/integrator_brownian_align.cpp integrators/integrator_langevin.cpp
  integrators/integrator_fire.cpp integrators/integrator_nve.cpp
  integrators/integrator_vicsek.cpp
)

inc=(-I"$here/ref_shim")
for d in system messenger utils potentials potentials/pair potentials/external potentials/bond \
         potentials/angle aligner aligner/pair aligner/external constraints integrators; do
  inc+=(-I"$src/$d")
done

strict_flags=(-std=c++17 -O2 -fPIC -ffp-contract=off -fno-fast-math -w)
fast_flags=(-std=c++17 -O3 -funroll-loops -ffast-math -DNDEBUG -march=x86-64-v3 -fPIC -w)

compile() {  # flavour file
  local flavour="$1" f="$2" obj extra=()
  obj="$out/$flavour/$(echo "$f" | tr '/' '_' | sed 's/\.cpp$/.o/')"
  [ "$f" = system/neighbour_list.cpp ] && extra=(-include "$here/ref_shim/cgal_stub.hpp")
  if [ "$flavour" = strict ]; then
    g++ "${strict_flags[@]}" "${inc[@]}" "${extra[@]}" -c "$src/$f" -o "$obj"
  else
    g++ "${fast_flags[@]}" "${inc[@]}" "${extra[@]}" -c "$src/$f" -o "$obj"
  fi
}

jobs_max="$(nproc 2>/dev/null || echo 4)"
pids=()
for flavour in strict fast; do
  for f in "${files[@]}"; do
    compile "$flavour" "$f" &
    pids+=($!)
    if [ "${#pids[@]}" -ge "$jobs_max" ]; then
      wait "${pids[0]}"
      pids=("${pids[@]:1}")
    fi
  done
done
for p in "${pids[@]}"; do wait "$p"; done

# the driver and the noise stream (always strict: the noise definition is the
# oracle's, shared with the CUDA path)
g++ "${strict_flags[@]}" "${inc[@]}" -c "$here/ref_driver.cpp" -o "$out/strict/ref_driver.o"
g++ "${fast_flags[@]}" "${inc[@]}" -c "$here/ref_driver.cpp" -o "$out/fast/ref_driver.o"
gcc -std=c11 -O2 -fPIC -ffp-contract=off -fno-fast-math -c "$here/samos_oracle.c" -o "$out/noise.o"

g++ -shared -o "$out/libsamos_ref.so" "$out"/strict/*.o "$out/noise.o" -lm
g++ -shared -o "$out/libsamos_ref_fast.so" "$out"/fast/*.o "$out/noise.o" -lm
echo "built $out/libsamos_ref.so and $out/libsamos_ref_fast.so"
