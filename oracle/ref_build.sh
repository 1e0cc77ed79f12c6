#!/usr/bin/env bash
# Builds the reference's own path (carlosduelo/visualTur) from its sources,
# where they lie, into oracle/_ref/vtref.  Test infrastructure only: the
# binary generates the golden vectors that pin the CPU oracle.
#
# Flags follow the reference Makefile (-G -O0 -g, Makefile:1-6) except the
# architecture: sm_20 is not supported by CUDA 12.9, so sm_100a is used.
# libhdf5 is absent on this image; oracle/ref_shim/ provides the few HDF5
# calls FileManager makes, over raw volume files.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${VT_REFERENCE_DIR:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -d "$REF/src" ]; then
    echo "ref_build: reference sources not found at $REF; keeping existing $OUT" >&2
    exit 0
fi
mkdir -p "$OUT/obj"
NVCC="${NVCC:-nvcc}"
FLAGS="-G -O0 -g -gencode arch=compute_100a,code=sm_100a -ccbin /usr/bin/g++ -w -I$REF/inc -I$HERE/ref_shim"
for f in Screen.cpp Camera.cu Octree.cu rayCaster.cu lruCache.cu FileManager.cu visualTur.cu; do
    $NVCC -c $FLAGS "$REF/src/$f" -o "$OUT/obj/${f%.*}.o"
done
$NVCC -c $FLAGS "$HERE/ref_shim/h5shim.cpp" -o "$OUT/obj/h5shim.o"
$NVCC -c $FLAGS -std=c++17 "$HERE/ref_driver.cu" -o "$OUT/obj/ref_driver.o"
O="$OUT/obj"
$NVCC $FLAGS $O/Screen.o $O/Camera.o $O/Octree.o $O/rayCaster.o $O/lruCache.o $O/FileManager.o \
    $O/visualTur.o $O/h5shim.o $O/ref_driver.o -o "$OUT/vtref" -lpthread
# The reference's own octree builder CLI (host code only; runs without a GPU).
$NVCC -c $FLAGS "$REF/src/CreateOctree.cu" -o "$O/CreateOctree.o"
$NVCC -c $FLAGS "$REF/src/VolumeToOctree.cu" -o "$O/VolumeToOctree.o"
$NVCC $FLAGS $O/CreateOctree.o $O/FileManager.o $O/h5shim.o $O/VolumeToOctree.o -o "$OUT/volumeToOctree"
echo "ref_build: built $OUT/vtref $OUT/volumeToOctree"
