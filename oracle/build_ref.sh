#!/bin/bash
# Builds the reference GustANN all-in-GPU (`search_mem -G`) path from its own
# sources, where they lie, into oracle/_ref/libgustann_ref.so (checker only).
#
#  * The reference's CMake build is not used; each translation unit that the
#    path links (src/CMakeLists.txt:3 minus the BaM/SPDK/io_uring/AIO options,
#    which are off by default, CMakeLists.txt:27-34) is compiled directly.
#  * spdlog (an empty submodule here) is replaced by the no-op logging header
#    in oracle/ref_shim: the reference uses it for log lines only.
#  * `-include cstdint`: some reference headers use int64_t without including it.
#  * pure_mem.cu alone gets -DNDEBUG, which removes the device-side assert at
#    src/impl/pure_mem.cuh:373 (it can only fire on an invalid merge state). It is
#    not applied elsewhere because src/nav_graph.cu:52 reads map.txt inside an
#    assert().
#  * Device code keeps nvcc's defaults (-fmad=true), like the reference build.
#
# Usage: oracle/build_ref.sh <reference_dir>   (or $GANN_REF_DIR)
set -euo pipefail
REF=${1:-${GANN_REF_DIR:-}}
if [ -z "$REF" ]; then
  echo "usage: build_ref.sh <reference_dir> (or set GANN_REF_DIR)" >&2
  exit 2
fi
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
OBJ="$OUT/obj"
SRC="$REF/src"
if [ ! -f "$SRC/pure_mem.cu" ]; then
  echo "build_ref: reference sources not found under $REF" >&2
  exit 2
fi
mkdir -p "$OBJ"
NVCC=${NVCC:-nvcc}
ARCH="-gencode arch=compute_100a,code=sm_100a"
COMMON="-std=c++17 -O2 -g -lineinfo -include cstdint -I$HERE/ref_shim -I$SRC"

compile_cu() {  # $1 = source relative to src/, $2 = extra flags
  local o="$OBJ/$(echo "$1" | tr '/' '_').o"
  $NVCC $ARCH $COMMON $2 -Xcompiler -fPIC -c "$SRC/$1" -o "$o"
  echo "$o"
}
compile_cpp() {
  local o="$OBJ/$(echo "$1" | tr '/' '_').o"
  g++ -std=c++17 -O2 -g -fPIC -include cstdint -I"$HERE/ref_shim" -I"$SRC" \
      -I/usr/local/cuda/include -c "$SRC/$1" -o "$o"
  echo "$o"
}

objs=()
objs+=("$(compile_cpp layout.cpp)")
objs+=("$(compile_cpp io/mem_io.cpp)")
objs+=("$(compile_cu pq_search.cu "")")
objs+=("$(compile_cu nav_graph.cu "")")
objs+=("$(compile_cu pure_mem.cu "-DNDEBUG")")
objs+=("$(compile_cu ssd_search.cu "")")
objs+=("$(compile_cu hybrid.cu "")")
objs+=("$(compile_cu hyd_task_runner.cu "")")
drv="$OBJ/ref_driver.o"
$NVCC $ARCH $COMMON -Xcompiler -fPIC -c "$HERE/ref_driver.cu" -o "$drv"
objs+=("$drv")
$NVCC $ARCH -shared -o "$OUT/libgustann_ref.so" "${objs[@]}" -lpthread
echo "built $OUT/libgustann_ref.so"
