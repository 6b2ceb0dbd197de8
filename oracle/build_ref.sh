#!/usr/bin/env bash
# Builds the reference implementation (mgowanlock/gpu_self_join) FROM ITS OWN
# SOURCES into oracle/_ref/<config>/main, one binary per params.h configuration.
# The reference bakes its switches into params.h at compile time, and its
# sources include "params.h" from their own directory, so each configuration is
# compiled in a throw-away temporary directory holding the reference sources and
# a params.h written here; only the binaries land in oracle/_ref/.  No reference
# source is kept in this repository.
#
# STAMP=1 is not built: the reference's main.cu does not compile with it
# (main.cu:556, 580 and 634 read neighborTableLookup members that exist only
# when STAMP=0), so unicomp configurations are pinned through their STAMP=0
# builds, which report the same pair set.
#
# The binaries are test infrastructure: the oracle's pin against the reference
# (tests/golden/make_ref_fixtures.py), the reference arm of bench.py, and the
# reference's own timing of the benchmarked workloads (tests/golden/time_ref_gpu.py).
#
# usage: oracle/build_ref.sh [REFERENCE_DIR]
#   (default: $GSJ_REFERENCE_DIR, else the checkout at /root/reference)
set -euo pipefail
REF=${1:-${GSJ_REFERENCE_DIR:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
[ -d "$REF" ] || { echo "reference sources not found at $REF" >&2; exit 1; }
mkdir -p "$OUT"
JOBS=${JOBS:-4}

# name  GPUNUMDIM NUMINDEXEDDIM DTYPE STAMP REORDER ILP SHORTCIRCUIT QUERYREORDER PRINTNEIGHBORTABLE [SORT]
CONFIGS=(
  "d2_plain        2  2 float  0 0 0 0 0 1"
  "d2_plain_f64    2  2 double 0 0 0 0 0 1"
  "d6_plain        6  6 float  0 0 0 0 0 1"
  "d18_k6_ilp8_sc 18  6 float  0 1 8 1 1 1"
  "d18_k6_ilp8    18  6 float  0 1 8 0 1 1"
  "d18_k6_ilp4_sc 18  6 float  0 1 4 1 0 1"
  "d90_k6_ilp8_sc 90  6 float  0 1 8 1 1 1"
  "d5_k3_f64_ilp2_sc 5 3 double 0 1 2 1 1 1"
  "d5_k3_f64_plain   5 3 double 0 1 0 0 0 1"
  "d18_k6_f64_ilp8  18 6 double 0 1 8 0 1 1"
  "d18_k6_f64_ilp8_sc 18 6 double 0 1 8 1 1 1"
  "d5_k3_f32_ilp8    5 3 float  0 1 8 0 0 1"
  "d5_k3_f64_ilp8    5 3 double 0 1 8 0 0 1"
  "d3_k3_f64_ilp2    3 3 double 0 0 2 0 0 1"
  "d5_k3_f32_ilp2_sc 5 3 float  0 1 2 1 1 1"
  "d2_sort           2 2 float  0 0 0 0 0 1 1"
  "d3_k2_sort        3 2 float  0 0 0 0 0 1 1"
  "d5_k3_f64_sort    5 3 double 0 1 2 1 0 1 1"
  # timing builds of the benchmarked workloads (no neighbour-table print)
  "t_d2   2 2 float 0 0 0 0 0 0"
  "t_d6   6 6 float 0 0 0 0 0 0"
  "t_d18 18 6 float 0 1 8 1 1 0"
  "t_d90 90 6 float 0 1 8 1 1 0"
)

write_params() {  # $1 dir, then the fields
  local d=$1 n=$2 k=$3 t=$4 st=$5 ro=$6 ilp=$7 sc=$8 qr=$9 pr=${10} so=${11:-0}
  cat > "$d/params.h" <<EOF
#define BLOCKSIZE 256
#define GPUNUMDIM $n
#define NUMINDEXEDDIM $k
#define DTYPE $t
#define PRINTNEIGHBORTABLE $pr
#define STAMP $st
#define LINEARSTAMP 0
#define SORT $so
#define REORDER $ro
#define ILP $ilp
#define SHORTCIRCUIT $sc
#define QUERYREORDER $qr
#define SEARCHFILTTIME 0
#define COUNTMETRICS 1
#define CTYPE unsigned long long
#define GPUBUFFERSIZE 100000000
#define GPUSTREAMS 3
#define MINBATCHES 3
#define SAMPLERATE 0.015
EOF
}

build_one() {
  local line=$1
  set -- $line
  local name=$1; shift
  local dst="$OUT/$name"
  if [ -x "$dst/main" ]; then echo "have $name"; return 0; fi
  local tmp
  tmp=$(mktemp -d)
  cp "$REF"/*.cu "$REF"/*.cpp "$REF"/*.h "$tmp"/
  write_params "$tmp" "$@"
  local FL="-std=c++14 -O3 -Xcompiler -fopenmp -lineinfo -arch=compute_100 -code=sm_100 -D_MWAITXINTRIN_H_INCLUDED -D_FORCE_INLINES"
  ( cd "$tmp" &&
    nvcc $FL -c import_dataset.cpp && nvcc $FL -c tree_index.cpp &&
    nvcc $FL -c main.cu && nvcc $FL -c kernel.cu && nvcc $FL -c GPU.cu &&
    nvcc -std=c++14 -O3 -Xcompiler -fopenmp -lcuda -arch=compute_100 -code=sm_100 \
         import_dataset.o tree_index.o GPU.o kernel.o main.o -o main ) > "$tmp/build.log" 2>&1 || {
      echo "build of $name failed:"; tail -20 "$tmp/build.log"; rm -rf "$tmp"; return 1; }
  mkdir -p "$dst"
  cp "$tmp/main" "$dst/main"
  rm -rf "$tmp"
  echo "built $name"
}

export -f build_one write_params
export REF OUT
printf '%s\n' "${CONFIGS[@]}" | xargs -P "$JOBS" -I{} bash -c 'build_one "$@"' _ {}

# The reference's CPU self-join (R-tree search + filter, tree_index.cpp and
# RTree.h) behind a timing harness (oracle/ref_rtree_harness.cpp), 2-D float:
# the reference arm of bench.py.  Plain g++ on the reference's own files.
build_harness() {
  local dst="$OUT/rtree_harness"
  if [ -x "$dst" ]; then echo "have rtree_harness"; return 0; fi
  local tmp
  tmp=$(mktemp -d)
  cp "$REF"/tree_index.cpp "$REF"/tree_index.h "$REF"/RTree.h "$tmp"/
  cp "$HERE/ref_rtree_harness.cpp" "$tmp"/
  write_params "$tmp" 2 2 float 0 0 0 0 0 0
  ( cd "$tmp" && g++ -O3 -std=c++14 -fopenmp tree_index.cpp ref_rtree_harness.cpp -o rtree_harness ) \
    > "$tmp/build.log" 2>&1 || { echo "harness build failed"; tail -20 "$tmp/build.log"; rm -rf "$tmp"; return 1; }
  cp "$tmp/rtree_harness" "$dst"
  rm -rf "$tmp"
  echo "built rtree_harness"
}
build_harness
