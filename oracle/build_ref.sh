#!/usr/bin/env bash
# Builds the reference's own CPU engine (Graph_Numa, the MULTI_CORE engine)
# into oracle/_ref/cgref_oracle, for use as the test oracle and the timed
# CPU baseline.  Test infrastructure only.
#
# The reference cannot be compiled as it ships (no Makefile, absolute
# CUDA-11.7 include paths, libnuma/TBB includes, comment-stripping damage).
# This recipe copies the few directories the CPU engine needs into a scratch
# folder under oracle/_ref/, applies seven one-line fixes there, builds the
# harness, and deletes the scratch copy again.  Nothing of the reference is
# written outside oracle/_ref/ and no reference source is kept.
#
# The seven fixes (paths relative to the reference's CGgraph/ folder):
#   1 Basic/GPU/cuda_include.cuh:8-10   absolute /usr/local/cuda-11.7 paths -> <...>
#   2 Basic/Thread/cpu_info.hpp (end)    class CPUInfo is never closed -> append "};"
#   3 Basic/Thread/omp_def.hpp:73        stray trailing "/" after a statement
#   4 Basic/Bitmap/fixed_bitset.cuh:152  stray trailing "/" after a statement
#   5 Basic/Bitmap/fixed_bitset.cuh:200  stripped comment left as "/" -> "//"
#   6 Basic/Other/generate_mtx.hpp:15    "..." + "_NATIVE.mtx" (pointer add) -> one literal
#   7 my_project/CGgraph/GraphNuma.cuh:53 member "active" used at :297 but never declared
# libnuma and TBB are replaced by the headers in oracle/refshim/.
#
# usage: oracle/build_ref.sh [reference root]
# The reference root is the argument, else $CGGRAPH_REFERENCE_ROOT, else
# /root/reference (where the build container mounts it).
set -euo pipefail

HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${CGGRAPH_REFERENCE_ROOT:-/root/reference}}/CGgraph"
OUT="$HERE/_ref"
SRC="$OUT/src"

if [ ! -d "$REF/Basic" ]; then
    echo "build_ref: reference not found at $REF; keeping any prebuilt oracle/_ref" >&2
    exit 0
fi

rm -rf "$SRC"
mkdir -p "$SRC/my_project"
# The vendored CUB (Basic/GPU/ThirdLib) is unused by the CPU engine.
(cd "$REF" && tar cf - --exclude='Basic/GPU/ThirdLib' Basic) | (cd "$SRC" && tar xf -)
cp -r "$REF/my_project/CGgraph" "$SRC/my_project/CGgraph"
chmod -R u+w "$SRC"

B="$SRC/Basic"
MP="$SRC/my_project/CGgraph"
sed -i 's#</usr/local/cuda-11.7/include/\([a-z_]*\.h\)>#<\1>#' "$B/GPU/cuda_include.cuh"        # 1
printf '\n};\n' >> "$B/Thread/cpu_info.hpp"                                                   # 2
sed -i '73s#;/[[:space:]]*$#;#' "$B/Thread/omp_def.hpp"                                       # 3
sed -i '152s#;/[[:space:]]*$#;#' "$B/Bitmap/fixed_bitset.cuh"                                 # 4
sed -i '200s#^\([[:space:]]*\)/\([^/]\)#\1//\2#' "$B/Bitmap/fixed_bitset.cuh"                 # 5
sed -i '15s#"\.\.\." + "_NATIVE\.mtx"#"..._NATIVE.mtx"#' "$B/Other/generate_mtx.hpp"          # 6
sed -i '53a\	DoubleBuffer<dense_bitset> active;' "$MP/GraphNuma.cuh"                             # 7

# Each fix must have applied exactly where expected.
grep -q '<cuda_runtime.h>' "$B/GPU/cuda_include.cuh"
! grep -q 'cuda-11.7' "$B/GPU/cuda_include.cuh"
! sed -n '73p' "$B/Thread/omp_def.hpp" | grep -q ';/'
! sed -n '152p' "$B/Bitmap/fixed_bitset.cuh" | grep -q ';/'
sed -n '200p' "$B/Bitmap/fixed_bitset.cuh" | grep -q '^[[:space:]]*//'
grep -q '"..._NATIVE.mtx"' "$B/Other/generate_mtx.hpp"
sed -n '54p' "$MP/GraphNuma.cuh" | grep -q 'DoubleBuffer<dense_bitset> active;'

NVCC="${NVCC:-nvcc}"
"$NVCC" -std=c++17 -O3 -x cu -Xcompiler -fopenmp -Xcompiler -w -w \
    -I"$HERE/refshim" -I"$SRC" -I"$MP" \
    "$HERE/ref_harness.cu" -o "$OUT/cgref_oracle.tmp" -lgomp
mv "$OUT/cgref_oracle.tmp" "$OUT/cgref_oracle"
rm -rf "$SRC"
echo "build_ref: built $OUT/cgref_oracle"
