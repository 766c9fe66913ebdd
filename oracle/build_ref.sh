#!/bin/sh
# Builds oracle/_ref/libazeban_ref.so: the reference's pointwise headers
# (from the reference tree, unmodified) behind the C entry points of
# oracle/ref/pointwise.cpp, with the stand-ins of oracle/ref for ZisaCore,
# ZisaMemory, fmt and the CMake-generated config.hpp.  TEST INFRASTRUCTURE.
# Usage: oracle/build_ref.sh [reference root, default /root/reference]
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${1:-/root/reference}
if [ ! -d "$REF/include/azeban" ]; then
  echo "reference sources not found under $REF" >&2
  exit 2
fi
mkdir -p "$HERE/_ref"
${CXX:-g++} -std=c++17 -O2 -fPIC -shared -ffp-contract=off \
  -I "$HERE/ref" -I "$REF/include" \
  "$HERE/ref/pointwise.cpp" -o "$HERE/_ref/libazeban_ref.so"
echo "$HERE/_ref/libazeban_ref.so"
