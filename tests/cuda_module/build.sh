#!/bin/sh
# Builds tests/cuda_module/_build/test_cuda_module: LELA code using
# Context<Modular<uint32>, CUDAModule<uint32>> (include/lela_cuda/cuda-module.h)
# against the reference headers and sources where they lie (REF), linked with
# lela_b200/liblela_cuda.so.  Needs the reference tree only to build.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
ROOT=$(cd "$HERE/../.." && pwd)
REF=${REF:-$(cd "$ROOT/.." && pwd)/reference}
if [ ! -d "$REF/lela" ]; then echo "reference tree not present; keeping prebuilt binary (if any)"; exit 0; fi
mkdir -p "$HERE/_build"
g++ -std=gnu++98 -O2 -fno-strict-aliasing -w \
    -I"$ROOT/oracle/shim" -I"$REF" -I"$ROOT/include" \
    -o "$HERE/_build/test_cuda_module" "$HERE/test_cuda_module.C" \
    "$REF/lela/util/commentator.C" "$REF/lela/util/debug.C" "$REF/lela/util/error.C" \
    "$REF/lela/util/timer.C" "$REF/lela/util/splicer.C" "$REF/lela/randiter/mersenne-twister.C" \
    -L"$ROOT/lela_b200" -llela_cuda -Wl,-rpath,'$ORIGIN/../../../lela_b200'
