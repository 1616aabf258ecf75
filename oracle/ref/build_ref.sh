#!/usr/bin/env bash
# Builds the reference's own CPU validators (from the read-only reference tree)
# into oracle/_ref/ for pinning the oracle.  Needs the reference tree, so it
# only runs where that tree is mounted; the products are git-ignored.
set -euo pipefail
REF=${GSW_REFERENCE_TREE:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/../_ref"
[ -d "$REF/src" ] || { echo "reference tree not found at $REF" >&2; exit 1; }
mkdir -p "$OUT"
for app in BFS SSSP CC BC PR GC; do
  lc=$(echo "$app" | tr 'A-Z' 'a-z')
  dst="$OUT/ref_$lc"
  if [ "$dst" -nt "$HERE/ref_driver.cu" ]; then continue; fi
  nvcc -std=c++14 -O2 --expt-extended-lambda -w \
    -gencode arch=compute_100a,code=sm_100a \
    -I "$REF" -I "$REF/src" -I "$REF/deps/moderngpu/src" \
    -Dmain=gsw_ref_app_main -DGSW_REF_$app -Xcompiler -pthread \
    "$HERE/ref_driver.cu" -o "$dst" &
done
wait
ls -1 "$OUT"
