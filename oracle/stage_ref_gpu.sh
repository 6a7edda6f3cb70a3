#!/usr/bin/env bash
# Stages the reference's own Numba kernel modules (src/kernels/*.py of
# Cosmo-NBody, unmodified) into oracle/_ref/ so that `bench.py --impl
# reference-gpu` can launch them on the GPU box.  oracle/_ref/ is git-ignored
# (the reference's files never enter this repository's history) and travels
# to the GPU box with the rest of the working tree.  Test infrastructure only.
set -euo pipefail
here="$(cd "$(dirname "$0")" && pwd)"
src="${1:-/root/reference}"
if [ ! -d "$src/src/kernels" ]; then
    echo "no reference checkout at $src" >&2
    exit 1
fi
dst="$here/_ref/src/kernels"
mkdir -p "$dst"
touch "$here/_ref/src/__init__.py"
for f in __init__.py morton.py tree_kernels.py physics_kernels.py render_kernels.py; do
    cp "$src/src/kernels/$f" "$dst/$f"
done
echo "staged $(ls "$dst" | wc -l) reference kernel modules in $dst"
