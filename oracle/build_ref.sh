#!/bin/sh
# Builds oracle/_ref/ref_timestep: oracle/ref_timestep.cu compiled against the
# reference's own header for its GPU time-step kernel, read where the reference
# is checked out (first argument, or $SPH3_REFERENCE, or /root/reference).
# Test infrastructure only; the binary stays out of the repository history.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${1:-${SPH3_REFERENCE:-/root/reference}}
INC="$REF/Particles_in_BH_Tree_III/Evrard_Collapse_2024"
[ -f "$INC/hfvCLibs_v7_hfv_v8.1.h" ] || { echo "reference header not found under $INC" >&2; exit 2; }
mkdir -p "$HERE/_ref"
NVCC=${CUDA_HOME:-/usr/local/cuda}/bin/nvcc
"$NVCC" -gencode arch=compute_100a,code=sm_100a -O3 -I "$INC" "$HERE/ref_timestep.cu" \
    -o "$HERE/_ref/ref_timestep.tmp$$" 2>"$HERE/_ref/build.log" || { cat "$HERE/_ref/build.log" >&2; exit 1; }
mv "$HERE/_ref/ref_timestep.tmp$$" "$HERE/_ref/ref_timestep"
echo "$HERE/_ref/ref_timestep"
