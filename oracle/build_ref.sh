#!/bin/sh
# Builds oracle/_ref/ref_timestep and oracle/_ref/ref_cooling: the small
# drivers oracle/ref_timestep.cu and oracle/ref_cooling.cu compiled against the
# reference's own header for its GPU time-step and heating/cooling kernels,
# read where the reference is checked out (first argument, or
# $SPH3_REFERENCE, or /root/reference).  Test infrastructure only; the
# binaries stay out of the repository history.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${1:-${SPH3_REFERENCE:-/root/reference}}
INC="$REF/Particles_in_BH_Tree_III/Evrard_Collapse_2024"
[ -f "$INC/hfvCLibs_v7_hfv_v8.1.h" ] || { echo "reference header not found under $INC" >&2; exit 2; }
mkdir -p "$HERE/_ref"
NVCC=${CUDA_HOME:-/usr/local/cuda}/bin/nvcc
for prog in ref_timestep ref_cooling; do
    "$NVCC" -gencode arch=compute_100a,code=sm_100a -O3 -I "$INC" "$HERE/$prog.cu" \
        -o "$HERE/_ref/$prog.tmp$$" 2>"$HERE/_ref/build_$prog.log" || { cat "$HERE/_ref/build_$prog.log" >&2; exit 1; }
    mv "$HERE/_ref/$prog.tmp$$" "$HERE/_ref/$prog"
    echo "$HERE/_ref/$prog"
done
