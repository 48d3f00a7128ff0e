#!/usr/bin/env bash
# Builds the reference ADDS binaries (UCLA-VAST/adds, ads_int/ and
# ads_float/) for sm_100a into oracle/_ref/.  TEST INFRASTRUCTURE ONLY: the
# binaries pin the oracle (tests/golden/make_ref_golden.py) and time the
# reference GPU kernel; the product never runs them.
#
# The sources are compiled from a scratch copy outside this repository
# because five harness edits are needed; nothing else is changed:
#   1. the vendored CUB 1.8.0 no longer compiles against CUDA 12.9's thrust:
#      kernel.cu includes the toolkit's <cub/cub.cuh> instead;
#   2. csr_graph.cu includes boost/mpl/if.hpp but never uses it: removed;
#   3. MAX_TB (wl.h:23 int 128, ads_float/wl.h:16 256) is below the worker
#      block count on 148 SMs (num_tb = tb_per_sm * (num_sm - 1)): 512;
#   4. gg_main aborts when cudaOccupancyMaxPotentialBlockSize (the block size
#      of best occupancy) is below its fixed TB_SIZE (kernel.cu:194-199); on a
#      2048-thread SM that size is smaller although TB_SIZE threads are
#      launchable, so the check uses the kernel's maxThreadsPerBlock;
#   5. float only, so its distances can be compared: copy_to_cpu copies
#      nnodes * sizeof(edge_data_type) bytes of 8-byte node records
#      (ads_float/csr_graph.cu:343-345) -> sizeof(node_data_type), and
#      output() prints the record through %f (ads_float/support.cu:93)
#      -> prints .dist, INF being dist == FLT_MAX.
# Outputs: oracle/_ref/ads_int_sssp, oracle/_ref/ads_float_sssp, and
# oracle/_ref/ref_ingest (the int csr_graph.cu reader and upload under the
# timing main oracle/ref_ingest_main.cu, for oracle/time_ingest.py).
set -euo pipefail
REF=${REF:-/root/reference}
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
[ -d "$REF/ads_int" ] || { echo "reference tree not found at $REF" >&2; exit 2; }
mkdir -p "$OUT"
WORK="$(mktemp -d /tmp/adds_ref_build.XXXXXX)"
trap 'rm -rf "$WORK"' EXIT
for v in int float; do
  cp -r "$REF/ads_$v" "$WORK/ads_$v"
  cd "$WORK/ads_$v"
  sed -i 's|#include "../cub-1.8.0/cub/cub.cuh"|#include <cub/cub.cuh>|' kernel.cu
  sed -i 's|#include <boost/mpl/if.hpp>||' csr_graph.cu
  sed -i -E 's|#define MAX_TB [0-9]+|#define MAX_TB 512|' wl.h
  sed -i 's|cudaOccupancyMaxPotentialBlockSize(&min_grid_size, &max_num_threads, sssp_kernel);|{ cudaFuncAttributes fa; cudaFuncGetAttributes(\&fa, sssp_kernel); max_num_threads = fa.maxThreadsPerBlock; (void)min_grid_size; }|' kernel.cu
  grep -q 'fa.maxThreadsPerBlock' kernel.cu || { echo "block-size check patch did not apply" >&2; exit 3; }
  if [ "$v" = float ]; then
    sed -i 's|nnodes \* sizeof(edge_data_type), cudaMemcpyDeviceToHost|nnodes * sizeof(node_data_type), cudaMemcpyDeviceToHost|' csr_graph.cu
    sed -i 's|nnodes \* sizeof(edge_data_type), cudaMemcpyHostToDevice|nnodes * sizeof(node_data_type), cudaMemcpyHostToDevice|' csr_graph.cu
    sed -i 's|if (g.node_data\[i\] == INF) {|if (g.node_data[i].dist == FLT_MAX) {|' support.cu
    sed -i 's|fprintf(f, "%d %f\\n", i, g.node_data\[i\]);|fprintf(f, "%d %f\\n", i, g.node_data[i].dist);|' support.cu
    grep -q 'node_data\[i\].dist);' support.cu || { echo "float output patch did not apply" >&2; exit 3; }
  fi
  grep -q '#define MAX_TB 512' wl.h || { echo "MAX_TB patch did not apply" >&2; exit 3; }
  "$NVCC" kernel.cu support.cu csr_graph.cu -O3 -gencode arch=compute_100a,code=sm_100a \
    -rdc=true -lcudadevrt -w -o "$OUT/ads_${v}_sssp"
  if [ "$v" = int ]; then
    # the reference's own reader and upload (csr_graph.cu) under a timing main
    "$NVCC" "$HERE/ref_ingest_main.cu" csr_graph.cu -I. -O3 \
      -gencode arch=compute_100a,code=sm_100a -w -o "$OUT/ref_ingest"
  fi
  cd - > /dev/null
done
echo "built: $OUT/ads_int_sssp $OUT/ads_float_sssp $OUT/ref_ingest"
