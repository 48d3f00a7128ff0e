/*
 * ref_ingest_main.cu — times the reference's graph ingest: CSRGraph::read
 * (readFromGR, ads_int/csr_graph.cu:203-296: mmap and a per-edge host loop)
 * and CSRGraph::copy_to_gpu (csr_graph.cu:309-328: pageable cudaMemcpy of
 * every array).  MEASUREMENT INFRASTRUCTURE ONLY: oracle/build_ref.sh links
 * it with the reference's own csr_graph.cu into oracle/_ref/ref_ingest;
 * oracle/time_ingest.py runs it beside adds_graph_load_gr.
 *
 *   ref_ingest graph.gr   ->  one JSON line on stdout (after the reader's own
 *                             progress output): read_s, upload_s, n, m
 */
#include <stdio.h>
#include <string.h>
#include <time.h>

#include <cuda_runtime.h>

#include "csr_graph.h"

static double now_s() {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return t.tv_sec + 1e-9 * t.tv_nsec;
}

int main(int argc, char **argv) {
  if (argc != 2) {
    fprintf(stderr, "usage: %s graph.gr\n", argv[0]);
    return 2;
  }
  static char path[4096];
  strncpy(path, argv[1], sizeof path - 1); /* read() tokenises its argument */
  cudaFree(0);                             /* context creation is not ingest */
  CSRGraph hg, dg;
  const double t0 = now_s();
  if (hg.read(path) != 0) return 1;
  const double t1 = now_s();
  hg.copy_to_gpu(dg);
  if (cudaDeviceSynchronize() != cudaSuccess) return 1;
  const double t2 = now_s();
  printf("\n{\"read_s\": %.6f, \"upload_s\": %.6f, \"n\": %u, \"m\": %u}\n", t1 - t0, t2 - t1,
         hg.nnodes, hg.nedges);
  return 0;
}
