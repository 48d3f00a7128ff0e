/*
 * sssp_cli.c — drop-in replacement for the reference `sssp` binaries
 * (ads_int/sssp and ads_float/sssp; main at ads_int/kernel.cu:290-305,
 * options at ads_int/support.cu:11-76).
 *
 *   sssp_int   [-q] [-g gpu] [-o out|-] [-b out.bin] [-s start] [-r runs] [-d shift] [-t]
 *              graph.gr
 *   sssp_float [same]
 *
 * Same flags, same distance file ("<v> <d>" / "<v> INF"), same fd-3 record
 * "<graph basename> <avg ms %.3f> <work %llu>" appended when fd 3 is open
 * (kernel.cu:215-216,282).  Like the reference, the int build averages 8
 * solves and counts popped vertices as work; the float build runs once and
 * counts scanned edges (ads_float/kernel.cu:59-60,225).  Extra flags:
 * -b raw distance words (n x 32-bit, little-endian; python -m
 * adds_b200.verify compares two such files bit for bit), -r runs, -d
 * bucket shift, -t autotune before timing.  Errors print a message and exit
 * non-zero instead of asserting.
 */
#include <errno.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "../../include/adds.h"

#ifdef ADDS_CLI_FLOAT
#define WT ADDS_F32
#define DEFAULT_RUNS 1
#else
#define WT ADDS_I32
#define DEFAULT_RUNS 8
#endif

static void usage(const char *prog) {
  fprintf(stderr,
          "usage: %s [-q] [-g gpunum] [-o output-file] [-b raw-output-file] [-s startNode] "
          "[-r runs] [-d shift] [-t] graph-file \n",
          prog);
}

static void die(const char *what, int rc) {
  fprintf(stderr, "%s: %s (%s)\n", what, adds_strerror(rc), adds_last_cuda_error());
  exit(1);
}

int main(int argc, char **argv) {
  int quiet = 0, gpu = 0, runs = DEFAULT_RUNS, shift = -1, tune = 0;
  long start = 0;
  const char *out = NULL, *out_bin = NULL;
  int c;
  if (argc == 1) {
    usage(argv[0]);
    return 1;
  }
  while ((c = getopt(argc, argv, "g:qo:b:s:r:d:tl")) != -1) {
    char *end = NULL;
    switch (c) {
      case 'q': quiet = 1; break;
      case 'o': out = optarg; break;
      case 'b': out_bin = optarg; break;
      case 'g':
        errno = 0;
        gpu = (int)strtol(optarg, &end, 10);
        if (errno || *end) {
          fprintf(stderr, "Invalid GPU device '%s'. An integer must be specified.\n", optarg);
          return EXIT_FAILURE;
        }
        break;
      case 's':
        start = strtol(optarg, &end, 10);
        if (*end || start < 0) {
          fprintf(stderr, "invalid start node '%s'\n", optarg);
          return 1;
        }
        break;
      case 'r': runs = atoi(optarg); if (runs < 1) runs = 1; break;
      case 'd': shift = atoi(optarg); break;
      case 't': tune = 1; break;
      case 'l': break; /* accepted for compatibility (prog_opts "ls:d:") */
      default: usage(argv[0]); return -1;
    }
  }
  if (optind >= argc) {
    usage(argv[0]);
    return -1;
  }
  const char *input = argv[optind];
  adds_graph *g = NULL;
  int rc = adds_graph_load_gr(input, WT, gpu, &g);
  if (rc) die("load graph", rc);
  adds_graph_info_t info;
  adds_graph_info(g, &info);
  if ((uint64_t)start >= info.n) {
    fprintf(stderr, "start node %ld out of range (n=%u)\n", start, info.n);
    return 1;
  }
  if (!quiet) printf("nnodes=%u, nedges=%llu.\n", info.n, (unsigned long long)info.m);
  adds_opts opts;
  adds_opts_init(&opts);
  opts.delta_shift = shift;
  if (tune) {
    uint32_t s = (uint32_t)start;
    rc = adds_tune(g, &s, 1, NULL, NULL);
    if (rc) die("tune", rc);
  }
  double total_ms = 0;
  unsigned long long total_work = 0;
  for (int r = 0; r < runs; ++r) {
    adds_stats st;
    rc = adds_sssp(g, (uint32_t)start, NULL, &opts, &st);
    if (rc) die("sssp", rc);
    total_ms += st.ms;
    total_work += (WT == ADDS_I32) ? st.items_popped : st.edges_scanned;
    if (!quiet) {
      printf("%s Measured time for sample = %.3fs\n", input, st.ms / 1000.0);
      printf("total work is %llu\n", (unsigned long long)((WT == ADDS_I32) ? st.items_popped : st.edges_scanned));
    }
  }
  const char *base = strrchr(input, '/');
  base = base ? base + 1 : input;
  FILE *d3 = fdopen(3, "a"); /* NULL when fd 3 is not open: no record */
  if (d3) {
    fprintf(d3, "%s %.3f %llu\n", base, total_ms / runs, total_work / (unsigned long long)runs);
    fflush(d3);
  }
  if (out || out_bin) {
    uint32_t *dist = (uint32_t *)malloc((size_t)info.n * 4);
    if (!dist) die("malloc", ADDS_ERR_OOM);
    rc = adds_graph_last_dist(g, dist);
    if (rc) die("copy distances", rc);
    if (out) {
      rc = adds_write_dist_text(out, info.n, dist, WT);
      if (rc) die("write output", rc);
    }
    if (out_bin) { /* raw 32-bit little-endian distance words, for bit checks */
      FILE *f = fopen(out_bin, "wb");
      if (!f || fwrite(dist, 4, info.n, f) != info.n || fclose(f) != 0)
        die("write binary output", ADDS_ERR_IO);
    }
    free(dist);
  }
  adds_graph_free(g);
  return 0;
}
