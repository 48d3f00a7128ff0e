/*
 * grio.cpp — distance text output in the reference formats.
 *
 * int:   "%d %d\n" or "%d INF\n" per vertex (ads_int/support.cu:78-97);
 * float: "%d %f\n" or "%d INF\n" (the Galois writer the float results are
 *        compared against, cpu_sssp_float.patch:241-247; the ADDS float
 *        writer itself prints the node struct through %f and is unusable).
 * Lines are formatted by several threads into private buffers and written
 * in order, so a 16.8M-vertex result does not take a serial printf pass.
 */
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <thread>
#include <vector>

#include "../../include/adds.h"

static void format_range(uint32_t lo, uint32_t hi, const uint32_t *d, adds_wtype wt,
                         std::string *out) {
  char line[96];
  out->reserve((size_t)(hi - lo) * 16);
  for (uint32_t v = lo; v < hi; ++v) {
    int len;
    if (wt == ADDS_I32) {
      if (d[v] == (uint32_t)ADDS_INF_I32) len = snprintf(line, sizeof line, "%d INF\n", (int)v);
      else len = snprintf(line, sizeof line, "%d %d\n", (int)v, (int)d[v]);
    } else {
      float f;
      memcpy(&f, d + v, 4);
      if (d[v] == ADDS_INF_F32_BITS) len = snprintf(line, sizeof line, "%d INF\n", (int)v);
      else len = snprintf(line, sizeof line, "%d %f\n", (int)v, (double)f);
    }
    out->append(line, (size_t)len);
  }
}

extern "C" int adds_write_dist_text(const char *path, uint32_t n, const void *dist, adds_wtype wt) {
  if (!path || (!dist && n) || (wt != ADDS_I32 && wt != ADDS_F32)) return ADDS_ERR_INVALID;
  FILE *f = strcmp(path, "-") == 0 ? stdout : fopen(path, "w");
  if (!f) return ADDS_ERR_IO;
  const uint32_t *d = (const uint32_t *)dist;
  unsigned nt = std::thread::hardware_concurrency();
  if (nt == 0) nt = 1;
  if (nt > 32) nt = 32;
  const uint32_t block = 1u << 20;
  bool ok = true;
  for (uint32_t base = 0; base < n && ok; base += block * nt) {
    std::vector<std::string> parts(nt);
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t) {
      const uint64_t lo64 = (uint64_t)base + (uint64_t)t * block;
      if (lo64 >= n) break;
      const uint32_t lo = (uint32_t)lo64;
      const uint32_t hi = (uint32_t)((lo64 + block < n) ? lo64 + block : n);
      th.emplace_back(format_range, lo, hi, d, wt, &parts[t]);
    }
    for (auto &x : th) x.join();
    for (auto &p : parts)
      if (!p.empty() && fwrite(p.data(), 1, p.size(), f) != p.size()) ok = false;
  }
  if (f != stdout) {
    if (fclose(f) != 0) ok = false;
  } else {
    fflush(f);
  }
  return ok ? ADDS_OK : ADDS_ERR_IO;
}
