// ref_driver_dheap.cpp -- Dijkstra with decrease-key on the reference's own
// d-ary heap class (common/dheap.h:55-78, common/dheap.cpp).
//
// TEST INFRASTRUCTURE ONLY: built into oracle/_ref/libref_sssp.so by
// oracle/Makefile.  The reference ships dheap with no SSSP driver; this driver
// is written here and cross-checks the d-heap restatement in sssp_oracle.c.
#include <chrono>
#include <cstdint>
#include <vector>

#include "dheap.h"

#define NPS_REF_INF 1073741824  // common/global.h:19

extern "C" {

// Dijkstra with decrease-key driven on the reference's own dheap class.
double nps_ref_dijkstra_dheap(int32_t n, const int32_t* row, const int32_t* col, const int32_t* w, int32_t src,
                              int32_t d, int32_t* cost) {
  auto t0 = std::chrono::steady_clock::now();
  for (int32_t i = 0; i < n; ++i) cost[i] = NPS_REF_INF;
  dheap h((unsigned long)n, d);
  std::vector<char> done((size_t)n, 0);
  cost[src] = 0;
  h.insert((item)src + 1, 0);
  while (!h.empty()) {
    item it = h.deletemin();
    int32_t u = (int32_t)(it - 1);
    done[u] = 1;
    for (int32_t e = row[u]; e < row[u + 1]; ++e) {
      int32_t v = col[e];
      if (done[v]) continue;
      long nd = (long)cost[u] + w[e];
      if (nd >= NPS_REF_INF || nd >= cost[v]) continue;
      cost[v] = (int32_t)nd;
      if (h.member((item)v + 1)) h.changekey((item)v + 1, nd);
      else h.insert((item)v + 1, nd);
    }
  }
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

}  // extern "C"
