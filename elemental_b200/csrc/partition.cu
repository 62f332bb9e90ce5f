// Sharding of independent systems across GPUs (host code).
//
// The batched and served forms solve independent systems, so N GPUs share a
// problem list without any device collective: every rank computes the same
// partition from the same list, solves the systems it owns, and only the
// statuses (and whatever results the caller wants) are gathered on the host.
// The partition balances the factorization work: system i costs
// c_i = w_kind * n_i^3 (w = 1/3 for an HPD solve, 2/3 for LU), and the systems
// are dealt out largest first to the currently least-loaded part (greedy
// longest-processing-time order).  Ties in cost keep the list order, ties in
// load go to the lowest part index, so the result depends only on the inputs.
#include <algorithm>
#include <numeric>
#include <queue>
#include <vector>

#include "internal.h"

extern "C" int egpu_partition_systems(int count, const int* n, const int* kind, int parts, int* owner,
                                      double* load) {
  if (count < 0 || parts < 1 || (count > 0 && (!n || !owner))) return EGPU_ERR_ARG;
  std::vector<double> cost(count);
  for (int i = 0; i < count; ++i) {
    if (n[i] < 0) return EGPU_ERR_ARG;
    const double w = (kind && kind[i] == 1) ? 2.0 / 3.0 : 1.0 / 3.0;
    cost[i] = w * (double)n[i] * n[i] * n[i];
  }
  std::vector<int> order(count);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  // min-heap of (load, part)
  using Slot = std::pair<double, int>;
  std::priority_queue<Slot, std::vector<Slot>, std::greater<Slot>> heap;
  for (int p = 0; p < parts; ++p) heap.push({0.0, p});
  std::vector<double> part_load(parts, 0.0);
  for (int i : order) {
    Slot s = heap.top();
    heap.pop();
    owner[i] = s.second;
    s.first += cost[i];
    part_load[s.second] = s.first;
    heap.push(s);
  }
  if (load)
    for (int p = 0; p < parts; ++p) load[p] = part_load[p];
  return EGPU_OK;
}
