// get_earliest_transport of one stop of one route for one query, shared by
// the batched route scan and the single-query no-allocation search.
#pragma once

#include "engine.cuh"

namespace b2r::dev {

// get_earliest_transport, raptor.h:1351-1442.  Event columns are ordered by
// minutes after midnight (loader/get_index.h), so the reference's
// linear_lb is a lower bound found by binary search; the scan that follows
// visits events in the reference's order with the same prune / skip / day
// rules.  Routes flagged unsorted use the reference's linear seek.
__device__ inline bool et_search(dtt const& T, bool fwd, uint32_t r, uint32_t si, uint16_t day_at_stop,
                          int mam, int lbv, int tad_k, uint16_t base, uint32_t& out_off,
                          uint16_t& out_day, uint32_t& n_ev, uint32_t& n_days) {
  auto const t0 = __ldg(T.route_tr_from + r);
  auto const n = __ldg(T.route_tr_to + r) - t0;
  auto const* col = T.st + __ldg(T.route_st_from + r) + n * (si * 2u - (fwd ? 0u : 1u));
  auto const sorted = __ldg(T.route_sorted + r) != 0;
  auto const rbf = __ldg(T.route_bf + r);
  for (auto i = 0u; i != 6u; ++i) {
    auto const day = static_cast<uint16_t>(fwd ? day_at_stop + i : day_at_stop - i);
    ++n_days;
    if (!bf_test(T, rbf, day)) continue;
    uint32_t j = 0;
    if (i == 0u) {
      if (sorted) {
        uint32_t lo = 0, hi = n;
        if (fwd) {  // first index with mam >= m
          while (lo < hi) {
            auto const mid = (lo + hi) >> 1;
            ++n_ev;
            if (static_cast<int>(__ldg(col + mid) >> 5) < mam) lo = mid + 1;
            else hi = mid;
          }
          j = lo;
        } else {  // first (from the end) with mam <= m: n - upper_bound(m)
          while (lo < hi) {
            auto const mid = (lo + hi) >> 1;
            ++n_ev;
            if (static_cast<int>(__ldg(col + mid) >> 5) <= mam) lo = mid + 1;
            else hi = mid;
          }
          j = n - lo;
        }
      } else {
        for (j = 0; j < n; ++j) {
          auto const em = static_cast<int>(__ldg(col + (fwd ? j : n - 1 - j)) >> 5);
          if (!(fwd ? em < mam : em > mam)) break;
        }
      }
    }
    for (; j < n; ++j) {
      auto const idx = fwd ? j : n - 1u - j;
      auto const e = __ldg(col + idx);
      ++n_ev;
      auto const em = static_cast<int>(e >> 5);
      if (to_delta_key(fwd, day, base, em) + lbv > tad_k) return false;
      if (i == 0u && !(fwd ? mam <= em : mam >= em)) continue;
      auto const sday = static_cast<uint16_t>(static_cast<int>(day) - static_cast<int>(e & 31u));
      if (!bf_test(T, __ldg(T.transport_bf + t0 + idx), sday)) continue;
      out_off = idx;
      out_day = sday;
      return true;
    }
  }
  return false;
}

}  // namespace b2r::dev
