// Parity harness in the style of nigiri's test/raptor_search.cc: the same
// queries run through the C++ mirror of nigiri's routing interface
// (b2r.hpp -> the B200 engine) and through the CPU oracle (test
// infrastructure), and the complete journeys (every leg) must be equal.
// Range queries also run through pong_search (walking allowed at the
// start, as at the destination), and the first queries again in the
// wheelchair profile.  The first one-to-one and range queries of each
// direction also run through search<Dir, Algo> (nigiri's driver restated
// in b2r.hpp) with the engine's Algo, b2r_algo.  One-to-all searches compare the round
// times of every location.
//
//   raptor_search_test            exit 0 when every query matches
#include <cstdio>
#include <cstring>
#include <vector>

#include "b2r.hpp"
#include "oracle.h"

namespace r = b2r::routing;

namespace {

r::query from_c(b2r_query const& c) { return r::query_of(c); }

void print(char const* who, std::vector<r::journey> const& js) {
  std::printf("  %s: %zu journeys\n", who, js.size());
  for (auto const& j : js) {
    std::printf("    [%d -> %d] transfers=%u dest=%u\n", j.start_time_, j.dest_time_, j.transfers_, j.dest_);
    for (auto const& l : j.legs_) {
      std::printf("      %u -> %u  %d .. %d  ", l.from_, l.to_, l.dep_time_, l.arr_time_);
      if (auto const* t = std::get_if<r::run_enter_exit>(&l.uses_)) {
        std::printf("transport %u day %u stops [%u, %u)\n", t->transport_, t->day_, t->stop_from_, t->stop_to_);
      } else if (auto const* f = std::get_if<r::footpath>(&l.uses_)) {
        std::printf("footpath %u min\n", f->duration_);
      } else {
        auto const& o = std::get<r::offset>(l.uses_);
        std::printf("offset %u min mode %d\n", o.duration_, o.transport_mode_id_);
      }
    }
  }
}

std::vector<r::journey> oracle_journeys(b2r_timetable_desc const& d, b2r_query const& q) {
  or_result* res = nullptr;
  b2r::check(or_search(&d, &q, &res), "or_search");
  b2r_result view{};
  or_result_view(res, &view, nullptr);
  auto out = r::journeys_of(view);
  or_result_free(res);
  return out;
}

int run_workload(uint32_t workload, uint32_t timetable_seed, uint32_t n, uint64_t query_seed,
                 uint32_t algo_queries) {
  b2r_host_timetable* h = nullptr;
  b2r::check(b2r_tt_generate(workload, timetable_seed, &h), "b2r_tt_generate");
  b2r_timetable_desc d{};
  b2r_tt_desc(h, &d);
  b2r_query_set* qs = nullptr;
  b2r::check(b2r_queries_generate(h, workload, query_seed, n, &qs), "b2r_queries_generate");
  auto const n_q = b2r_queries_count(qs);

  b2r::timetable tt{d};
  b2r::engine eng{tt};
  int bad = 0;
  size_t n_journeys = 0, n_algo = 0;
  for (auto dir : {r::direction::kForward, r::direction::kBackward}) {
    std::vector<r::query> batch;
    std::vector<b2r_query const*> cq;
    for (auto i = 0U; i != n_q; ++i) {
      auto const* c = b2r_queries_get(qs, i);
      if (c->kind != B2R_ONE_TO_ONE || c->direction != static_cast<uint8_t>(dir)) continue;
      batch.push_back(from_c(*c));
      cq.push_back(c);
    }
    if (batch.empty()) continue;
    auto const got = r::raptor_search(eng, batch, dir);
    for (auto i = 0U; i != batch.size(); ++i) {
      auto const want = oracle_journeys(d, *cq[i]);
      n_journeys += want.size();
      if (got[i].status_ != B2R_OK || got[i].journeys_ != want) {
        ++bad;
        std::printf("workload %u query %u (%s) differs\n", workload, i,
                    dir == r::direction::kForward ? "forward" : "backward");
        print("engine", got[i].journeys_);
        print("oracle", want);
      }
      // the same query through search<Dir, Algo> with the engine's Algo
      // (nigiri's own driver loop over reset_arrivals .. reconstruct)
      if (i < algo_queries) {
        r::b2r_algo_state state;
        auto const via_algo =
            dir == r::direction::kForward
                ? r::search<r::direction::kForward, r::b2r_algo<r::direction::kForward>>{tt, state, batch[i]}.execute()
                : r::search<r::direction::kBackward, r::b2r_algo<r::direction::kBackward>>{tt, state, batch[i]}
                      .execute();
        ++n_algo;
        if (via_algo.status_ != B2R_OK || via_algo.journeys_ != want) {
          ++bad;
          std::printf("workload %u query %u (%s) differs through search<Dir, b2r_algo>\n", workload, i,
                      dir == r::direction::kForward ? "forward" : "backward");
          print("search<Dir, b2r_algo>", via_algo.journeys_);
          print("oracle", want);
        }
      }
    }
    // pong_search on the range queries
    std::vector<r::query> ranges;
    std::vector<b2r_query> cr;
    for (auto i = 0U; i != batch.size(); ++i) {
      if (cq[i]->is_interval == 0) continue;
      auto c = *cq[i];
      c.use_start_footpaths = 1;
      c.algorithm = B2R_ALGO_PONG;
      cr.push_back(c);
      ranges.push_back(from_c(c));
    }
    if (ranges.empty()) continue;
    auto const pongs = r::pong_search(eng, ranges, dir);
    for (auto i = 0U; i != ranges.size(); ++i) {
      auto const want = oracle_journeys(d, cr[i]);
      n_journeys += want.size();
      if (pongs[i].status_ != B2R_OK || pongs[i].journeys_ != want) {
        ++bad;
        std::printf("workload %u pong query %u (%s) differs\n", workload, i,
                    dir == r::direction::kForward ? "forward" : "backward");
        print("engine", pongs[i].journeys_);
        print("oracle", want);
      }
    }
  }
  // the wheelchair profile on the first one-to-one queries, both directions
  for (auto dir : {r::direction::kForward, r::direction::kBackward}) {
    std::vector<r::query> batch;
    std::vector<b2r_query> cw;
    for (auto i = 0U; i != n_q && cw.size() != 20U; ++i) {
      auto c = *b2r_queries_get(qs, i);
      if (c.kind != B2R_ONE_TO_ONE || c.direction != static_cast<uint8_t>(dir)) continue;
      c.prf_idx = B2R_PROFILE_WHEELCHAIR;
      cw.push_back(c);
      batch.push_back(from_c(c));
    }
    if (batch.empty()) continue;
    auto const got = r::raptor_search(eng, batch, dir);
    for (auto i = 0U; i != batch.size(); ++i) {
      auto const want = oracle_journeys(d, cw[i]);
      n_journeys += want.size();
      if (got[i].status_ != B2R_OK || got[i].journeys_ != want) {
        ++bad;
        std::printf("workload %u wheelchair query %u differs\n", workload, i);
        print("engine", got[i].journeys_);
        print("oracle", want);
      }
    }
  }
  // one-to-all on the first queries of the set, both directions
  for (auto i = 0U; i != 4U && i < n_q; ++i) {
    auto c = *b2r_queries_get(qs, i);
    c.kind = B2R_ONE_TO_ALL;
    c.n_destination = 0;
    c.is_interval = 0;
    c.direction = static_cast<uint8_t>(i % 2U);
    auto const state = r::one_to_all(eng, from_c(c), static_cast<r::direction>(c.direction));
    or_result* res = nullptr;
    b2r::check(or_search(&d, &c, &res), "or_search");
    int16_t const* rows = nullptr;
    int16_t const* best = nullptr;
    int32_t base_day = 0;
    or_result_state(res, &rows, &best, &base_day);
    auto const same = base_day == state.base_day_ &&
                      std::memcmp(rows, state.round_times_.data(), state.round_times_.size() * 2) == 0;
    or_result_free(res);
    if (!same) {
      ++bad;
      std::printf("workload %u one_to_all %u differs\n", workload, i);
    }
  }
  std::printf("workload %u: %u queries (%zu also through search<Dir, b2r_algo>), %zu journeys, %d differ\n",
              workload, n_q, n_algo, n_journeys, bad);
  b2r_queries_destroy(qs);
  b2r_tt_destroy(h);
  return bad;
}

}  // namespace

int main() {
  try {
    auto bad = run_workload(1, 1, 200, 4711, 60);  // city, forward one-to-one
    bad += run_workload(3, 2, 48, 4712, 12);        // regional, range, both directions
    std::printf(bad == 0 ? "ok\n" : "FAILED\n");
    return bad == 0 ? 0 : 1;
  } catch (b2r::error const& e) {
    std::printf("error %d: %s\n", e.status, e.what());
    return 2;
  }
}
