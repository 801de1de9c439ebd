// Seeded synthetic query streams for workloads 1..5 (definitions in
// generator.cc).  A query set owns the offset arrays its b2r_query structs
// point to.
#include <algorithm>
#include <cmath>
#include <memory>
#include <random>
#include <vector>

#include "host_tt.h"
#include "queries.h"

namespace b2r {

namespace {

struct rng {
  std::mt19937_64 g;
  explicit rng(uint64_t s) : g(s) {}
  int64_t uni(int64_t lo, int64_t hi) {
    auto const span = static_cast<uint64_t>(hi - lo + 1);
    return lo + static_cast<int64_t>(g() % span);
  }
  double unit() { return (g() >> 11) * (1.0 / 9007199254740992.0); }
};

}  // namespace

query_set make_queries(host_timetable const& t, uint32_t config, uint64_t seed,
                       uint32_t n) {
  rng rnd{seed * 0x2545F4914F6CDD1Dull + 7U * config};
  query_set qs;
  qs.queries.resize(n);
  qs.offsets.resize(n);

  // stops served by at least one route
  std::vector<uint32_t> served;
  for (auto l = B2R_N_SPECIAL_STATIONS; l < t.n_locations; ++l) {
    if (t.location_routes_index[l + 1] != t.location_routes_index[l]) {
      served.push_back(l);
    }
  }
  auto const n_days = static_cast<int64_t>(t.date_range_to - t.date_range_from);
  auto const pick = [&]() {
    return served[static_cast<size_t>(rnd.uni(0, static_cast<int64_t>(served.size()) - 1))];
  };
  auto const pick_time = [&]() {
    auto const day = t.date_range_from + static_cast<int32_t>(rnd.uni(0, n_days - 1));
    auto const mam = static_cast<int32_t>(rnd.uni(6 * 60, 22 * 60));
    return day * 1440 + mam;
  };
  // the k served stops nearest to `c` (c included), brute force over a
  // window of neighbouring indices (indices follow a Morton curve)
  auto const nearest = [&](uint32_t c, uint32_t k) {
    std::vector<std::pair<float, uint32_t>> cand;
    auto const it = std::lower_bound(served.begin(), served.end(), c);
    auto const pos = static_cast<int64_t>(it - served.begin());
    for (auto i = std::max<int64_t>(0, pos - 200);
         i < std::min<int64_t>(static_cast<int64_t>(served.size()), pos + 200); ++i) {
      auto const l = served[static_cast<size_t>(i)];
      auto const dx = t.x[l] - t.x[c], dy = t.y[l] - t.y[c];
      cand.emplace_back(dx * dx + dy * dy, l);
    }
    std::sort(cand.begin(), cand.end());
    std::vector<uint32_t> out;
    for (auto i = 0U; i < std::min<size_t>(k, cand.size()); ++i) out.push_back(cand[i].second);
    return out;
  };

  // a served stop at a distance drawn uniformly from [1, 12] km (urban and
  // regional trip lengths) from `s`
  auto const pick_near = [&](uint32_t s) {
    auto const target = 1000.0 + rnd.unit() * 11000.0;
    for (auto attempt = 0; attempt != 64; ++attempt) {
      auto const a = rnd.unit() * 6.283185307179586;
      auto const px = t.x[s] + target * std::cos(a), py = t.y[s] + target * std::sin(a);
      // nearest served stop to (px, py) among a random sample
      auto best = s;
      auto best_d = 1e300;
      for (auto c = 0; c != 256; ++c) {
        auto const l = pick();
        auto const dx = t.x[l] - px, dy = t.y[l] - py;
        auto const dd = static_cast<double>(dx) * dx + static_cast<double>(dy) * dy;
        if (dd < best_d) {
          best_d = dd;
          best = l;
        }
      }
      if (best != s && best_d < 4.0e6) return best;
    }
    auto d = pick();
    while (d == s) d = pick();
    return d;
  };

  for (auto i = 0U; i != n; ++i) {
    auto& q = qs.queries[i];
    b2r_query_init(&q);
    auto& off = qs.offsets[i];
    auto const single = [&](uint32_t& s, uint32_t& d) {
      s = pick();
      if (config == 1) {
        do {
          d = pick();
        } while (d == s);
      } else {
        d = pick_near(s);
      }
    };
    switch (config) {
      case 1: {
        uint32_t s, d;
        single(s, d);
        off.start = {{s, 0, 0, 0}};
        off.dest = {{d, 0, 0, 0}};
        q.max_transfers = 7;
        q.start_time = pick_time();
        break;
      }
      case 2: {
        auto const sc = pick();
        auto const dc = pick_near(sc);
        for (auto l : nearest(sc, static_cast<uint32_t>(rnd.uni(1, 10)))) {
          off.start.push_back({l, static_cast<int16_t>(rnd.uni(0, 15)), 0, 0});
        }
        for (auto l : nearest(dc, static_cast<uint32_t>(rnd.uni(1, 10)))) {
          off.dest.push_back({l, static_cast<int16_t>(rnd.uni(0, 15)), 0, 0});
        }
        q.start_match_mode = B2R_MATCH_INTERMODAL;
        q.dest_match_mode = B2R_MATCH_INTERMODAL;
        q.start_time = pick_time();
        break;
      }
      case 3: {
        uint32_t s, d;
        single(s, d);
        off.start = {{s, 0, 0, 0}};
        off.dest = {{d, 0, 0, 0}};
        q.direction = (rnd.unit() < 0.5) ? B2R_FORWARD : B2R_BACKWARD;
        q.is_interval = 1;
        q.interval_from = pick_time();
        q.interval_to = q.interval_from + static_cast<int32_t>(rnd.uni(30, 240));
        break;
      }
      default: {  // 4, 5: 70% one-to-one, 20% range, 10% one-to-all
        auto const u = rnd.unit();
        uint32_t s, d;
        single(s, d);
        off.start = {{s, 0, 0, 0}};
        if (u < 0.7) {
          off.dest = {{d, 0, 0, 0}};
          q.start_time = pick_time();
        } else if (u < 0.9) {
          off.dest = {{d, 0, 0, 0}};
          q.direction = (rnd.unit() < 0.5) ? B2R_FORWARD : B2R_BACKWARD;
          q.is_interval = 1;
          q.interval_from = pick_time();
          q.interval_to = q.interval_from + (config == 4 ? 60 : 120);
        } else {
          q.kind = B2R_ONE_TO_ALL;
          q.start_time = pick_time();
        }
        break;
      }
    }
  }
  for (auto i = 0U; i != n; ++i) {
    auto& q = qs.queries[i];
    q.start = qs.offsets[i].start.data();
    q.n_start = static_cast<uint32_t>(qs.offsets[i].start.size());
    q.destination = qs.offsets[i].dest.data();
    q.n_destination = static_cast<uint32_t>(qs.offsets[i].dest.size());
  }
  return qs;
}

}  // namespace b2r
