// Seeded synthetic timetables and query streams standing in for the real
// GTFS feeds nigiri's own benchmark reads (exe/benchmark.cc:80-97).
//
// Workloads (timetable seed = config index, query seed = 1000 + config):
//  1: 1,000 stops in a 20x20 km square, 120 routes of 10-40 stops,
//     30-150 transports per route, 7-day range, 80% weekday-only routes.
//     Queries: one-to-one forward ontrip, 06:00-22:00, max 7 transfers.
//  2: 40,000 stops, 4,000 routes, ~400k transports, 365-day range with 5%
//     holiday days on which weekday-only routes do not run.  Queries:
//     intermodal offset sets of 1-10 stops with 0-15 min walks, ontrip.
//  3: the workload-2 timetable; range queries with 30-240 min windows,
//     50% forward / 50% backward, station to station.
//  4: 300,000 stops, 25,000 routes, ~2.5M transports, <= 20 footpaths per
//     stop, 5% of transports in longer stay-seated chain routes.  Query
//     mix: 70% one-to-one, 20% 1 h range, 10% one-to-all.
//  5: the workload-4 timetable, same mix with 2 h ranges (served stream).
// Stops lie uniformly in a square whose side grows with sqrt(n) (constant
// density); routes are nearest-neighbour random walks over distinct stops;
// hop (1-4 min) and dwell (0-1 min) times are fixed per segment so
// transports of a route never overtake; departures run 05:00-24:00 UTC at
// the first stop with a per-route headway of 5-20 min, so late trips cross
// midnight.  Footpaths link stops within 400 m at 1.2 m/s (ceil, >= 2 min);
// every stop has a 2 min transfer time.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <unordered_map>

#include "host_tt.h"

namespace b2r {

namespace {

struct rng {
  std::mt19937_64 g;
  explicit rng(uint64_t s) : g(s) {}
  uint64_t next() { return g(); }
  // uniform integer in [lo, hi]
  int64_t uni(int64_t lo, int64_t hi) {
    auto const span = static_cast<uint64_t>(hi - lo + 1);
    return lo + static_cast<int64_t>(next() % span);
  }
  double unit() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
};

struct workload {
  uint32_t n_stops, n_routes;
  uint32_t min_stops, max_stops;
  uint32_t min_t, max_t;  // transports per route clamp
  uint32_t n_days;
  double holiday_frac;
  uint32_t max_fp;
  double chain_frac;
};

workload get_workload(uint32_t config) {
  switch (config) {
    case 1: return {1000, 120, 10, 40, 30, 150, 7, 0.0, 20, 0.0};
    case 2:
    case 3: return {40000, 4000, 10, 40, 1, 100000, 365, 0.05, 20, 0.0};
    case 4:
    case 5: return {300000, 25000, 10, 40, 1, 100000, 365, 0.05, 20, 0.05};
    default: return {1000, 120, 10, 40, 30, 150, 7, 0.0, 20, 0.0};
  }
}

constexpr int32_t kEpochMonday20240101 = 19723;  // 2024-01-01, a Monday

uint32_t morton(uint32_t x, uint32_t y) {
  auto const spread = [](uint32_t v) {
    v &= 0xFFFF;
    v = (v | (v << 8)) & 0x00FF00FF;
    v = (v | (v << 4)) & 0x0F0F0F0F;
    v = (v | (v << 2)) & 0x33333333;
    v = (v | (v << 1)) & 0x55555555;
    return v;
  };
  return spread(x) | (spread(y) << 1);
}

struct grid {
  double cell;
  uint32_t n;
  std::vector<std::vector<uint32_t>> cells;
  std::vector<float> const& x;
  std::vector<float> const& y;
  grid(std::vector<float> const& xs, std::vector<float> const& ys, double side,
       double cell_size)
      : cell{cell_size},
        n{std::max(1U, static_cast<uint32_t>(std::ceil(side / cell_size)))},
        cells(static_cast<size_t>(n) * n),
        x{xs},
        y{ys} {}
  uint32_t cx(float v) const {
    return std::min(n - 1, static_cast<uint32_t>(std::max(0.0, v / cell)));
  }
  void insert(uint32_t i) { cells[cx(y[i]) * n + cx(x[i])].push_back(i); }
  template <typename Fn>
  void for_each_within(uint32_t i, double radius, Fn&& fn) const {
    auto const r = static_cast<int>(std::ceil(radius / cell));
    auto const gx = static_cast<int>(cx(x[i])), gy = static_cast<int>(cx(y[i]));
    for (auto yy = std::max(0, gy - r); yy <= std::min<int>(n - 1, gy + r); ++yy) {
      for (auto xx = std::max(0, gx - r); xx <= std::min<int>(n - 1, gx + r); ++xx) {
        for (auto j : cells[yy * n + xx]) {
          auto const dx = x[j] - x[i], dy = y[j] - y[i];
          auto const d = std::sqrt(static_cast<double>(dx) * dx + static_cast<double>(dy) * dy);
          if (d <= radius) fn(j, d);
        }
      }
    }
  }
};

}  // namespace

host_timetable generate(uint32_t config, uint64_t seed) {
  auto const w = get_workload(config);
  rng rnd{seed * 0x9E3779B97F4A7C15ull + config};
  host_timetable t;

  // ---- stops (special stations 0..8 first, special_stations.h:7-19)
  auto const side = std::sqrt(w.n_stops / 1000.0) * 20000.0;  // metres
  std::vector<float> px(w.n_stops), py(w.n_stops);
  for (auto i = 0U; i != w.n_stops; ++i) {
    px[i] = static_cast<float>(rnd.unit() * side);
    py[i] = static_cast<float>(rnd.unit() * side);
  }
  // order stops along a Morton curve so that nearby stops get nearby
  // indices (locality of the [location] arrays on the device)
  std::vector<uint32_t> order(w.n_stops);
  std::iota(order.begin(), order.end(), 0U);
  {
    auto const cell = side / 4096.0;
    std::vector<uint32_t> code(w.n_stops);
    for (auto i = 0U; i != w.n_stops; ++i) {
      code[i] = morton(static_cast<uint32_t>(px[i] / cell),
                       static_cast<uint32_t>(py[i] / cell));
    }
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return code[a] < code[b]; });
  }
  t.n_locations = w.n_stops + B2R_N_SPECIAL_STATIONS;
  t.x.assign(t.n_locations, 0.0F);
  t.y.assign(t.n_locations, 0.0F);
  for (auto i = 0U; i != w.n_stops; ++i) {
    t.x[B2R_N_SPECIAL_STATIONS + i] = px[order[i]];
    t.y[B2R_N_SPECIAL_STATIONS + i] = py[order[i]];
  }
  t.transfer_time.assign(t.n_locations, 2U);
  for (auto i = 0U; i != B2R_N_SPECIAL_STATIONS; ++i) t.transfer_time[i] = 0U;
  t.date_range_from = kEpochMonday20240101;
  t.date_range_to = kEpochMonday20240101 + static_cast<int32_t>(w.n_days);

  // spatial index over real stops
  auto const spacing = side / std::sqrt(static_cast<double>(w.n_stops));
  grid g{t.x, t.y, side, std::max(400.0, spacing)};
  for (auto i = B2R_N_SPECIAL_STATIONS; i != t.n_locations; ++i) g.insert(i);

  // ---- footpaths: stops within 400 m, ceil(d / 72 m/min), >= 2 min,
  //      the `max_fp` nearest kept, sorted by duration
  t.fp_out_index.assign(1, 0U);
  for (auto i = 0U; i != t.n_locations; ++i) {
    std::vector<std::pair<double, uint32_t>> nb;
    if (i >= B2R_N_SPECIAL_STATIONS) {
      g.for_each_within(i, 400.0, [&](uint32_t j, double d) {
        if (j != i) nb.emplace_back(d, j);
      });
      std::sort(nb.begin(), nb.end());
      if (nb.size() > w.max_fp) nb.resize(w.max_fp);
    }
    std::vector<uint32_t> fps;
    for (auto const& [d, j] : nb) {
      auto const dur = std::max(2U, static_cast<uint32_t>(std::ceil(d / 72.0)));
      fps.push_back((j & 0x7FFFFFu) | (dur << 23));
    }
    std::stable_sort(fps.begin(), fps.end(), [](uint32_t a, uint32_t b) {
      return B2R_FP_DURATION(a) < B2R_FP_DURATION(b);
    });
    t.fp_out.insert(t.fp_out.end(), fps.begin(), fps.end());
    t.fp_out_index.push_back(static_cast<uint32_t>(t.fp_out.size()));
  }

  // ---- wheelchair profile: about one location in five is not accessible
  //      (from the location index; no draws from the random stream, so the
  //      rest of the timetable does not change); its footpaths are the walks
  //      into accessible locations, half as long again
  auto const accessible = [](uint32_t l) { return ((l * 2654435761u) >> 28) % 5u != 0u; };
  {
    auto& wp = t.profiles[B2R_PROFILE_WHEELCHAIR - 1U];
    wp.fp_out_index.assign(1, 0U);
    for (auto i = 0U; i != t.n_locations; ++i) {
      std::vector<uint32_t> fps;
      for (auto x = t.fp_out_index[i]; x != t.fp_out_index[i + 1]; ++x) {
        auto const tgt = B2R_FP_TARGET(t.fp_out[x]);
        if (!accessible(tgt)) continue;
        auto const dur = std::min(511U, (B2R_FP_DURATION(t.fp_out[x]) * 3U + 1U) / 2U);
        fps.push_back((tgt & 0x7FFFFFu) | (dur << 23));
      }
      std::stable_sort(fps.begin(), fps.end(), [](uint32_t a, uint32_t b) {
        return B2R_FP_DURATION(a) < B2R_FP_DURATION(b);
      });
      wp.fp_out.insert(wp.fp_out.end(), fps.begin(), fps.end());
      wp.fp_out_index.push_back(static_cast<uint32_t>(wp.fp_out.size()));
    }
  }

  // ---- service day bitfields (bit 0 = date_range_from - 5 days)
  std::vector<uint8_t> holiday(w.n_days, 0U);
  if (w.holiday_frac > 0.0) {
    auto const n_hol = static_cast<uint32_t>(std::lround(w.n_days * w.holiday_frac));
    for (auto h = 0U; h < n_hol;) {
      auto const d = static_cast<uint32_t>(rnd.uni(0, w.n_days - 1));
      if (!holiday[d]) {
        holiday[d] = 1U;
        ++h;
      }
    }
  }
  auto const make_bf = [&](bool weekday_only) {
    std::vector<uint64_t> bf(8, 0ULL);
    for (auto d = 0U; d != w.n_days; ++d) {
      auto const dow = (d % 7U);  // 0 = Monday
      if (weekday_only && (dow >= 5U || holiday[d])) continue;
      auto const bit = d + B2R_TIMETABLE_OFFSET_DAYS;
      bf[bit / 64] |= 1ULL << (bit % 64);
    }
    return bf;
  };
  t.bitfields.assign(8, 0ULL);  // bitfield 0 = empty (init_finish.cc:33)
  auto const bf_weekday = t.n_bitfields();
  {
    auto b = make_bf(true);
    t.bitfields.insert(t.bitfields.end(), b.begin(), b.end());
  }
  auto const bf_daily = t.n_bitfields();
  {
    auto b = make_bf(false);
    t.bitfields.insert(t.bitfields.end(), b.begin(), b.end());
  }

  // ---- base routes: stop sequences (random walks)
  auto const n_chain_routes =
      static_cast<uint32_t>(std::lround(w.n_routes * w.chain_frac));
  std::vector<std::vector<uint32_t>> base_seq;
  std::vector<uint8_t> visited(t.n_locations, 0U);
  while (base_seq.size() < w.n_routes) {
    auto const is_chain = base_seq.size() >= w.n_routes - n_chain_routes;
    // stay-seated chains: two to three trips joined into one longer run
    auto const n_stops = static_cast<uint32_t>(
        is_chain ? rnd.uni(2 * w.min_stops, 3 * w.max_stops / 2)
                 : rnd.uni(w.min_stops, w.max_stops));
    std::vector<uint32_t> seq;
    auto cur = static_cast<uint32_t>(
        rnd.uni(B2R_N_SPECIAL_STATIONS, t.n_locations - 1));
    seq.push_back(cur);
    visited[cur] = 1U;
    auto radius = std::max(400.0, 1.5 * spacing);
    auto heading = rnd.unit() * 6.283185307179586;
    while (seq.size() < n_stops) {
      std::vector<std::pair<double, uint32_t>> nb;
      g.for_each_within(cur, radius, [&](uint32_t j, double d) {
        if (!visited[j]) nb.emplace_back(d, j);
      });
      if (nb.size() < 2U) {
        if (radius > side) break;
        radius *= 2.0;
        continue;
      }
      // among the 4 nearest unvisited stops take the one best aligned
      // with the route's (slowly drifting) heading: line-like routes
      std::sort(nb.begin(), nb.end());
      auto const k = std::min<size_t>(4U, nb.size());
      heading += (rnd.unit() - 0.5) * 0.6;
      auto best_j = nb[0].second;
      auto best_score = -2.0;
      for (auto c = 0U; c != k; ++c) {
        auto const j = nb[c].second;
        auto const dx = t.x[j] - t.x[cur], dy = t.y[j] - t.y[cur];
        auto const len = std::sqrt(static_cast<double>(dx) * dx + static_cast<double>(dy) * dy) + 1e-9;
        auto const score = (dx * std::cos(heading) + dy * std::sin(heading)) / len;
        if (score > best_score) {
          best_score = score;
          best_j = j;
        }
      }
      cur = best_j;
      seq.push_back(cur);
      visited[cur] = 1U;
      radius = std::max(400.0, 1.5 * spacing);
    }
    for (auto x : seq) visited[x] = 0U;
    if (seq.size() >= 2U) base_seq.push_back(std::move(seq));
  }

  // ---- transports.  Every trip of a base route shares hop/dwell times and
  // the traffic-day pattern; trips are grouped into routes by nigiri's rule
  // that minutes after midnight are ordered at every stop
  // (loader/get_index.h:8-29), so trips crossing midnight at different stops
  // land in separate sub-routes (gtfs/load_timetable.cc:288-309).
  struct trip {
    std::vector<int> times;  // dep(0), arr(1), dep(1), ..., arr(n-1)
  };
  auto const get_index = [](std::vector<trip const*> const& route,
                            trip const& s) -> int64_t {
    auto const key = s.times[0] % 1440;
    size_t index = 0;
    while (index < route.size() && route[index]->times[0] % 1440 < key) ++index;
    for (auto i = 0U; i != s.times.size(); ++i) {
      auto const x = s.times[i] % 1440;
      if ((index > 0 && x < route[index - 1]->times[i] % 1440) ||
          (index < route.size() && x > route[index]->times[i] % 1440)) {
        return -1;
      }
    }
    return static_cast<int64_t>(index);
  };
  auto const enc = [](int minutes) {
    auto const days = static_cast<uint16_t>(minutes / 1440);
    auto const mam = static_cast<uint16_t>(minutes % 1440);
    return static_cast<uint16_t>((days & 0x1Fu) | (mam << 5));
  };
  // route classes and flags come from a stream of their own, so that the
  // network and its trips are the same with or without them.  Classes: bus
  // mostly, then tram, subway, suburban, regional.  Flags per section
  // (bikes, cars, wheelchair, no reservation): a route carries a flag on
  // all, some or none of its sections.
  rng frnd{seed * 0xD1B54A32D192ED03ull + config + 1U};
  struct flag_mix {
    double all, some;
  };
  static constexpr flag_mix kFlagMix[4] = {
      {0.55, 0.20}, {0.05, 0.05}, {0.50, 0.20}, {0.80, 0.10}};
  t.route_stop_index.assign(1, 0U);
  for (auto const& seq : base_seq) {
    auto const n = static_cast<uint32_t>(seq.size());
    uint8_t clasz = 10U;
    {
      auto const u = frnd.unit();
      clasz = u < 0.60 ? 10U : u < 0.75 ? 9U : u < 0.85 ? 8U : u < 0.95 ? 7U : 6U;
    }
    std::vector<uint8_t> sections(n, 0U);  // section s: stop s -> s + 1
    for (auto f = 0U; f != 4U; ++f) {
      auto const u = frnd.unit();
      auto const some = u >= kFlagMix[f].all && u < kFlagMix[f].all + kFlagMix[f].some;
      for (auto s = 0U; s + 1U < n; ++s) {
        auto const on = u < kFlagMix[f].all || (some && frnd.unit() < 0.6);
        if (on) sections[s] = static_cast<uint8_t>(sections[s] | (1U << f));
      }
    }
    std::vector<int> hop(n, 0), dwell(n, 0);
    for (auto s = 1U; s < n; ++s) hop[s] = static_cast<int>(rnd.uni(1, 4));
    for (auto s = 1U; s + 1U < n; ++s) dwell[s] = static_cast<int>(rnd.uni(0, 1));
    auto const headway = static_cast<int>(rnd.uni(5, 20));
    // first departures 05:00 .. 23:59
    auto n_t = static_cast<uint32_t>((24 * 60 - 1 - 5 * 60) / headway + 1);
    n_t = std::clamp(n_t, w.min_t, w.max_t);
    auto const weekday_only = rnd.unit() < 0.8;
    auto const bf = weekday_only ? bf_weekday : bf_daily;
    std::vector<trip> trips(n_t);
    for (auto j = 0U; j != n_t; ++j) {
      auto& tm = trips[j].times;
      tm.reserve(2 * (n - 1));
      auto cur = 5 * 60 + static_cast<int>(j) * headway;
      for (auto s = 0U; s + 1U < n; ++s) {
        if (s != 0U) cur += dwell[s];
        tm.push_back(cur);   // dep(s)
        cur += hop[s + 1];
        tm.push_back(cur);   // arr(s + 1)
      }
    }
    std::vector<std::vector<trip const*>> subs;
    for (auto const& tr : trips) {
      auto placed = false;
      for (auto& sub : subs) {
        auto const idx = get_index(sub, tr);
        if (idx >= 0) {
          sub.insert(sub.begin() + idx, &tr);
          placed = true;
          break;
        }
      }
      if (!placed) subs.push_back({&tr});
    }
    for (auto const& sub : subs) {
      for (auto x : seq) {
        t.route_stops.push_back((x & 0x0FFFFFFFu) | (1u << 28) | (1u << 29) |
                                (accessible(x) ? (1u << 30) | (1u << 31) : 0u));
      }
      t.route_stop_index.push_back(static_cast<uint32_t>(t.route_stops.size()));
      t.route_transport_from.push_back(static_cast<uint32_t>(t.transport_traffic_days.size()));
      for (auto j = 0U; j != sub.size(); ++j) t.transport_traffic_days.push_back(bf);
      t.route_transport_to.push_back(static_cast<uint32_t>(t.transport_traffic_days.size()));
      t.route_stop_time_from.push_back(static_cast<uint32_t>(t.route_stop_times.size()));
      t.route_clasz.push_back(clasz);
      t.route_section_flags.insert(t.route_section_flags.end(), sections.begin(),
                                   sections.end());
      for (auto slot = 0U; slot != 2 * (n - 1); ++slot) {
        for (auto const* tr : sub) t.route_stop_times.push_back(enc(tr->times[slot]));
      }
    }
  }
  t.n_routes = static_cast<uint32_t>(t.route_transport_from.size());
  t.n_transports = static_cast<uint32_t>(t.transport_traffic_days.size());

  finalize(t);
  return t;
}

}  // namespace b2r
