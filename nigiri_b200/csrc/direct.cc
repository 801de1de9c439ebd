// Direct journeys of an exact-match one-to-one query (the part of
// src/routing/direct.cc that pong's earlier-alternative pass uses: no
// real-time transports, no time-dependent footpaths, profile 0).
#include "direct.h"

#include <algorithm>
#include <iterator>
#include <optional>
#include <queue>
#include <vector>

namespace b2r {
namespace {

constexpr int kMaxFootpath = 511;  // footpath::kMaxDuration (9 duration bits)

template <typename T>
T adjusted_tt(tts_norm const& s, T d) {  // adjusted_transfer_time, transfer_time_settings.h:20-47
  if (s.is_default) return d;
  return static_cast<T>(static_cast<T>(s.additional_time) +
                        std::max(static_cast<T>(s.min_transfer_time),
                                 static_cast<T>(static_cast<float>(d) * s.factor)));
}

struct tt_access {
  b2r_timetable_desc const& d;
  int32_t internal_from() const { return (d.date_range_from - B2R_TIMETABLE_OFFSET_DAYS) * 1440; }
  uint32_t n_t(uint32_t r) const { return d.route_transport_to[r] - d.route_transport_from[r]; }
  uint32_t stop(uint32_t r, uint32_t i) const { return d.route_stops[d.route_stop_index[r] + i]; }
  uint16_t ev(uint32_t r, uint32_t x, uint32_t s, bool arr) const {
    return d.route_stop_times[d.route_stop_time_from[r] + n_t(r) * (s * 2 - (arr ? 1 : 0)) + x];
  }
  bool bit(uint32_t bf, uint32_t i) const {
    return i < B2R_MAX_DAYS && ((d.bitfields[8ull * bf + i / 64] >> (i % 64)) & 1ULL) != 0ULL;
  }
  int32_t event_time(uint32_t r, uint32_t x, uint16_t day, uint32_t s, bool arr) const {
    auto const e = ev(r, x, s, arr);
    return internal_from() + (static_cast<int32_t>(day) + B2R_DELTA_DAYS(e)) * 1440 + B2R_DELTA_MAM(e);
  }
  uint8_t clasz(uint32_t r) const { return d.route_clasz != nullptr ? d.route_clasz[r] : 10U; }
  uint8_t flags(uint32_t r) const { return d.route_flags != nullptr ? d.route_flags[r] : 0U; }
  uint8_t section(uint32_t r, uint32_t s) const {
    return d.route_section_flags != nullptr ? d.route_section_flags[d.route_stop_index[r] + s] : 0U;
  }
};

// lookup_footpath (direct.cc:65-160) for one exact-match offset of
// duration 0 at `anchor`: the reflexive transfer time if loc is the anchor,
// or the shortest footpath between them.
std::optional<b2r_leg> access_walk(tt_access const& t, tts_norm const& tts, uint32_t prf, uint32_t anchor,
                                   uint32_t loc, int32_t time, bool boarding) {
  int best = kMaxFootpath;
  if (anchor == loc) best = adjusted_tt<uint8_t>(tts, t.d.transfer_time[anchor]);
  auto eff = kMaxFootpath;
  auto const [fb, fe] = footpaths_at(t.d, prf, boarding, anchor);
  for (auto const* f = fb; f != fe; ++f) {
    if (B2R_FP_TARGET(*f) != loc) continue;
    auto const a = adjusted_tt<int16_t>(tts, static_cast<int16_t>(B2R_FP_DURATION(*f)));
    if (a < eff) eff = a;
  }
  if (eff < kMaxFootpath && eff < best) best = eff;
  if (best >= kMaxFootpath) return std::nullopt;
  b2r_leg l{};
  l.rt_transport = B2R_INVALID_IDX;
  l.kind = B2R_LEG_FOOTPATH;
  l.from = boarding ? anchor : loc;
  l.to = boarding ? loc : anchor;
  l.dep_time = boarding ? time - best : time;
  l.arr_time = boarding ? time : time + best;
  l.transport = l.to;
  l.duration = static_cast<int16_t>(best);
  return l;
}

}  // namespace

bool earliest_alternative(host_view const& hv, tts_norm const& tts, uint32_t prf, uint32_t allowed_claszes,
                          uint8_t required_flags, uint32_t from, uint32_t to, int32_t from_arr,
                          int32_t to_dep, std::array<b2r_leg, 3>& out) {
  tt_access const t{hv.d};
  auto const& d = hv.d;
  // collect_locations (direct.cc:183-240): the anchors and their footpath
  // neighbours in the query's profile (out of `from`, into `to`)
  std::vector<uint32_t> boarding{from}, alighting{to};
  for (auto [f, e] = footpaths_at(d, prf, true, from); f != e; ++f) boarding.push_back(B2R_FP_TARGET(*f));
  for (auto [f, e] = footpaths_at(d, prf, false, to); f != e; ++f) alighting.push_back(B2R_FP_TARGET(*f));
  auto const contains = [](std::vector<uint32_t> const& v, uint32_t x) {
    return std::find(v.begin(), v.end(), x) != v.end();
  };
  auto const routes_at = [&](std::vector<uint32_t> const& locs) {
    std::vector<uint32_t> rs;
    for (auto const l : locs) {
      rs.insert(rs.end(), d.location_routes + d.location_routes_index[l],
                d.location_routes + d.location_routes_index[l + 1]);
    }
    std::sort(rs.begin(), rs.end());
    rs.erase(std::unique(rs.begin(), rs.end()), rs.end());
    return rs;
  };
  auto const a = routes_at(boarding), b = routes_at(alighting);
  std::vector<uint32_t> routes;
  std::set_intersection(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(routes));

  // per (route, boarding, alighting) pair the first journey route_gen
  // (direct.cc:281-376) yields
  auto const last_day = d.date_range_to + 1 - (d.date_range_from - B2R_TIMETABLE_OFFSET_DAYS);
  std::vector<std::array<b2r_leg, 3>> heads;
  for (auto const r : routes) {
    auto const fl = t.flags(r);
    auto allowed = ((allowed_claszes >> t.clasz(r)) & 1U) != 0U;  // direct.cc:503-513
    for (auto f = 0U; f != 4U; ++f) {
      if (((required_flags >> f) & 1U) != 0U && ((fl >> (2U * f)) & 3U) == 0U) allowed = false;
    }
    if (!allowed) continue;
    auto const flag_on_section = [&](uint32_t f, uint32_t s) {  // run_stop::is_flag_set(f, kDep)
      if ((fl >> (2U * f)) & 1U) return true;
      if (((fl >> (2U * f + 1U)) & 1U) == 0U) return false;
      return ((t.section(r, s) >> f) & 1U) != 0U;
    };
    auto const n = d.route_stop_index[r + 1] - d.route_stop_index[r];
    std::optional<uint32_t> board;  // for_each_pair, direct.cc:429-450
    for (auto i = 0U; i != n; ++i) {
      auto const stp = t.stop(r, i);
      auto const loc = B2R_STOP_LOC(stp);
      if (!board.has_value()) {
        if (contains(boarding, loc) && stop_in(stp, prf)) board = i;  // stop::in_allowed(prf_idx)
        continue;
      }
      if (!contains(alighting, loc) || !stop_out(stp, prf)) continue;
      auto const s_from = *board, s_to = i;
      board.reset();
      auto violates = false;  // sections_violate_constraints, direct.cc:242-260
      for (auto s = s_from; s != s_to && !violates; ++s) {
        for (auto f = 0U; f != 4U; ++f) {
          if (((required_flags >> f) & 1U) != 0U && !flag_on_section(f, s)) violates = true;
        }
      }
      if (violates) continue;
      auto const board_loc = B2R_STOP_LOC(t.stop(r, s_from)), alight_loc = B2R_STOP_LOC(t.stop(r, s_to));
      auto found = false;
      for (auto day = (from_arr - t.internal_from()) / 1440; !found && day <= last_day; ++day) {
        if (!t.bit(d.route_traffic_days[r], static_cast<uint32_t>(day))) continue;
        for (auto x = 0U; x != t.n_t(r); ++x) {
          auto const start_day = day - static_cast<int>(B2R_DELTA_DAYS(t.ev(r, x, s_from, false)));
          if (start_day < 0 || start_day >= B2R_MAX_DAYS) continue;
          auto const tr = d.route_transport_from[r] + x;
          if (!t.bit(d.transport_traffic_days[tr], static_cast<uint32_t>(start_day))) continue;
          auto const sd = static_cast<uint16_t>(start_day);
          auto const dep = t.event_time(r, x, sd, s_from, false), arr = t.event_time(r, x, sd, s_to, true);
          auto const bw = access_walk(t, tts, prf, from, board_loc, dep, true);
          auto const aw = access_walk(t, tts, prf, to, alight_loc, arr, false);
          if (!bw.has_value() || !aw.has_value() || bw->dep_time < from_arr) continue;
          b2r_leg ride{};
          ride.rt_transport = B2R_INVALID_IDX;
          ride.kind = B2R_LEG_TRANSPORT;
          ride.from = board_loc;
          ride.to = alight_loc;
          ride.dep_time = dep;
          ride.arr_time = arr;
          ride.transport = tr;
          ride.day = sd;
          ride.stop_from = static_cast<uint16_t>(s_from);
          ride.stop_to = static_cast<uint16_t>(s_to + 1U);
          heads.push_back({*bw, ride, *aw});
          found = true;
          break;
        }
      }
    }
  }
  if (heads.empty()) return false;
  // the generators merged by arrival (direct.cc:578-604): the reference's
  // binary heap picks the first among equal arrivals
  auto const later = [&](size_t x, size_t y) { return heads[x][2].arr_time > heads[y][2].arr_time; };
  std::priority_queue<size_t, std::vector<size_t>, decltype(later)> heap{later};
  for (auto i = size_t{0}; i != heads.size(); ++i) heap.push(i);
  auto legs = heads[heap.top()];
  if (legs[2].arr_time > to_dep) return false;
  auto const walk = legs[0].arr_time - legs[0].dep_time;  // the walk starts on arrival (pong.cc:53-58)
  legs[0].dep_time = from_arr;
  legs[0].arr_time = from_arr + walk;
  out = legs;
  return true;
}

}  // namespace b2r
