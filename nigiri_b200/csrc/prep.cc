// Host-side query preparation (see prep.h).  Reference semantics are cited
// per function; the code is the engine's own.
#include "prep.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <unordered_map>

namespace b2r {

// std::chrono::round<days> of a minute time point (ties to even)
int32_t round_to_days(int64_t m) {
  int64_t const d0 = m >= 0 ? m / 1440 : -((-m + 1439) / 1440);
  int64_t const r0 = m - d0 * 1440, r1 = 1440 - r0;
  if (r0 == r1) return static_cast<int32_t>((d0 & 1) ? d0 + 1 : d0);
  return static_cast<int32_t>(r0 < r1 ? d0 : d0 + 1);
}

namespace {

// interval_estimator::clamp (interval_estimate.h:138-146): into the
// timetable's external interval, the data type's window, then the query's
// max_interval_, one after another (std::clamp, both ends inclusive)
int32_t clamp_interval_end(prepped_query const& p, int32_t ext_from, int32_t ext_to, int32_t x) {
  x = std::clamp(x, ext_from, ext_to);
  x = std::clamp(x, p.data_max_from, p.data_max_to);
  if (p.has_max_interval) x = std::clamp(x, p.max_iv_from, p.max_iv_to);
  return x;
}

constexpr uint16_t kUnreach = 0xFFFFu;
constexpr int kMaxDur = 511;  // footpath::kMaxDuration

// the route flags a query requires (raptor.h:251-257, direct.cc:503-513):
// bikes, cars, no compulsory reservation, and wheelchair accessibility for
// the wheelchair profile
uint8_t required_flags(b2r_query const& q) {
  return static_cast<uint8_t>((q.require_bike_transport != 0 ? 1U << B2R_FLAG_BIKES : 0U) |
                              (q.require_car_transport != 0 ? 1U << B2R_FLAG_CARS : 0U) |
                              (q.prf_idx == B2R_PROFILE_WHEELCHAIR ? 1U << B2R_FLAG_WHEELCHAIR : 0U) |
                              (q.no_compulsory_reservation != 0 ? 1U << B2R_FLAG_RESERVATION_NOT_REQUIRED : 0U));
}

template <typename T>
T adjust(tts_norm const& s, T d) {  // transfer_time_settings.h:20-31
  if (s.is_default) return d;
  return static_cast<T>(static_cast<T>(s.additional_time) +
                        std::max(static_cast<T>(s.min_transfer_time),
                                 static_cast<T>(static_cast<float>(d) * s.factor)));
}

struct view {
  b2r_timetable_desc const& d;
  rt_host const* rt{nullptr};
  // timetable / rt_timetable::is_transport_active: the overlay's days for
  // a transport it changed
  bool transport_active(uint32_t t, uint32_t day) const;
  template <typename Fn>
  void kids(uint32_t l, Fn&& fn) const {
    if (d.children_index == nullptr) return;
    for (auto i = d.children_index[l]; i != d.children_index[l + 1]; ++i) fn(d.children[i]);
  }
  uint32_t root(uint32_t idx) const {  // timetable.h:62-76
    if (d.parent == nullptr) return idx;
    auto l = idx;
    for (auto i = 0, p = static_cast<int>(0); ; ++i) {
      auto const par = d.parent[l];
      if (par == B2R_INVALID_IDX) break;
      if (par == idx || i > 20) {
        l = d.parent[idx];
        break;
      }
      l = par;
      (void)p;
    }
    return l;
  }
  // for_each_meta, for_each_meta.h:8-45 (no equivalence lists in the image)
  template <typename Fn>
  void metas(uint8_t mode, uint32_t l, Fn&& fn) const {
    switch (mode) {
      case B2R_MATCH_EXACT: fn(l); break;
      case B2R_MATCH_INTERMODAL:
        fn(l);
        kids(l, [&](uint32_t c) {
          if (d.location_type != nullptr && d.location_type[c] == B2R_LOC_GENERATED_TRACK) fn(c);
        });
        break;
      case B2R_MATCH_ONLY_CHILDREN:
        fn(l);
        kids(l, [&](uint32_t c) {
          fn(c);
          kids(c, fn);
        });
        break;
      default: {
        auto const r = root(l);
        fn(r);
        kids(r, [&](uint32_t c) {
          fn(c);
          kids(c, fn);
        });
      }
    }
  }
  int32_t internal_from_min() const { return (d.date_range_from - 5) * 1440; }
};

// get_fastest_direct.cc:12-100 -- footpath-only walk from the start set to
// destination offsets.
int16_t fastest_direct(view const& v, b2r_query const& q, std::vector<b2r_offset> const& st,
                       std::vector<b2r_offset> const& de, tts_norm const& raw, bool fwd) {
  if (q.has_fastest_direct) return q.fastest_direct;
  std::vector<std::pair<uint32_t, uint16_t>> dist;  // insertion ordered
  std::unordered_map<uint32_t, size_t> at;
  auto const get = [&](uint32_t l) -> uint16_t& {
    auto it = at.find(l);
    if (it == at.end()) {
      it = at.emplace(l, dist.size()).first;
      dist.emplace_back(l, uint16_t{32767});
    }
    return dist[it->second].second;
  };
  for (auto const& s : st) {
    v.metas(q.start_match_mode, s.target, [&](uint32_t l) {
      auto& x = get(l);
      x = std::min(static_cast<uint16_t>(s.duration), x);
    });
  }
  // bucket queue over distances [0, 65535)
  std::map<uint32_t, std::vector<uint32_t>> buckets;
  for (auto const& [l, dd] : dist) buckets[dd].push_back(l);
  std::unordered_map<uint32_t, uint16_t> dest_off;
  for (auto const& o : de) {
    auto const dd = static_cast<uint16_t>(o.duration);
    auto it = dest_off.find(o.target);
    if (it == dest_off.end()) dest_off.emplace(o.target, dd);
    else if (it->second > dd) it->second = dd;
  }
  uint32_t end_dist = 32767;
  while (!buckets.empty()) {
    auto it = buckets.begin();
    auto const dcur = it->first;
    auto const l = it->second.back();
    it->second.pop_back();
    if (it->second.empty()) buckets.erase(it);
    if (l == B2R_SPECIAL_END) break;
    if (get(l) < dcur) continue;
    auto const [fb, fe] = footpaths_at(v.d, q.prf_idx, fwd, l);
    for (auto const* f = fb; f != fe; ++f) {
      auto const nd = dcur + adjust<uint16_t>(raw, static_cast<uint16_t>(B2R_FP_DURATION(*f)));
      if (nd > 65535u) continue;
      auto const tgt = B2R_FP_TARGET(*f);
      if (!dest_off.contains(tgt)) continue;
      auto& td = get(tgt);
      if (nd < td && nd < 65535u) {
        td = static_cast<uint16_t>(nd);
        buckets[nd].push_back(tgt);
      }
    }
    if (auto jt = dest_off.find(l); jt != dest_off.end()) {
      auto const nd = dcur + jt->second;
      if (nd < 65535u && nd < end_dist) end_dist = nd;
    }
  }
  if (end_dist == 32767) return 32767;
  return static_cast<int16_t>(std::ceil(end_dist * q.fastest_direct_factor));
}

// dijkstra.cc:18-67 over the precomputed lower-bound graph: a bucket queue
// over distances 0..kMaxTravelTime (dial.h) whose buckets are reused across
// queries of the same thread.  Shortest distances do not depend on the pop
// order inside a bucket.
// Dijkstra seeds: per root location the minimum offset, then every meta of
// the root with that distance (dijkstra.cc:26-48).
void lb_seeds(view const& v, prepped_query const& p,
              std::vector<std::pair<uint32_t, uint16_t>>& out) {
  std::map<uint32_t, uint16_t> seed;
  for (auto const& o : p.dest_offsets) {
    v.metas(p.dest_mode, o.target, [&](uint32_t x) {
      auto const r = v.root(x);
      auto it = seed.find(r);
      if (it == seed.end()) it = seed.emplace(r, kUnreach).first;
      it->second = std::min(static_cast<uint16_t>(o.duration), it->second);
    });
  }
  out.clear();
  for (auto const& [l, dd] : seed) {
    v.metas(p.dest_mode, l, [&](uint32_t m) { out.emplace_back(m, dd); });
  }
}

void lower_bounds(view const& v, prepped_query const& p, std::vector<uint16_t>& dist) {
  auto const n = v.d.n_locations;
  dist.assign(n, kUnreach);
  std::map<uint32_t, uint16_t> seed;
  for (auto const& o : p.dest_offsets) {
    v.metas(p.dest_mode, o.target, [&](uint32_t x) {
      auto const r = v.root(x);
      auto it = seed.find(r);
      if (it == seed.end()) it = seed.emplace(r, dist[r]).first;
      it->second = std::min(static_cast<uint16_t>(o.duration), it->second);
    });
  }
  constexpr uint32_t kBuckets = B2R_MAX_TRAVEL_TIME_MIN + 1;
  thread_local std::vector<std::vector<uint32_t>> bucket(kBuckets);
  size_t cur = kBuckets, size = 0, hi = 0;
  auto const push = [&](uint32_t l, uint32_t d) {
    bucket[d].push_back(l);
    cur = std::min<size_t>(cur, d);
    hi = std::max<size_t>(hi, d);
    ++size;
  };
  for (auto const& [l, dd] : seed) {
    v.metas(p.dest_mode, l, [&](uint32_t m) {
      push(m, dd);
      dist[m] = std::min(dd, dist[m]);
    });
  }
  while (size != 0) {
    while (bucket[cur].empty()) ++cur;
    auto const l = bucket[cur].back();
    bucket[cur].pop_back();
    --size;
    if (dist[l] < cur) continue;
    auto const [eb, ee] = lb_edges_at(v.d, p.prf, p.fwd, l);  // the profile's graph
    for (auto const* e = eb; e != ee; ++e) {
      auto const tgt = B2R_FP_TARGET(*e);
      auto const nd = static_cast<uint32_t>(cur) + B2R_FP_DURATION(*e);
      if (nd < dist[tgt] && nd < kBuckets) {
        dist[tgt] = static_cast<uint16_t>(nd);
        push(tgt, nd);
      }
    }
  }
  for (auto i = 0U; i != n; ++i) {
    auto const lb = dist[i];
    v.kids(i, [&](uint32_t c) { dist[c] = std::min(lb, dist[c]); });
  }
}

}  // namespace

// One row of the all-pairs lower-bound table: the Dijkstra of
// lower_bounds() from the single seed `src` at distance 0, without the
// children step (applied per query after the rows are combined).
void lb_table_row(host_view const& hv, bool fwd, uint32_t src, uint16_t* row) {
  auto const n = hv.d.n_locations;
  std::fill(row, row + n, kUnreach);
  constexpr uint32_t kBuckets = B2R_MAX_TRAVEL_TIME_MIN + 1;
  thread_local std::vector<std::vector<uint32_t>> bucket(kBuckets);
  size_t cur = 0, size = 1;
  bucket[0].push_back(src);
  row[src] = 0;
  auto const* gi = fwd ? hv.d.lb_fwd_index : hv.d.lb_bwd_index;
  auto const* gd = fwd ? hv.d.lb_fwd : hv.d.lb_bwd;
  while (size != 0) {
    while (bucket[cur].empty()) ++cur;
    auto const l = bucket[cur].back();
    bucket[cur].pop_back();
    --size;
    if (row[l] < cur) continue;
    for (auto e = gi[l]; e != gi[l + 1]; ++e) {
      auto const tgt = B2R_FP_TARGET(gd[e]);
      auto const nd = static_cast<uint32_t>(cur) + B2R_FP_DURATION(gd[e]);
      if (nd < row[tgt] && nd < kBuckets) {
        row[tgt] = static_cast<uint16_t>(nd);
        bucket[nd].push_back(tgt);
        ++size;
      }
    }
  }
}

namespace {

uint16_t event(b2r_timetable_desc const& d, uint32_t r, uint32_t t, uint32_t s, bool arr) {
  auto const n_t = d.route_transport_to[r] - d.route_transport_from[r];
  return d.route_stop_times[d.route_stop_time_from[r] + n_t * (s * 2 - (arr ? 1U : 0U)) +
                            (t - d.route_transport_from[r])];
}

bool bf_test(b2r_timetable_desc const& d, uint32_t bf, uint32_t i) {
  return i < B2R_MAX_DAYS && ((d.bitfields[8ull * bf + i / 64] >> (i % 64)) & 1ULL);
}

bool view::transport_active(uint32_t t, uint32_t day) const {
  if (rt != nullptr) {
    auto const it = rt->changed.find(t);
    if (it != rt->changed.end()) {
      return day < B2R_MAX_DAYS && ((rt->changed_days[8ull * it->second + day / 64] >> (day % 64)) & 1ULL);
    }
  }
  return bf_test(d, d.transport_traffic_days[t], day);
}

// add_starts_in_interval + add_start_times_at_stop, start_times.cc:40-239
void interval_starts(view const& v, prepped_query const& p, int32_t iv_from, int32_t iv_to,
                     uint32_t l, int16_t off, bool add_ontrip, std::vector<start_label>& out) {
  auto const& d = v.d;
  auto const fwd = p.fwd;
  auto const day_of = [&](int32_t t) {
    return static_cast<uint16_t>((t - v.internal_from_min()) / 1440);
  };
  for (auto ri = d.location_routes_index[l]; ri != d.location_routes_index[l + 1]; ++ri) {
    auto const r = d.location_routes[ri];
    auto const s0 = d.route_stop_index[r];
    auto const n = d.route_stop_index[r + 1] - s0;
    for (auto i = 0U; i != n; ++i) {
      auto const stp = d.route_stops[s0 + i];
      if (B2R_STOP_LOC(stp) != l) continue;
      if ((!fwd && (i == 0U || !stop_out(stp, p.prf))) || (fwd && (i + 1U == n || !stop_in(stp, p.prf)))) {
        continue;
      }
      auto const st_from = fwd ? iv_from : iv_from - p.max_start_offset_;
      auto const st_to = fwd ? iv_to + p.max_start_offset_ : iv_to;
      auto const first = day_of(st_from), last = day_of(st_to);
      for (auto t = d.route_transport_from[r]; t != d.route_transport_to[r]; ++t) {
        auto const ev = event(d, r, t, i, !fwd);
        auto const cnt = static_cast<int16_t>(B2R_DELTA_DAYS(ev) * 1440 + B2R_DELTA_MAM(ev));
        auto const day_off = static_cast<uint16_t>(cnt / 1440);
        auto const mam = cnt % 1440;
        for (uint32_t day = first; day <= last; ++day) {
          auto const ev_time = v.internal_from_min() + static_cast<int32_t>(day) * 1440 + mam;
          if (!v.transport_active(t, static_cast<uint16_t>(day - day_off)) || ev_time < st_from ||
              ev_time >= st_to) {
            continue;
          }
          if (off == kMaxDur) continue;
          auto const tas = fwd ? ev_time - off : ev_time + off;
          if (tas < iv_from || tas >= iv_to) continue;
          if (!out.empty() && out.back().time_at_start == tas &&
              (fwd ? out.back().time_at_stop <= ev_time : out.back().time_at_stop >= ev_time)) {
            continue;
          }
          out.push_back({tas, ev_time, l});
        }
      }
    }
  }
  if (v.rt != nullptr) {  // real-time starts, start_times.cc:177-215
    auto const& rt = *v.rt;
    for (auto xi = rt.loc_idx[l]; xi != rt.loc_idx[l + 1]; ++xi) {
      auto const x = rt.loc_rt[xi];
      auto const n = rt.n_stops(x);
      for (auto i = 0U; i != n; ++i) {
        auto const stp = rt.stop(x, i);
        if (B2R_STOP_LOC(stp) != l) continue;
        if ((!fwd && (i == 0U || !stop_out(stp, p.prf))) || (fwd && (i + 1U == n || !stop_in(stp, p.prf)))) continue;
        auto const ev_time = rt.event(x, i, !fwd);
        auto const tas = fwd ? ev_time - off : ev_time + off;
        if (tas < iv_from || tas >= iv_to) continue;
        out.push_back({tas, ev_time, l});
      }
    }
  }
  if (add_ontrip) {
    auto const tas = fwd ? iv_to : iv_from - 1;
    if (off != kMaxDur) out.push_back({tas, fwd ? iv_to + off : iv_from - 1 - off, l});
  }
}


// get_starts, start_times.cc:241-319: shortest offset per start location
// (insertion ordered), then ontrip labels or interval departures.
void collect_starts(view const& v, prepped_query const& p, bool interval, int32_t t,
                    int32_t iv_from, int32_t iv_to, bool use_fp, bool add_ontrip,
                    std::vector<start_label>& out) {
  std::vector<std::pair<uint32_t, int16_t>> shortest;
  std::unordered_map<uint32_t, size_t> at;
  auto const upd = [&](uint32_t l, int16_t dd) {
    auto it = at.find(l);
    if (it == at.end()) {
      at.emplace(l, shortest.size());
      shortest.emplace_back(l, dd);
    } else {
      shortest[it->second].second = std::min(shortest[it->second].second, dd);
    }
  };
  for (auto const& o : p.start_offsets) {
    v.metas(p.start_mode, o.target, [&](uint32_t l) {
      upd(l, o.duration);
      if (use_fp) {
        auto const [fb, fe] = footpaths_at(v.d, p.prf, p.fwd, l);
        for (auto const* f = fb; f != fe; ++f) {
          upd(B2R_FP_TARGET(*f),
              static_cast<int16_t>(o.duration + adjust<int16_t>(p.tts, static_cast<int16_t>(B2R_FP_DURATION(*f)))));
        }
      }
    });
  }
  for (auto const& [l, o] : shortest) {
    if (interval) {
      interval_starts(v, p, iv_from, iv_to, l, o, add_ontrip, out);
    } else {
      out.push_back({t, p.fwd ? t + o : t - o, l});
    }
  }
}

void sort_starts(bool fwd, std::vector<start_label>& s) {  // search.h:408-410
  auto const lt = [](start_label const& a, start_label const& b) {
    if (a.time_at_start != b.time_at_start) return a.time_at_start < b.time_at_start;
    if (a.time_at_stop != b.time_at_stop) return a.time_at_stop < b.time_at_stop;
    return a.stop < b.stop;
  };
  std::sort(s.begin(), s.end(), [&](start_label const& a, start_label const& b) {
    return fwd ? lt(b, a) : lt(a, b);
  });
}

}  // namespace

// destination sets of a search: distances of intermodal offsets, or the
// matching locations of station offsets (collect_destinations,
// start_times.cc:321-353)
void collect_dests(view const& v, prepped_query& p) {
  p.intermodal_dest = p.dest_mode == B2R_MATCH_INTERMODAL;
  if (p.intermodal_dest) {
    std::map<uint32_t, uint16_t> dd;
    for (auto const& o : p.dest_offsets) {
      v.metas(B2R_MATCH_INTERMODAL, o.target, [&](uint32_t l) {
        auto it = dd.find(l);
        auto const val = static_cast<uint16_t>(o.duration);
        if (it == dd.end()) dd.emplace(l, val);
        else it->second = std::min(it->second, val);
      });
    }
    for (auto const& [l, x] : dd) {
      if (x != kUnreach) p.dest_dist.emplace_back(l, x);
    }
  } else {
    for (auto const& o : p.dest_offsets) {
      v.metas(p.dest_mode, o.target, [&](uint32_t l) { p.dest_locs.push_back(l); });
    }
    std::sort(p.dest_locs.begin(), p.dest_locs.end());
    p.dest_locs.erase(std::unique(p.dest_locs.begin(), p.dest_locs.end()), p.dest_locs.end());
  }
}

// pong_search, pong.cc:63-230: the sanitised query, its fastest direct
// connection and base day, and the templates of the ping (the query's
// direction, with the Dijkstra lower bounds) and of the pong (flipped,
// without lower bounds: kPruneWithPingBounds).  Transfer time settings stay
// as given: pong hands q.transfer_time_settings_ to both searches without
// search::init's normalisation.
void prepare_pong(host_view const& hv, b2r_query const& q, int lb_mode, prepped_query& out) {
  view const v{hv.d, hv.rt};
  out = prepped_query{};
  if (q.kind != B2R_ONE_TO_ONE || (q.start_match_mode == B2R_MATCH_INTERMODAL && q.use_start_footpaths != 0)) {
    out.status = B2R_ERR_INVALID_ARGUMENT;  // query::sanitize's verify (query.cc:59-62)
    return;
  }
  auto plan = std::make_shared<pong_plan>();
  auto const fwd = q.direction == B2R_FORWARD;
  std::vector<b2r_offset> so(q.start, q.start + q.n_start), de(q.destination, q.destination + q.n_destination);
  for (auto const* offs : {&so, &de}) {
    for (auto const& o : *offs) {
      if (o.target >= hv.d.n_locations) {
        out.status = B2R_ERR_INVALID_ARGUMENT;
        return;
      }
    }
  }
  auto const by_dur = [](b2r_offset const& a, b2r_offset const& b) { return a.duration < b.duration; };
  std::sort(so.begin(), so.end(), by_dur);
  std::sort(de.begin(), de.end(), by_dur);
  tts_norm const raw{q.tts_default, q.tts_min_transfer_time, q.tts_additional_time, q.tts_factor};
  auto const mtt = (q.max_travel_time < 0 || q.max_travel_time > B2R_MAX_TRAVEL_TIME_MIN)
                       ? static_cast<int16_t>(B2R_MAX_TRAVEL_TIME_MIN)
                       : q.max_travel_time;
  auto const iv_from = q.is_interval != 0 ? q.interval_from : q.start_time;
  auto const iv_to = q.is_interval != 0 ? q.interval_to : q.start_time;
  auto const mid = static_cast<int64_t>(iv_from) + (iv_to - iv_from) / 2;
  auto const base = static_cast<uint16_t>(round_to_days(mid) - hv.internal_from_days());
  auto const fdirect = fastest_direct(v, q, so, de, raw, fwd);

  auto const tmpl = [&](bool dir, uint8_t smode, uint8_t dmode, std::vector<b2r_offset> const& st,
                        std::vector<b2r_offset> const& dt, prepped_query& t) {
    t.fwd = dir;
    t.one_to_all = false;
    t.ontrip = q.is_interval == 0;
    t.start_mode = smode;
    t.dest_mode = dmode;
    t.max_transfers = q.max_transfers;
    t.max_start_offset_ = q.max_start_offset;
    t.end_k = static_cast<uint8_t>(std::min<int>(q.max_transfers, B2R_MAX_TRANSFERS) + 2);
    t.allowed_claszes = static_cast<uint16_t>(q.allowed_claszes & 0xFFFFU);
    t.req_flags = required_flags(q);
    t.prf = q.prf_idx;
    t.start_offsets = st;
    t.dest_offsets = dt;
    t.tts_raw = raw;
    t.tts = raw;
    t.max_travel_time = mtt;
    t.fastest_direct = fdirect;
    t.base = base;
    t.base_days = hv.internal_from_days() + base;
    t.iv_from = iv_from;
    t.iv_to = iv_to;
    collect_dests(v, t);
  };
  auto& ping = plan->ping;
  tmpl(fwd, q.start_match_mode, q.dest_match_mode, so, de, ping);
  // the device lower-bound tables and solver cover profile 0; other
  // profiles take the host Dijkstra over their own graph
  auto const host_lb = lb_mode == 1 || (lb_mode >= 2 && ping.prf != 0U);
  if (host_lb) lower_bounds(v, ping, ping.lb);
  if (!host_lb && (lb_mode == 2 || lb_mode == 3)) lb_seeds(v, ping, ping.lb_seeds);
  ping.use_start_footpaths = q.use_start_footpaths != 0;
  ping.span = static_cast<int16_t>(std::min<int>(mtt + 1440, B2R_MAX_TRAVEL_TIME_MIN));  // kMinLookAhead
  ping.recon_mode = 2;
  auto& pong = plan->pong;
  tmpl(!fwd, q.dest_match_mode, q.start_match_mode, de, so, pong);
  pong.no_lb = true;
  pong.keep_lb = true;
  pong.use_start_footpaths = q.dest_match_mode != B2R_MATCH_INTERMODAL;  // pong.cc:291-295
  pong.recon_mode = 1;
  plan->iv_from = iv_from;
  plan->iv_to = iv_to;
  plan->ext_from = hv.d.date_range_from * 1440;
  plan->ext_to = hv.d.date_range_to * 1440;
  plan->fastest_direct = fdirect;
  plan->max_travel_time = mtt;
  plan->max_transfers = q.max_transfers;
  plan->min_connection_count = q.min_connection_count;
  plan->fwd = fwd;
  plan->extend_earlier = q.extend_interval_earlier != 0;
  plan->extend_later = q.extend_interval_later != 0;

  // the first ping, at the first start time of the sweep
  out = ping;
  auto const t0 = fwd ? iv_from : iv_to - 1;
  if (!(plan->ext_from <= t0 && t0 < plan->ext_to)) {  // pong.cc:243: no iteration at all
    out.empty_result = true;
    out.iv_from = fwd ? iv_from : t0 + 1;
    out.iv_to = fwd ? t0 : iv_to;
  } else {
    collect_starts(v, out, false, t0, 0, 0, out.use_start_footpaths, false, out.starts);
  }
  out.pong = std::move(plan);
}

void phase_starts(host_view const& hv, prepped_query const& tmpl, int32_t t, std::vector<start_label>& out) {
  view const v{hv.d, hv.rt};
  out.clear();
  collect_starts(v, tmpl, false, t, 0, 0, tmpl.use_start_footpaths, false, out);
}

void prepare(host_view const& hv, b2r_query const& q, int lb_mode, prepped_query& p) {
  if (q.prf_idx >= B2R_N_PROFILES) {  // profile_idx_t below kNProfiles (types.h:204-210)
    p = prepped_query{};
    p.status = B2R_ERR_INVALID_ARGUMENT;
    return;
  }
  if (q.algorithm == B2R_ALGO_PONG) {
    if (hv.rt != nullptr) {  // pong over a real-time overlay is not implemented
      p = prepped_query{};
      p.status = B2R_ERR_UNSUPPORTED;
      return;
    }
    prepare_pong(hv, q, lb_mode, p);
    return;
  }
  if (q.algorithm != B2R_ALGO_RAPTOR) {
    p = prepped_query{};
    p.status = B2R_ERR_INVALID_ARGUMENT;
    return;
  }
  view const v{hv.d, hv.rt};
  p = prepped_query{};
  p.fwd = q.direction == B2R_FORWARD;
  p.one_to_all = q.kind == B2R_ONE_TO_ALL;
  p.ontrip = q.is_interval == 0;
  p.start_mode = q.start_match_mode;
  p.dest_mode = q.dest_match_mode;
  p.max_transfers = q.max_transfers;
  p.max_start_offset_ = q.max_start_offset;
  p.end_k = static_cast<uint8_t>(std::min<int>(q.max_transfers, B2R_MAX_TRANSFERS) + 2);
  p.min_connection_count = q.min_connection_count;
  p.extend_earlier = q.extend_interval_earlier != 0;
  p.extend_later = q.extend_interval_later != 0;
  p.allowed_claszes = static_cast<uint16_t>(q.allowed_claszes & 0xFFFFU);  // 16 classes
  p.req_flags = required_flags(q);
  p.prf = q.prf_idx;
  p.start_offsets.assign(q.start, q.start + q.n_start);
  p.dest_offsets.assign(q.destination, q.destination + q.n_destination);
  p.tts_raw = {q.tts_default, q.tts_min_transfer_time, q.tts_additional_time, q.tts_factor};

  for (auto const& o : p.start_offsets) {
    if (o.target >= hv.d.n_locations) {
      p.status = B2R_ERR_INVALID_ARGUMENT;
      return;
    }
  }
  for (auto const& o : p.dest_offsets) {
    if (o.target >= hv.d.n_locations) {
      p.status = B2R_ERR_INVALID_ARGUMENT;
      return;
    }
  }

  if (p.one_to_all) {  // one_to_all.cc:18-104
    p.max_travel_time = q.max_travel_time;
    p.tts = p.tts_raw;
    p.base = static_cast<uint16_t>(round_to_days(q.start_time) - hv.internal_from_days());
    p.base_days = hv.internal_from_days() + p.base;
    p.iv_from = p.iv_to = q.start_time;
    for (auto const& s : p.start_offsets) {
      auto const t = p.fwd ? q.start_time + s.duration : q.start_time - s.duration;
      v.metas(p.start_mode, s.target, [&](uint32_t l) {
        p.starts.push_back({q.start_time, t, l});
      });
    }
    p.lb.clear();  // one_to_all runs without lower bounds (lb = 0)
    p.span = p.max_travel_time;  // one_to_all.cc:44-46
    return;
  }

  // query::sanitize (query.cc:59-67), applied by raptor_search_with_dir
  p.max_travel_time = (q.max_travel_time < 0 || q.max_travel_time > B2R_MAX_TRAVEL_TIME_MIN)
                          ? B2R_MAX_TRAVEL_TIME_MIN
                          : q.max_travel_time;
  auto const by_dur = [](b2r_offset const& a, b2r_offset const& b) { return a.duration < b.duration; };
  std::sort(p.start_offsets.begin(), p.start_offsets.end(), by_dur);
  std::sort(p.dest_offsets.begin(), p.dest_offsets.end(), by_dur);

  p.iv_from = p.ontrip ? q.start_time : q.interval_from;
  p.iv_to = p.ontrip ? q.start_time : q.interval_to;
  p.fastest_direct = fastest_direct(v, q, p.start_offsets, p.dest_offsets, p.tts_raw, p.fwd);

  // search::init, search.h:84-172
  p.tts.factor = std::max(p.tts_raw.factor, 1.0F);
  p.tts.min_transfer_time = std::max<int16_t>(p.tts_raw.min_transfer_time, 0);
  p.tts.additional_time = std::max<int16_t>(p.tts_raw.additional_time, 0);
  p.tts.is_default = p.tts.factor == 1.0F && p.tts.min_transfer_time == 0 && p.tts.additional_time == 0;
  collect_dests(v, p);
  p.span = static_cast<int16_t>(std::min<int>(p.fastest_direct, p.max_travel_time) + 1);  // search.h:426-429
  auto const host_lb = lb_mode == 1 || (lb_mode >= 2 && p.prf != 0U);  // as for pong's ping
  if (host_lb) lower_bounds(v, p, p.lb);
  if (!host_lb && (lb_mode == 2 || lb_mode == 3)) lb_seeds(v, p, p.lb_seeds);
  auto const mid = static_cast<int64_t>(p.iv_from) + (p.iv_to - p.iv_from) / 2;
  p.base = static_cast<uint16_t>(round_to_days(mid) - hv.internal_from_days());
  p.base_days = hv.internal_from_days() + p.base;

  // start_dest_overlap, search.h:354-378
  if (p.start_mode != B2R_MATCH_INTERMODAL && p.dest_mode != B2R_MATCH_INTERMODAL) {
    auto overlap = false;
    for (auto const& o : p.dest_offsets) {
      v.metas(p.dest_mode, o.target, [&](uint32_t eq) {
        for (auto const& s : p.start_offsets) {
          v.metas(p.start_mode, s.target, [&](uint32_t x) { overlap = overlap || x == eq; });
        }
      });
    }
    if (overlap) {
      p.empty_result = true;
      return;
    }
  }

  // interval_estimator, interval_estimate.h:12-80
  auto const ext_from = hv.d.date_range_from * 1440, ext_to = hv.d.date_range_to * 1440;
  {
    auto const w = q.has_fastest_direct ? 1 : 2;
    constexpr int kMaxIv = (32767 / 1440 - 7) * 1440;
    p.data_max_from = std::max(round_to_days(static_cast<int64_t>(p.iv_from) - w * 1440) * 1440,
                               round_to_days(static_cast<int64_t>(p.iv_from) +
                                             (p.iv_to - p.iv_from - kMaxIv) / 2) * 1440);
    p.data_max_to = std::min(round_to_days(static_cast<int64_t>(p.iv_to) + w * 1440) * 1440,
                             round_to_days(static_cast<int64_t>(p.iv_from) +
                                           (p.iv_to - p.iv_from + kMaxIv) / 2) * 1440);
  }
  p.has_max_interval = q.has_max_interval != 0;
  p.max_iv_from = q.max_interval_from;
  p.max_iv_to = q.max_interval_to;
  auto const clampi = [&](int32_t x) { return clamp_interval_end(p, ext_from, ext_to, x); };
  if (!p.ontrip && p.min_connection_count != 0 && (p.extend_earlier || p.extend_later)) {
    auto nf = p.iv_from, nt = p.iv_to;
    auto const ext = 60 * static_cast<int>(p.min_connection_count);
    auto const can_earlier = p.extend_earlier && p.iv_from != ext_from;
    auto const can_later = p.extend_later && p.iv_to != ext_to;
    if (p.fwd ? can_later : can_earlier) {
      if (p.fwd) {
        if (can_earlier) nf -= 60;
        else nt += 60;
        nt += ext;
      } else {
        if (can_later) nt += 60;
        else nf -= 60;
        nf -= ext;
      }
    } else {
      if (p.fwd && p.extend_earlier) nf -= 60 + ext;
      if (!p.fwd && p.extend_later) nt += 60 + ext;
    }
    p.iv_from = clampi(nf);
    p.iv_to = clampi(nt);
  }

  // add_start_labels, search.h:220-225, 401-411
  if (p.iv_to - p.iv_from != 0) {
    collect_starts(v, p, true, 0, p.iv_from, p.iv_to, q.use_start_footpaths != 0, true, p.starts);
  } else {
    collect_starts(v, p, !p.ontrip, q.start_time, q.interval_from, q.interval_to,
                   q.use_start_footpaths != 0, true, p.starts);
  }
  sort_starts(p.fwd, p.starts);
}

void add_interval_starts(host_view const& hv, prepped_query const& p, int32_t from, int32_t to,
                         bool add_ontrip, std::vector<start_label>& starts) {
  view const v{hv.d, hv.rt};
  collect_starts(v, p, true, 0, from, to, false, add_ontrip, starts);
  sort_starts(p.fwd, starts);
}

bool extend_interval(prepped_query const& p, int32_t ext_from, int32_t ext_to,
                     uint32_t num_con_req, int32_t& from, int32_t& to) {
  if (num_con_req == 0 || (!p.extend_earlier && !p.extend_later)) return false;
  auto nf = from, nt = to;
  auto const ext = (to - from) * static_cast<int>(num_con_req);
  auto const can_earlier = p.extend_earlier && from != ext_from;
  auto const can_later = p.extend_later && to != ext_to;
  if (can_earlier && can_later) {
    nf -= ext / 2;
    nt += ext / 2;
  } else {
    if (p.extend_earlier) nf -= ext;
    if (p.extend_later) nt += ext;
  }
  auto const clampi = [&](int32_t x) { return clamp_interval_end(p, ext_from, ext_to, x); };
  nf = clampi(nf);
  nt = clampi(nt);
  auto const changed = nf != from || nt != to;
  from = nf;
  to = nt;
  return changed;
}

bool rt_host::init(b2r_rt_desc const& src, uint32_t n_loc, uint32_t n_transports) {
  auto const n_rt = src.n_rt_transports;
  if ((src.n_changed != 0 && (src.changed_transport == nullptr || src.changed_days == nullptr)) ||
      (n_rt != 0 && (src.rt_stop_index == nullptr || src.rt_stops == nullptr || src.rt_event_times == nullptr))) {
    return false;
  }
  changed_transport.assign(src.changed_transport, src.changed_transport + src.n_changed);
  changed_days.assign(src.changed_days, src.changed_days + 8ull * src.n_changed);
  for (auto i = 0U; i != src.n_changed; ++i) {
    if (changed_transport[i] >= n_transports) return false;
    changed[changed_transport[i]] = i;
  }
  if (n_rt != 0) {
    stop_index.assign(src.rt_stop_index, src.rt_stop_index + n_rt + 1);
  } else {
    stop_index.assign(1, 0U);
  }
  if (stop_index[0] != 0U) return false;
  for (auto x = 0U; x != n_rt; ++x) {
    if (stop_index[x + 1] < stop_index[x] + 2U) return false;  // a run has two stops at least
  }
  auto const n_stops_all = stop_index.back();
  stops.assign(src.rt_stops, src.rt_stops + n_stops_all);
  for (auto w : stops) {
    if (B2R_STOP_LOC(w) >= n_loc) return false;
  }
  times.assign(src.rt_event_times, src.rt_event_times + 2ull * (n_stops_all - n_rt));
  static_transport.assign(n_rt, B2R_INVALID_IDX);
  if (src.rt_static_transport != nullptr) static_transport.assign(src.rt_static_transport, src.rt_static_transport + n_rt);
  static_day.assign(n_rt, 0U);
  if (src.rt_static_day != nullptr) static_day.assign(src.rt_static_day, src.rt_static_day + n_rt);
  clasz.assign(n_rt, 10U);
  if (src.rt_clasz != nullptr) clasz.assign(src.rt_clasz, src.rt_clasz + n_rt);
  for (auto c : clasz) {
    if (c >= 16U) return false;
  }
  flags.assign(n_rt, 0U);
  if (src.rt_flags != nullptr) flags.assign(src.rt_flags, src.rt_flags + n_rt);
  section_flags.assign(n_stops_all, 0U);
  if (src.rt_section_flags != nullptr) section_flags.assign(src.rt_section_flags, src.rt_section_flags + n_stops_all);
  // location_rt_transports_: each run once per location, in run order
  std::vector<std::vector<uint32_t>> by_loc(n_loc);
  for (auto x = 0U; x != n_rt; ++x) {
    for (auto i = stop_index[x]; i != stop_index[x + 1]; ++i) {
      auto& v = by_loc[B2R_STOP_LOC(stops[i])];
      if (v.empty() || v.back() != x) v.push_back(x);
    }
  }
  loc_idx.assign(n_loc + 1U, 0U);
  loc_rt.clear();
  for (auto l = 0U; l != n_loc; ++l) {
    loc_idx[l + 1U] = loc_idx[l] + static_cast<uint32_t>(by_loc[l].size());
    loc_rt.insert(loc_rt.end(), by_loc[l].begin(), by_loc[l].end());
  }
  d = src;
  d.changed_transport = changed_transport.data();
  d.changed_days = changed_days.data();
  d.rt_stop_index = stop_index.data();
  d.rt_stops = stops.data();
  d.rt_event_times = times.data();
  d.rt_static_transport = static_transport.data();
  d.rt_static_day = static_day.data();
  d.rt_clasz = clasz.data();
  d.rt_flags = flags.data();
  d.rt_section_flags = section_flags.data();
  return true;
}

}  // namespace b2r
