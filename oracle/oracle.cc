// TEST INFRASTRUCTURE ONLY -- CPU restatement of nigiri's RAPTOR search
// (see oracle.h for the list of restated reference files).  Compiled with
// -ffp-contract=off so that the double arithmetic of get_penalty matches the
// reference bit for bit.
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <optional>
#include <queue>
#include <array>
#include <iterator>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace oracle {

using unixtime = int32_t;  // minutes since epoch (unixtime_t)
using delta_t = int16_t;
constexpr int kK = B2R_K;
constexpr int kMaxTransfers = B2R_MAX_TRANSFERS;
constexpr int kMaxTravelTime = B2R_MAX_TRAVEL_TIME_MIN;
constexpr int kFpMaxDuration = 511;  // footpath::kMaxDuration
constexpr uint32_t kInvalidIdx = 0xFFFFFFFFu;
constexpr uint16_t kUnreachable = 0xFFFFu;
constexpr uint32_t kEnd = B2R_SPECIAL_END;
constexpr uint32_t kStart = B2R_SPECIAL_START;

// ----------------------------------------------------------- delta_t.h
inline delta_t clamp16(int t) {
  return static_cast<delta_t>(std::clamp(t, -32768, 32767));
}
inline delta_t unix_to_delta(int32_t base_days, unixtime t) {
  return clamp16(t - base_days * 1440);
}
inline unixtime delta_to_unix(int32_t base_days, delta_t d) {
  return base_days * 1440 + d;
}
inline std::pair<uint16_t, int16_t> split_day_mam(uint16_t base, delta_t x) {
  auto const minutes = static_cast<int>(base) * 1440 + x;
  return {static_cast<uint16_t>(minutes / 1440),
          static_cast<int16_t>(minutes % 1440)};
}

// std::chrono::round<days> on a minute time point (ties to even)
inline int32_t round_days(int64_t minutes) {
  auto const d0 = minutes >= 0 ? minutes / 1440 : -((-minutes + 1439) / 1440);
  auto const d1 = d0 + 1;
  auto const diff0 = minutes - d0 * 1440;
  auto const diff1 = d1 * 1440 - minutes;
  if (diff0 == diff1) return static_cast<int32_t>((d0 & 1) ? d1 : d0);
  return static_cast<int32_t>(diff0 < diff1 ? d0 : d1);
}

// ------------------------------------------------- timetable accessors
// the real-time overlay (rt_timetable, rt/rt_timetable.h:48-311): the
// description and the lookups rt_timetable keeps (changed traffic days by
// transport, location_rt_transports_)
struct rt_overlay {
  b2r_rt_desc const* d{nullptr};
  std::unordered_map<uint32_t, uint32_t> changed;  // transport -> its row of changed_days
  std::vector<uint32_t> loc_idx, loc_rt;            // location_rt_transports_ (CSR)

  rt_overlay(b2r_rt_desc const* desc, uint32_t n_loc) : d{desc} {
    if (d == nullptr) return;
    for (auto i = 0U; i != d->n_changed; ++i) changed[d->changed_transport[i]] = i;
    std::vector<std::vector<uint32_t>> by_loc(n_loc);
    for (auto x = 0U; x != d->n_rt_transports; ++x) {
      for (auto i = d->rt_stop_index[x]; i != d->rt_stop_index[x + 1]; ++i) {
        auto const l = B2R_STOP_LOC(d->rt_stops[i]);
        if (by_loc[l].empty() || by_loc[l].back() != x) by_loc[l].push_back(x);
      }
    }
    loc_idx.assign(n_loc + 1U, 0U);
    for (auto l = 0U; l != n_loc; ++l) {
      loc_idx[l + 1U] = loc_idx[l] + static_cast<uint32_t>(by_loc[l].size());
      loc_rt.insert(loc_rt.end(), by_loc[l].begin(), by_loc[l].end());
    }
  }
};

struct tt_view {
  b2r_timetable_desc const& d;
  uint32_t prf{0};  // the query's footpath profile (query::prf_idx_)
  rt_overlay const* rt{nullptr};
  mutable std::vector<uint32_t> zero_{};

  // footpaths_out_[prf] (out) or footpaths_in_[prf] (timetable.h:97-98) and
  // fwd / bwd_search_lb_graph_[prf] (:421-422): CSR index and words; a
  // profile without them reads as an all-zero index
  uint32_t const* zero_index() const {
    if (zero_.empty()) zero_.assign(d.n_locations + 1U, 0U);
    return zero_.data();
  }
  uint32_t const* fp_index(bool out) const {
    auto const* x = prf == 0U ? (out ? d.footpaths_out_index : d.footpaths_in_index)
                              : (out ? d.profile_footpaths_out_index[prf - 1U] : d.profile_footpaths_in_index[prf - 1U]);
    return x != nullptr ? x : zero_index();
  }
  uint32_t const* fp_words(bool out) const {
    auto const* x = prf == 0U ? (out ? d.footpaths_out : d.footpaths_in)
                              : (out ? d.profile_footpaths_out[prf - 1U] : d.profile_footpaths_in[prf - 1U]);
    return x != nullptr ? x : zero_index();
  }
  uint32_t const* lb_index(bool fwd) const {
    auto const* x = prf == 0U ? (fwd ? d.lb_fwd_index : d.lb_bwd_index)
                              : (fwd ? d.profile_lb_fwd_index[prf - 1U] : d.profile_lb_bwd_index[prf - 1U]);
    return x != nullptr ? x : zero_index();
  }
  uint32_t const* lb_words(bool fwd) const {
    auto const* x = prf == 0U ? (fwd ? d.lb_fwd : d.lb_bwd)
                              : (fwd ? d.profile_lb_fwd[prf - 1U] : d.profile_lb_bwd[prf - 1U]);
    return x != nullptr ? x : zero_index();
  }
  // stop::in_allowed(p) / out_allowed(p) (stop.h:44-49)
  bool stop_in(uint32_t w) const { return (prf == B2R_PROFILE_WHEELCHAIR ? B2R_STOP_IN_WC(w) : B2R_STOP_IN(w)) != 0U; }
  bool stop_out(uint32_t w) const { return (prf == B2R_PROFILE_WHEELCHAIR ? B2R_STOP_OUT_WC(w) : B2R_STOP_OUT(w)) != 0U; }

  int32_t internal_from_days() const {
    return d.date_range_from - B2R_TIMETABLE_OFFSET_DAYS;
  }
  unixtime internal_from() const { return internal_from_days() * 1440; }
  unixtime external_from() const { return d.date_range_from * 1440; }
  unixtime external_to() const { return d.date_range_to * 1440; }

  bool bf_test(uint32_t bf, uint32_t i) const {  // cista::bitset::test
    if (i >= B2R_MAX_DAYS) return false;
    return ((d.bitfields[8ull * bf + i / 64] >> (i % 64)) & 1ULL) != 0ULL;
  }
  // timetable / rt_timetable::is_transport_active (rt_timetable.h:210-213):
  // the overlay's days for a transport it changed
  bool transport_active(uint32_t t, uint16_t day) const {
    if (has_rt()) {
      auto const it = rt->changed.find(t);
      if (it != rt->changed.end()) {
        return day < B2R_MAX_DAYS && ((rt->d->changed_days[8ull * it->second + day / 64] >> (day % 64)) & 1ULL);
      }
    }
    return bf_test(d.transport_traffic_days[t], day);
  }
  // rt transports: stop sequence, unix event times (rt_timetable::
  // unix_event_time), class, flags and section flags
  bool has_rt() const { return rt != nullptr && rt->d != nullptr; }
  uint32_t n_rt() const { return has_rt() ? rt->d->n_rt_transports : 0U; }
  uint32_t rt_n_stops(uint32_t x) const { return rt->d->rt_stop_index[x + 1] - rt->d->rt_stop_index[x]; }
  uint32_t rt_stop(uint32_t x, uint32_t i) const { return rt->d->rt_stops[rt->d->rt_stop_index[x] + i]; }
  unixtime rt_event(uint32_t x, uint32_t i, bool arr) const {
    return rt->d->rt_event_times[2ull * (rt->d->rt_stop_index[x] - x) + 2ull * i - (arr ? 1U : 0U)];
  }
  uint8_t rt_clasz(uint32_t x) const { return rt->d->rt_clasz == nullptr ? 10U : rt->d->rt_clasz[x]; }
  uint8_t rt_flags(uint32_t x) const { return rt->d->rt_flags == nullptr ? 0U : rt->d->rt_flags[x]; }
  uint8_t rt_section_flags(uint32_t x, uint32_t section) const {
    return rt->d->rt_section_flags == nullptr ? 0U : rt->d->rt_section_flags[rt->d->rt_stop_index[x] + section];
  }
  template <typename Fn>
  void location_rt(uint32_t l, Fn&& fn) const {
    if (!has_rt()) return;
    for (auto i = rt->loc_idx[l]; i != rt->loc_idx[l + 1]; ++i) fn(rt->loc_rt[i]);
  }
  bool route_active(uint32_t r, uint16_t day) const {
    return bf_test(d.route_traffic_days[r], day);
  }
  uint32_t n_t(uint32_t r) const {
    return d.route_transport_to[r] - d.route_transport_from[r];
  }
  uint32_t n_stops(uint32_t r) const {
    return d.route_stop_index[r + 1] - d.route_stop_index[r];
  }
  uint32_t stop(uint32_t r, uint32_t i) const {
    return d.route_stops[d.route_stop_index[r] + i];
  }
  // route_clasz_ / route_flags_ / route_flags_per_section_
  // (timetable.h:348-361); absent arrays: bus, no flags
  uint8_t clasz(uint32_t r) const {
    return d.route_clasz == nullptr ? 10U : d.route_clasz[r];
  }
  uint8_t flags(uint32_t r) const {
    return d.route_flags == nullptr ? 0U : d.route_flags[r];
  }
  uint8_t section_flags(uint32_t r, uint32_t section) const {
    return d.route_section_flags == nullptr
               ? 0U
               : d.route_section_flags[d.route_stop_index[r] + section];
  }
  // event_times_at_stop, timetable.h:155-164
  uint16_t const* event_times(uint32_t r, uint32_t s, bool arr) const {
    auto const idx = d.route_stop_time_from[r] + n_t(r) * (s * 2 - (arr ? 1 : 0));
    return d.route_stop_times + idx;
  }
  // event_mam, timetable.h:166-177
  uint16_t event_mam(uint32_t r, uint32_t t, uint32_t s, bool arr) const {
    return event_times(r, s, arr)[t - d.route_transport_from[r]];
  }
  uint16_t event_mam(uint32_t t, uint32_t s, bool arr) const {
    return event_mam(d.transport_route[t], t, s, arr);
  }
  // timetable::event_time, timetable.h:183-188
  unixtime event_time(uint32_t t, uint16_t day, uint32_t s, bool arr) const {
    auto const ev = event_mam(t, s, arr);
    return internal_from() + day * 1440 + B2R_DELTA_DAYS(ev) * 1440 +
           B2R_DELTA_MAM(ev);
  }
  // day_idx_mam, timetable.h:200-208
  std::pair<uint16_t, int> day_idx_mam(unixtime t) const {
    auto const m = t - internal_from();
    return {static_cast<uint16_t>(m / 1440), m % 1440};
  }
  unixtime to_unixtime(uint16_t day, int mam) const {
    return internal_from() + day * 1440 + mam;
  }
  uint32_t root(uint32_t idx) const {  // get_root_idx, timetable.h:62-76
    if (d.parent == nullptr) return idx;
    auto l = idx;
    auto i = 0;
    for (auto p = d.parent[l]; p != kInvalidIdx; p = d.parent[l]) {
      if (p == idx || i > 20) {
        l = d.parent[idx];
        break;
      }
      l = p;
      ++i;
    }
    return l;
  }
  template <typename Fn>
  void children(uint32_t l, Fn&& fn) const {
    if (d.children_index == nullptr) return;
    for (auto i = d.children_index[l]; i != d.children_index[l + 1]; ++i) {
      fn(d.children[i]);
    }
  }
  uint8_t type(uint32_t l) const {
    return d.location_type == nullptr ? 0 : d.location_type[l];
  }
};

// for_each_meta, for_each_meta.h:8-45 (equivalences are not part of the
// flattened image; kEquivalent reduces to root + children)
template <typename Fn>
void for_each_meta(tt_view const& tt, uint8_t mode, uint32_t l, Fn&& fn) {
  auto const handle_children = [&](uint32_t loc) {
    tt.children(loc, [&](uint32_t c) {
      fn(c);
      tt.children(c, [&](uint32_t cc) { fn(cc); });
    });
  };
  if (mode == B2R_MATCH_EXACT) {
    fn(l);
  } else if (mode == B2R_MATCH_INTERMODAL) {
    fn(l);
    tt.children(l, [&](uint32_t c) {
      if (tt.type(c) == B2R_LOC_GENERATED_TRACK) fn(c);
    });
  } else if (mode == B2R_MATCH_ONLY_CHILDREN) {
    fn(l);
    handle_children(l);
  } else {
    auto const root = tt.root(l);
    fn(root);
    handle_children(root);
  }
}

bool matches(tt_view const& tt, uint8_t mode, uint32_t a, uint32_t b) {
  if (mode == B2R_MATCH_EXACT) return a == b;
  if (a == b) return true;
  auto m = false;
  for_each_meta(tt, mode, a, [&](uint32_t c) { m = m || c == b; });
  return m;
}

// ------------------------------------------------------ query / settings
struct tts_t {  // transfer_time_settings.h:8-18
  bool default_{true};
  int16_t min_transfer_time{0};
  int16_t additional_time{0};
  float factor{1.0F};
};

// adjusted_transfer_time<T>, transfer_time_settings.h:20-31
template <typename T>
T adjusted(tts_t const& s, T const duration) {
  if (s.default_) return duration;
  return static_cast<T>(
      static_cast<T>(s.additional_time) +
      std::max(static_cast<T>(s.min_transfer_time),
               static_cast<T>(static_cast<float>(duration) * s.factor)));
}

struct offset_t {
  uint32_t target;
  int16_t duration;
  int32_t mode_id;
};

struct query_t {
  bool is_interval{false};
  unixtime start_time{0};
  unixtime iv_from{0}, iv_to{0};
  uint8_t start_mode{B2R_MATCH_EXACT}, dest_mode{B2R_MATCH_EXACT};
  bool use_start_footpaths{false};
  std::vector<offset_t> start, dest;
  int16_t max_start_offset{kMaxTravelTime};
  uint8_t max_transfers{kMaxTransfers};
  int16_t max_travel_time{kMaxTravelTime};
  uint32_t min_connection_count{0};
  bool extend_earlier{false}, extend_later{false};
  bool has_max_interval{false};  // query::max_interval_, query.h:89
  int32_t max_interval_from{0}, max_interval_to{0};
  tts_t tts;
  bool has_fastest_direct{false};
  int16_t fastest_direct{0};
  double fastest_direct_factor{1.0};
  uint32_t allowed_claszes{B2R_ALL_CLASZ};
  uint8_t required_flags{0};  // bit f: route flag f required
  bool pong{false};           // pong_search instead of search<raptor>

  void flip_dir() {  // query.cc:52-57
    std::swap(start, dest);
    std::swap(start_mode, dest_mode);
  }
  void sanitize() {  // query.cc:59-67 (no vias)
    if (max_travel_time < 0 || max_travel_time > kMaxTravelTime) {
      max_travel_time = kMaxTravelTime;
    }
    auto const cmp = [](offset_t const& a, offset_t const& b) {
      return a.duration < b.duration;
    };
    std::sort(start.begin(), start.end(), cmp);
    std::sort(dest.begin(), dest.end(), cmp);
  }
};

query_t to_query(b2r_query const& q) {
  query_t r;
  r.is_interval = q.is_interval != 0;
  r.start_time = q.start_time;
  r.iv_from = q.interval_from;
  r.iv_to = q.interval_to;
  r.start_mode = q.start_match_mode;
  r.dest_mode = q.dest_match_mode;
  r.use_start_footpaths = q.use_start_footpaths != 0;
  for (auto i = 0U; i != q.n_start; ++i) {
    r.start.push_back({q.start[i].target, q.start[i].duration,
                       q.start[i].transport_mode_id});
  }
  for (auto i = 0U; i != q.n_destination; ++i) {
    r.dest.push_back({q.destination[i].target, q.destination[i].duration,
                      q.destination[i].transport_mode_id});
  }
  r.max_start_offset = q.max_start_offset;
  r.max_transfers = q.max_transfers;
  r.max_travel_time = q.max_travel_time;
  r.min_connection_count = q.min_connection_count;
  r.extend_earlier = q.extend_interval_earlier != 0;
  r.extend_later = q.extend_interval_later != 0;
  r.has_max_interval = q.has_max_interval != 0;
  r.max_interval_from = q.max_interval_from;
  r.max_interval_to = q.max_interval_to;
  r.tts = {q.tts_default != 0, q.tts_min_transfer_time, q.tts_additional_time,
           q.tts_factor};
  r.has_fastest_direct = q.has_fastest_direct != 0;
  r.fastest_direct = q.fastest_direct;
  r.fastest_direct_factor = q.fastest_direct_factor;
  r.allowed_claszes = q.allowed_claszes;
  r.required_flags = static_cast<uint8_t>(
      (q.require_bike_transport != 0 ? 1U << B2R_FLAG_BIKES : 0U) |
      (q.require_car_transport != 0 ? 1U << B2R_FLAG_CARS : 0U) |
      // is_wheelchair: the wheelchair-accessible route filter (raptor.h:256)
      (q.prf_idx == B2R_PROFILE_WHEELCHAIR ? 1U << B2R_FLAG_WHEELCHAIR : 0U) |
      (q.no_compulsory_reservation != 0
           ? 1U << B2R_FLAG_RESERVATION_NOT_REQUIRED
           : 0U));
  r.pong = q.algorithm == B2R_ALGO_PONG;
  return r;
}

// ------------------------------------------------------ journey / pareto
struct leg_t {
  uint32_t from{0}, to{0};
  unixtime dep{0}, arr{0};
  uint8_t kind{B2R_LEG_FOOTPATH};
  uint32_t transport{0};
  uint16_t day{0};
  uint16_t stop_from{0}, stop_to{0};  // [from, to)
  uint32_t target{0};
  int16_t duration{0};
  int32_t mode_id{0};
  uint32_t rt_transport{kInvalidIdx};  // rt::run::rt_ of a real-time run
};

// journey::leg ctor, journey.h:45-60
leg_t make_leg(bool fwd, uint32_t a, uint32_t b, unixtime ta, unixtime tb) {
  leg_t l;
  l.from = fwd ? a : b;
  l.to = fwd ? b : a;
  l.dep = fwd ? ta : tb;
  l.arr = fwd ? tb : ta;
  return l;
}
void set_run(leg_t& l, uint32_t t, uint16_t day, uint16_t a, uint16_t b) {
  l.kind = B2R_LEG_TRANSPORT;
  l.rt_transport = kInvalidIdx;
  l.transport = t;
  l.day = day;
  l.stop_from = std::min(a, b);
  l.stop_to = static_cast<uint16_t>(std::max(a, b) + 1U);
}
void set_fp(leg_t& l, uint32_t target, int dur) {
  l.kind = B2R_LEG_FOOTPATH;
  l.target = target;
  l.duration = static_cast<int16_t>(std::min(dur, kFpMaxDuration));
}
void set_offset(leg_t& l, offset_t const& o) {
  l.kind = B2R_LEG_OFFSET;
  l.target = o.target;
  l.duration = o.duration;
  l.mode_id = o.mode_id;
}

struct journey_t {
  std::vector<leg_t> legs;
  unixtime start_time{0}, dest_time{0};
  uint32_t dest{0};
  uint8_t transfers{0};
  bool error{false};
  bool reconstructed{false};

  bool dominates(journey_t const& o) const {  // journey.h:84-92
    if (start_time <= dest_time) {
      return transfers <= o.transfers && start_time >= o.start_time &&
             dest_time <= o.dest_time;
    }
    return transfers <= o.transfers && start_time <= o.start_time &&
           dest_time >= o.dest_time;
  }
  int travel_time() const { return std::abs(dest_time - start_time); }
};

struct pareto_t {  // pareto_set.h:17-37
  std::vector<journey_t> els;
  bool is_dominated(journey_t const& el) const {
    for (auto const& x : els) {
      if (x.dominates(el)) return true;
    }
    return false;
  }
  bool add(journey_t&& el) {
    auto n_removed = size_t{0};
    for (auto i = 0U; i < els.size(); ++i) {
      if (els[i].dominates(el)) return false;
      if (el.dominates(els[i])) {
        ++n_removed;
        continue;
      }
      els[i - n_removed] = els[i];
    }
    els.resize(els.size() - n_removed + 1);
    els.back() = std::move(el);
    return true;
  }
};

// ------------------------------------------------------------ bitvec
struct bitvec {
  std::vector<uint64_t> b;
  void resize(uint32_t n) { b.assign((n + 63) / 64, 0ULL); }
  void clear() { std::fill(b.begin(), b.end(), 0ULL); }
  void set(uint32_t i) { b[i / 64] |= 1ULL << (i % 64); }
  bool test(uint32_t i) const { return (b[i / 64] >> (i % 64)) & 1ULL; }
  bool any() const {
    for (auto w : b)
      if (w) return true;
    return false;
  }
  template <typename Fn>
  void for_each(Fn&& fn) const {
    for (auto w = 0U; w != b.size(); ++w) {
      auto x = b[w];
      while (x) {
        auto const bit = static_cast<uint32_t>(__builtin_ctzll(x));
        fn(w * 64 + bit);
        x &= x - 1;
      }
    }
  }
};

// The route filters of loop_routes (raptor.h:499-545) and get_transport
// (reconstruct.cc:456-498): false if route r's class is not allowed or a
// required flag is on none of its sections; `sections` receives the
// required flags set on some but not all sections, which the walk along the
// route then checks section by section.
bool route_allowed(tt_view const& tt, uint32_t allowed_claszes, uint8_t required_flags,
                   uint32_t r, uint8_t& sections) {
  sections = 0U;
  auto const c = tt.clasz(r);
  if (c >= 32U || ((allowed_claszes >> c) & 1U) == 0U) return false;
  auto const fl = tt.flags(r);
  for (auto f = 0U; f != 4U; ++f) {
    if (((required_flags >> f) & 1U) == 0U) continue;
    if ((fl >> (2U * f)) & 1U) continue;                     // on all sections
    if (((fl >> (2U * f + 1U)) & 1U) == 0U) return false;  // on none
    sections = static_cast<uint8_t>(sections | (1U << f));
  }
  return true;
}

// the same filters for rt transport x: the class of its first section and
// its route flags (raptor.h:583-626, reconstruct.cc:382-429)
bool rt_allowed(tt_view const& tt, uint32_t allowed_claszes, uint8_t required_flags,
                uint32_t x, uint8_t& sections) {
  sections = 0U;
  auto const c = tt.rt_clasz(x);
  if (c >= 32U || ((allowed_claszes >> c) & 1U) == 0U) return false;
  auto const fl = tt.rt_flags(x);
  for (auto f = 0U; f != 4U; ++f) {
    if (((required_flags >> f) & 1U) == 0U) continue;
    if ((fl >> (2U * f)) & 1U) continue;
    if (((fl >> (2U * f + 1U)) & 1U) == 0U) return false;
    sections = static_cast<uint8_t>(sections | (1U << f));
  }
  return true;
}

// whether the section from stop s to stop s + 1 of route r carries every
// flag in `sections`
bool section_ok(tt_view const& tt, uint32_t r, uint32_t s, uint8_t sections) {
  return (tt.section_flags(r, s) & sections) == sections;
}

// ---------------------------------------------------------------- raptor
// raptor<Dir, false, 0, Mode>, raptor.h:25-1535
struct raptor_t {
  tt_view const& tt;
  bool fwd;
  bool one_to_all;
  uint32_t n_loc, n_routes;
  std::vector<delta_t> tmp, best, rt;  // rt[k * n_loc + l]
  bitvec station_mark, prev_station_mark, route_mark, rt_transport_mark;
  bitvec const& is_dest;
  std::vector<uint16_t> const& dist_to_end;
  std::vector<uint16_t> const& lb;
  bitvec end_reachable;
  std::array<delta_t, kK> time_at_dest{};
  uint16_t base_;
  tts_t tts;
  or_stats& st;
  uint32_t allowed_claszes{B2R_ALL_CLASZ};  // query filters
  uint8_t required_flags{0U};
  // pong's pruning bounds (raptor_state::bounds_storage_, raptor.h:117-172):
  // rows [k][location] folded from another search's round times
  std::vector<delta_t> bounds;
  unsigned bounds_last_k{0U};

  delta_t kInvalid() const { return fwd ? 32767 : -32768; }
  bool is_better(int a, int b) const { return fwd ? a < b : a > b; }
  bool is_better_or_eq(int a, int b) const { return fwd ? a <= b : a >= b; }
  int get_best(int a, int b) const { return is_better(a, b) ? a : b; }
  int dir(int a) const { return fwd ? a : -a; }
  int32_t base_days() const { return tt.internal_from_days() + base_; }

  raptor_t(tt_view const& t, bool f, bool ota, bitvec const& dest,
           std::vector<uint16_t> const& dte, std::vector<uint16_t> const& l,
           uint16_t base, tts_t const& s, or_stats& stats)
      : tt{t},
        fwd{f},
        one_to_all{ota},
        n_loc{t.d.n_locations},
        n_routes{t.d.n_routes},
        is_dest{dest},
        dist_to_end{dte},
        lb{l},
        base_{base},
        tts{s},
        st{stats} {
    tmp.assign(n_loc, kInvalid());
    best.assign(n_loc, kInvalid());
    rt.assign(static_cast<size_t>(kK) * n_loc, kInvalid());
    station_mark.resize(n_loc);
    prev_station_mark.resize(n_loc);
    route_mark.resize(n_routes);
    rt_transport_mark.resize(std::max(1U, t.n_rt()));
    reset_arrivals();
    if (!dist_to_end.empty()) {  // raptor.h:101-112
      end_reachable.resize(n_loc);
      for (auto i = 0U; i != dist_to_end.size(); ++i) {
        if (dist_to_end[i] != kUnreachable) end_reachable.set(i);
      }
    }
  }

  delta_t& RT(int k, uint32_t l) { return rt[static_cast<size_t>(k) * n_loc + l]; }

  void reset_arrivals() {  // raptor.h:174-177
    time_at_dest.fill(kInvalid());
    std::fill(rt.begin(), rt.end(), kInvalid());
  }

  void next_start_time() {  // raptor.h:179-188
    std::fill(best.begin(), best.end(), kInvalid());
    std::fill(tmp.begin(), tmp.end(), kInvalid());
    prev_station_mark.clear();
    station_mark.clear();
    route_mark.clear();
    rt_transport_mark.clear();
  }

  void add_start(uint32_t l, unixtime t) {  // raptor.h:190-203
    best[l] = static_cast<delta_t>(get_best(unix_to_delta(base_days(), t), best[l]));
    RT(0, l) = static_cast<delta_t>(get_best(unix_to_delta(base_days(), t), RT(0, l)));
    station_mark.set(l);
  }

  // fill_bounds, raptor.h:117-170 (no vias, no td footpaths): row 0 is
  // round 0, row k the best of rounds 0..k
  void fill_bounds(size_t n_rows, std::vector<delta_t>& dst) const {
    dst.resize(static_cast<size_t>(kK) * n_loc);
    for (auto x = 0U; x != n_loc; ++x) dst[x] = rt[x];
    for (auto k = size_t{1U}; k < n_rows; ++k) {
      for (auto x = 0U; x != n_loc; ++x) {
        auto const s = rt[k * n_loc + x], d = dst[(k - 1) * n_loc + x];
        dst[k * n_loc + x] = fwd ? std::min(s, d) : std::max(s, d);
      }
    }
  }
  // within_bounds, raptor.h:458-489: the label t at l in round k may not
  // beat the bounding search's row (last_k - k) at l by less than l's
  // transfer time
  bool within_bounds(unsigned k, uint32_t l, int t) const {
    if (bounds_last_k == 0U) return true;
    auto const row = bounds[static_cast<size_t>(bounds_last_k - k) * n_loc + l];
    auto const transfer = dir(adjusted<int>(tts, tt.d.transfer_time[l]));
    return is_better_or_eq(t, row + transfer);
  }

  uint16_t get_lb(uint32_t i) const { return lb[i]; }
  bool lb_reachable(uint32_t i) const { return lb[i] != kUnreachable; }
  bool is_intermodal_dest() const { return !dist_to_end.empty(); }

  void update_time_at_dest(unsigned k, delta_t t) {  // raptor.h:1479-1486
    if (one_to_all) return;
    for (auto i = k; i != time_at_dest.size(); ++i) {
      time_at_dest[i] = static_cast<delta_t>(get_best(time_at_dest[i], t));
    }
  }

  delta_t to_delta(uint16_t day, int mam) const {  // raptor.h:1467-1469
    return clamp16((static_cast<int>(day) - static_cast<int>(base_)) * 1440 + mam);
  }
  // raptor.h:1452-1458 (event_mam(...).count() = days * 1440 + mam)
  delta_t time_at_stop(uint32_t r, uint32_t t, uint16_t day, uint32_t s, bool arr) const {
    auto const ev = tt.event_mam(r, t, s, arr);
    auto const cnt = static_cast<int16_t>(B2R_DELTA_DAYS(ev) * 1440 + B2R_DELTA_MAM(ev));
    return to_delta(day, cnt);
  }

  void execute(unixtime start_time, uint8_t max_transfers,
               unixtime worst_time_at_dest, pareto_t& results) {
    // raptor.h:205-414
    auto const end_k = std::min<unsigned>(max_transfers, kMaxTransfers) + 2U;
    auto const d_worst = unix_to_delta(base_days(), worst_time_at_dest);
    for (auto& t : time_at_dest) t = static_cast<delta_t>(get_best(d_worst, t));

    for (auto k = 1U; k != end_k; ++k) {
      ++st.n_rounds;
      st.n_sweep_locations += n_loc;
      for (auto i = 0U; i != n_loc; ++i) {
        best[i] = static_cast<delta_t>(get_best(RT(k, i), best[i]));
      }
      is_dest.for_each([&](uint32_t i) { update_time_at_dest(k, best[i]); });

      auto any_marked = false;
      station_mark.for_each([&](uint32_t i) {
        ++st.n_marked_stations;
        for (auto ri = tt.d.location_routes_index[i];
             ri != tt.d.location_routes_index[i + 1]; ++ri) {
          ++st.n_location_routes_read;
          any_marked = true;
          route_mark.set(tt.d.location_routes[ri]);
        }
        tt.location_rt(i, [&](uint32_t x) {  // raptor.h:234-240
          any_marked = true;
          rt_transport_mark.set(x);
        });
      });
      if (!any_marked) break;

      std::swap(prev_station_mark, station_mark);
      station_mark.clear();

      route_mark.for_each([&](uint32_t r) {
        uint8_t sections = 0U;
        if (!route_allowed(tt, allowed_claszes, required_flags, r, sections)) return;
        ++st.n_routes_visited;
        any_marked |= update_route(k, r, sections);
      });
      rt_transport_mark.for_each([&](uint32_t x) {  // loop_rt_routes, raptor.h:577-678
        uint8_t sections = 0U;
        if (!rt_allowed(tt, allowed_claszes, required_flags, x, sections)) return;
        ++st.n_routes_visited;
        any_marked |= update_rt_transport(k, x, sections);
      });
      if (!any_marked) break;

      route_mark.clear();
      rt_transport_mark.clear();
      std::swap(prev_station_mark, station_mark);
      station_mark.clear();

      update_transfers(k);
      update_intermodal_footpaths(k);
      update_footpaths(k);
    }

    if (one_to_all) return;

    is_dest.for_each([&](uint32_t i) {  // raptor.h:393-413
      for (auto k = 1U; k != end_k; ++k) {
        auto const dest_time = RT(k, i);
        if (dest_time != kInvalid()) {
          journey_t j;
          j.start_time = start_time;
          j.dest_time = delta_to_unix(base_days(), dest_time);
          j.dest = i;
          j.transfers = static_cast<uint8_t>(k - 1);
          results.add(std::move(j));
        }
      }
    });
  }

  void update_transfers(unsigned k) {  // raptor.h:680-743
    prev_station_mark.for_each([&](uint32_t i) {
      ++st.n_fp_stations;
      auto const tmp_time = tmp[i];
      if (tmp_time == kInvalid()) return;
      auto const dest = is_dest.test(i);
      auto const transfer_time =
          (!is_intermodal_dest() && dest)
              ? 0
              : dir(adjusted<int>(tts, tt.d.transfer_time[i]));
      auto const fp_target_time = clamp16(tmp_time + transfer_time);
      if (bounds_last_k == 0U && is_better(fp_target_time, best[i])) {
        RT(k, i) = static_cast<delta_t>(get_best(fp_target_time, RT(k, i)));
        ++st.n_label_writes;
      }
      if (is_better(fp_target_time, best[i]) &&
          is_better_or_eq(fp_target_time, time_at_dest[k])) {
        if (!lb_reachable(i) ||
            !is_better_or_eq(fp_target_time + dir(get_lb(i)), time_at_dest[k])) {
          return;
        }
        if (!within_bounds(k, i, fp_target_time)) return;
        RT(k, i) = fp_target_time;
        best[i] = fp_target_time;
        st.n_label_writes += 2;
        station_mark.set(i);
        if (dest) update_time_at_dest(k, fp_target_time);
      }
    });
  }

  void update_footpaths(unsigned k) {  // raptor.h:745-845
    prev_station_mark.for_each([&](uint32_t i) {
      auto const* idx = tt.fp_index(fwd);
      auto const* fps = tt.fp_words(fwd);
      for (auto fi = idx[i]; fi != idx[i + 1]; ++fi) {
        ++st.n_footpaths_visited;
        auto const fp = fps[fi];
        auto const target = B2R_FP_TARGET(fp);
        auto const tmp_time = tmp[i];
        if (tmp_time == kInvalid()) continue;
        auto const fp_target_time = clamp16(
            tmp_time + dir(adjusted<int>(tts, static_cast<int>(B2R_FP_DURATION(fp)))));
        if (bounds_last_k == 0U && is_better(fp_target_time, best[target])) {
          RT(k, target) = static_cast<delta_t>(get_best(fp_target_time, RT(k, target)));
          ++st.n_label_writes;
        }
        if (is_better(fp_target_time, best[target]) &&
            is_better_or_eq(fp_target_time, time_at_dest[k])) {
          if (!lb_reachable(target) ||
              !is_better_or_eq(fp_target_time + dir(get_lb(target)),
                               time_at_dest[k])) {
            continue;
          }
          if (!within_bounds(k, target, fp_target_time)) continue;
          RT(k, target) = fp_target_time;
          best[target] = fp_target_time;
          st.n_label_writes += 2;
          station_mark.set(target);
          if (is_dest.test(target)) update_time_at_dest(k, fp_target_time);
        }
      }
    });
  }

  void update_intermodal_footpaths(unsigned k) {  // raptor.h:954-1026
    if (dist_to_end.empty()) return;
    prev_station_mark.for_each([&](uint32_t i) {
      if (!end_reachable.test(i)) return;
      if (dist_to_end[i] != kUnreachable) {
        auto const tmp_time = tmp[i];
        if (tmp_time == kInvalid()) return;
        auto const end_time = clamp16(tmp_time + dir(dist_to_end[i]));
        if (is_better_or_eq(end_time, time_at_dest[k])) {
          RT(k, kEnd) = end_time;
          best[kEnd] = end_time;
          st.n_label_writes += 2;
          update_time_at_dest(k, end_time);
        }
      }
    });
  }

  bool update_route(unsigned k, uint32_t r, uint8_t sections) {  // raptor.h:1177-1349
    auto const n_stops = tt.n_stops(r);
    auto any_marked = false;
    bool et_valid = false;
    uint32_t et_t = 0;
    uint16_t et_day = 0;
    st.n_route_stops_visited += n_stops;

    for (auto i = 0U; i != n_stops; ++i) {
      auto const stop_idx = fwd ? i : n_stops - i - 1U;
      auto const stp = tt.stop(r, stop_idx);
      auto const l = B2R_STOP_LOC(stp);
      auto const is_last = i == n_stops - 1U;
      // stop::can_finish / can_start (stop.h:51-67) with is_wheelchair
      auto const can_finish = fwd ? tt.stop_out(stp) : tt.stop_in(stp);
      auto const can_start = fwd ? tt.stop_in(stp) : tt.stop_out(stp);

      // section filters, raptor.h:1194-1217: the trip carried into this
      // stop is dropped if the section it rode lacks a required flag
      if (sections != 0U && i != 0U &&
          !section_ok(tt, r, fwd ? stop_idx - 1U : stop_idx, sections)) {
        et_valid = false;
      }

      delta_t current_best = kInvalid();
      if (et_valid && can_finish) {
        auto const by_transport = time_at_stop(r, et_t, et_day, stop_idx, fwd);
        current_best = static_cast<delta_t>(
            get_best(get_best(RT(k - 1, l), tmp[l]), best[l]));
        if (is_better_or_eq(by_transport, time_at_dest[k]) && lb_reachable(l) &&
            is_better_or_eq(by_transport + dir(get_lb(l)), time_at_dest[k]) &&
            within_bounds(k, l, by_transport)) {
          tmp[l] = static_cast<delta_t>(get_best(by_transport, tmp[l]));
          ++st.n_label_writes;
          station_mark.set(l);
          if (is_better(by_transport, current_best)) current_best = by_transport;
          any_marked = true;
        }
      }

      if (is_last || !can_start || !prev_station_mark.test(l)) continue;
      if (!lb_reachable(l)) break;

      auto const et_time_at_stop =
          et_valid ? time_at_stop(r, et_t, et_day, stop_idx, !fwd) : kInvalid();
      auto const prev_round_time = RT(k - 1, l);
      if (prev_round_time != kInvalid() &&
          is_better_or_eq(prev_round_time, et_time_at_stop)) {
        auto const [day, mam] = split_day_mam(base_, prev_round_time);
        uint32_t nt = 0;
        uint16_t nd = 0;
        auto const found = get_earliest_transport(k, r, stop_idx, day, mam, l, nt, nd);
        current_best = static_cast<delta_t>(
            get_best(get_best(current_best, best[l]), tmp[l]));
        if (found && (current_best == kInvalid() ||
                      is_better_or_eq(time_at_stop(r, nt, nd, stop_idx, !fwd),
                                      et_time_at_stop))) {
          et_valid = true;
          et_t = nt;
          et_day = nd;
        }
      }
    }
    return any_marked;
  }

  // update_rt_transport, raptor.h:1068-1175 (no vias): et is whether the
  // query rides the run when it passes the stop
  bool update_rt_transport(unsigned k, uint32_t x, uint8_t sections) {
    auto const n_stops = tt.rt_n_stops(x);
    auto any_marked = false;
    auto et = false;
    st.n_route_stops_visited += n_stops;
    for (auto i = 0U; i != n_stops; ++i) {
      auto const stop_idx = fwd ? i : n_stops - i - 1U;
      auto const stp = tt.rt_stop(x, stop_idx);
      auto const l = B2R_STOP_LOC(stp);
      auto const is_last = i == n_stops - 1U;
      if (sections != 0U && i != 0U &&
          (tt.rt_section_flags(x, fwd ? stop_idx - 1U : stop_idx) & sections) != sections) {
        et = false;
      }
      if ((fwd && stop_idx != 0U) || (!fwd && stop_idx != n_stops - 1U)) {
        auto const by_transport = unix_to_delta(base_days(), tt.rt_event(x, stop_idx, fwd));
        if (et && (fwd ? tt.stop_out(stp) : tt.stop_in(stp))) {
          if (is_better_or_eq(by_transport, time_at_dest[k]) && lb_reachable(l) &&
              is_better_or_eq(by_transport + dir(get_lb(l)), time_at_dest[k]) &&
              within_bounds(k, l, by_transport)) {
            tmp[l] = static_cast<delta_t>(get_best(by_transport, tmp[l]));
            ++st.n_label_writes;
            station_mark.set(l);
            any_marked = true;
          }
        }
      }
      if (!lb_reachable(l)) break;
      if (is_last || !(fwd ? tt.stop_in(stp) : tt.stop_out(stp)) || !prev_station_mark.test(l)) continue;
      auto const by_transport = unix_to_delta(base_days(), tt.rt_event(x, stop_idx, !fwd));
      if (is_better_or_eq(RT(k - 1, l), by_transport)) et = true;
    }
    return any_marked;
  }

  // raptor.h:1351-1442
  bool get_earliest_transport(unsigned k, uint32_t r, uint32_t stop_idx,
                              uint16_t day_at_stop, int16_t mam_at_stop,
                              uint32_t l, uint32_t& out_t, uint16_t& out_day) {
    ++st.n_et_calls;
    auto const n = tt.n_t(r);
    auto const* ev = tt.event_times(r, stop_idx, !fwd);
    // linear_lb over the column in search direction, comparing mam only
    auto const at = [&](uint32_t j) { return ev[fwd ? j : n - 1U - j]; };
    auto const seek_first_day = [&]() {
      for (auto j = 0U; j != n; ++j) {
        if (!is_better(B2R_DELTA_MAM(at(j)), mam_at_stop)) return j;
      }
      return n;
    };
    constexpr auto n_days_to_iterate = kMaxTravelTime / 1440 + 1;
    for (auto i = 0U; i != n_days_to_iterate; ++i) {
      auto const day = static_cast<uint16_t>(fwd ? day_at_stop + i : day_at_stop - i);
      ++st.n_et_days;
      if (!tt.route_active(r, day)) continue;
      auto const from = i == 0U ? seek_first_day() : 0U;
      for (auto j = from; j < n; ++j) {
        ++st.n_et_events;
        auto const e = at(j);
        auto const ev_mam = B2R_DELTA_MAM(e);
        if (!is_better_or_eq(to_delta(day, ev_mam) + dir(get_lb(l)), time_at_dest[k])) {
          return false;
        }
        auto const t_offset = fwd ? j : n - 1U - j;
        auto const t = tt.d.route_transport_from[r] + t_offset;
        if (i == 0U && !is_better_or_eq(mam_at_stop, ev_mam)) continue;
        auto const start_day =
            static_cast<uint16_t>(static_cast<int>(day) - B2R_DELTA_DAYS(e));
        if (!tt.transport_active(t, start_day)) continue;
        out_t = t;
        out_day = start_day;
        return true;
      }
    }
    return false;
  }
};

// ------------------------------------------------------------ start labels
struct start_t {
  unixtime time_at_start, time_at_stop;
  uint32_t stop;
  bool operator<(start_t const& o) const {
    return std::tie(time_at_start, time_at_stop, stop) <
           std::tie(o.time_at_start, o.time_at_stop, o.stop);
  }
};

struct interval_t {
  unixtime from, to;
  bool contains(unixtime t) const { return from <= t && t < to; }
  int size() const { return to - from; }
  unixtime clamp(unixtime t) const { return std::clamp(t, from, to); }
  bool operator==(interval_t const& o) const { return from == o.from && to == o.to; }
};

// start_times.cc:40-121
void add_start_times_at_stop(tt_view const& tt, bool fwd, uint32_t r,
                             uint32_t stop_idx, uint32_t l,
                             interval_t const& iv_at_start,
                             interval_t const& iv_at_stop, int16_t offset,
                             std::vector<start_t>& starts) {
  auto const better_eq = [&](int a, int b) { return fwd ? a <= b : a >= b; };
  auto const first_day = tt.day_idx_mam(iv_at_stop.from).first;
  auto const last_day = tt.day_idx_mam(iv_at_stop.to).first;
  for (auto t = tt.d.route_transport_from[r]; t != tt.d.route_transport_to[r]; ++t) {
    auto const ev = tt.event_mam(t, stop_idx, !fwd);
    auto const cnt = static_cast<int16_t>(B2R_DELTA_DAYS(ev) * 1440 + B2R_DELTA_MAM(ev));
    auto const day_offset = static_cast<uint16_t>(cnt / 1440);
    auto const stop_time_mam = cnt % 1440;
    for (auto day = first_day; day <= last_day; ++day) {
      // the overlay's traffic days where it changed them (start_times.cc:64-65)
      if (tt.transport_active(t, static_cast<uint16_t>(day - day_offset)) &&
          iv_at_stop.contains(tt.to_unixtime(day, stop_time_mam))) {
        auto const ev_time = tt.to_unixtime(day, stop_time_mam);
        auto const d = offset;
        if (d == kFpMaxDuration) continue;
        auto const time_at_start = fwd ? ev_time - d : ev_time + d;
        if (!iv_at_start.contains(time_at_start)) continue;
        if (!starts.empty() && starts.back().time_at_start == time_at_start &&
            better_eq(starts.back().time_at_stop, ev_time)) {
          continue;
        }
        starts.push_back({time_at_start, ev_time, l});
      }
      if (day == 0xFFFF) break;
    }
  }
}

// start_times.cc:123-239 (static timetable)
void add_starts_in_interval(tt_view const& tt, bool fwd, interval_t const& iv,
                            uint32_t l, int16_t offset, int16_t max_start_offset,
                            std::vector<start_t>& starts, bool add_ontrip) {
  for (auto ri = tt.d.location_routes_index[l]; ri != tt.d.location_routes_index[l + 1];
       ++ri) {
    auto const r = tt.d.location_routes[ri];
    auto const n = tt.n_stops(r);
    for (auto i = 0U; i != n; ++i) {
      auto const stp = tt.stop(r, i);
      if (B2R_STOP_LOC(stp) != l) continue;
      if ((!fwd && (i == 0U || !tt.stop_out(stp))) ||  // out_allowed(prf_idx)
          (fwd && (i == n - 1U || !tt.stop_in(stp)))) {
        continue;
      }
      add_start_times_at_stop(
          tt, fwd, r, i, l, iv,
          fwd ? interval_t{iv.from, iv.to + max_start_offset}
              : interval_t{iv.from - max_start_offset, iv.to},
          offset, starts);
    }
  }
  // real-time starts, start_times.cc:177-215
  tt.location_rt(l, [&](uint32_t x) {
    auto const n = tt.rt_n_stops(x);
    for (auto i = 0U; i != n; ++i) {
      auto const stp = tt.rt_stop(x, i);
      if (B2R_STOP_LOC(stp) != l) continue;
      if ((!fwd && (i == 0U || !tt.stop_out(stp))) || (fwd && (i == n - 1U || !tt.stop_in(stp)))) continue;
      auto const ev_time = tt.rt_event(x, i, !fwd);
      auto const time_at_start = fwd ? ev_time - offset : ev_time + offset;
      if (!iv.contains(time_at_start)) continue;
      starts.push_back({time_at_start, ev_time, l});
    }
  });
  if (add_ontrip) {
    auto const time_at_start = fwd ? iv.to : iv.from - 1;
    auto const d = offset;
    if (d != kFpMaxDuration) {
      starts.push_back({time_at_start, fwd ? iv.to + d : iv.from - 1 - d, l});
    }
  }
}

struct start_time_v {  // start_time_t variant
  bool is_interval;
  unixtime t;
  interval_t iv;
};

// start_times.cc:241-319
void get_starts(tt_view const& tt, bool fwd, start_time_v const& st,
                query_t const& q, tts_t const& tts, std::vector<start_t>& starts,
                bool add_ontrip) {
  std::vector<std::pair<uint32_t, int16_t>> shortest;  // insertion ordered
  std::unordered_map<uint32_t, size_t> pos;
  auto const update = [&](uint32_t l, int16_t d) {
    auto it = pos.find(l);
    if (it == pos.end()) {
      pos.emplace(l, shortest.size());
      shortest.emplace_back(l, d);
    } else {
      shortest[it->second].second = std::min(shortest[it->second].second, d);
    }
  };
  for (auto const& o : q.start) {
    for_each_meta(tt, q.start_mode, o.target, [&](uint32_t l) {
      update(l, o.duration);
      if (q.use_start_footpaths) {
        auto const* idx = tt.fp_index(fwd);
        auto const* fps = tt.fp_words(fwd);
        for (auto fi = idx[l]; fi != idx[l + 1]; ++fi) {
          update(B2R_FP_TARGET(fps[fi]),
                 static_cast<int16_t>(
                     o.duration + adjusted<int16_t>(
                                      tts, static_cast<int16_t>(B2R_FP_DURATION(fps[fi])))));
        }
      }
    });
  }
  for (auto const& [l, o] : shortest) {
    if (st.is_interval) {
      add_starts_in_interval(tt, fwd, st.iv, l, o, q.max_start_offset, starts,
                             add_ontrip);
    } else {
      starts.push_back({st.t, fwd ? st.t + o : st.t - o, l});
    }
  }
}

// start_times.cc:321-353
void collect_destinations(tt_view const& tt, query_t const& q, bitvec& is_dest,
                          std::vector<uint16_t>& dist_to_dest) {
  is_dest.resize(tt.d.n_locations);
  if (q.dest_mode == B2R_MATCH_INTERMODAL) {
    is_dest.set(kEnd);
    dist_to_dest.assign(tt.d.n_locations, kUnreachable);
  } else {
    dist_to_dest.clear();
  }
  for (auto const& d : q.dest) {
    for_each_meta(tt, q.dest_mode, d.target, [&](uint32_t l) {
      if (q.dest_mode == B2R_MATCH_INTERMODAL) {
        dist_to_dest[l] = std::min(dist_to_dest[l], static_cast<uint16_t>(d.duration));
      } else {
        is_dest.set(l);
      }
    });
  }
}

// dial.h bucket queue
struct dial_t {
  struct label {
    uint32_t l;
    uint16_t d;
  };
  std::vector<std::vector<label>> buckets;
  size_t cur{0}, size{0};
  explicit dial_t(size_t n_buckets) : buckets(n_buckets) {}
  void push(label x) {
    buckets[x.d].push_back(x);
    cur = std::min<size_t>(cur, x.d);
    ++size;
  }
  size_t next() const {
    auto b = cur;
    while (b < buckets.size() && buckets[b].empty()) ++b;
    return b;
  }
  label top() {
    cur = next();
    return buckets[cur].back();
  }
  void pop() {
    cur = next();
    buckets[cur].pop_back();
    --size;
  }
  bool empty() const { return size == 0; }
};

// dijkstra.cc:18-67 + dijkstra.h:31-70
void dijkstra_lb(tt_view const& tt, query_t const& q, bool fwd,
                 std::vector<uint16_t>& dists) {
  dists.assign(tt.d.n_locations, kUnreachable);
  std::map<uint32_t, uint16_t> mn;
  auto const update_min = [&](uint32_t x, int16_t d) {
    auto const l = tt.root(x);
    auto it = mn.find(l);
    if (it == mn.end()) it = mn.emplace(l, dists[l]).first;
    it->second = std::min(static_cast<uint16_t>(d), it->second);
  };
  for (auto const& s : q.dest) {
    for_each_meta(tt, q.dest_mode, s.target, [&](uint32_t x) { update_min(x, s.duration); });
  }
  dial_t pq{kMaxTravelTime + 1};
  for (auto const& [l, d] : mn) {
    for_each_meta(tt, q.dest_mode, l, [&](uint32_t meta) {
      pq.push({meta, d});
      dists[meta] = std::min(d, dists[meta]);
    });
  }
  auto const* gi = tt.lb_index(fwd);
  auto const* gd = tt.lb_words(fwd);
  while (!pq.empty()) {
    auto const l = pq.top();
    pq.pop();
    if (dists[l.l] < l.d) continue;
    for (auto e = gi[l.l]; e != gi[l.l + 1]; ++e) {
      auto const target = B2R_FP_TARGET(gd[e]);
      auto const new_dist = static_cast<uint32_t>(l.d) + B2R_FP_DURATION(gd[e]);
      if (new_dist < dists[target] && new_dist < pq.buckets.size() &&
          new_dist < 65535u) {
        dists[target] = static_cast<uint16_t>(new_dist);
        pq.push({target, static_cast<uint16_t>(new_dist)});
      }
    }
  }
  for (auto i = 0U; i != tt.d.n_locations; ++i) {
    auto const lb = dists[i];
    tt.children(i, [&](uint32_t c) { dists[c] = std::min(lb, dists[c]); });
  }
}

// get_fastest_direct.cc:12-100
int16_t get_fastest_direct(tt_view const& tt, query_t const& q, bool fwd) {
  if (q.has_fastest_direct) return q.fastest_direct;
  constexpr uint32_t max_dist = 65535;
  std::vector<std::pair<uint32_t, uint16_t>> dist_v;
  std::unordered_map<uint32_t, size_t> dpos;
  auto const get_dist = [&](uint32_t l) -> uint16_t& {
    auto it = dpos.find(l);
    if (it == dpos.end()) {
      it = dpos.emplace(l, dist_v.size()).first;
      dist_v.emplace_back(l, static_cast<uint16_t>(32767));
    }
    return dist_v[it->second].second;
  };
  dial_t pq{max_dist};
  for (auto const& s : q.start) {
    for_each_meta(tt, q.start_mode, s.target, [&](uint32_t start) {
      auto& d = get_dist(start);
      d = std::min(static_cast<uint16_t>(s.duration), d);
    });
  }
  for (auto i = 0U; i != dist_v.size(); ++i) pq.push({dist_v[i].first, dist_v[i].second});
  std::unordered_map<uint32_t, uint16_t> dest_offsets;
  for (auto const& o : q.dest) {
    auto const d = static_cast<uint16_t>(o.duration);
    auto it = dest_offsets.find(o.target);
    if (it != dest_offsets.end() && it->second > d) {
      it->second = d;
    } else {
      dest_offsets.emplace(o.target, d);
    }
  }
  constexpr uint16_t kUnreachableDirect = 32767;
  uint16_t end_dist = kUnreachableDirect;
  while (!pq.empty()) {
    auto const l = pq.top();
    pq.pop();
    if (l.l == kEnd) break;
    if (get_dist(l.l) < l.d) continue;
    auto const* idx = tt.fp_index(fwd);
    auto const* fps = tt.fp_words(fwd);
    for (auto fi = idx[l.l]; fi != idx[l.l + 1]; ++fi) {
      auto const new_dist =
          static_cast<uint32_t>(l.d) +
          adjusted<uint16_t>(q.tts, static_cast<uint16_t>(B2R_FP_DURATION(fps[fi])));
      if (new_dist > max_dist) continue;
      auto const target = B2R_FP_TARGET(fps[fi]);
      if (!dest_offsets.contains(target)) continue;
      auto& td = get_dist(target);
      if (new_dist < td && new_dist < pq.buckets.size() && new_dist < max_dist) {
        td = static_cast<uint16_t>(new_dist);
        pq.push({target, static_cast<uint16_t>(new_dist)});
      }
    }
    if (auto it = dest_offsets.find(l.l); it != dest_offsets.end()) {
      auto const new_dist = static_cast<uint32_t>(l.d) + it->second;
      if (new_dist < max_dist && new_dist < end_dist) {
        end_dist = static_cast<uint16_t>(new_dist);
      }
    }
  }
  return end_dist == kUnreachableDirect
             ? kUnreachableDirect
             : static_cast<int16_t>(std::ceil(end_dist * q.fastest_direct_factor));
}

// ------------------------------------------------------- reconstruction
struct reconstructor {
  tt_view const& tt;
  query_t const& q;  // search query (sanitized, normalised tts)
  raptor_t& state;
  journey_t& j;
  bool fwd;
  int32_t base;  // days
  uint16_t base_day_idx;
  bool is_ontrip;

  int dir(int a) const { return fwd ? a : -a; }
  bool better_eq(int a, int b) const { return fwd ? a <= b : a >= b; }
  bool start_matches(int a, int b) const {
    return is_ontrip ? better_eq(a, b) : a == b;
  }
  delta_t rt(unsigned k, uint32_t l) const { return state.rt[k * state.n_loc + l]; }
  bool is_journey_start(uint32_t cand) const {  // reconstruct.cc:22-28
    for (auto const& o : q.start) {
      if (matches(tt, q.start_mode, o.target, cand)) return true;
    }
    return false;
  }
  unixtime stop_time(uint32_t t, uint16_t day, uint32_t s, bool arr) const {
    return tt.event_time(t, day, s, arr);
  }

  // reconstruct.cc:180-280 (Vias = 0: only the first pass runs)
  std::optional<leg_t> find_start_in_prev_round(unsigned k, uint32_t t, uint16_t day,
                                                uint32_t finish, uint8_t sections) {
    auto const r = tt.d.transport_route[t];
    auto const size = tt.n_stops(r);
    auto const n_stops = fwd ? finish + 1U : size - finish;
    for (auto i = 1U; i < n_stops; ++i) {
      auto const stop_idx = fwd ? finish - i : finish + i;
      auto const stp = tt.stop(r, stop_idx);
      auto const l = B2R_STOP_LOC(stp);
      // reconstruct.cc:239-250: a section without a required flag ends the
      // ride (departure section forward, arrival section backward)
      if (sections != 0U &&
          !section_ok(tt, r, fwd ? stop_idx : stop_idx - 1U, sections)) {
        break;
      }
      // reconstruct.cc:252-253 passes the bool is_wheelchair where
      // stop::in_allowed takes a profile index: profile 0 or 1, never the
      // wheelchair profile, so reconstruction reads the plain bits
      if ((fwd && !B2R_STOP_IN(stp)) || (!fwd && !B2R_STOP_OUT(stp))) continue;
      auto const event_time = unix_to_delta(base, stop_time(t, day, stop_idx, !fwd));
      auto const round_time = rt(k - 1, l);
      if (better_eq(round_time, event_time) ||
          (k == 1 && q.start_mode == B2R_MATCH_EQUIVALENT && is_journey_start(l) &&
           start_matches(round_time, event_time))) {
        auto leg = make_leg(fwd, l, B2R_STOP_LOC(tt.stop(r, finish)),
                            delta_to_unix(base, event_time),
                            stop_time(t, day, finish, fwd));
        set_run(leg, t, day, static_cast<uint16_t>(stop_idx),
                static_cast<uint16_t>(finish));
        return leg;
      }
    }
    return std::nullopt;
  }

  // find_start_in_prev_round (reconstruct.cc:186-280) on a real-time run:
  // its own stops and event times (rt::frun::from_rt)
  std::optional<leg_t> find_start_in_prev_round_rt(unsigned k, uint32_t x, uint32_t finish, uint8_t sections) {
    auto const size = tt.rt_n_stops(x);
    auto const n_stops = fwd ? finish + 1U : size - finish;
    for (auto i = 1U; i < n_stops; ++i) {
      auto const stop_idx = fwd ? finish - i : finish + i;
      auto const stp = tt.rt_stop(x, stop_idx);
      auto const l = B2R_STOP_LOC(stp);
      if (sections != 0U &&
          (tt.rt_section_flags(x, fwd ? stop_idx : stop_idx - 1U) & sections) != sections) {
        break;
      }
      if ((fwd && !B2R_STOP_IN(stp)) || (!fwd && !B2R_STOP_OUT(stp))) continue;
      auto const event_time = unix_to_delta(base, tt.rt_event(x, stop_idx, !fwd));
      auto const round_time = rt(k - 1, l);
      if (better_eq(round_time, event_time) ||
          (k == 1 && q.start_mode == B2R_MATCH_EQUIVALENT && is_journey_start(l) &&
           start_matches(round_time, event_time))) {
        auto leg = make_leg(fwd, l, B2R_STOP_LOC(tt.rt_stop(x, finish)), delta_to_unix(base, event_time),
                            tt.rt_event(x, finish, fwd));
        auto const st = tt.rt->d->rt_static_transport;
        set_run(leg, st != nullptr ? st[x] : kInvalidIdx,
                tt.rt->d->rt_static_day != nullptr ? tt.rt->d->rt_static_day[x] : uint16_t{0},
                static_cast<uint16_t>(stop_idx), static_cast<uint16_t>(finish));
        leg.rt_transport = x;
        return leg;
      }
    }
    return std::nullopt;
  }

  // reconstruct.cc:292-373
  std::optional<leg_t> get_route_transport(unsigned k, delta_t time, uint32_t r,
                                           uint32_t stop_idx, uint8_t sections) {
    auto const [day, mam] = split_day_mam(base_day_idx, time);
    for (auto t = tt.d.route_transport_from[r]; t != tt.d.route_transport_to[r]; ++t) {
      auto const ev = tt.event_mam(t, stop_idx, fwd);
      auto const cnt = static_cast<int16_t>(B2R_DELTA_DAYS(ev) * 1440 + B2R_DELTA_MAM(ev));
      if (static_cast<int16_t>(cnt % 1440) != mam) continue;
      auto const traffic_day = static_cast<int>(day) - cnt / 1440;
      auto const tday = static_cast<uint16_t>(traffic_day);
      if (!tt.transport_active(t, tday)) continue;
      auto leg = find_start_in_prev_round(k, t, tday, stop_idx, sections);
      if (leg.has_value()) return leg;
    }
    return std::nullopt;
  }

  // reconstruct.cc:375-545: real-time runs first (381-452; an earlier
  // arrival than the label is accepted), then the routes
  std::optional<leg_t> get_transport(unsigned k, uint32_t l, delta_t time) {
    std::optional<leg_t> found;
    tt.location_rt(l, [&](uint32_t x) {
      if (found.has_value()) return;
      uint8_t sections = 0U;
      if (!rt_allowed(tt, q.allowed_claszes, q.required_flags, x, sections)) return;
      auto const n = tt.rt_n_stops(x);
      for (auto i = 0U; i != n && !found.has_value(); ++i) {
        auto const stp = tt.rt_stop(x, i);
        if (B2R_STOP_LOC(stp) != l || (fwd && (i == 0U || !B2R_STOP_OUT(stp))) ||
            (!fwd && (i == n - 1U || !B2R_STOP_IN(stp))) ||
            !better_eq(tt.rt_event(x, i, fwd), delta_to_unix(base, time))) {
          continue;
        }
        found = find_start_in_prev_round_rt(k, x, i, sections);
      }
    });
    if (found.has_value()) return found;
    for (auto ri = tt.d.location_routes_index[l]; ri != tt.d.location_routes_index[l + 1];
         ++ri) {
      auto const r = tt.d.location_routes[ri];
      uint8_t sections = 0U;
      if (!route_allowed(tt, q.allowed_claszes, q.required_flags, r, sections)) continue;
      auto const n = tt.n_stops(r);
      for (auto i = 0U; i != n; ++i) {
        auto const stp = tt.stop(r, i);
        // plain bits as above (reconstruct.cc:505-509)
        if (B2R_STOP_LOC(stp) != l || (fwd && (i == 0U || !B2R_STOP_OUT(stp))) ||
            (!fwd && (i == n - 1U || !B2R_STOP_IN(stp)))) {
          continue;
        }
        auto leg = get_route_transport(k, time, r, i, sections);
        if (leg.has_value()) return leg;
      }
    }
    return std::nullopt;
  }

  // reconstruct.cc:547-666 (Vias = 0: the adjust_via attempt is a no-op)
  std::optional<std::pair<leg_t, leg_t>> check_fp(unsigned k, uint32_t l,
                                                  delta_t curr_time,
                                                  uint32_t fp_target, int fp_dur_raw,
                                                  bool adjust_transfer_time) {
    auto const fp_duration =
        adjust_transfer_time ? adjusted<int16_t>(q.tts, static_cast<int16_t>(fp_dur_raw))
                             : static_cast<int16_t>(fp_dur_raw);
    auto const fp_start = static_cast<delta_t>(curr_time - dir(fp_duration));
    auto transport_leg = get_transport(k, fp_target, fp_start);
    if (transport_leg.has_value()) {
      auto fp_leg = make_leg(fwd, fp_target, l, delta_to_unix(base, fp_start),
                             delta_to_unix(base, fp_start + dir(fp_duration)));
      set_fp(fp_leg, fp_target, fp_dur_raw);
      return std::pair{fp_leg, *transport_leg};
    }
    return std::nullopt;
  }

  // reconstruct.cc:668-698
  std::optional<std::pair<leg_t, leg_t>> find_dest_leg(unsigned k, uint32_t l,
                                                       offset_t const& dest_offset) {
    if (dest_offset.duration >= kFpMaxDuration) return std::nullopt;
    std::optional<std::pair<leg_t, leg_t>> ret;
    auto const curr_time = rt(k, l);
    for_each_meta(tt, B2R_MATCH_INTERMODAL, dest_offset.target, [&](uint32_t eq) {
      auto res = check_fp(k, l, curr_time, eq, dest_offset.duration, false);
      if (res.has_value()) {
        set_offset(res->first, {eq, dest_offset.duration, dest_offset.mode_id});
        ret = std::move(res);
      }
    });
    return ret;
  }

  // reconstruct.cc:700-790
  std::pair<leg_t, leg_t> get_legs(unsigned k, uint32_t l) {
    auto const curr_time = rt(k, l);
    if (q.dest_mode == B2R_MATCH_INTERMODAL && k == j.transfers + 1U) {
      for (auto const& dest_offset : q.dest) {
        auto ret = find_dest_leg(k, l, dest_offset);
        if (ret.has_value()) return *ret;
      }
      throw std::runtime_error("intermodal destination reconstruction failed");
    }
    auto const same_stop_dur =
        (k == j.transfers + 1U)
            ? 0
            : static_cast<int>(adjusted<uint8_t>(q.tts, tt.d.transfer_time[l]));
    auto transfer = check_fp(k, l, curr_time, l, same_stop_dur, false);
    if (transfer.has_value()) return *transfer;
    auto const* idx = tt.fp_index(!fwd);
    auto const* fps = tt.fp_words(!fwd);
    for (auto fi = idx[l]; fi != idx[l + 1]; ++fi) {
      auto res = check_fp(k, l, curr_time, B2R_FP_TARGET(fps[fi]),
                          static_cast<int>(B2R_FP_DURATION(fps[fi])), true);
      if (res.has_value()) return *res;
    }
    throw std::runtime_error("reconstruction failed");
  }

  // reconstruct.cc:30-160 (Vias = 0)
  std::optional<leg_t> find_start_footpath() {
    auto const& back = j.legs.back();
    auto const leg_start_location = fwd ? back.from : back.to;
    auto const leg_start_time = fwd ? back.dep : back.arr;
    if (q.start_mode != B2R_MATCH_INTERMODAL && is_journey_start(leg_start_location) &&
        better_eq(j.start_time, leg_start_time)) {
      return std::nullopt;
    }
    auto const* idx = tt.fp_index(!fwd);
    auto const* fps = tt.fp_words(!fwd);
    auto const j_start_time = unix_to_delta(base, j.start_time);
    auto const fp_target_time = rt(0, leg_start_location);
    if (q.start_mode == B2R_MATCH_INTERMODAL) {
      for (auto const& o : q.start) {
        if (matches(tt, q.start_mode, o.target, leg_start_location) &&
            better_eq(j.start_time, leg_start_time - dir(o.duration))) {
          auto leg = make_leg(fwd, kStart, leg_start_location,
                              leg_start_time - dir(o.duration), leg_start_time);
          set_offset(leg, o);
          return leg;
        }
      }
    } else {
      for (auto fi = idx[leg_start_location]; fi != idx[leg_start_location + 1]; ++fi) {
        auto const target = B2R_FP_TARGET(fps[fi]);
        auto const fp_duration =
            adjusted<int16_t>(q.tts, static_cast<int16_t>(B2R_FP_DURATION(fps[fi])));
        if (is_journey_start(target) && fp_target_time != state.kInvalid() &&
            start_matches(j_start_time + dir(fp_duration), fp_target_time)) {
          auto leg = make_leg(fwd, target, leg_start_location, j.start_time,
                              delta_to_unix(base, fp_target_time));
          set_fp(leg, target, fp_duration);
          return leg;
        }
      }
    }
    throw std::runtime_error("no valid journey start found");
  }

  void run() {  // reconstruct.cc:792-877
    auto l = j.dest;
    for (auto i = 0U; i <= j.transfers; ++i) {
      auto const k = j.transfers + 1U - i;
      auto [fp_leg, transport_leg] = get_legs(k, l);
      l = fwd ? transport_leg.from : transport_leg.to;
      if (i != 0 || fp_leg.from != fp_leg.to || fp_leg.dep != fp_leg.arr) {
        j.legs.push_back(fp_leg);
      }
      j.legs.push_back(transport_leg);
    }
    auto init_fp = find_start_footpath();
    if (init_fp.has_value()) j.legs.push_back(*init_fp);
    if (fwd) {
      std::reverse(j.legs.begin(), j.legs.end());
    } else {
      for (auto i = 1U; i < j.legs.size(); ++i) {
        auto& it = j.legs[i];
        if (it.kind != B2R_LEG_FOOTPATH) continue;
        auto const diff = it.dep - j.legs[i - 1].arr;
        it.dep -= diff;
        it.arr -= diff;
      }
    }
    auto jq = q;
    if (!fwd) jq.flip_dir();
    optimize_footpaths(jq);
    j.reconstructed = true;
  }

  // ---------------------------------------------- optimize_footpaths.cc
  // the stops and event times of a leg's run (rt::frun: a real-time run's
  // own, else the static trip's)
  unixtime stime(leg_t const& transport_leg, uint32_t s, bool arr) const {
    if (transport_leg.rt_transport != kInvalidIdx) return tt.rt_event(transport_leg.rt_transport, s, arr);
    return tt.event_time(transport_leg.transport, transport_leg.day, s, arr);
  }
  uint32_t sword(leg_t const& transport_leg, uint32_t s) const {
    if (transport_leg.rt_transport != kInvalidIdx) return tt.rt_stop(transport_leg.rt_transport, s);
    return tt.stop(tt.d.transport_route[transport_leg.transport], s);
  }
  uint32_t sloc(leg_t const& transport_leg, uint32_t s) const { return B2R_STOP_LOC(sword(transport_leg, s)); }
  uint32_t run_size(leg_t const& transport_leg) const {
    if (transport_leg.rt_transport != kInvalidIdx) return tt.rt_n_stops(transport_leg.rt_transport);
    return tt.n_stops(tt.d.transport_route[transport_leg.transport]);
  }

  void optimize_initial_departure(query_t const& jq) {  // :15-60
    auto& L = j.legs;
    if (L.size() <= 1 || L[0].kind != B2R_LEG_OFFSET || L[1].kind != B2R_LEG_TRANSPORT) return;
    auto& offset_leg = L[0];
    auto& transport_leg = L[1];
    auto offset_dur_best = offset_leg.duration;
    auto const end = static_cast<uint32_t>(transport_leg.stop_to - 1U);
    for (auto s = 0U; s < end; ++s) {
      if (!B2R_STOP_IN(sword(transport_leg, s))) continue;
      for (auto const& o : jq.start) {
        if (offset_dur_best <= o.duration || o.target != sloc(transport_leg, s)) continue;
        auto const dep = stime(transport_leg, s, false);
        auto const o_start = dep - o.duration;
        if (offset_leg.dep <= o_start) {
          offset_leg.to = sloc(transport_leg, s);
          offset_leg.dep = o_start;
          offset_leg.arr = dep;
          set_offset(offset_leg, o);
          transport_leg.from = sloc(transport_leg, s);
          transport_leg.dep = dep;
          transport_leg.stop_from = static_cast<uint16_t>(s);
          offset_dur_best = o.duration;
        }
      }
    }
  }

  void optimize_initial_start_footpath(query_t const& jq) {  // :62-120
    auto& L = j.legs;
    if (L.size() <= 1 || L[0].kind != B2R_LEG_FOOTPATH || L[1].kind != B2R_LEG_TRANSPORT) {
      return;
    }
    auto& fp_leg = L[0];
    auto& transport_leg = L[1];
    auto const start_loc = fp_leg.from;
    auto fp_dur_best = adjusted<int16_t>(jq.tts, fp_leg.duration);
    auto const end = static_cast<uint32_t>(transport_leg.stop_to - 1U);
    for (auto s = 0U; s < end; ++s) {
      if (!B2R_STOP_IN(sword(transport_leg, s))) continue;
      for (auto fi = tt.fp_index(true)[start_loc];
           fi != tt.fp_index(true)[start_loc + 1]; ++fi) {
        auto const fp = tt.fp_words(true)[fi];
        if (B2R_FP_TARGET(fp) != sloc(transport_leg, s)) continue;
        auto const fp_dur =
            adjusted<int16_t>(jq.tts, static_cast<int16_t>(B2R_FP_DURATION(fp)));
        if (fp_dur < fp_dur_best) {
          auto const dep = stime(transport_leg, s, false);
          auto const fp_start = dep - fp_dur;
          if (fp_leg.dep <= fp_start) {
            fp_leg.to = sloc(transport_leg, s);
            fp_leg.dep = fp_start;
            fp_leg.arr = dep;
            set_fp(fp_leg, sloc(transport_leg, s), fp_dur);
            transport_leg.from = sloc(transport_leg, s);
            transport_leg.dep = dep;
            transport_leg.stop_from = static_cast<uint16_t>(s);
            fp_dur_best = fp_dur;
          }
        }
        break;
      }
    }
  }

  void optimize_last_arrival(query_t const& jq) {  // :122-187
    auto& L = j.legs;
    if (L.size() <= 1 || L.back().kind != B2R_LEG_OFFSET ||
        L[L.size() - 2].kind != B2R_LEG_TRANSPORT) {
      return;
    }
    auto& offset_leg = L.back();
    auto& transport_leg = L[L.size() - 2];
    auto offset_dur_best = offset_leg.duration;
    auto const range_from = static_cast<uint32_t>(transport_leg.stop_from + 1U);
    auto const size = run_size(transport_leg);
    for (auto s = range_from; s < size; ++s) {
      if (!B2R_STOP_OUT(sword(transport_leg, s))) continue;
      for (auto const& o : jq.dest) {
        if (offset_dur_best <= o.duration || o.target != sloc(transport_leg, s)) continue;
        auto const arr = stime(transport_leg, s, true);
        auto const o_end = arr + o.duration;
        if (o_end <= offset_leg.arr) {
          offset_leg.from = sloc(transport_leg, s);
          offset_leg.dep = arr;
          offset_leg.arr = o_end;
          set_offset(offset_leg, o);
          transport_leg.to = sloc(transport_leg, s);
          transport_leg.arr = arr;
          transport_leg.stop_to = static_cast<uint16_t>(s + 1U);
          offset_dur_best = o.duration;
        }
      }
    }
  }

  void optimize_final_egress_footpath(query_t const& jq) {  // :189-257
    auto& L = j.legs;
    if (L.size() <= 1 || L.back().kind != B2R_LEG_FOOTPATH ||
        L[L.size() - 2].kind != B2R_LEG_TRANSPORT) {
      return;
    }
    auto& fp_leg = L.back();
    auto& transport_leg = L[L.size() - 2];
    auto const dest_loc = fp_leg.to;
    auto fp_dur_best = adjusted<int16_t>(jq.tts, fp_leg.duration);
    auto const range_from = static_cast<uint32_t>(transport_leg.stop_from + 1U);
    auto const size = run_size(transport_leg);
    for (auto s = range_from; s < size; ++s) {
      if (!B2R_STOP_OUT(sword(transport_leg, s))) continue;
      for (auto fi = tt.fp_index(false)[dest_loc];
           fi != tt.fp_index(false)[dest_loc + 1]; ++fi) {
        auto const fp = tt.fp_words(false)[fi];
        if (B2R_FP_TARGET(fp) != sloc(transport_leg, s)) continue;
        auto const fp_dur =
            adjusted<int16_t>(jq.tts, static_cast<int16_t>(B2R_FP_DURATION(fp)));
        if (fp_dur < fp_dur_best) {
          auto const arr = stime(transport_leg, s, true);
          auto const fp_end = arr + fp_dur;
          if (fp_end <= fp_leg.arr) {
            fp_leg.from = sloc(transport_leg, s);
            fp_leg.dep = arr;
            fp_leg.arr = fp_end;
            set_fp(fp_leg, dest_loc, fp_dur);
            transport_leg.to = sloc(transport_leg, s);
            transport_leg.arr = arr;
            transport_leg.stop_to = static_cast<uint16_t>(s + 1U);
            fp_dur_best = fp_dur;
          }
        }
        break;
      }
    }
  }

  double get_penalty(int duration, int buffer, uint32_t from, uint32_t to) const {
    // optimize_footpaths.cc:259-283
    auto weight = static_cast<double>(duration);
    if (matches(tt, B2R_MATCH_EQUIVALENT, from, to)) {
      auto const x = tt.root(from);
      auto const imp = tt.d.importance == nullptr ? 0U : tt.d.importance[x];
      weight -= (static_cast<double>(imp) / tt.d.max_importance) * 3U;
    }
    constexpr auto kBufferWeight = 0.2;
    weight -= kBufferWeight * static_cast<double>(std::clamp(buffer, 0, 15));
    return weight;
  }

  void optimize_transfers(query_t const& jq) {  // :285-450 (no vias)
    auto& L = j.legs;
    for (auto i = 0U; i + 2 < L.size(); ++i) {
      auto& leg_from = L[i];
      auto& leg_fp = L[i + 1];
      auto& leg_to = L[i + 2];
      if (leg_from.kind != B2R_LEG_TRANSPORT || leg_fp.kind != B2R_LEG_FOOTPATH ||
          leg_to.kind != B2R_LEG_TRANSPORT) {
        continue;
      }
      auto const from_start = static_cast<uint32_t>(leg_from.stop_from + 1U);
      auto const from_size = run_size(leg_from);
      auto const to_end = static_cast<uint32_t>(leg_to.stop_to - 1U);
      auto penalty_best = get_penalty(leg_fp.duration, leg_to.dep - leg_fp.arr,
                                      leg_from.from, leg_to.to);
      for (auto sf = from_start; sf < from_size; ++sf) {
        if (!B2R_STOP_OUT(sword(leg_from, sf))) continue;
        for (auto stt = 0U; stt < to_end; ++stt) {
          if (!B2R_STOP_IN(sword(leg_to, stt))) continue;
          auto const lf = sloc(leg_from, sf);
          auto const lt = sloc(leg_to, stt);
          for (auto fi = tt.fp_index(true)[lf];
               fi != tt.fp_index(true)[lf + 1]; ++fi) {
            auto const fp = tt.fp_words(true)[fi];
            if (B2R_FP_TARGET(fp) != lt) continue;
            auto const fp_dur =
                adjusted<int16_t>(jq.tts, static_cast<int16_t>(B2R_FP_DURATION(fp)));
            auto const arr = stime(leg_from, sf, true);
            auto const dep = stime(leg_to, stt, false);
            auto const arr_fp = arr + fp_dur;
            if (arr_fp <= dep) {
              auto const penalty = get_penalty(fp_dur, dep - arr_fp, lf, lt);
              if (penalty < penalty_best) {
                leg_from.to = lf;
                leg_from.arr = arr;
                leg_from.stop_to = static_cast<uint16_t>(sf + 1U);
                leg_to.from = lt;
                leg_to.dep = dep;
                leg_to.stop_from = static_cast<uint16_t>(stt);
                leg_fp.from = lf;
                leg_fp.to = lt;
                leg_fp.dep = arr;
                leg_fp.arr = arr_fp;
                set_fp(leg_fp, B2R_FP_TARGET(fp), static_cast<int>(B2R_FP_DURATION(fp)));
                penalty_best = penalty;
              }
            }
            break;
          }
        }
      }
    }
  }

  void optimize_footpaths(query_t const& jq) {  // :452-457
    optimize_initial_departure(jq);
    optimize_initial_start_footpath(jq);
    optimize_last_arrival(jq);
    optimize_final_egress_footpath(jq);
    optimize_transfers(jq);
  }
};

// ----------------------------------------------------------------- search
struct search_result {
  std::vector<journey_t> journeys;
  interval_t interval{0, 0};
  or_stats stats{};
  // final state
  std::vector<delta_t> rt, best;
  int32_t base_day{0};
  uint32_t n_rows{0};
  std::vector<int16_t> ota_rows;
};

// search.h:78-505 for Algo = raptor<Dir, false, 0, kOneToOne>
void run_search(tt_view const& tt, query_t q, bool fwd, search_result& res) {
  q.sanitize();  // raptor_search.cc:57 (raptor_search_with_dir)
  auto& st = res.stats;
  auto const is_ontrip = !q.is_interval;
  interval_t search_interval = q.is_interval ? interval_t{q.iv_from, q.iv_to}
                                             : interval_t{q.start_time, q.start_time};
  // fastest_direct_ is computed before init() normalises the settings
  auto const fastest_direct = get_fastest_direct(tt, q, fwd);
  // init(), search.h:84-172
  auto& tts = q.tts;
  tts.factor = std::max(tts.factor, 1.0F);
  tts.min_transfer_time = std::max<int16_t>(tts.min_transfer_time, 0);
  tts.additional_time = std::max<int16_t>(tts.additional_time, 0);
  tts.default_ = tts.factor == 1.0F && tts.min_transfer_time == 0 &&
                 tts.additional_time == 0;
  bitvec is_dest;
  std::vector<uint16_t> dist_to_dest, lb;
  collect_destinations(tt, q, is_dest, dist_to_dest);
  dijkstra_lb(tt, q, fwd, lb);
  auto const mid = static_cast<int64_t>(search_interval.from) +
                   (search_interval.to - search_interval.from) / 2;
  auto const base_idx =
      static_cast<uint16_t>(round_days(mid) - tt.internal_from_days());
  raptor_t algo{tt, fwd, false, is_dest, dist_to_dest, lb, base_idx, tts, st};
  algo.allowed_claszes = q.allowed_claszes;
  algo.required_flags = q.required_flags;
  q.sanitize();  // search ctor body

  pareto_t results;
  // start_dest_overlap, search.h:354-378
  auto overlap = false;
  if (q.start_mode != B2R_MATCH_INTERMODAL && q.dest_mode != B2R_MATCH_INTERMODAL) {
    for (auto const& o : q.dest) {
      for_each_meta(tt, q.dest_mode, o.target, [&](uint32_t eq) {
        for (auto const& s : q.start) {
          for_each_meta(tt, q.start_mode, s.target, [&](uint32_t x) {
            overlap = overlap || x == eq;
          });
        }
      });
    }
  }
  if (overlap) {
    res.interval = search_interval;
    return;
  }

  // interval_estimator, interval_estimate.h:12-151
  auto const ext_from = tt.external_from(), ext_to = tt.external_to();
  auto const window = q.has_fastest_direct ? 1 : 2;
  constexpr int kMaxSearchIntervalSize = (32767 / 1440 - 7) * 1440;  // limits.h:11-13
  auto const start_itv = search_interval;
  interval_t data_max{
      std::max(round_days(static_cast<int64_t>(start_itv.from) - window * 1440) * 1440,
               round_days(static_cast<int64_t>(start_itv.from) +
                          (start_itv.to - start_itv.from - kMaxSearchIntervalSize) / 2) *
                   1440),
      std::min(round_days(static_cast<int64_t>(start_itv.to) + window * 1440) * 1440,
               round_days(static_cast<int64_t>(start_itv.from) +
                          (start_itv.to - start_itv.from + kMaxSearchIntervalSize) / 2) *
                   1440)};
  auto const clamp_itv = [&](interval_t& itv) {
    itv.from = std::clamp(itv.from, ext_from, ext_to);
    itv.to = std::clamp(itv.to, ext_from, ext_to);
    itv.from = std::clamp(itv.from, data_max.from, data_max.to);
    itv.to = std::clamp(itv.to, data_max.from, data_max.to);
    if (q.has_max_interval) {  // interval_estimate.h:142-145
      itv.from = std::clamp(itv.from, q.max_interval_from, q.max_interval_to);
      itv.to = std::clamp(itv.to, q.max_interval_from, q.max_interval_to);
    }
  };
  auto const can_extend_earlier = [&](interval_t const& itv) {
    return q.extend_earlier && itv.from != ext_from;
  };
  auto const can_extend_later = [&](interval_t const& itv) {
    return q.extend_later && itv.to != ext_to;
  };
  auto const initial = [&](interval_t itv) {
    if (q.min_connection_count == 0 || (!q.extend_earlier && !q.extend_later)) return itv;
    auto new_itv = itv;
    auto const ext = 60 * static_cast<int>(q.min_connection_count);
    auto const bad_dir = fwd ? can_extend_later(itv) : can_extend_earlier(itv);
    if (bad_dir) {
      if (fwd) {
        if (can_extend_earlier(itv)) new_itv.from -= 60;
        else new_itv.to += 60;
        new_itv.to += ext;
      } else {
        if (can_extend_later(itv)) new_itv.to += 60;
        else new_itv.from -= 60;
        new_itv.from -= ext;
      }
    } else {
      if (fwd) {
        if (q.extend_earlier) new_itv.from -= 60 + ext;
      } else {
        if (q.extend_later) new_itv.to += 60 + ext;
      }
    }
    clamp_itv(new_itv);
    return new_itv;
  };
  auto const extension = [&](interval_t const& itv, uint32_t num_con_req) {
    if (num_con_req == 0 || (!q.extend_earlier && !q.extend_later)) return itv;
    auto new_itv = itv;
    auto const ext = itv.size() * static_cast<int>(num_con_req);
    if (can_extend_earlier(itv) && can_extend_later(itv)) {
      new_itv.from -= ext / 2;
      new_itv.to += ext / 2;
    } else {
      if (q.extend_earlier) new_itv.from -= ext;
      if (q.extend_later) new_itv.to += ext;
    }
    clamp_itv(new_itv);
    return new_itv;
  };

  std::vector<start_t> starts;
  auto const add_start_labels = [&](start_time_v const& sv, bool add_ontrip) {
    get_starts(tt, fwd, sv, q, tts, starts, add_ontrip);
    std::sort(starts.begin(), starts.end(), [&](start_t const& a, start_t const& b) {
      return fwd ? b < a : a < b;
    });
  };
  auto const n_results_in_interval = [&]() {
    if (q.is_interval) {
      auto c = 0U;
      for (auto const& j : results.els) c += search_interval.contains(j.start_time) ? 1U : 0U;
      return c;
    }
    return static_cast<unsigned>(results.els.size());
  };

  if (!is_ontrip) search_interval = initial(search_interval);
  starts.clear();
  if (search_interval.size() != 0) {
    add_start_labels({true, 0, search_interval}, true);
  } else {
    add_start_labels({q.is_interval, q.start_time, {q.iv_from, q.iv_to}}, true);
  }

  auto const search_interval_fn = [&]() {  // search.h:419-494
    auto early_termination = false;
    for (size_t from = 0; from < starts.size();) {
      auto to = from + 1;
      while (to < starts.size() && starts[to].time_at_start == starts[from].time_at_start) ++to;
      if (early_termination) {
        from = to;
        continue;
      }
      ++st.n_start_times;
      algo.next_start_time();
      auto const start_time = starts[from].time_at_start;
      for (auto i = from; i != to; ++i) algo.add_start(starts[i].stop, starts[i].time_at_stop);
      auto const worst_time_at_dest =
          start_time + (fwd ? 1 : -1) *
                           (std::min<int>(fastest_direct, q.max_travel_time) + 1);
      algo.execute(start_time, q.max_transfers, worst_time_at_dest, results);
      for (auto& j : results.els) {
        if (!j.reconstructed && !j.error &&
            (is_ontrip || search_interval.contains(j.start_time)) &&
            j.travel_time() < fastest_direct) {
          try {
            reconstructor rc{tt, q, algo, j, fwd, algo.base_days(), base_idx, is_ontrip};
            rc.run();
          } catch (std::exception const&) {
            j.error = true;
          }
        }
      }
      if (q.min_connection_count > 0 && n_results_in_interval() >= q.min_connection_count &&
          ((fwd && q.extend_earlier && !q.extend_later) ||
           (!fwd && !q.extend_earlier && q.extend_later))) {
        early_termination = true;
        if (fwd) search_interval.from = start_time;
        else search_interval.to = start_time + 1;
      }
      from = to;
    }
  };

  while (true) {
    search_interval_fn();
    if (results.els.empty() || is_ontrip ||
        n_results_in_interval() >= q.min_connection_count) {
      break;
    }
    starts.clear();
    auto const new_interval =
        extension(search_interval, q.min_connection_count - n_results_in_interval());
    if (new_interval == search_interval) break;
    if (new_interval.from != search_interval.from) {
      add_start_labels({true, 0, {new_interval.from, search_interval.from}}, !fwd);
      if (!fwd) {
        algo.reset_arrivals();
        std::erase_if(results.els, [&](journey_t const& j) {
          return !search_interval.contains(j.start_time);
        });
      }
    }
    if (new_interval.to != search_interval.to) {
      add_start_labels({true, 0, {search_interval.to, new_interval.to}}, fwd);
      if (fwd) {
        algo.reset_arrivals();
        std::erase_if(results.els, [&](journey_t const& j) {
          return !search_interval.contains(j.start_time);
        });
      }
    }
    search_interval = new_interval;
  }

  if (!is_ontrip) {
    std::erase_if(results.els, [&](journey_t const& j) {
      return !search_interval.contains(j.start_time) || j.travel_time() >= fastest_direct ||
             j.travel_time() > q.max_travel_time;
    });
    std::sort(results.els.begin(), results.els.end(),
              [](journey_t const& a, journey_t const& b) {
                return std::tie(a.start_time, a.transfers) < std::tie(b.start_time, b.transfers);
              });
  }
  std::erase_if(results.els, [](journey_t const& j) { return !j.reconstructed; });
  res.journeys = std::move(results.els);
  res.interval = search_interval;
  res.rt = algo.rt;
  res.best = algo.best;
  res.base_day = algo.base_days();
}

// one_to_all.cc:18-104
void run_one_to_all(tt_view const& tt, query_t const& q, bool fwd, search_result& res) {
  auto& st = res.stats;
  bitvec is_dest;
  is_dest.resize(tt.d.n_locations);
  std::vector<uint16_t> dist_to_dest;
  std::vector<uint16_t> lb(tt.d.n_locations, 0U);
  auto const base = static_cast<uint16_t>(round_days(q.start_time) - tt.internal_from_days());
  raptor_t r{tt, fwd, true, is_dest, dist_to_dest, lb, base, q.tts, st};
  r.allowed_claszes = q.allowed_claszes;
  r.required_flags = q.required_flags;
  pareto_t results;
  r.next_start_time();
  ++st.n_start_times;
  for (auto const& s : q.start) {
    auto const t = fwd ? q.start_time + s.duration : q.start_time - s.duration;
    for_each_meta(tt, q.start_mode, s.target, [&](uint32_t l) { r.add_start(l, t); });
  }
  auto const worst = q.start_time + (fwd ? 1 : -1) * q.max_travel_time;
  r.execute(q.start_time, q.max_transfers, worst, results);
  res.rt = r.rt;
  res.best = r.best;
  res.base_day = r.base_days();
}

// ------------------------------------------------------------------- pong
// lookup_footpath, direct.cc:65-160, for the exact-match offsets of an
// alternative query (no td footpaths, profile 0): the shortest way from an
// offset's location to `loc` (boarding) or from `loc` to it (alighting),
// either the reflexive transfer time or a footpath.
std::optional<leg_t> lookup_footpath(tt_view const& tt, query_t const& q, uint32_t loc,
                                     unixtime t, bool boarding) {
  auto const& offs = boarding ? q.start : q.dest;
  auto const use_footpaths = boarding ? q.use_start_footpaths : true;
  int best_dur = kFpMaxDuration;
  uint32_t best_source = 0U;
  for (auto const& o : offs) {
    auto const l = o.target;  // for_each_meta of kExact
    if (l == loc && o.duration < best_dur) {
      best_dur = o.duration + adjusted<uint8_t>(q.tts, tt.d.transfer_time[l]);
      best_source = o.target;
    }
    if (!use_footpaths) continue;
    auto eff = kFpMaxDuration;
    auto const* idx = tt.fp_index(boarding);
    auto const* fps = tt.fp_words(boarding);
    for (auto fi = idx[l]; fi != idx[l + 1]; ++fi) {
      if (B2R_FP_TARGET(fps[fi]) != loc) continue;
      auto const adj =
          adjusted<int16_t>(q.tts, static_cast<int16_t>(B2R_FP_DURATION(fps[fi])));
      if (adj < eff) eff = adj;
    }
    if (eff >= kFpMaxDuration) continue;
    auto const total = o.duration + eff;
    if (total < best_dur) {
      best_dur = total;
      best_source = o.target;
    }
  }
  if (best_dur >= kFpMaxDuration) return std::nullopt;
  leg_t l;
  l.from = boarding ? best_source : loc;
  l.to = boarding ? loc : best_source;
  l.dep = boarding ? t - best_dur : t;
  l.arr = boarding ? t : t + best_dur;
  set_fp(l, l.to, best_dur);
  return l;
}

// The first journey get_direct_journeys<kForward> (direct.cc:454-605)
// yields for an exact-match one-to-one query departing at `time` or later:
// per (route, boarding stop, alighting stop) the first departure route_gen
// (direct.cc:281-376) accepts, merged by arrival time in a binary heap as
// the reference's priority queue does.  Returns walk, transit, walk.
std::optional<std::array<leg_t, 3>> first_direct_journey(tt_view const& tt, query_t const& q,
                                                         unixtime time) {
  auto const from = q.start.front().target, to = q.dest.front().target;
  std::vector<uint32_t> boarding{from}, alighting{to};
  for (auto fi = tt.fp_index(true)[from]; fi != tt.fp_index(true)[from + 1]; ++fi) {
    boarding.push_back(B2R_FP_TARGET(tt.fp_words(true)[fi]));
  }
  for (auto fi = tt.fp_index(false)[to]; fi != tt.fp_index(false)[to + 1]; ++fi) {
    alighting.push_back(B2R_FP_TARGET(tt.fp_words(false)[fi]));
  }
  auto const has = [](std::vector<uint32_t> const& v, uint32_t x) {
    return std::find(v.begin(), v.end(), x) != v.end();
  };
  auto const routes_of = [&](std::vector<uint32_t> const& locs) {
    std::vector<uint32_t> rs;
    for (auto const l : locs) {
      for (auto ri = tt.d.location_routes_index[l]; ri != tt.d.location_routes_index[l + 1]; ++ri) {
        rs.push_back(tt.d.location_routes[ri]);
      }
    }
    std::sort(rs.begin(), rs.end());
    rs.erase(std::unique(rs.begin(), rs.end()), rs.end());
    return rs;
  };
  auto const from_routes = routes_of(boarding), to_routes = routes_of(alighting);
  std::vector<uint32_t> both;
  std::set_intersection(from_routes.begin(), from_routes.end(), to_routes.begin(),
                        to_routes.end(), std::back_inserter(both));

  auto const day_hi = tt.d.date_range_to + 1 - tt.internal_from_days();
  std::vector<std::array<leg_t, 3>> heads;
  for (auto const r : both) {
    // route filters of direct.cc:503-513: class, flag on some or all sections
    if (((q.allowed_claszes >> tt.clasz(r)) & 1U) == 0U) continue;
    auto const fl = tt.flags(r);
    auto skip = false;
    for (auto f = 0U; f != 4U; ++f) {
      if (((q.required_flags >> f) & 1U) != 0U && ((fl >> (2U * f)) & 3U) == 0U) skip = true;
    }
    if (skip) continue;
    // run_stop::is_flag_set(f, kDep) of section s (rt/frun.cc:453-475)
    auto const flag_set = [&](uint32_t f, uint32_t s) {
      if ((fl >> (2U * f)) & 1U) return true;
      if (((fl >> (2U * f + 1U)) & 1U) == 0U) return false;
      return ((tt.section_flags(r, s) >> f) & 1U) != 0U;
    };
    auto const n = tt.n_stops(r);
    // for_each_pair, direct.cc:429-450
    std::optional<uint32_t> board;
    for (auto i = 0U; i != n; ++i) {
      auto const stp = tt.stop(r, i);
      auto const loc = B2R_STOP_LOC(stp);
      if (board.has_value()) {
        if (!has(alighting, loc) || !tt.stop_out(stp)) continue;  // out_allowed(prf_idx)
        auto const a = *board, b = i;
        board.reset();
        // sections_violate_constraints, direct.cc:242-260
        auto violates = false;
        for (auto s = a; s != b && !violates; ++s) {
          for (auto f = 0U; f != 4U; ++f) {
            if (((q.required_flags >> f) & 1U) != 0U && !flag_set(f, s)) violates = true;
          }
        }
        if (violates) continue;
        // route_gen<kForward>: days from time's day on, transports in order
        auto const boarding_loc = B2R_STOP_LOC(tt.stop(r, a));
        auto const alighting_loc = B2R_STOP_LOC(tt.stop(r, b));
        auto const* ev = tt.event_times(r, a, false);
        auto const n_t = tt.n_t(r);
        auto found = false;
        for (auto day = (time - tt.internal_from()) / 1440; !found && day <= day_hi; ++day) {
          if (!tt.route_active(r, static_cast<uint16_t>(day))) continue;
          for (auto x = 0U; x != n_t; ++x) {
            auto const day_off = day - static_cast<int>(B2R_DELTA_DAYS(ev[x]));
            if (day_off < 0 || day_off >= B2R_MAX_DAYS) continue;
            auto const t = tt.d.route_transport_from[r] + x;
            auto const sd = static_cast<uint16_t>(day_off);
            if (!tt.transport_active(t, sd)) continue;
            auto const bt = tt.event_time(t, sd, a, false), at = tt.event_time(t, sd, b, true);
            auto const bw = lookup_footpath(tt, q, boarding_loc, bt, true);
            auto const aw = lookup_footpath(tt, q, alighting_loc, at, false);
            if (!bw.has_value() || !aw.has_value() || bw->dep < time) continue;
            leg_t transit = make_leg(true, boarding_loc, alighting_loc, bt, at);
            set_run(transit, t, sd, static_cast<uint16_t>(a), static_cast<uint16_t>(b));
            heads.push_back({*bw, transit, *aw});
            found = true;
            break;
          }
        }
      } else if (has(boarding, loc) && tt.stop_in(stp)) {
        board = i;
      }
    }
  }
  if (heads.empty()) return std::nullopt;
  auto const cmp = [&](size_t a, size_t b) { return heads[a][2].arr > heads[b][2].arr; };
  std::priority_queue<size_t, std::vector<size_t>, decltype(cmp)> heap{cmp};
  for (auto i = size_t{0}; i != heads.size(); ++i) heap.push(i);
  return heads[heap.top()];
}

// get_earliest_alternative, pong.cc:35-61: the earliest direct journey from
// `from` (reached at from_arr) to `to` that arrives by to_dep, its walk
// moved to start at from_arr.
std::optional<std::array<leg_t, 3>> get_earliest_alternative(tt_view const& tt,
                                                             query_t const& q, uint32_t from,
                                                             uint32_t to, unixtime from_arr,
                                                             unixtime to_dep) {
  query_t dq;  // make_alternative_query, leg_alternatives.cc:27-45
  dq.start_mode = B2R_MATCH_EXACT;
  dq.dest_mode = B2R_MATCH_EXACT;
  dq.use_start_footpaths = true;
  dq.start = {{from, 0, 0}};
  dq.dest = {{to, 0, 0}};
  dq.allowed_claszes = q.allowed_claszes;
  dq.required_flags = q.required_flags;
  dq.tts = q.tts;
  auto legs = first_direct_journey(tt, dq, from_arr);
  if (!legs.has_value() || (*legs)[2].arr > to_dep) return std::nullopt;
  auto const walk = (*legs)[0].arr - (*legs)[0].dep;
  (*legs)[0].dep = from_arr;
  (*legs)[0].arr = from_arr + walk;
  return legs;
}

// pong.cc:63-475 for Rt = false, Vias = 0, no td offsets: a ping search from
// the current start time, then for each of its results (most transfers
// first) a pong search back from its arrival, bounded by the ping's round
// times, that finds the latest departure; the sweep continues one minute
// after the earliest such departure.
void run_pong(tt_view const& tt, query_t q, bool fwd, search_result& res) {
  auto& st = res.stats;
  q.sanitize();
  auto const fastest_direct = get_fastest_direct(tt, q, fwd);
  auto const search_interval = q.is_interval ? interval_t{q.iv_from, q.iv_to}
                                             : interval_t{q.start_time, q.start_time};
  auto const mid = static_cast<int64_t>(search_interval.from) +
                   (search_interval.to - search_interval.from) / 2;
  auto const base_idx = static_cast<uint16_t>(round_days(mid) - tt.internal_from_days());

  bitvec ping_is_dest;
  std::vector<uint16_t> ping_dist, ping_lb;
  collect_destinations(tt, q, ping_is_dest, ping_dist);
  dijkstra_lb(tt, q, fwd, ping_lb);
  raptor_t ping{tt, fwd, false, ping_is_dest, ping_dist, ping_lb, base_idx, q.tts, st};
  ping.allowed_claszes = q.allowed_claszes;
  ping.required_flags = q.required_flags;

  auto qf = q;
  qf.flip_dir();
  bitvec pong_is_dest;
  std::vector<uint16_t> pong_dist;
  collect_destinations(tt, qf, pong_is_dest, pong_dist);
  std::vector<uint16_t> const pong_lb(tt.d.n_locations, 0U);  // kPruneWithPingBounds
  raptor_t pong{tt, !fwd, false, pong_is_dest, pong_dist, pong_lb, base_idx, q.tts, st};
  pong.allowed_claszes = q.allowed_claszes;
  pong.required_flags = q.required_flags;
  // the pong's start labels walk only for station starts (pong.cc:291-295)
  qf.use_start_footpaths = qf.start_mode != B2R_MATCH_INTERMODAL;

  pareto_t results;
  std::vector<start_t> starts;
  auto start_time = fwd ? search_interval.from : search_interval.to - 1;
  auto const end_time = fwd ? search_interval.to : search_interval.from - 1;
  auto const is_better = [&](int a, int b) { return fwd ? a < b : a > b; };
  auto const is_validated = [&](journey_t const& j) { return is_better(j.dest_time, start_time); };
  auto const result_count = [&](bool include_too_slow) {
    auto c = 0U;
    for (auto const& j : results.els) {
      c += (is_validated(j) && (include_too_slow || (j.travel_time() < fastest_direct &&
                                                     j.travel_time() <= q.max_travel_time)))
               ? 1U
               : 0U;
    }
    return c;
  };
  auto const ext_from = tt.external_from(), ext_to = tt.external_to();
  while ((is_better(start_time, end_time) ||
          result_count(true) + result_count(false) < 2U * q.min_connection_count) &&
         ext_from <= start_time && start_time < ext_to) {
    // ping
    starts.clear();
    get_starts(tt, fwd, {false, start_time, {}}, q, q.tts, starts, false);
    ping.reset_arrivals();
    ping.next_start_time();
    ++st.n_start_times;
    for (auto const& s : starts) ping.add_start(s.stop, s.time_at_stop);
    auto const worst_time_at_dest =
        start_time + (fwd ? 1 : -1) * std::min(q.max_travel_time + 1440, int{kMaxTravelTime});
    pareto_t ping_results;
    ping.execute(start_time, q.max_transfers, worst_time_at_dest, ping_results);
    if (ping_results.els.empty()) break;
    std::erase_if(ping_results.els,
                  [&](journey_t const& x) { return results.is_dominated(x); });
    if (ping_results.els.empty()) break;
    std::sort(ping_results.els.begin(), ping_results.els.end(),
              [](journey_t const& a, journey_t const& b) { return a.transfers > b.transfers; });

    // pongs
    ping.fill_bounds(ping_results.els.front().transfers + size_t{1U}, pong.bounds);
    pong.reset_arrivals();
    for (auto& ping_j : ping_results.els) {
      pong.bounds_last_k = ping_j.transfers + 1U;
      starts.clear();
      get_starts(tt, !fwd, {false, ping_j.dest_time, {}}, qf, q.tts, starts, false);
      pong.next_start_time();
      ++st.n_start_times;
      for (auto const& s : starts) pong.add_start(s.stop, s.time_at_stop);
      pong.execute(ping_j.dest_time, ping_j.transfers, ping_j.start_time, results);
      auto const match = std::find_if(results.els.begin(), results.els.end(), [&](journey_t const& p) {
        return p.transfers == ping_j.transfers && p.start_time == ping_j.dest_time;
      });
      if (match == results.els.end()) throw std::runtime_error{"no pong"};
      if (!match->reconstructed && !match->error) {
        reconstructor rc{tt, qf, pong, *match, !fwd, pong.base_days(), base_idx, !q.is_interval};
        rc.run();
      }
      ping_j.start_time = match->dest_time;
    }

    // next start time
    auto const first_it = std::min_element(
        ping_results.els.begin(), ping_results.els.end(),
        [&](journey_t const& a, journey_t const& b) { return is_better(a.start_time, b.start_time); });
    auto const next = first_it->start_time + (fwd ? 1 : -1);
    if (!is_better(start_time, next)) throw std::runtime_error{"no pong progress"};
    start_time = next;
  }

  std::erase_if(results.els, [&](journey_t const& j) {
    auto const j_start = j.dest_time;
    auto const out_of_interval =
        fwd ? !q.extend_later && j_start >= search_interval.to
            : !q.extend_earlier && j_start < search_interval.from;
    return !j.reconstructed || !is_validated(j) || out_of_interval ||
           j.travel_time() >= fastest_direct || j.travel_time() > q.max_travel_time;
  });
  for (auto& j : results.els) std::swap(j.start_time, j.dest_time);
  res.interval = {fwd ? search_interval.from : start_time + 1,
                  fwd ? start_time : search_interval.to};
  for (auto& j : results.els) {
    auto const swap = [](uint32_t l) { return l == kStart ? kEnd : l == kEnd ? kStart : l; };
    j.legs.front().from = swap(j.legs.front().from);
    j.legs.back().to = swap(j.legs.back().to);
  }
  std::sort(results.els.begin(), results.els.end(), [](journey_t const& a, journey_t const& b) {
    return std::tie(a.start_time, a.transfers) < std::tie(b.start_time, b.transfers);
  });
  if (fwd) {  // pong.cc:433-472: earlier alternatives for inner rides
    for (auto& j : results.els) {
      for (auto w = size_t{0}; w + 5U <= j.legs.size(); ++w) {
        auto& l = j.legs;
        if (l[w].kind != B2R_LEG_TRANSPORT || l[w + 2].kind != B2R_LEG_TRANSPORT ||
            l[w + 4].kind != B2R_LEG_TRANSPORT) {
          continue;
        }
        auto const& front = l[w];
        auto const from_stop = static_cast<uint32_t>(front.stop_to - 1U);
        auto const from = B2R_STOP_LOC(tt.stop(tt.d.transport_route[front.transport], from_stop));
        auto const arr_time = tt.event_time(front.transport, front.day, from_stop, true);
        auto const& back = l[w + 4];
        auto const to = B2R_STOP_LOC(tt.stop(tt.d.transport_route[back.transport], back.stop_from));
        auto const dep_time = tt.event_time(back.transport, back.day, back.stop_from, false);
        auto const earlier = get_earliest_alternative(tt, q, from, to, arr_time, dep_time);
        if (earlier.has_value()) {
          l[w + 1] = (*earlier)[0];
          l[w + 2] = (*earlier)[1];
          l[w + 3] = (*earlier)[2];
        }
      }
    }
  }
  res.journeys = std::move(results.els);
  res.rt = pong.rt;
  res.best = pong.best;
  res.base_day = pong.base_days();
}

uint64_t byte_model(or_stats const& s) {
  // algorithmic bytes of the hot path (bytes the reference loop must touch):
  //  route phase: 4 B stop word + 2 B previous-round label + 2 B event per
  //  visited route stop; earliest-trip: 2 B per examined event + 8 B per
  //  examined day (bitfield word); label writes 2 B; marking 4 B per
  //  location_routes entry; footpath phase 2 B tmp + 1 B transfer time per
  //  station and 4 B + 2 B per footpath; sweep 4 B per location and round.
  return s.n_route_stops_visited * 8ull + s.n_et_events * 2ull + s.n_et_days * 8ull +
         s.n_label_writes * 2ull + s.n_location_routes_read * 4ull +
         s.n_fp_stations * 3ull + s.n_footpaths_visited * 6ull +
         s.n_sweep_locations * 4ull;
}

}  // namespace oracle

// ===================================================================== C ABI
struct or_result {
  oracle::search_result r;
  std::vector<b2r_journey> journeys;
  std::vector<b2r_leg> legs;
};

namespace {
thread_local std::string g_error;  // what the last failed or_search threw
}  // namespace

extern "C" {

int or_search(const b2r_timetable_desc* tt, const b2r_query* q, or_result** out) {
  return or_search_rt(tt, nullptr, q, out);
}

int or_search_rt(const b2r_timetable_desc* tt, const b2r_rt_desc* rtd, const b2r_query* q, or_result** out) {
  if (tt == nullptr || q == nullptr || out == nullptr) return B2R_ERR_INVALID_ARGUMENT;
  if (q->prf_idx >= B2R_N_PROFILES) return B2R_ERR_INVALID_ARGUMENT;  // profile_idx_t < kNProfiles
  try {
    auto res = std::make_unique<or_result>();
    oracle::rt_overlay const ov{rtd, tt->n_locations};
    oracle::tt_view const v{*tt, q->prf_idx, rtd != nullptr ? &ov : nullptr};
    auto const qq = oracle::to_query(*q);
    auto const fwd = q->direction == B2R_FORWARD;
    if (q->kind == B2R_ONE_TO_ALL) {
      oracle::run_one_to_all(v, qq, fwd, res->r);
      auto const end_k = std::min<unsigned>(q->max_transfers, B2R_MAX_TRANSFERS) + 2U;
      res->r.n_rows = end_k;
      res->r.ota_rows.assign(res->r.rt.begin(),
                             res->r.rt.begin() + static_cast<size_t>(end_k) * tt->n_locations);
    } else if (qq.pong) {
      oracle::run_pong(v, qq, fwd, res->r);
    } else {
      oracle::run_search(v, qq, fwd, res->r);
    }
    for (auto const& j : res->r.journeys) {
      b2r_journey bj{};
      bj.start_time = j.start_time;
      bj.dest_time = j.dest_time;
      bj.dest = j.dest;
      bj.transfers = j.transfers;
      bj.error = j.error ? 1 : 0;
      bj.n_legs = static_cast<uint16_t>(j.legs.size());
      bj.first_leg = static_cast<uint32_t>(res->legs.size());
      for (auto const& l : j.legs) {
        b2r_leg bl{};
        bl.from = l.from;
        bl.to = l.to;
        bl.dep_time = l.dep;
        bl.arr_time = l.arr;
        bl.kind = l.kind;
        bl.rt_transport = B2R_INVALID_IDX;
        if (l.kind == B2R_LEG_TRANSPORT) {
          bl.transport = l.transport;
          bl.day = l.day;
          bl.stop_from = l.stop_from;
          bl.stop_to = l.stop_to;
          bl.rt_transport = l.rt_transport;
        } else {
          bl.transport = l.target;
          bl.duration = l.duration;
          bl.transport_mode_id = l.kind == B2R_LEG_OFFSET ? l.mode_id : 0;
        }
        res->legs.push_back(bl);
      }
      res->journeys.push_back(bj);
    }
    res->r.stats.algorithmic_bytes = oracle::byte_model(res->r.stats);
    *out = res.release();
    return B2R_OK;
  } catch (std::exception const& ex) {
    g_error = ex.what();
    return B2R_ERR_INTERNAL;
  }
}

const char* or_last_error(void) { return g_error.c_str(); }

int or_result_view(const or_result* r, b2r_result* view, or_stats* stats) {
  if (r == nullptr) return B2R_ERR_INVALID_ARGUMENT;
  if (view != nullptr) {
    std::memset(view, 0, sizeof(*view));
    view->status = B2R_OK;
    view->n_journeys = static_cast<uint32_t>(r->journeys.size());
    view->journeys = r->journeys.data();
    view->legs = r->legs.data();
    view->interval_from = r->r.interval.from;
    view->interval_to = r->r.interval.to;
    view->n_rows = r->r.n_rows;
    view->base_day = r->r.base_day;
    view->round_times = r->r.ota_rows.empty() ? nullptr : r->r.ota_rows.data();
    view->n_rounds = r->r.stats.n_rounds;
    view->n_start_times = r->r.stats.n_start_times;
  }
  if (stats != nullptr) *stats = r->r.stats;
  return B2R_OK;
}

int or_result_state(const or_result* r, const int16_t** round_times,
                    const int16_t** best, int32_t* base_day) {
  if (r == nullptr) return B2R_ERR_INVALID_ARGUMENT;
  *round_times = r->r.rt.data();
  *best = r->r.best.data();
  *base_day = r->r.base_day;
  return B2R_OK;
}

void or_result_free(or_result* r) { delete r; }

// get_earliest_alternative (pong.cc:35-61) with the filters and transfer
// time settings of q: 1 and three legs if found, 0 if not.
int or_earliest_alternative(const b2r_timetable_desc* tt, const b2r_query* q, uint32_t from,
                            uint32_t to, int32_t from_arr, int32_t to_dep, b2r_leg* legs) {
  if (tt == nullptr || q == nullptr || legs == nullptr) return B2R_ERR_INVALID_ARGUMENT;
  try {
    oracle::tt_view const v{*tt, q->prf_idx};
    auto const qq = oracle::to_query(*q);
    auto const r = oracle::get_earliest_alternative(v, qq, from, to, from_arr, to_dep);
    if (!r.has_value()) return 0;
    for (auto i = 0U; i != 3U; ++i) {
      auto const& l = (*r)[i];
      b2r_leg bl{};
      bl.from = l.from;
      bl.to = l.to;
      bl.dep_time = l.dep;
      bl.arr_time = l.arr;
      bl.kind = l.kind;
      bl.rt_transport = B2R_INVALID_IDX;
      if (l.kind == B2R_LEG_TRANSPORT) {
        bl.transport = l.transport;
        bl.day = l.day;
        bl.stop_from = l.stop_from;
        bl.stop_to = l.stop_to;
      } else {
        bl.transport = l.target;
        bl.duration = l.duration;
      }
      legs[i] = bl;
    }
    return 1;
  } catch (std::exception const&) {
    return B2R_ERR_INTERNAL;
  }
}

int or_get_starts(const b2r_timetable_desc* tt, const b2r_query* q, int32_t* tas,
                  int32_t* tst, uint32_t* stop, uint32_t capacity, uint32_t* n) {
  try {
    oracle::tt_view const v{*tt, q->prf_idx};
    auto qq = oracle::to_query(*q);
    qq.sanitize();
    auto const fwd = q->direction == B2R_FORWARD;
    std::vector<oracle::start_t> starts;
    oracle::start_time_v sv{qq.is_interval != 0, qq.start_time, {qq.iv_from, qq.iv_to}};
    oracle::get_starts(v, fwd, sv, qq, qq.tts, starts, true);
    std::sort(starts.begin(), starts.end(),
              [&](oracle::start_t const& a, oracle::start_t const& b) {
                return fwd ? b < a : a < b;
              });
    *n = static_cast<uint32_t>(starts.size());
    for (auto i = 0U; i < std::min<size_t>(capacity, starts.size()); ++i) {
      tas[i] = starts[i].time_at_start;
      tst[i] = starts[i].time_at_stop;
      stop[i] = starts[i].stop;
    }
    return B2R_OK;
  } catch (...) {
    return B2R_ERR_INTERNAL;
  }
}

int or_lower_bounds(const b2r_timetable_desc* tt, const b2r_query* q, uint16_t* dists) {
  try {
    oracle::tt_view const v{*tt, q->prf_idx};
    auto qq = oracle::to_query(*q);
    qq.sanitize();
    std::vector<uint16_t> lb;
    oracle::dijkstra_lb(v, qq, q->direction == B2R_FORWARD, lb);
    std::memcpy(dists, lb.data(), lb.size() * sizeof(uint16_t));
    return B2R_OK;
  } catch (...) {
    return B2R_ERR_INTERNAL;
  }
}

int or_run_many(const b2r_timetable_desc* tt, const b2r_query* qs, uint32_t n,
                uint32_t threads, double* latencies_us, uint64_t* journeys, double* wall_s) {
  std::atomic<uint32_t> next{0};
  std::atomic<uint64_t> n_journeys{0};
  auto const t0 = std::chrono::steady_clock::now();
  auto worker = [&]() {
    for (auto i = next++; i < n; i = next++) {
      auto const a = std::chrono::steady_clock::now();
      or_result* r = nullptr;
      if (or_search(tt, &qs[i], &r) == B2R_OK) {
        n_journeys += r->journeys.size();
        or_result_free(r);
      }
      auto const b = std::chrono::steady_clock::now();
      if (latencies_us != nullptr) {
        latencies_us[i] = std::chrono::duration<double, std::micro>(b - a).count();
      }
    }
  };
  std::vector<std::thread> pool;
  for (auto t = 0U; t < std::max(1U, threads); ++t) pool.emplace_back(worker);
  for (auto& t : pool) t.join();
  if (wall_s != nullptr) {
    *wall_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  if (journeys != nullptr) *journeys = n_journeys;
  return B2R_OK;
}

}  // extern "C"
