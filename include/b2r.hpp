/*
 * b2r.hpp -- C++ mirror of nigiri's routing interface over the C ABI of
 * b2r.h (header only).
 *
 * Names and meanings follow nigiri so that code written against
 * nigiri::routing reads the same here:
 *  - routing::query             include/nigiri/routing/query.h:70-100
 *  - routing::offset            query.h:28-48
 *  - routing::journey / leg     include/nigiri/routing/journey.h:20-118
 *  - routing::routing_result    include/nigiri/routing/search.h:71-76
 *  - routing::raptor_search     include/nigiri/routing/raptor_search.h:9-17
 *  - routing::pong_search       include/nigiri/routing/raptor/pong.h:21-29
 *  - routing::one_to_all        include/nigiri/routing/one_to_all.h:22-25
 *  - routing::raptor_state      round_times_ of raptor_state.h:22-111
 * restricted to what the engine runs: the static timetable (no real-time
 * overlay), no vias, no time-dependent offsets; footpath profiles (the
 * wheelchair profile among them) and the class, bike, car and reservation
 * filters included.  Times are minutes since the epoch
 * (unixtime_t), durations minutes.
 *
 * Errors: every call that fails throws b2r::error with the C ABI's status
 * and message (nigiri reports errors by exception as well).  A query whose
 * own search fails is returned with routing_result::status_ != B2R_OK.
 */
#pragma once

#include <algorithm>
#include <cstdint>
#include <iterator>
#include <optional>
#include <span>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <variant>
#include <vector>

#include "b2r.h"

namespace b2r {

struct error : std::runtime_error {
  error(int s, std::string const& what) : std::runtime_error{what}, status{s} {}
  int status;
};

inline void check(int rc, char const* what) {
  if (rc != B2R_OK) throw error{rc, std::string{what} + ": " + b2r_last_error()};
}

namespace routing {

using unixtime_t = int32_t;  // minutes since 1970-01-01
using duration_t = int16_t;  // minutes

enum class direction : uint8_t { kForward = B2R_FORWARD, kBackward = B2R_BACKWARD };

enum class location_match_mode : uint8_t {
  kExact = B2R_MATCH_EXACT,
  kOnlyChildren = B2R_MATCH_ONLY_CHILDREN,
  kEquivalent = B2R_MATCH_EQUIVALENT,
  kIntermodal = B2R_MATCH_INTERMODAL
};

struct interval {
  unixtime_t from_{0}, to_{0};
  friend bool operator==(interval const&, interval const&) = default;
};

struct offset {
  uint32_t target_{0};
  duration_t duration_{0};
  int32_t transport_mode_id_{0};
  friend bool operator==(offset const&, offset const&) = default;
};

struct transfer_time_settings {
  bool default_{true};
  duration_t min_transfer_time_{0};
  duration_t additional_time_{0};
  float factor_{1.0F};
};

struct query {
  std::variant<unixtime_t, interval> start_time_{unixtime_t{0}};
  location_match_mode start_match_mode_{location_match_mode::kExact};
  location_match_mode dest_match_mode_{location_match_mode::kExact};
  bool use_start_footpaths_{false};
  std::vector<offset> start_{}, destination_{};
  duration_t max_start_offset_{B2R_MAX_TRAVEL_TIME_MIN};
  uint8_t max_transfers_{B2R_MAX_TRANSFERS};
  duration_t max_travel_time_{B2R_MAX_TRAVEL_TIME_MIN};
  unsigned min_connection_count_{0U};
  bool extend_interval_earlier_{false};
  bool extend_interval_later_{false};
  std::optional<interval> max_interval_{};  // clamp of every interval extension
  uint8_t prf_idx_{0U};                      // footpath profile (B2R_PROFILE_*)
  std::optional<duration_t> fastest_direct_{};
  double fastest_direct_factor_{1.0};
  transfer_time_settings transfer_time_settings_{};
  uint16_t allowed_claszes_{0xFFFFU};  // clasz_mask_t: bit c = class c allowed
  bool require_bike_transport_{false};
  bool require_car_transport_{false};
  bool no_compulsory_reservation_{false};
};

struct run_enter_exit {  // journey::run_enter_exit (transport, day, stops, real-time run)
  uint32_t transport_{0};
  uint16_t day_{0};
  uint16_t stop_from_{0}, stop_to_{0};  // stop_range_ [from, to)
  uint32_t rt_transport_{B2R_INVALID_IDX};  // rt::run::rt_
  friend bool operator==(run_enter_exit const&, run_enter_exit const&) = default;
};

struct footpath {
  uint32_t target_{0};
  duration_t duration_{0};
  friend bool operator==(footpath const&, footpath const&) = default;
};

struct leg {
  uint32_t from_{0}, to_{0};
  unixtime_t dep_time_{0}, arr_time_{0};
  std::variant<run_enter_exit, footpath, offset> uses_{};
  friend bool operator==(leg const&, leg const&) = default;
};

struct journey {
  unixtime_t travel_time() const { return dest_time_ > start_time_ ? dest_time_ - start_time_ : start_time_ - dest_time_; }
  std::vector<leg> legs_{};
  unixtime_t start_time_{0}, dest_time_{0};
  uint32_t dest_{0};
  uint8_t transfers_{0};
  bool error_{false};
  bool is_reconstructed_{false};
  friend bool operator==(journey const&, journey const&) = default;

  // journey::dominates, journey.h:84-92
  bool dominates(journey const& o) const {
    if (start_time_ <= dest_time_) {
      return transfers_ <= o.transfers_ && start_time_ >= o.start_time_ && dest_time_ <= o.dest_time_;
    }
    return transfers_ <= o.transfers_ && start_time_ <= o.start_time_ && dest_time_ >= o.dest_time_;
  }
};

// routing::pareto_set, pareto_set.h:13-60: add() keeps only undominated
// elements, in insertion order.
template <typename T>
struct pareto_set {
  using iterator = typename std::vector<T>::iterator;
  std::tuple<bool, iterator, iterator> add(T&& el) {
    auto n_removed = std::size_t{0};
    for (auto i = std::size_t{0}; i < els_.size(); ++i) {
      if (els_[i].dominates(el)) return {false, end(), begin() + static_cast<std::ptrdiff_t>(i)};
      if (el.dominates(els_[i])) {
        ++n_removed;
        continue;
      }
      els_[i - n_removed] = els_[i];
    }
    els_.resize(els_.size() - n_removed);
    els_.emplace_back(std::move(el));
    return {true, std::prev(end()), end()};
  }
  iterator begin() { return els_.begin(); }
  iterator end() { return els_.end(); }
  std::size_t size() const { return els_.size(); }
  bool empty() const { return els_.empty(); }
  void clear() { els_.clear(); }
  template <typename Fn>
  void erase_if(Fn&& fn) {
    els_.erase(std::remove_if(els_.begin(), els_.end(), fn), els_.end());
  }
  std::vector<T> els_;
};

struct routing_result {
  int status_{B2R_OK};
  std::vector<journey> journeys_{};
  interval interval_{};
  uint64_t n_rounds_{0}, n_start_times_{0};
};

// The round times one_to_all leaves in raptor_state: rows k = 0..n_rows-1
// of delta_t minutes relative to base_day (kInvalidDelta where unreached).
struct raptor_state {
  int16_t at(uint32_t k, uint32_t l) const { return round_times_[static_cast<size_t>(k) * n_locations_ + l]; }
  std::vector<int16_t> round_times_{};
  uint32_t n_rows_{0}, n_locations_{0};
  int32_t base_day_{0};  // days since the epoch
};

}  // namespace routing

// Device-resident timetable image (b2r_timetable_upload); the description's
// arrays are copied, so they may be freed after construction.
class timetable {
public:
  explicit timetable(b2r_timetable_desc const& d, int device = 0)
      : n_locations_{d.n_locations}, internal_from_days_{d.date_range_from - B2R_TIMETABLE_OFFSET_DAYS} {
    check(b2r_timetable_upload(&d, device, &h_), "b2r_timetable_upload");
  }
  // an image uploaded elsewhere (from description d), not destroyed here
  timetable(b2r_timetable* uploaded, b2r_timetable_desc const& d)
      : h_{uploaded},
        n_locations_{d.n_locations},
        internal_from_days_{d.date_range_from - B2R_TIMETABLE_OFFSET_DAYS},
        owned_{false} {}
  timetable(timetable const&) = delete;
  timetable& operator=(timetable const&) = delete;
  ~timetable() {
    if (owned_) b2r_timetable_destroy(h_);
  }
  b2r_timetable* handle() const { return h_; }
  uint32_t n_locations() const { return n_locations_; }
  // first day of timetable::internal_interval(), days since the epoch
  int32_t internal_from_days() const { return internal_from_days_; }

private:
  b2r_timetable* h_{nullptr};
  uint32_t n_locations_;
  int32_t internal_from_days_;
  bool owned_{true};
};

// Resident query slots on one GPU (b2r_engine_create).  Like nigiri's
// search state, an engine serves one host thread at a time.
class engine {
public:
  explicit engine(timetable& tt, std::optional<b2r_engine_config> cfg = std::nullopt) : tt_{&tt} {
    b2r_engine_config c;
    b2r_engine_config_init(&c);
    if (cfg) c = *cfg;
    check(b2r_engine_create(tt.handle(), &c, &h_), "b2r_engine_create");
  }
  engine(engine const&) = delete;
  engine& operator=(engine const&) = delete;
  ~engine() { b2r_engine_destroy(h_); }
  b2r_engine* handle() const { return h_; }
  timetable const& tt() const { return *tt_; }

private:
  timetable* tt_;
  b2r_engine* h_{nullptr};
};

namespace routing {
namespace detail {

// A query in the C ABI's layout; owns the offset arrays it points to.
struct c_query {
  c_query(query const& q, direction dir, uint8_t kind, uint8_t algorithm = B2R_ALGO_RAPTOR)
      : start{to_c(q.start_)}, dest{to_c(q.destination_)} {
    b2r_query_init(&c);
    c.kind = kind;
    c.algorithm = algorithm;
    c.direction = static_cast<uint8_t>(dir);
    if (auto const* t = std::get_if<unixtime_t>(&q.start_time_)) {
      c.start_time = *t;
    } else {
      auto const& iv = std::get<interval>(q.start_time_);
      c.is_interval = 1;
      c.interval_from = iv.from_;
      c.interval_to = iv.to_;
    }
    c.start_match_mode = static_cast<uint8_t>(q.start_match_mode_);
    c.dest_match_mode = static_cast<uint8_t>(q.dest_match_mode_);
    c.use_start_footpaths = q.use_start_footpaths_ ? 1 : 0;
    c.extend_interval_earlier = q.extend_interval_earlier_ ? 1 : 0;
    c.extend_interval_later = q.extend_interval_later_ ? 1 : 0;
    c.prf_idx = q.prf_idx_;
    if (q.max_interval_) {
      c.has_max_interval = 1;
      c.max_interval_from = q.max_interval_->from_;
      c.max_interval_to = q.max_interval_->to_;
    }
    c.start = start.data();
    c.n_start = static_cast<uint32_t>(start.size());
    c.destination = dest.data();
    c.n_destination = static_cast<uint32_t>(dest.size());
    c.max_start_offset = q.max_start_offset_;
    c.max_transfers = q.max_transfers_;
    c.max_travel_time = q.max_travel_time_;
    c.min_connection_count = q.min_connection_count_;
    c.has_fastest_direct = q.fastest_direct_.has_value() ? 1 : 0;
    c.fastest_direct = q.fastest_direct_.value_or(0);
    c.fastest_direct_factor = q.fastest_direct_factor_;
    auto const& s = q.transfer_time_settings_;
    c.tts_default = s.default_ ? 1 : 0;
    c.tts_min_transfer_time = s.min_transfer_time_;
    c.tts_additional_time = s.additional_time_;
    c.tts_factor = s.factor_;
    c.allowed_claszes = q.allowed_claszes_;
    c.require_bike_transport = q.require_bike_transport_ ? 1 : 0;
    c.require_car_transport = q.require_car_transport_ ? 1 : 0;
    c.no_compulsory_reservation = q.no_compulsory_reservation_ ? 1 : 0;
  }
  static std::vector<b2r_offset> to_c(std::vector<offset> const& v) {
    std::vector<b2r_offset> out;
    out.reserve(v.size());
    for (auto const& o : v) out.push_back(b2r_offset{o.target_, o.duration_, 0, o.transport_mode_id_});
    return out;
  }
  std::vector<b2r_offset> start, dest;
  b2r_query c{};
};

}  // namespace detail

// A C ABI query in nigiri's terms (the inverse of detail::c_query).
inline query query_of(b2r_query const& c) {
  query q;
  if (c.is_interval != 0) q.start_time_ = interval{c.interval_from, c.interval_to};
  else q.start_time_ = c.start_time;
  q.start_match_mode_ = static_cast<location_match_mode>(c.start_match_mode);
  q.dest_match_mode_ = static_cast<location_match_mode>(c.dest_match_mode);
  q.use_start_footpaths_ = c.use_start_footpaths != 0;
  for (auto i = 0U; i != c.n_start; ++i) {
    q.start_.push_back({c.start[i].target, c.start[i].duration, c.start[i].transport_mode_id});
  }
  for (auto i = 0U; i != c.n_destination; ++i) {
    q.destination_.push_back({c.destination[i].target, c.destination[i].duration,
                              c.destination[i].transport_mode_id});
  }
  q.max_start_offset_ = c.max_start_offset;
  q.max_transfers_ = c.max_transfers;
  q.max_travel_time_ = c.max_travel_time;
  q.min_connection_count_ = c.min_connection_count;
  q.extend_interval_earlier_ = c.extend_interval_earlier != 0;
  q.extend_interval_later_ = c.extend_interval_later != 0;
  if (c.has_fastest_direct != 0) q.fastest_direct_ = c.fastest_direct;
  q.fastest_direct_factor_ = c.fastest_direct_factor;
  q.transfer_time_settings_ = {c.tts_default != 0, c.tts_min_transfer_time, c.tts_additional_time, c.tts_factor};
  q.allowed_claszes_ = static_cast<uint16_t>(c.allowed_claszes);
  q.require_bike_transport_ = c.require_bike_transport != 0;
  q.require_car_transport_ = c.require_car_transport != 0;
  q.no_compulsory_reservation_ = c.no_compulsory_reservation != 0;
  q.prf_idx_ = c.prf_idx;
  if (c.has_max_interval != 0) q.max_interval_ = interval{c.max_interval_from, c.max_interval_to};
  return q;
}

// One C ABI leg as a routing::journey::leg.
inline leg leg_of(b2r_leg const& l) {
  leg y{l.from, l.to, l.dep_time, l.arr_time, {}};
  switch (l.kind) {
    case B2R_LEG_TRANSPORT:
      y.uses_ = run_enter_exit{l.transport, l.day, l.stop_from, l.stop_to, l.rt_transport};
      break;
    case B2R_LEG_FOOTPATH: y.uses_ = footpath{l.transport, l.duration}; break;
    default: y.uses_ = offset{l.transport, l.duration, l.transport_mode_id};
  }
  return y;
}

// The journeys of one C ABI result, as routing::journey values.
inline std::vector<journey> journeys_of(b2r_result const& r) {
  std::vector<journey> out;
  out.reserve(r.n_journeys);
  for (auto i = 0U; i != r.n_journeys; ++i) {
    auto const& j = r.journeys[i];
    journey x;
    x.start_time_ = j.start_time;
    x.dest_time_ = j.dest_time;
    x.dest_ = j.dest;
    x.transfers_ = j.transfers;
    x.error_ = j.error != 0;
    x.is_reconstructed_ = true;  // the engine returns rebuilt journeys only
    for (auto k = 0U; k != j.n_legs; ++k) x.legs_.push_back(leg_of(r.legs[j.first_leg + k]));
    out.push_back(std::move(x));
  }
  return out;
}

namespace detail {
inline std::vector<routing_result> search(engine& e, std::span<query const> qs, direction dir,
                                          uint8_t algorithm) {
  std::vector<detail::c_query> cq;
  cq.reserve(qs.size());
  for (auto const& q : qs) cq.emplace_back(q, dir, static_cast<uint8_t>(B2R_ONE_TO_ONE), algorithm);
  std::vector<b2r_query> arr;
  arr.reserve(cq.size());
  for (auto const& x : cq) arr.push_back(x.c);
  std::vector<b2r_result> res(arr.size());
  check(b2r_search_batch(e.handle(), arr.data(), static_cast<uint32_t>(arr.size()), res.data()),
        "b2r_search_batch");
  std::vector<routing_result> out(res.size());
  for (auto i = 0U; i != res.size(); ++i) {
    out[i].status_ = res[i].status;
    out[i].journeys_ = journeys_of(res[i]);
    out[i].interval_ = {res[i].interval_from, res[i].interval_to};
    out[i].n_rounds_ = res[i].n_rounds;
    out[i].n_start_times_ = res[i].n_start_times;
  }
  return out;
}
}  // namespace detail

// routing::raptor_search for many queries in one engine call (continuous
// batching over the engine's resident slots).
inline std::vector<routing_result> raptor_search(engine& e, std::span<query const> qs, direction dir) {
  return detail::search(e, qs, dir, B2R_ALGO_RAPTOR);
}

inline routing_result raptor_search(engine& e, query const& q, direction dir) {
  return raptor_search(e, std::span<query const>{&q, 1U}, dir).front();
}

// routing::pong_search: the same range search by alternating forward and
// backward searches.  A sweep that fails as the reference's would ("no
// pong") returns status_ == B2R_ERR_INTERNAL instead of throwing.
inline std::vector<routing_result> pong_search(engine& e, std::span<query const> qs, direction dir) {
  return detail::search(e, qs, dir, B2R_ALGO_PONG);
}

inline routing_result pong_search(engine& e, query const& q, direction dir) {
  return pong_search(e, std::span<query const>{&q, 1U}, dir).front();
}

// routing::one_to_all: the round times of every location.
inline raptor_state one_to_all(engine& e, query const& q, direction dir) {
  detail::c_query cq{q, dir, static_cast<uint8_t>(B2R_ONE_TO_ALL)};
  b2r_result r{};
  check(b2r_search_batch(e.handle(), &cq.c, 1U, &r), "b2r_search_batch");
  check(r.status, "one_to_all");
  raptor_state s;
  s.n_rows_ = r.n_rows;
  s.n_locations_ = e.tt().n_locations();
  s.base_day_ = r.base_day;
  s.round_times_.assign(r.round_times, r.round_times + static_cast<size_t>(r.n_rows) * s.n_locations_);
  return s;
}

// ---------------------------------------------------------------------------
// The Algo concept of routing::search<Dir, Algo> over the engine.
//
// search<Dir, Algo> constructs its Algo with the query's prepared state
// (search.h:148-171) and drives it through reset_arrivals, next_start_time,
// add_start, execute and reconstruct.  b2r_algo is that Algo for the
// B200 engine: one query's raptor_state resident on the device (the C ABI's
// b2r_raptor), each execute the rounds of one start time; the search
// direction is a template parameter as in raptor<SearchDir, ...>.  Its constructor
// takes raptor's arguments (raptor.h:56-73) for the static timetable: the
// real-time overlay, vias and time-dependent offsets must be absent
// (b2r::error B2R_ERR_UNSUPPORTED otherwise).

struct b2r_algo_state {};  // raptor_state's place: the device state is the algo's own

struct b2r_algo_stats {
  uint64_t n_rounds_{0};
};

struct via_stop {};   // vias are not supported: the list must be empty
struct td_offset {};  // time-dependent offsets are not supported

template <direction SearchDir>
class b2r_algo {
public:
  using algo_state_t = b2r_algo_state;
  using algo_stats_t = b2r_algo_stats;
  static constexpr bool kUseLowerBounds = true;

  b2r_algo(b2r::timetable& tt, void const* rtt, algo_state_t&, std::vector<bool> const& is_dest,
           std::vector<std::vector<bool>> const& is_via, std::vector<uint16_t> const& dist_to_dest,
           std::vector<std::pair<uint32_t, std::vector<td_offset>>> const& td_dist_to_dest,
           std::vector<uint16_t> const& lb, std::vector<via_stop> const& via_stops, uint16_t base,
           uint16_t allowed_claszes, bool require_bike_transport, bool require_car_transport, bool is_wheelchair,
           bool no_compulsory_reservation, transfer_time_settings const& tts, uint8_t prf_idx) {
    if (rtt != nullptr || !via_stops.empty() || !td_dist_to_dest.empty()) {
      throw error{B2R_ERR_UNSUPPORTED, "b2r_algo: real-time overlay, vias and time-dependent offsets"};
    }
    for (auto const& v : is_via) {
      if (std::find(v.begin(), v.end(), true) != v.end()) throw error{B2R_ERR_UNSUPPORTED, "b2r_algo: vias"};
    }
    (void)is_wheelchair;  // the wheelchair profile (prf_idx) carries it
    std::vector<uint32_t> dests;
    for (auto l = std::size_t{0}; l < is_dest.size(); ++l) {
      if (is_dest[l]) dests.push_back(static_cast<uint32_t>(l));
    }
    b2r_raptor_args a{};
    a.direction = static_cast<uint8_t>(SearchDir);
    a.prf_idx = prf_idx;
    a.require_bike_transport = require_bike_transport ? 1 : 0;
    a.require_car_transport = require_car_transport ? 1 : 0;
    a.no_compulsory_reservation = no_compulsory_reservation ? 1 : 0;
    a.tts_default = tts.default_ ? 1 : 0;
    a.allowed_claszes = allowed_claszes;
    a.tts_min_transfer_time = tts.min_transfer_time_;
    a.tts_additional_time = tts.additional_time_;
    a.tts_factor = tts.factor_;
    a.base_day = tt.internal_from_days() + base;
    a.n_destinations = static_cast<uint32_t>(dests.size());
    a.destinations = dests.data();
    a.dist_to_dest = dist_to_dest.empty() ? nullptr : dist_to_dest.data();
    a.lower_bounds = lb.empty() ? nullptr : lb.data();
    check(b2r_raptor_create(tt.handle(), &a, &h_), "b2r_raptor_create");
  }
  b2r_algo(b2r_algo const&) = delete;
  b2r_algo& operator=(b2r_algo const&) = delete;
  ~b2r_algo() { b2r_raptor_destroy(h_); }

  void reset_arrivals() { check(b2r_raptor_reset_arrivals(h_), "reset_arrivals"); }
  void next_start_time() { check(b2r_raptor_next_start_time(h_), "next_start_time"); }
  void add_start(uint32_t l, unixtime_t t) { check(b2r_raptor_add_start(h_, l, t), "add_start"); }

  void execute(unixtime_t start_time, uint8_t max_transfers, unixtime_t worst_time_at_dest,
               pareto_set<journey>& results) {
    std::vector<b2r_journey> js(B2R_K * 64U);
    uint32_t n = 0;
    check(b2r_raptor_execute(h_, start_time, max_transfers, worst_time_at_dest, js.data(),
                             static_cast<uint32_t>(js.size()), &n),
          "execute");
    for (auto i = 0U; i != n; ++i) {  // raptor.h:393-413
      journey j;
      j.start_time_ = js[i].start_time;
      j.dest_time_ = js[i].dest_time;
      j.dest_ = js[i].dest;
      j.transfers_ = js[i].transfers;
      results.add(std::move(j));
    }
  }

  void reconstruct(query const& q, journey& j) {
    detail::c_query cq{q, SearchDir, static_cast<uint8_t>(B2R_ONE_TO_ONE)};
    b2r_journey bj{j.start_time_, j.dest_time_, j.dest_, j.transfers_, 0, 0, 0};
    std::vector<b2r_leg> legs(64);
    check(b2r_raptor_reconstruct(h_, &cq.c, &bj, legs.data(), static_cast<uint32_t>(legs.size())),
          "reconstruct");
    if (bj.error != 0) throw error{B2R_ERR_INTERNAL, "reconstruct failed"};
    j.legs_.clear();
    for (auto i = 0U; i != bj.n_legs; ++i) j.legs_.push_back(leg_of(legs[i]));
    j.is_reconstructed_ = true;
  }

  algo_stats_t get_stats() const { return {b2r_raptor_rounds(h_)}; }

private:
  b2r_raptor* h_{nullptr};
};

// routing::search<SearchDir, Algo> (search.h:78-505) for the static
// timetable: search::init's preparation (b2r_search_prepare), the start
// times in groups with early termination, reconstruction of the new
// journeys, interval extension, and the final filtering and ordering.
template <direction SearchDir, typename Algo>
class search {
  static constexpr bool kFwd = SearchDir == direction::kForward;

public:
  search(b2r::timetable& tt, typename Algo::algo_state_t& state, query q)
      : tt_{tt}, state_{state}, q_{std::move(q)} {}

  routing_result execute() {
    detail::c_query cq{q_, SearchDir, static_cast<uint8_t>(B2R_ONE_TO_ONE)};
    b2r_search_plan* plan = nullptr;
    check(b2r_search_prepare(tt_.handle(), &cq.c, &plan), "b2r_search_prepare");
    struct free_plan {
      b2r_search_plan* p;
      ~free_plan() { b2r_search_plan_free(p); }
    } guard{plan};
    routing_result res;
    res.status_ = plan->status;
    res.interval_ = {plan->interval_from, plan->interval_to};
    if (plan->status != B2R_OK || plan->start_dest_overlap != 0) return res;

    std::vector<bool> is_dest(tt_.n_locations(), false);
    for (auto i = 0U; i != plan->n_destinations; ++i) is_dest[plan->destinations[i]] = true;
    std::vector<uint16_t> dist, lb;
    if (plan->dist_to_dest != nullptr) dist.assign(plan->dist_to_dest, plan->dist_to_dest + tt_.n_locations());
    if (plan->lower_bounds != nullptr) lb.assign(plan->lower_bounds, plan->lower_bounds + tt_.n_locations());
    transfer_time_settings const tts{plan->tts_default != 0, plan->tts_min_transfer_time,
                                     plan->tts_additional_time, plan->tts_factor};
    Algo algo{tt_, nullptr, state_, is_dest, {}, dist, {}, lb, {},
              static_cast<uint16_t>(plan->base_day - tt_.internal_from_days()), q_.allowed_claszes_,
              q_.require_bike_transport_, q_.require_car_transport_, q_.prf_idx_ == B2R_PROFILE_WHEELCHAIR,
              q_.no_compulsory_reservation_, tts, q_.prf_idx_};

    ontrip_ = plan->ontrip != 0;
    interval_ = {plan->interval_from, plan->interval_to};
    fastest_direct_ = plan->fastest_direct;
    max_travel_time_ = plan->max_travel_time;
    while (true) {  // search.h:227-317
      search_interval(algo, *plan);
      if (results_.empty() || ontrip_ || n_results_in_interval() >= q_.min_connection_count_) break;
      uint8_t changed = 0, reset = 0;
      check(b2r_search_extend(tt_.handle(), plan, q_.min_connection_count_ - n_results_in_interval(), &changed,
                              &reset),
            "b2r_search_extend");
      if (changed == 0) break;
      if (reset != 0) {
        algo.reset_arrivals();
        results_.erase_if([&](journey const& j) { return !contains(j.start_time_); });  // remove_ontrip_results
      }
      interval_ = {plan->interval_from, plan->interval_to};
    }
    if (!ontrip_) {  // search.h:319-336
      results_.erase_if([&](journey const& j) {
        return !contains(j.start_time_) || j.travel_time() >= fastest_direct_ || j.travel_time() > max_travel_time_;
      });
      std::sort(results_.begin(), results_.end(), [](journey const& a, journey const& b) {
        return std::tie(a.start_time_, a.transfers_) < std::tie(b.start_time_, b.transfers_);
      });
    }
    results_.erase_if([](journey const& j) { return !j.is_reconstructed_; });
    res.journeys_ = results_.els_;
    res.interval_ = interval_;
    res.n_rounds_ = algo.get_stats().n_rounds_;
    res.n_start_times_ = n_start_times_;
    return res;
  }

private:
  bool contains(unixtime_t t) const { return interval_.from_ <= t && t < interval_.to_; }

  unsigned n_results_in_interval() {  // search.h:380-389
    if (ontrip_) return static_cast<unsigned>(results_.size());
    return static_cast<unsigned>(
        std::count_if(results_.begin(), results_.end(), [&](journey const& j) { return contains(j.start_time_); }));
  }

  // search.h:419-494: one execute per group of start labels with the same
  // time at start
  void search_interval(Algo& algo, b2r_search_plan const& plan) {
    auto early_termination = false;
    for (auto i = 0U; i < plan.n_starts;) {
      auto j = i;
      while (j != plan.n_starts && plan.starts[j].time_at_start == plan.starts[i].time_at_start) ++j;
      if (!early_termination) {
        algo.next_start_time();
        auto const start_time = plan.starts[i].time_at_start;
        for (auto x = i; x != j; ++x) algo.add_start(plan.starts[x].location, plan.starts[x].time_at_stop);
        auto const worst_time_at_dest =
            start_time + (kFwd ? 1 : -1) * (std::min(fastest_direct_, max_travel_time_) + 1);
        algo.execute(start_time, q_.max_transfers_, worst_time_at_dest, results_);
        ++n_start_times_;
        for (auto& jr : results_) {
          if (!jr.is_reconstructed_ && !jr.error_ && (ontrip_ || contains(jr.start_time_)) &&
              jr.travel_time() < fastest_direct_) {
            try {
              algo.reconstruct(q_, jr);
            } catch (error const&) {
              jr.error_ = true;
            }
          }
        }
        if (q_.min_connection_count_ > 0 && n_results_in_interval() >= q_.min_connection_count_ &&
            ((kFwd && q_.extend_interval_earlier_ && !q_.extend_interval_later_) ||
             (!kFwd && !q_.extend_interval_earlier_ && q_.extend_interval_later_))) {
          early_termination = true;
          if (kFwd) interval_.from_ = start_time;
          else interval_.to_ = start_time + 1;
        }
      }
      i = j;
    }
  }

  b2r::timetable& tt_;
  typename Algo::algo_state_t& state_;
  query q_;
  pareto_set<journey> results_;
  bool ontrip_{true};
  interval interval_{};
  int fastest_direct_{0}, max_travel_time_{0};
  uint64_t n_start_times_{0};
};

}  // namespace routing
}  // namespace b2r
