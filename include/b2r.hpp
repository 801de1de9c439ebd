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

#include <cstdint>
#include <optional>
#include <span>
#include <stdexcept>
#include <string>
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

struct run_enter_exit {  // journey::run_enter_exit (transport, day, stops)
  uint32_t transport_{0};
  uint16_t day_{0};
  uint16_t stop_from_{0}, stop_to_{0};  // stop_range_ [from, to)
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
  friend bool operator==(journey const&, journey const&) = default;
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
  explicit timetable(b2r_timetable_desc const& d, int device = 0) : n_locations_{d.n_locations} {
    check(b2r_timetable_upload(&d, device, &h_), "b2r_timetable_upload");
  }
  timetable(timetable const&) = delete;
  timetable& operator=(timetable const&) = delete;
  ~timetable() { b2r_timetable_destroy(h_); }
  b2r_timetable* handle() const { return h_; }
  uint32_t n_locations() const { return n_locations_; }

private:
  b2r_timetable* h_{nullptr};
  uint32_t n_locations_;
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
    for (auto k = 0U; k != j.n_legs; ++k) {
      auto const& l = r.legs[j.first_leg + k];
      leg y{l.from, l.to, l.dep_time, l.arr_time, {}};
      switch (l.kind) {
        case B2R_LEG_TRANSPORT: y.uses_ = run_enter_exit{l.transport, l.day, l.stop_from, l.stop_to}; break;
        case B2R_LEG_FOOTPATH: y.uses_ = footpath{l.transport, l.duration}; break;
        default: y.uses_ = offset{l.transport, l.duration, l.transport_mode_id};
      }
      x.legs_.push_back(std::move(y));
    }
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

}  // namespace routing
}  // namespace b2r
