// Host-side per-query preparation for the device engine: everything
// routing::search<Dir, Algo> does before and between the Algo calls
// (include/nigiri/routing/search.h:84-172, 204-345, 401-417) for the static
// instantiation.  The device runs the start-time groups, the rounds, the
// result collection and the reconstruction.
#pragma once

#include <cstdint>
#include <memory>
#include <unordered_map>
#include <utility>
#include <vector>

#include "b2r.h"

namespace b2r {

struct host_view;

struct start_label {  // routing::start, start_times.h:21-26
  int32_t time_at_start;
  int32_t time_at_stop;
  uint32_t stop;
};

struct tts_norm {  // transfer_time_settings after search::init()
  uint8_t is_default{1};
  int16_t min_transfer_time{0};
  int16_t additional_time{0};
  float factor{1.0F};
};

struct pong_plan;

struct prepped_query {
  int status{B2R_OK};
  bool empty_result{false};  // start and destination overlap
  bool fwd{true};
  bool one_to_all{false};
  bool ontrip{true};
  bool intermodal_dest{false};
  uint8_t start_mode{0}, dest_mode{0};
  uint8_t max_transfers{14};
  uint8_t end_k{16};
  int16_t max_travel_time{7200};
  int16_t max_start_offset_{7200};
  int16_t fastest_direct{32767};
  uint16_t base{0};        // day index relative to the internal interval
  int32_t base_days{0};    // days since epoch
  int32_t iv_from{0}, iv_to{0};  // search interval
  uint32_t min_connection_count{0};
  bool extend_earlier{false}, extend_later{false};
  uint16_t allowed_claszes{0xFFFFU};  // bit c: transport class c allowed
  uint8_t req_flags{0U};              // bit f: route flag f required
  uint8_t prf{0U};                    // query::prf_idx_
  int32_t data_max_from{0}, data_max_to{0};  // interval_estimator clamp
  bool has_max_interval{false};               // query::max_interval_
  int32_t max_iv_from{0}, max_iv_to{0};
  tts_norm tts;
  tts_norm tts_raw;  // as given (fastest-direct uses it)
  std::vector<b2r_offset> start_offsets, dest_offsets;  // sanitized order
  std::vector<start_label> starts;                      // sorted
  std::vector<uint32_t> dest_locs;                      // ascending
  std::vector<std::pair<uint32_t, uint16_t>> dest_dist; // intermodal, ascending
  std::vector<uint16_t> lb;                             // [n_locations]
  // Dijkstra seeds (location, distance) for lower bounds computed on the
  // device (dijkstra.cc:26-48)
  std::vector<std::pair<uint32_t, uint16_t>> lb_seeds;
  // worst time at destination of a start-time group = its start + dir(span)
  // (search.h:426-429; pong.cc:262-265 for a ping, the ping's departure
  // for a pong)
  int16_t span{0};
  bool no_lb{false};      // run without lower bounds (a pong phase)
  bool keep_lb{false};    // leave the slot's lower-bound column as it is
  bool need_sweep{false}; // round times of an earlier phase stay in effect
  uint8_t blast{0};       // pong bounds (raptor.h:172)
  uint8_t recon_mode{0};  // 0: journeys of the interval, 1: one journey, 2: none
  uint8_t recon_transfers{0};
  int32_t recon_start{0};
  bool use_start_footpaths{false};
  // B2R_ALGO_PONG: the whole sweep (this query is then its first ping)
  std::shared_ptr<pong_plan const> pong;
};

// pong_search (pong.cc:63-475): everything the host needs between the
// phases.  `ping` and `pong` are phase templates (the query in its own and
// in the flipped direction); a phase is a template plus its start labels and
// bounds.
struct pong_plan {
  prepped_query ping, pong;
  int32_t iv_from{0}, iv_to{0};  // search interval
  int32_t ext_from{0}, ext_to{0};  // timetable::external_interval, minutes
  int16_t fastest_direct{0};
  int16_t max_travel_time{0};
  uint8_t max_transfers{0};
  uint32_t min_connection_count{0};
  bool fwd{true}, extend_earlier{false}, extend_later{false};
};

// Row `src` of the all-pairs lower-bound table: shortest distances from
// src over the forward- or backward-search lower-bound graph, 0xFFFF beyond
// kMaxTravelTime (row must hold n_locations values).
void lb_table_row(host_view const& tt, bool fwd, uint32_t src, uint16_t* row);

// std::chrono::round<days> of a minute time point (ties to even).
int32_t round_to_days(int64_t minutes);

// Computes everything above.  lb_mode: 0 = no lower bounds (lb = 0),
// 1 = Dijkstra on the host (lb filled), 2 = on the device and 3 = from the
// all-pairs table on the device (lb_seeds filled).
void prepare(host_view const& tt, b2r_query const& q, int lb_mode,
             prepped_query& out);

// The start labels of one phase of a pong search at time t: get_starts
// with a single start time (start_times.cc:241-319) over the phase
// template's offsets.
void phase_starts(host_view const& tt, prepped_query const& tmpl, int32_t t,
                  std::vector<start_label>& out);

// Start labels of [from, to) for an interval extension (search.h:294-312).
void add_interval_starts(host_view const& tt, prepped_query const& p,
                         int32_t from, int32_t to, bool add_ontrip,
                         std::vector<start_label>& starts);
// interval_estimator::extension, interval_estimate.h:82-106
bool extend_interval(prepped_query const& p, int32_t ext_from, int32_t ext_to,
                     uint32_t num_con_req, int32_t& from, int32_t& to);

// A real-time overlay on the host: a copy of its description and the
// lookups rt_timetable keeps (the changed traffic days by transport,
// location_rt_transports_ in rt transport order, rt_timetable.cc:54-59).
struct rt_host {
  b2r_rt_desc d{};
  std::vector<uint32_t> changed_transport, stop_index, stops, static_transport;
  std::vector<uint64_t> changed_days;
  std::vector<int32_t> times;
  std::vector<uint16_t> static_day;
  std::vector<uint8_t> clasz, flags, section_flags;
  std::unordered_map<uint32_t, uint32_t> changed;  // transport -> row of changed_days
  std::vector<uint32_t> loc_idx, loc_rt;

  // copies d's arrays; false if d is malformed for a timetable of n_loc
  // locations and n_transports transports
  bool init(b2r_rt_desc const& src, uint32_t n_loc, uint32_t n_transports);
  uint32_t n_stops(uint32_t x) const { return stop_index[x + 1] - stop_index[x]; }
  uint32_t stop(uint32_t x, uint32_t i) const { return stops[stop_index[x] + i]; }
  int32_t event(uint32_t x, uint32_t i, bool arr) const {  // rt_timetable::unix_event_time
    return times[2ull * (stop_index[x] - x) + 2ull * i - (arr ? 1U : 0U)];
  }
};

// The flattened timetable as seen by host code (plain pointers), with the
// real-time overlay the searching engine is bound to, if any.
struct host_view {
  b2r_timetable_desc d;
  rt_host const* rt{nullptr};
  int32_t internal_from_days() const { return d.date_range_from - 5; }
};

// footpaths_out_[prf][l] (out) or footpaths_in_[prf][l] as [begin, end);
// empty for a profile without footpaths
inline std::pair<uint32_t const*, uint32_t const*> footpaths_at(b2r_timetable_desc const& d, uint32_t prf,
                                                                bool out, uint32_t l) {
  auto const* idx = prf == 0U ? (out ? d.footpaths_out_index : d.footpaths_in_index)
                              : (out ? d.profile_footpaths_out_index[prf - 1U] : d.profile_footpaths_in_index[prf - 1U]);
  auto const* dat = prf == 0U ? (out ? d.footpaths_out : d.footpaths_in)
                              : (out ? d.profile_footpaths_out[prf - 1U] : d.profile_footpaths_in[prf - 1U]);
  if (idx == nullptr) return {nullptr, nullptr};
  return {dat + idx[l], dat + idx[l + 1]};
}

// fwd / bwd_search_lb_graph_[prf][l]; empty for a profile without a graph
inline std::pair<uint32_t const*, uint32_t const*> lb_edges_at(b2r_timetable_desc const& d, uint32_t prf, bool fwd,
                                                               uint32_t l) {
  auto const* idx = prf == 0U ? (fwd ? d.lb_fwd_index : d.lb_bwd_index)
                              : (fwd ? d.profile_lb_fwd_index[prf - 1U] : d.profile_lb_bwd_index[prf - 1U]);
  auto const* dat = prf == 0U ? (fwd ? d.lb_fwd : d.lb_bwd)
                              : (fwd ? d.profile_lb_fwd[prf - 1U] : d.profile_lb_bwd[prf - 1U]);
  if (idx == nullptr) return {nullptr, nullptr};
  return {dat + idx[l], dat + idx[l + 1]};
}

// stop::in_allowed(p) / out_allowed(p), stop.h:44-49: the wheelchair bits
// for the wheelchair profile
inline bool stop_in(uint32_t w, uint32_t prf) {
  return prf == B2R_PROFILE_WHEELCHAIR ? B2R_STOP_IN_WC(w) != 0U : B2R_STOP_IN(w) != 0U;
}
inline bool stop_out(uint32_t w, uint32_t prf) {
  return prf == B2R_PROFILE_WHEELCHAIR ? B2R_STOP_OUT_WC(w) != 0U : B2R_STOP_OUT(w) != 0U;
}

}  // namespace b2r
