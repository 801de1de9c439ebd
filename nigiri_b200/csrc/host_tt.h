// Host-side flattened timetable (owning std::vector storage) and the
// derivations nigiri's loader performs in finalize():
//   footpaths_in, location_routes      (gtfs/load_timetable.cc:405-415)
//   route traffic days                  (loader/init_finish.cc:168-198)
//   lower-bound graphs                  (loader/build_lb_graph.h:11-99)
//   location importance                 (loader/init_finish.cc:64-102)
// This is timetable construction, not the routing hot path.
#pragma once

#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "b2r.h"

namespace b2r {

struct host_timetable {
  uint32_t n_locations{0}, n_routes{0}, n_transports{0};
  int32_t date_range_from{0}, date_range_to{0};

  std::vector<uint8_t> transfer_time;
  std::vector<uint32_t> parent;
  std::vector<uint8_t> location_type;
  std::vector<uint32_t> children_index, children;
  std::vector<uint32_t> importance;
  uint32_t max_importance{0};
  std::vector<uint32_t> fp_out_index, fp_out, fp_in_index, fp_in;

  std::vector<uint32_t> route_stop_index, route_stops;
  std::vector<uint8_t> route_clasz;
  // per route: bit 2f = flag f on all sections, 2f+1 = on some sections;
  // per route stop index (section s -> s+1): the flag bits of that section
  std::vector<uint8_t> route_flags, route_section_flags;
  std::vector<uint32_t> route_transport_from, route_transport_to;
  std::vector<uint32_t> route_stop_time_from;
  std::vector<uint16_t> route_stop_times;
  std::vector<uint32_t> route_traffic_days, transport_traffic_days,
      transport_route;
  std::vector<uint64_t> bitfields;  // n_bitfields * 8
  std::vector<uint32_t> location_routes_index, location_routes;
  std::vector<uint32_t> lb_fwd_index, lb_fwd, lb_bwd_index, lb_bwd;
  // footpath profiles 1..4 at index p - 1: footpaths (out as given, in
  // derived) and their lower-bound graphs; empty vectors: no footpaths
  struct profile {
    std::vector<uint32_t> fp_out_index, fp_out, fp_in_index, fp_in;
    std::vector<uint32_t> lb_fwd_index, lb_fwd, lb_bwd_index, lb_bwd;
  };
  std::array<profile, B2R_N_PROFILES - 1> profiles;

  // generator metadata (coordinates in metres, for query generation)
  std::vector<float> x, y;
  // feed identifiers of a loaded feed (GTFS stop_id per location, the
  // display name of each transport), empty for generated timetables
  std::vector<std::string> location_ids, transport_names;

  uint32_t n_bitfields() const {
    return static_cast<uint32_t>(bitfields.size() / 8U);
  }
  b2r_timetable_desc desc() const;
};

// Computes every derived array from the base arrays already present in t
// (locations, footpaths_out, routes, route_stop_times, transport bitfields).
void finalize(host_timetable& t);

// Synthetic workloads 1..5 (see generator.cc for the exact definitions).
host_timetable generate(uint32_t config, uint64_t seed);

bool save(host_timetable const& t, std::string const& path);
bool load(std::string const& path, host_timetable& t);

}  // namespace b2r

// the C ABI's host timetable handle
struct b2r_host_timetable {
  b2r::host_timetable t;
};
