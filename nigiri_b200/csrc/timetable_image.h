// The device image of an uploaded timetable (b2r_timetable of the C ABI)
// together with the host copies the query preparation reads.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <vector>

#include "b2r.h"
#include "engine.cuh"
#include "prep.h"

struct b2r_timetable {
  int device{0};
  b2r_timetable_desc host{};  // pointers are NOT retained (sizes only)
  b2r::dev::dtt d{};
  std::vector<void*> allocs;
  uint64_t bytes{0};
  // host copies needed by the query preparation
  std::vector<uint8_t> transfer_time;
  std::vector<uint32_t> parent, children_index, children, fp_out_index, fp_out, fp_in_index,
      fp_in, route_stop_index, route_stops, route_transport_from, route_transport_to,
      route_stop_time_from, transport_traffic_days, route_traffic_days, location_routes_index,
      location_routes, lb_fwd_index, lb_fwd, lb_bwd_index, lb_bwd, transport_route;
  std::vector<uint8_t> location_type, route_clasz, route_flags, route_section_flags;
  std::vector<uint16_t> route_stop_times;
  std::vector<uint64_t> bitfields;
  // footpath profiles 1..4: footpaths (out, in) and lower-bound graphs
  // (fwd, bwd), CSR index then words, empty when the profile has none
  struct profile_copy {
    std::vector<uint32_t> lists[8];
  };
  profile_copy profiles[B2R_N_PROFILES - 1];
  b2r::host_view view{};
  // all-pairs lower-bound tables [source][location] (u16 minutes, 0xFFFF
  // unreachable) for forward and backward searches, built by the first
  // engine that uses them
  uint16_t* lb_table[2]{nullptr, nullptr};
  uint32_t lb_stride{0};  // row length: n_locations rounded up to a multiple of 8
  std::mutex lb_table_mutex;

  ~b2r_timetable() {
    for (auto* p : allocs) cudaFree(p);
  }
};
