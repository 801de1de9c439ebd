#pragma once

#include <vector>

#include "b2r.h"

namespace b2r {

struct host_timetable;

struct query_offsets {
  std::vector<b2r_offset> start, dest;
};

struct query_set {
  std::vector<b2r_query> queries;
  std::vector<query_offsets> offsets;
};

query_set make_queries(host_timetable const& t, uint32_t config, uint64_t seed,
                       uint32_t n);

}  // namespace b2r
