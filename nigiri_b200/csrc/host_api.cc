// C-ABI for host-side timetable construction and query generation.
#include <cstring>
#include <exception>
#include <new>
#include <string>

#include "b2r.h"
#include "errors.h"
#include "host_tt.h"
#include "queries.h"


struct b2r_query_set {
  b2r::query_set s;
};

namespace b2r {
thread_local std::string g_last_error;
void set_error(std::string msg) { g_last_error = std::move(msg); }
}  // namespace b2r

extern "C" {

const char* b2r_last_error(void) { return b2r::g_last_error.c_str(); }

void b2r_query_init(b2r_query* q) {
  std::memset(q, 0, sizeof(*q));
  q->kind = B2R_ONE_TO_ONE;
  q->direction = B2R_FORWARD;
  q->start_match_mode = B2R_MATCH_EXACT;
  q->dest_match_mode = B2R_MATCH_EXACT;
  q->max_start_offset = B2R_MAX_TRAVEL_TIME_MIN;
  q->max_transfers = B2R_MAX_TRANSFERS;
  q->max_travel_time = B2R_MAX_TRAVEL_TIME_MIN;
  q->fastest_direct_factor = 1.0;
  q->tts_default = 1;
  q->tts_factor = 1.0F;
  q->allowed_claszes = B2R_ALL_CLASZ;
}

void b2r_engine_config_init(b2r_engine_config* c) {
  std::memset(c, 0, sizeof(*c));
  c->max_slots = 1024;
  c->hbm_budget = 64ull << 30;
  c->max_journeys = 128;
  c->host_threads = 0;
  c->use_lower_bounds = 3;
  c->use_graphs = 1;
  c->route_block = 4;
}

int b2r_tt_generate(uint32_t config, uint64_t seed, b2r_host_timetable** out) {
  B2R_API_GUARD({
    if (out == nullptr || config < 1 || config > 5) {
      return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "b2r_tt_generate: bad args");
    }
    auto* h = new b2r_host_timetable{};
    h->t = b2r::generate(config, seed);
    *out = h;
    return B2R_OK;
  });
}

int b2r_tt_build(const b2r_tt_base* b, b2r_host_timetable** out) {
  B2R_API_GUARD({
    if (b == nullptr || out == nullptr) {
      return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "b2r_tt_build: null");
    }
    auto* h = new b2r_host_timetable{};
    auto& t = h->t;
    t.n_locations = b->n_locations;
    t.date_range_from = b->date_range_from;
    t.date_range_to = b->date_range_to;
    t.transfer_time.assign(b->transfer_time, b->transfer_time + b->n_locations);
    if (b->parent != nullptr) t.parent.assign(b->parent, b->parent + b->n_locations);
    if (b->location_type != nullptr) {
      t.location_type.assign(b->location_type, b->location_type + b->n_locations);
    }
    t.fp_out_index.assign(b->footpaths_out_index,
                          b->footpaths_out_index + b->n_locations + 1);
    t.fp_out.assign(b->footpaths_out,
                    b->footpaths_out + b->footpaths_out_index[b->n_locations]);
    for (auto p = 0U; p != B2R_N_PROFILES - 1U; ++p) {
      if (b->profile_footpaths_out_index[p] == nullptr) continue;
      auto const* idx = b->profile_footpaths_out_index[p];
      auto& x = t.profiles[p];
      x.fp_out_index.assign(idx, idx + b->n_locations + 1);
      auto ok = b->profile_footpaths_out[p] != nullptr || idx[b->n_locations] == 0U;
      for (auto l = 0U; ok && l != b->n_locations; ++l) ok = idx[l] <= idx[l + 1];
      if (ok && idx[b->n_locations] != 0U) {
        x.fp_out.assign(b->profile_footpaths_out[p], b->profile_footpaths_out[p] + idx[b->n_locations]);
        for (auto const fp : x.fp_out) ok = ok && B2R_FP_TARGET(fp) < b->n_locations;
      }
      if (!ok) {
        delete h;
        return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "b2r_tt_build: malformed profile footpaths");
      }
    }
    t.n_routes = b->n_routes;
    t.route_stop_index.assign(b->route_stop_index, b->route_stop_index + b->n_routes + 1);
    t.route_stops.assign(b->route_stops, b->route_stops + b->route_stop_index[b->n_routes]);
    if (b->route_clasz != nullptr) {
      for (auto r = 0U; r != b->n_routes; ++r) {
        if (b->route_clasz[r] >= 16U) {  // clasz::kNumClasses (types.h:394-412)
          delete h;
          return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "b2r_tt_build: route_clasz out of range (0..15)");
        }
      }
      t.route_clasz.assign(b->route_clasz, b->route_clasz + b->n_routes);
    }
    if (b->route_flags != nullptr) {
      t.route_flags.assign(b->route_flags, b->route_flags + b->n_routes);
    }
    if (b->route_section_flags != nullptr) {
      t.route_section_flags.assign(b->route_section_flags,
                                   b->route_section_flags + b->route_stop_index[b->n_routes]);
    }
    t.route_transport_from.resize(b->n_routes);
    t.route_transport_to.resize(b->n_routes);
    t.route_stop_time_from.resize(b->n_routes);
    uint32_t n_t = 0;
    uint64_t st = 0;
    for (auto r = 0U; r != b->n_routes; ++r) {
      auto const n_stops = b->route_stop_index[r + 1] - b->route_stop_index[r];
      t.route_transport_from[r] = n_t;
      n_t += b->route_n_transports[r];
      t.route_transport_to[r] = n_t;
      t.route_stop_time_from[r] = static_cast<uint32_t>(st);
      st += static_cast<uint64_t>(b->route_n_transports[r]) * 2U * (n_stops - 1U);
    }
    t.route_stop_times.assign(b->route_stop_times, b->route_stop_times + st);
    t.transport_traffic_days.assign(b->transport_bitfield, b->transport_bitfield + n_t);
    t.bitfields.assign(b->bitfields, b->bitfields + 8ull * b->n_bitfields);
    b2r::finalize(t);
    *out = h;
    return B2R_OK;
  });
}

int b2r_tt_save(const b2r_host_timetable* t, const char* path) {
  B2R_API_GUARD({
    if (t == nullptr || path == nullptr || !b2r::save(t->t, path)) {
      return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "b2r_tt_save failed");
    }
    return B2R_OK;
  });
}

int b2r_tt_load(const char* path, b2r_host_timetable** out) {
  B2R_API_GUARD({
    auto* h = new b2r_host_timetable{};
    if (path == nullptr || !b2r::load(path, h->t)) {
      delete h;
      return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "b2r_tt_load failed");
    }
    *out = h;
    return B2R_OK;
  });
}

int b2r_tt_desc(const b2r_host_timetable* t, b2r_timetable_desc* out) {
  if (t == nullptr || out == nullptr) {
    return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "b2r_tt_desc: null");
  }
  *out = t->t.desc();
  return B2R_OK;
}

int b2r_tt_destroy(b2r_host_timetable* t) {
  delete t;
  return B2R_OK;
}

int b2r_queries_generate(const b2r_host_timetable* t, uint32_t config,
                         uint64_t seed, uint32_t n, b2r_query_set** out) {
  B2R_API_GUARD({
    if (t == nullptr || out == nullptr) {
      return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "b2r_queries_generate: null");
    }
    auto* s = new b2r_query_set{};
    s->s = b2r::make_queries(t->t, config, seed, n);
    *out = s;
    return B2R_OK;
  });
}

uint32_t b2r_queries_count(const b2r_query_set* s) {
  return s == nullptr ? 0U : static_cast<uint32_t>(s->s.queries.size());
}

const b2r_query* b2r_queries_get(const b2r_query_set* s, uint32_t i) {
  if (s == nullptr || i >= s->s.queries.size()) return nullptr;
  return &s->s.queries[i];
}

int b2r_queries_destroy(b2r_query_set* s) {
  delete s;
  return B2R_OK;
}

}  // extern "C"
