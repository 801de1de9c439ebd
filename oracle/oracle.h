/*
 * oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of nigiri's RAPTOR search path, used as the parity
 * checker of the B200 engine and as the timed CPU baseline.  Nothing in the
 * product (nigiri_b200/) links or calls this code; only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * The restatement follows (paths relative to the nigiri source tree):
 *   include/nigiri/routing/raptor/raptor.h:56-489, 680-845, 954-1062,
 *     1177-1486   (raptor<Dir, false, 0, kOneToOne|kOneToAll>)
 *   include/nigiri/routing/search.h:84-494        (search<Dir, raptor>)
 *   src/routing/start_times.cc:40-353              (get_starts, dests)
 *   src/routing/dijkstra.cc:18-67, dijkstra.h:31-70 (lower bounds)
 *   src/routing/get_fastest_direct.cc:12-100
 *   include/nigiri/routing/interval_estimate.h:12-151
 *   src/routing/raptor/reconstruct.cc:22-160, 162-877 (Vias = 0)
 *   raptor.h:1068-1175 (update_rt_transport), rt branches of raptor.h,
 *     start_times.cc:40-215 and reconstruct.cc:297-452 (Rt = true)
 *   src/routing/raptor/optimize_footpaths.cc:15-457
 *   src/routing/one_to_all.cc:26-104
 *   include/nigiri/routing/pareto_set.h:21-37, journey.h:84-118
 * Parity is pinned by the reference's golden journey printouts
 * (tests/golden/, generated by tests/golden/make_fixtures.py).
 */
#ifndef B2R_ORACLE_H_
#define B2R_ORACLE_H_

#include "b2r.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_result or_result;

/* Per-query work counters (raptor_stats.h:9-52 plus the byte model). */
typedef struct or_stats {
  uint64_t n_rounds;
  uint64_t n_start_times;
  uint64_t n_routes_visited;
  uint64_t n_route_stops_visited;
  uint64_t n_et_calls;
  uint64_t n_et_days;
  uint64_t n_et_events;
  uint64_t n_label_writes;
  uint64_t n_marked_stations;      /* route marking phase */
  uint64_t n_location_routes_read; /* route marking phase */
  uint64_t n_fp_stations;          /* transfer/footpath phase */
  uint64_t n_footpaths_visited;
  uint64_t n_sweep_locations;
  uint64_t algorithmic_bytes; /* byte model of the hot path */
} or_stats;

/* Run one query exactly as raptor_search / one_to_all would. */
int or_search(const b2r_timetable_desc* tt, const b2r_query* q,
              or_result** out);
/* The same with a real-time overlay (raptor<Dir, Rt = true>, the rt
 * branches of start_times.cc and reconstruct.cc); rt may be NULL. */
int or_search_rt(const b2r_timetable_desc* tt, const b2r_rt_desc* rt,
                 const b2r_query* q, or_result** out);
int or_result_view(const or_result* r, b2r_result* view, or_stats* stats);
/* Final raptor_state: round_times [B2R_K][n_locations] and best
 * [n_locations] as int16 deltas (for state-level parity). */
int or_result_state(const or_result* r, const int16_t** round_times,
                    const int16_t** best, int32_t* base_day);
void or_result_free(or_result* r);

/* Start labels of a query (get_starts + the search's sort), for the
 * start_times known-answer tests: arrays of n entries. */
int or_get_starts(const b2r_timetable_desc* tt, const b2r_query* q,
                  int32_t* time_at_start, int32_t* time_at_stop,
                  uint32_t* stop, uint32_t capacity, uint32_t* n);

/* Dijkstra lower bounds of a query (dists[n_locations]). */
int or_lower_bounds(const b2r_timetable_desc* tt, const b2r_query* q,
                    uint16_t* dists);

/* Timed CPU baseline: run n queries on `threads` host threads (one query
 * per thread at a time, pulled from an atomic counter like
 * exe/benchmark.cc:209-270).  latencies_us[n] receives per-query times. */
int or_run_many(const b2r_timetable_desc* tt, const b2r_query* qs, uint32_t n,
                uint32_t threads, double* latencies_us, uint64_t* journeys,
                double* wall_s);

#ifdef __cplusplus
}
#endif

#endif
