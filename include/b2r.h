/*
 * b2r.h -- C ABI of the B200 RAPTOR engine (drop-in behind nigiri's routing
 * seam).
 *
 * Everything crosses this boundary as plain pointers, sizes and PODs; every
 * entry point returns an int status (B2R_OK == 0, negative on error) and never
 * throws.  The last error message of the calling thread is available through
 * b2r_last_error().
 *
 * Reference seam being replaced (paths relative to the nigiri source tree):
 *  - routing::raptor_search(tt, rtt, search_state&, AlgoState&, query, dir)
 *      src/routing/raptor_search.cc:94-159, instantiated for raptor_state and
 *      gpu::gpu_raptor_state at src/routing/raptor_search.cc:161-177
 *  - the Algo concept driven by routing::search<Dir, Algo>
 *      include/nigiri/routing/search.h:148-171 (construction),
 *      search.h:436-475 (next_start_time / add_start / execute / reconstruct)
 *  - routing::one_to_all<Dir>  src/routing/one_to_all.cc:52-104
 *  - routing::gpu::gpu_timetable / gpu_raptor_state (device image + state)
 *      include/nigiri/routing/gpu/raptor.h:23-129
 *
 * Time conventions follow nigiri: unixtime = int32 minutes since 1970-01-01
 * (unixtime_t, include/nigiri/types.h:360); days = int32 days since
 * 1970-01-01 (date::sys_days); round times are int16 minutes relative to a
 * per-query base day (delta_t, include/nigiri/common/delta_t.h:11-59).
 */
#ifndef B2R_H_
#define B2R_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum b2r_status {
  B2R_OK = 0,
  B2R_ERR_INVALID_ARGUMENT = -1,
  B2R_ERR_CUDA = -2,
  B2R_ERR_OUT_OF_MEMORY = -3, /* HBM budget or device allocation exhausted */
  B2R_ERR_CAPACITY = -4,      /* a per-query fixed-size buffer overflowed */
  B2R_ERR_NOT_READY = -5,     /* b2r_poll: ticket still running */
  B2R_ERR_DEVICE_STATUS = -6, /* a kernel wrote an error status word */
  B2R_ERR_UNSUPPORTED = -7,
  B2R_ERR_INTERNAL = -8
};

/* Message of the last failing call on this thread ("" if none). */
const char* b2r_last_error(void);

/* ------------------------------------------------------- constants */
#define B2R_MAX_TRANSFERS 14 /* routing/limits.h:9 kMaxTransfers */
#define B2R_K 16             /* kMaxTransfers + 2 round rows */
#define B2R_MAX_TRAVEL_TIME_MIN 7200 /* routing/limits.h:10 kMaxTravelTime */
#define B2R_MAX_DAYS 512             /* types.h:62 kMaxDays */
#define B2R_TIMETABLE_OFFSET_DAYS 5  /* types.h:53 kTimetableOffset */
#define B2R_N_SPECIAL_STATIONS 9     /* special_stations.h:7-19 */
#define B2R_SPECIAL_START 0u
#define B2R_SPECIAL_END 1u
#define B2R_INVALID_IDX 0xFFFFFFFFu
#define B2R_UNREACHABLE 0xFFFFu

/* Route flags (types.h:417-423 route_flag) and the all-classes mask
 * (routing/clasz_mask.h:13-25: bit c = transport class c allowed). */
#define B2R_FLAG_BIKES 0u
#define B2R_FLAG_CARS 1u
#define B2R_FLAG_WHEELCHAIR 2u
#define B2R_FLAG_RESERVATION_NOT_REQUIRED 3u
#define B2R_ALL_CLASZ 0xFFFFFFFFu

/* Footpath profiles (types.h:204-210 profile_idx_t): profile 0 is the
 * timetable's own footpaths; profile 2 (wheelchair) also boards and alights
 * by the stops' wheelchair bits and needs wheelchair-accessible routes. */
#define B2R_N_PROFILES 5u
#define B2R_PROFILE_DEFAULT 0u
#define B2R_PROFILE_FOOT 1u
#define B2R_PROFILE_WHEELCHAIR 2u
#define B2R_PROFILE_CAR 3u
#define B2R_PROFILE_BIKE 4u

/* Search algorithms (b2r_query::algorithm). */
#define B2R_ALGO_RAPTOR 0u
#define B2R_ALGO_PONG 1u

/* Location types used by location_match_mode::kIntermodal
 * (for_each_meta.h:29-35 reads kGeneratedTrack children). */
#define B2R_LOC_STATION 0u
#define B2R_LOC_TRACK 1u
#define B2R_LOC_GENERATED_TRACK 2u

/* Packed words, bit-identical to nigiri's:
 *  stop      (stop.h:86-89):      location:28 | in:1 | out:1 | in_wc:1 | out_wc:1
 *  footpath  (footpath.h:81-82):  target:23 | duration:9
 *  delta     (types.h:619-620):   days:5 | mam:11 (days in the low bits) */
#define B2R_STOP_LOC(w) ((w)&0x0FFFFFFFu)
#define B2R_STOP_IN(w) (((w) >> 28) & 1u)
#define B2R_STOP_OUT(w) (((w) >> 29) & 1u)
#define B2R_STOP_IN_WC(w) (((w) >> 30) & 1u)
#define B2R_STOP_OUT_WC(w) (((w) >> 31) & 1u)
#define B2R_FP_TARGET(w) ((w)&0x7FFFFFu)
#define B2R_FP_DURATION(w) ((w) >> 23)
#define B2R_DELTA_DAYS(d) ((int)((d)&0x1Fu))
#define B2R_DELTA_MAM(d) ((int)((d) >> 5))

/* ------------------------------------------------------- timetable image */
/*
 * Flattened timetable: the arrays the RAPTOR hot path reads
 * (timetable.h:341-398, locations_ 89-98).  CSR pairs are (index[n+1], data).
 * All pointers are host memory owned by the caller; b2r_timetable_upload
 * copies them into one device-resident image.
 */
typedef struct b2r_timetable_desc {
  uint32_t n_locations; /* incl. the 9 special stations at 0..8 */
  uint32_t n_routes;
  uint32_t n_transports;
  uint32_t n_bitfields;
  int32_t date_range_from; /* days since epoch, timetable::date_range_.from_ */
  int32_t date_range_to;   /* days since epoch, exclusive */

  /* locations */
  const uint8_t* transfer_time;   /* [n_locations] minutes (u8_minutes) */
  const uint32_t* parent;         /* [n_locations] or NULL (no parents) */
  const uint8_t* location_type;   /* [n_locations] or NULL (all stations) */
  const uint32_t* children_index; /* CSR or NULL */
  const uint32_t* children;
  const uint32_t* importance; /* [n_locations] or NULL (assign_importance) */
  uint32_t max_importance;
  const uint32_t* footpaths_out_index; /* CSR, footpaths_out_[0] */
  const uint32_t* footpaths_out;
  const uint32_t* footpaths_in_index; /* CSR, footpaths_in_[0] */
  const uint32_t* footpaths_in;

  /* routes */
  const uint32_t* route_stop_index; /* CSR route_location_seq_ */
  const uint32_t* route_stops;
  const uint32_t* route_transport_from; /* [n_routes] first transport */
  const uint32_t* route_transport_to;   /* [n_routes] one past last */
  const uint32_t* route_stop_time_from; /* [n_routes] route_stop_time_ranges_ */
  const uint16_t* route_stop_times;     /* packed delta */
  uint64_t n_route_stop_times;
  const uint32_t* route_traffic_days;     /* [n_routes] bitfield index */
  const uint32_t* transport_traffic_days; /* [n_transports] bitfield index */
  const uint32_t* transport_route;        /* [n_transports] */
  const uint64_t* bitfields;              /* [n_bitfields * 8] 512-bit sets */
  const uint32_t* location_routes_index;  /* CSR location_routes_ */
  const uint32_t* location_routes;

  /* lower-bound graphs (build_lb_graph.h:11-99), packed footpath words */
  const uint32_t* lb_fwd_index;
  const uint32_t* lb_fwd;
  const uint32_t* lb_bwd_index;
  const uint32_t* lb_bwd;

  /* route filters (timetable.h:348-361): class per route, and per route flag
   * f (B2R_FLAG_*) bit 2f = set on all sections, bit 2f+1 = set on some
   * (route_flags_), plus per section s of route r the flag bits at
   * route_section_flags[route_stop_index[r] + s] (route_flags_per_section_).
   * NULL: class 0, no flags. */
  const uint8_t* route_clasz;
  const uint8_t* route_flags;
  const uint8_t* route_section_flags;

  /* profiles 1..4 at index p - 1 (timetable.h:97-98 footpaths_out_[p] /
   * footpaths_in_[p], :421-422 fwd / bwd_search_lb_graph_[p]), in the
   * layout of profile 0's arrays above.  NULL: the profile has no footpaths
   * (and, for the lower-bound graphs, no graph). */
  const uint32_t* profile_footpaths_out_index[B2R_N_PROFILES - 1];
  const uint32_t* profile_footpaths_out[B2R_N_PROFILES - 1];
  const uint32_t* profile_footpaths_in_index[B2R_N_PROFILES - 1];
  const uint32_t* profile_footpaths_in[B2R_N_PROFILES - 1];
  const uint32_t* profile_lb_fwd_index[B2R_N_PROFILES - 1];
  const uint32_t* profile_lb_fwd[B2R_N_PROFILES - 1];
  const uint32_t* profile_lb_bwd_index[B2R_N_PROFILES - 1];
  const uint32_t* profile_lb_bwd[B2R_N_PROFILES - 1];
} b2r_timetable_desc;

/* ------------------------------------------------------------- queries */
enum b2r_direction { B2R_FORWARD = 0, B2R_BACKWARD = 1 };
enum b2r_match_mode { /* location_match_mode.h:5-10 */
  B2R_MATCH_EXACT = 0,
  B2R_MATCH_ONLY_CHILDREN = 1,
  B2R_MATCH_EQUIVALENT = 2,
  B2R_MATCH_INTERMODAL = 3
};
enum b2r_query_kind {
  B2R_ONE_TO_ONE = 0, /* search<Dir, raptor<..., kOneToOne>> */
  B2R_ONE_TO_ALL = 1  /* one_to_all<Dir> */
};

/* routing::offset, query.h:28-48 */
typedef struct b2r_offset {
  uint32_t target;
  int16_t duration; /* minutes */
  int16_t pad_;
  int32_t transport_mode_id;
} b2r_offset;

/* routing::query, query.h:70-100, restricted to the static (no rtt, no
 * vias, no td offsets) instantiation. */
typedef struct b2r_query {
  uint8_t kind;      /* b2r_query_kind */
  uint8_t direction; /* b2r_direction */
  uint8_t is_interval;
  uint8_t start_match_mode;
  uint8_t dest_match_mode;
  uint8_t use_start_footpaths;
  uint8_t extend_interval_earlier;
  uint8_t extend_interval_later;
  int32_t start_time;    /* ontrip start (unixtime) */
  int32_t interval_from; /* pretrip start interval [from, to) */
  int32_t interval_to;
  const b2r_offset* start;
  uint32_t n_start;
  const b2r_offset* destination;
  uint32_t n_destination;
  int16_t max_start_offset; /* default 7200 */
  uint8_t max_transfers;    /* default 14 */
  uint8_t has_fastest_direct;
  int16_t max_travel_time; /* default 7200 */
  int16_t fastest_direct;
  uint32_t min_connection_count;
  double fastest_direct_factor; /* default 1.0 */
  /* transfer_time_settings, transfer_time_settings.h:8-18 */
  uint8_t tts_default; /* 1 = identity */
  uint8_t pad_[3];
  int16_t tts_min_transfer_time;
  int16_t tts_additional_time;
  float tts_factor;
  /* filters (query.h:91-94): allowed transport classes, and routes / sections
   * that must carry bikes, carry cars, need no reservation */
  uint32_t allowed_claszes; /* default B2R_ALL_CLASZ */
  uint8_t require_bike_transport;
  uint8_t require_car_transport;
  uint8_t no_compulsory_reservation;
  /* B2R_ALGO_RAPTOR: routing::raptor_search (search<raptor>, raptor_search.cc);
   * B2R_ALGO_PONG: routing::pong_search (pong.cc:63-475), one-to-one only */
  uint8_t algorithm;
  /* query::max_interval_ (query.h:89): when set, every search interval the
   * interval estimator produces (interval_estimate.h:138-146) is clamped
   * into [max_interval_from, max_interval_to] (unixtime minutes) */
  uint8_t has_max_interval;
  /* query::prf_idx_ (query.h:90): footpaths, lower bounds and -- for
   * B2R_PROFILE_WHEELCHAIR -- stop and route accessibility of the profile */
  uint8_t prf_idx;
  uint8_t pad2_[2];
  int32_t max_interval_from;
  int32_t max_interval_to;
} b2r_query;

/* Fill a query with nigiri's defaults (query.h:84-99). */
void b2r_query_init(b2r_query* q);

/* ------------------------------------------------------------- results */
enum b2r_leg_kind {
  B2R_LEG_TRANSPORT = 0, /* journey::run_enter_exit */
  B2R_LEG_FOOTPATH = 1,  /* footpath */
  B2R_LEG_OFFSET = 2     /* routing::offset (first / last mile) */
};

/* journey::leg, journey.h:42-82 */
typedef struct b2r_leg {
  uint32_t from;
  uint32_t to;
  int32_t dep_time; /* unixtime */
  int32_t arr_time;
  uint8_t kind;
  uint8_t pad_;
  uint16_t day;        /* transport: traffic day index */
  uint32_t transport;  /* transport idx | footpath/offset target */
  uint16_t stop_from;  /* transport: stop_range_ [from, to) */
  uint16_t stop_to;
  int16_t duration;    /* footpath / offset duration */
  int16_t pad2_;
  int32_t transport_mode_id; /* offset */
  uint32_t rt_transport;     /* transport: the real-time run ridden
                                (rt::run::rt_), B2R_INVALID_IDX for a static
                                one; `transport` and `day` then name the
                                static trip it runs for, B2R_INVALID_IDX for
                                an added trip */
} b2r_leg;

/* journey, journey.h:84-118 */
typedef struct b2r_journey {
  int32_t start_time;
  int32_t dest_time;
  uint32_t dest;
  uint8_t transfers;
  uint8_t error;
  uint16_t n_legs;
  uint32_t first_leg; /* index into the result's leg array */
} b2r_journey;

/* Per-query result.  journeys/legs point into engine-owned memory valid
 * until the next call on the same engine (or b2r_result_release). */
typedef struct b2r_result {
  int32_t status; /* B2R_OK or an error for this query alone */
  uint32_t n_journeys;
  const b2r_journey* journeys;
  const b2r_leg* legs;
  int32_t interval_from; /* routing_result::interval_ */
  int32_t interval_to;
  /* one_to_all: round_times rows k = 0..n_rows-1, each n_locations int16
   * deltas relative to base_day (raptor_state::round_times_). */
  uint32_t n_rows;
  int32_t base_day; /* days since epoch */
  const int16_t* round_times;
  /* counters (raptor_stats) */
  uint64_t n_rounds;
  uint64_t n_start_times;
  /* time from the batch call to this query's completion (host clock) */
  double latency_ms;
} b2r_result;

/* ---------------------------------------------------------------- engine */
typedef struct b2r_timetable b2r_timetable; /* device image handle */
typedef struct b2r_engine b2r_engine;       /* state pool + streams */

/* Upload the flattened timetable once; the handle owns the device copy. */
int b2r_timetable_upload(const b2r_timetable_desc* desc, int device,
                         b2r_timetable** out);
int b2r_timetable_destroy(b2r_timetable* tt);
/* Device bytes held by the image. */
uint64_t b2r_timetable_device_bytes(const b2r_timetable* tt);

/* Largest all-pairs lower-bound tables an engine builds (both directions):
 * 16 GiB, i.e. up to 65,536 locations. */
#define B2R_LB_TABLE_MAX_BYTES (16ull << 30)

typedef struct b2r_engine_config {
  uint32_t max_slots;       /* queries resident at once (multiple of 32) */
  uint64_t hbm_budget;      /* bytes of raptor state the pool may hold */
  uint32_t max_journeys;    /* per-query pareto set capacity (default 128) */
  uint32_t host_threads;    /* host prep threads (0 = hardware) */
  uint32_t use_lower_bounds;/* Dijkstra lower bounds for target pruning
                               (raptor.h:33 kUseLowerBounds): 0 = off (lb = 0,
                               like nigiri's GPU raptor), 1 = on the host,
                               2 = solved on the device, 3 = from all-pairs
                               tables on the device (default; built once per
                               timetable on the host threads, 2 * n_locations^2
                               * 2 bytes; falls back to 0 above
                               B2R_LB_TABLE_MAX_BYTES, where the host
                               Dijkstra would cost more than the pruning
                               saves).  Journeys are the same in every mode. */
  uint32_t use_graphs;      /* 1 = capture the super-step in a CUDA graph */
  uint32_t route_block;     /* launch shape: warps per CTA in the route scan */
  uint32_t max_starts;      /* start labels per query (default 4096) */
  uint32_t steps_per_sync;  /* super-steps between host checks (default 4) */
  uint32_t profile;         /* 1 = time route scans with CUDA events around
                               every launch and count their work (a
                               counting build of the scan; no graphs);
                               2 = time them only: the build the launch
                               shape selects, events inside the super-step
                               graph, one super-step per host check */
  uint32_t reserved[4];
} b2r_engine_config;

void b2r_engine_config_init(b2r_engine_config* c);

/* Create an engine bound to one timetable image.  Admission is bounded by
 * cfg->hbm_budget: the slot count is min(max_slots, budget / bytes_per_slot). */
int b2r_engine_create(b2r_timetable* tt, const b2r_engine_config* cfg,
                      b2r_engine** out);
int b2r_engine_destroy(b2r_engine* e);
/* Bytes of device state one resident query needs. */
uint64_t b2r_engine_bytes_per_slot(const b2r_engine* e);
uint32_t b2r_engine_slots(const b2r_engine* e);

/* Batched search: runs n queries (any mix of kinds and directions) through
 * the resident slot pool with continuous admission and blocks until all are
 * done.  out[i] receives query i's result. */
int b2r_search_batch(b2r_engine* e, const b2r_query* qs, uint32_t n,
                     b2r_result* out);

/* Plain engine: one query, per-round kernel launches from the host and a
 * synchronisation per query (the launch pattern of nigiri's
 * src/routing/gpu/raptor.cu:894-990).  Same results as b2r_search_batch. */
int b2r_search_plain(b2r_engine* e, const b2r_query* q, b2r_result* out);

/* One-to-all search of ONE query that allocates nothing.  This entry point
 * has no counterpart in the reference.
 *
 * For callers that cannot allocate device memory on the query path:
 * request handlers of a serving process whose device memory is owned by
 * another allocator (a framework's caching allocator, or a fixed pool that
 * reserves the HBM), and latency-critical paths that must not call
 * cudaMalloc / cudaFree because cudaFree synchronises the whole device and
 * stalls every other stream of the process (the batched engine included).
 * The call uses no engine, calls no cudaMalloc, cudaFree or other allocating
 * routine, and keeps its working state in one fixed device array of
 * B2R_NOALLOC_SCRATCH_BYTES that lives in the library.
 *
 * - q->kind must be B2R_ONE_TO_ALL.  The timetable may have at most
 *   B2R_NOALLOC_MAX_LOCATIONS locations and B2R_NOALLOC_MAX_ROUTES routes,
 *   the query at most B2R_NOALLOC_MAX_OFFSETS start offsets; larger inputs
 *   are rejected with B2R_ERR_CAPACITY and a message (b2r_last_error).
 * - round_times (host memory, capacity elements) receives n_rows rows of
 *   n_locations int16 deltas relative to *base_day, exactly the rows
 *   b2r_search_batch returns for the same query.
 *   n_rows = min(max_transfers, B2R_MAX_TRANSFERS) + 2.
 * - stream: a cudaStream_t on tt's device, or NULL for the default stream.
 *   The call returns when the rows are in round_times.
 * - Set-up: the first call on a device, with that device current, loads the
 *   library's device module (the driver reserves the scratch array then)
 *   and looks up the array's address; later calls reuse it.  Make the first
 *   call on each device before any stream capture.  The address is kept per
 *   device for the life of the process: a caller that resets a device
 *   (cudaDeviceReset) must not call this entry point on it again.
 * - Every call on a device shares the one scratch array: calls that overlap
 *   on the GPU (from two streams or two host threads) race and corrupt each
 *   other's results.  Issue them one at a time per device.
 * - A rejected call records its error message for b2r_last_error on the
 *   host heap; a call that succeeds touches no allocator. */
#define B2R_NOALLOC_MAX_LOCATIONS 65536u
#define B2R_NOALLOC_MAX_ROUTES 65536u
#define B2R_NOALLOC_MAX_OFFSETS 64u
#define B2R_NOALLOC_SCRATCH_BYTES (8388608u + 256u) /* 8 MiB + counters */
int b2r_one_to_all_noalloc(const b2r_timetable* tt, const b2r_query* q,
                           int16_t* round_times, uint64_t capacity,
                           uint32_t* n_rows, int32_t* base_day, void* stream);

/* ------------------------------------------------------------------------
 * Real-time overlay: what rt_timetable (include/nigiri/rt/rt_timetable.h:
 * 48-311) holds for routing, after the real-time updates are applied.
 * - Static transports whose service changed on some days get new traffic
 *   days (transport_traffic_days_ with kRtBitfieldFlag, bitfields_).
 * - Every delayed, rerouted or added run is an rt transport with its own
 *   stop sequence and event times (rt_transport_location_seq_,
 *   rt_transport_stop_times_), class and route flags
 *   (rt_transport_section_clasz_, rt_transport_flags_,
 *   rt_flags_per_section_).
 * An engine bound to an overlay (b2r_engine_set_rt) searches with it as
 * raptor<Dir, Rt = true> does: rt transports are marked from their stations
 * (raptor.h:228-241), scanned by update_rt_transport (raptor.h:1068-1175),
 * taken first by reconstruction (reconstruct.cc:381-452) and boarded by
 * interval start times (start_times.cc:177-215). */
typedef struct b2r_rt_desc {
  uint32_t n_changed;                /* static transports with new traffic days */
  const uint32_t* changed_transport; /* their indices */
  const uint64_t* changed_days;      /* n_changed x 8 words: their 512-bit days */
  uint32_t n_rt_transports;
  const uint32_t* rt_stop_index;     /* n_rt_transports + 1 */
  const uint32_t* rt_stops;          /* stop words (B2R_STOP_*) */
  const int32_t* rt_event_times;     /* per rt transport 2 (n_stops - 1) times,
                                        minutes since the epoch, in the order of
                                        rt_transport_stop_times_: departure at
                                        stop 0, arrival at stop 1, departure at
                                        stop 1, ..., arrival at the last stop;
                                        rt transport i starts at
                                        2 (rt_stop_index[i] - i) */
  const uint32_t* rt_static_transport; /* the static trip it runs for, or
                                          B2R_INVALID_IDX (added) */
  const uint16_t* rt_static_day;     /* that trip's traffic day index */
  const uint8_t* rt_clasz;           /* class of its first section; NULL: 10 */
  const uint8_t* rt_flags;           /* route flags as route_flags; NULL: none */
  const uint8_t* rt_section_flags;   /* per rt stop like route_section_flags;
                                        NULL: none */
} b2r_rt_desc;

typedef struct b2r_rt b2r_rt;
/* Uploads an overlay for timetable tt (the arrays are copied). */
int b2r_rt_upload(b2r_timetable* tt, const b2r_rt_desc* d, b2r_rt** out);
int b2r_rt_destroy(b2r_rt* rt);
/* Searches of this engine use the overlay from the next call on (NULL: the
 * static timetable).  The overlay must outlive the binding.  While one is
 * bound the engine prunes without lower bounds (lb = 0): the timetable's
 * bounds do not cover added runs, and bounds only prune, so the journeys
 * are the same. */
int b2r_engine_set_rt(b2r_engine* e, const b2r_rt* rt);

/* ------------------------------------------------------------------------
 * The Algo concept of routing::search<Dir, Algo>.
 *
 * nigiri's search<Dir, Algo> (search.h:78-505) prepares a query
 * (search::init, search.h:84-172: transfer-time normalisation, destination
 * set, lower bounds, base day; add_start_labels, search.h:401-411) and then
 * drives an Algo through reset_arrivals / next_start_time / add_start /
 * execute / reconstruct (raptor.h:56-73, 174-203, 205-414, 416-452).
 * b2r_search_prepare is that preparation on the host; b2r_raptor is the
 * Algo: one query's raptor_state resident on the device, each execute the
 * rounds of one start time.  Static timetable, no vias, no time-dependent
 * offsets. */
typedef struct b2r_start {     /* routing::start, start_times.h:21-26 */
  int32_t time_at_start;       /* minutes since the epoch */
  int32_t time_at_stop;
  uint32_t location;
} b2r_start;

typedef struct b2r_search_plan {
  int32_t status;              /* B2R_OK, or why the query cannot be searched */
  uint8_t direction;
  uint8_t ontrip;              /* start_time_ is a point in time */
  uint8_t start_dest_overlap;  /* search.h:354-378: the result is empty */
  uint8_t max_transfers;
  int32_t base_day;            /* days since the epoch (search.h:148-160) */
  int32_t interval_from, interval_to; /* search_interval_ after
                                         interval_estimator::initial */
  int16_t fastest_direct;      /* fastest_direct_ (minutes) */
  int16_t max_travel_time;     /* query::max_travel_time_ after sanitize */
  uint8_t tts_default;         /* transfer_time_settings after search::init */
  uint8_t pad2;
  int16_t tts_min_transfer_time, tts_additional_time;
  float tts_factor;
  uint32_t n_starts;           /* state_.starts_ in search order */
  const b2r_start* starts;
  uint32_t n_destinations;     /* is_destination_: set bits, ascending */
  const uint32_t* destinations;
  const uint16_t* dist_to_dest;/* n_locations entries (0xFFFF: none), or NULL
                                  for a station-to-station query */
  const uint16_t* lower_bounds;/* n_locations: travel_time_lower_bound_
                                  (0xFFFF: unreachable) */
} b2r_search_plan;

/* The host part of search::init for query q (raptor queries; q->kind
 * B2R_ONE_TO_ONE).  The plan owns its arrays; free it with
 * b2r_search_plan_free. */
int b2r_search_prepare(const b2r_timetable* tt, const b2r_query* q, b2r_search_plan** out);
void b2r_search_plan_free(b2r_search_plan* p);
/* One interval extension of search::execute (search.h:275-316): the search
 * interval grown for n_missing more results (interval_estimator::
 * extension), and plan->starts replaced by the start labels of the new
 * parts in search order.  *changed = 0: the interval cannot grow, the
 * search ends.  *reset_arrivals = 1: the Algo's arrivals are to be reset
 * and the results outside the old interval removed first
 * (remove_ontrip_results). */
int b2r_search_extend(const b2r_timetable* tt, b2r_search_plan* plan, uint32_t n_missing,
                      uint8_t* changed, uint8_t* reset_arrivals);

/* The Algo's constructor arguments (raptor.h:56-73), static instantiation:
 * no real-time overlay, no vias, no time-dependent offsets. */
typedef struct b2r_raptor_args {
  uint8_t direction;
  uint8_t prf_idx;             /* footpath profile; B2R_PROFILE_WHEELCHAIR
                                  is the reference's is_wheelchair */
  uint8_t require_bike_transport, require_car_transport;
  uint8_t no_compulsory_reservation;
  uint8_t tts_default;
  uint16_t allowed_claszes;    /* clasz_mask_t */
  int16_t tts_min_transfer_time, tts_additional_time;
  float tts_factor;
  int32_t base_day;            /* the base day, days since the epoch */
  uint32_t n_destinations;     /* is_dest: set bits */
  const uint32_t* destinations;
  const uint16_t* dist_to_dest;/* n_locations entries, or NULL */
  const uint16_t* lower_bounds;/* n_locations entries, or NULL: lb = 0 */
} b2r_raptor_args;

typedef struct b2r_raptor b2r_raptor;
/* A raptor state on tt's device with the constructor's arguments (copied).
 * One host thread at a time, like the reference's per-thread search
 * state. */
int b2r_raptor_create(b2r_timetable* tt, const b2r_raptor_args* args, b2r_raptor** out);
int b2r_raptor_destroy(b2r_raptor* r);
/* raptor::reset_arrivals (raptor.h:174-177): round times and
 * time_at_dest invalid before the next execute. */
int b2r_raptor_reset_arrivals(b2r_raptor* r);
/* raptor::next_start_time (raptor.h:179-188): best / tmp and the marks
 * reset, the start labels of the next execute start empty. */
int b2r_raptor_next_start_time(b2r_raptor* r);
/* raptor::add_start (raptor.h:190-203): a start label at location l at
 * time t (minutes since the epoch). */
int b2r_raptor_add_start(b2r_raptor* r, uint32_t location, int32_t time);
/* raptor::execute (raptor.h:205-414): the rounds from the start labels
 * added since next_start_time, then the journeys of every round that
 * reaches a destination, as the reference adds them to its pareto set
 * (start_time, dest_time, dest, transfers; no legs).  At most `capacity`
 * are written; *n receives their number (B2R_ERR_CAPACITY if more). */
int b2r_raptor_execute(b2r_raptor* r, int32_t start_time, uint8_t max_transfers,
                       int32_t worst_time_at_dest, b2r_journey* results,
                       uint32_t capacity, uint32_t* n);
/* raptor::reconstruct (raptor.h:416-452, reconstruct.cc:162-902): the legs
 * of journey j (its start_time, dest_time, dest and transfers) from the
 * round times of the last execute, for query q (offsets, match modes).
 * On success j->n_legs legs go to legs[0..] (capacity at least 40); a
 * journey the reference could not rebuild comes back with j->error = 1. */
int b2r_raptor_reconstruct(b2r_raptor* r, const b2r_query* q, b2r_journey* j,
                           b2r_leg* legs, uint32_t capacity);
/* Rounds run so far (raptor_stats::n_rounds_). */
uint64_t b2r_raptor_rounds(const b2r_raptor* r);

/* Serving: asynchronous submission.  Queries are admitted into free slots at
 * super-step boundaries by a driver thread; results are fetched by ticket. */
int b2r_serve_start(b2r_engine* e);
int b2r_serve_stop(b2r_engine* e);
int b2r_submit(b2r_engine* e, const b2r_query* q, uint64_t* ticket);
/* B2R_OK when done (result copied into *out, valid until b2r_release),
 * B2R_ERR_NOT_READY otherwise. */
int b2r_poll(b2r_engine* e, uint64_t ticket, b2r_result* out);
int b2r_wait(b2r_engine* e, uint64_t ticket, b2r_result* out);
int b2r_release(b2r_engine* e, uint64_t ticket);

/* Timing of the last b2r_search_batch: device milliseconds (CUDA events:
 * the union of the intervals in which super-step chunks and the
 * finished-slot kernels, deferred reconstruction and result export, ran;
 * host-only gaps between them are excluded), wall time of the call, and the
 * number of kernel launches issued (graph nodes included). */
typedef struct b2r_batch_stats {
  double device_ms;
  double host_prep_ms; /* wall time of the whole call */
  uint64_t kernel_launches;
  uint64_t super_steps;
  uint64_t route_scan_launches;
  double route_scan_ms;     /* summed CUDA-event time of the route scans
                               (profiling engines only) */
  uint64_t route_stop_visits; /* (route, query) stop steps scanned */
  uint64_t et_events;         /* event times examined by trip searches */
  uint64_t et_days;           /* service days examined by trip searches */
  uint64_t label_writes;      /* tmp label improvements */
  uint64_t route_scan_bytes;  /* algorithmic bytes of the route scans */
  double lb_ms;               /* wall time of device lower-bound solves */
  uint64_t lb_iterations;     /* solver iterations (8 per chunk) */
  uint64_t lb_relaxations;    /* improving edge relaxations */
  uint64_t h2d_bytes;         /* host->device bytes the call copied */
  uint64_t d2h_bytes;         /* device->host bytes the call copied */
  uint64_t route_warp_steps;  /* stop steps of route-scan warps (32 lanes
                                 each; profiling engines only) */
  double recon_ms;            /* summed CUDA-event time of the reconstruction
                                 launches (profiling engines only) */
  double recon_max_journey_us; /* longest single journey reconstruction */
  uint64_t recon_journeys;    /* journeys reconstructed */
  double host_prep_cpu_ms;    /* query preparation, summed over the workers */
  double host_admit_ms;       /* admission (staging + copies), driver thread */
  double host_export_ms;      /* export, finalisation and retirement */
  double host_idle_ms;        /* driver waiting for preparation, no slot busy */
} b2r_batch_stats;
int b2r_last_batch_stats(const b2r_engine* e, b2r_batch_stats* s);
/* Counters of the serving loop since b2r_serve_start (the engine's current
 * or last serving run): super_steps and kernel_launches run, and host
 * milliseconds spent admitting (host_admit_ms), exporting, finalising and
 * retiring finished slots (host_export_ms), waiting for prepared queries
 * with nothing resident (host_idle_ms), preparing queries summed over the
 * preparation threads (host_prep_cpu_ms), and waiting for super-step
 * chunks to end (device_ms).  Other fields are 0. */
int b2r_serve_stats(const b2r_engine* e, b2r_batch_stats* out);

/* Launch shape of the super-step's main kernels.  Results do not depend on
 * it; throughput does, with the timetable, the query mix and the slot
 * count.  The counterpart of the reference's fixed GPU launch configuration
 * (src/routing/gpu/raptor.cu:894-990). */
typedef struct b2r_launch_shape {
  uint32_t scan_blocks_per_sm;  /* route scan grid = SMs x this (default 8) */
  uint32_t scan_threads;        /* route scan block: 32..256 threads, x32 (256) */
  uint32_t pair_blocks_per_sm;  /* route marking, transfers, footpaths (8) */
  uint32_t recon_blocks_per_sm; /* reconstruction, 128-thread blocks (4) */
  uint32_t steps_per_sync;      /* super-steps between host checks (4) */
  uint32_t scan_occupancy;      /* route scan build: 4, 5 or 6 resident
                                   blocks of 256 threads per SM (0, 1, 2;
                                   fewer registers per thread, the last two
                                   keep a few values in local memory) (0) */
} b2r_launch_shape;
int b2r_engine_get_shape(const b2r_engine* e, b2r_launch_shape* out);
/* Rejects values out of range; re-captures the super-step graph. */
int b2r_engine_set_shape(b2r_engine* e, const b2r_launch_shape* shape);

/* Autotuner: runs `sample` (n queries, results discarded) three times per
 * candidate launch shape, one knob at a time over a small grid of values
 * (coordinate descent, repeated until a pass changes nothing, at most three
 * passes), then measures the starting shape and the pick once more side by
 * side and keeps the faster (so best_ms <= start_ms), and reports what it
 * tried.  The last-batch results and statistics are overwritten. */
typedef struct b2r_tune_report {
  uint32_t n_tried;
  b2r_launch_shape start, best;
  double start_ms, best_ms; /* wall time of the sample batch */
} b2r_tune_report;
int b2r_engine_autotune(b2r_engine* e, const b2r_query* sample, uint32_t n,
                        b2r_tune_report* report);

/* Profiling engines (b2r_engine_config::profile = 1): per route-scan launch of
 * the last b2r_search_batch, its CUDA-event time, the marked (route, query
 * group) entries it scanned and the (route, query) stop steps it made.  *n
 * receives the number of launches; at most cap are written. */
int b2r_last_batch_scan_profile(const b2r_engine* e, double* scan_ms, uint64_t* entries,
                                uint64_t* stop_visits, uint32_t cap, uint32_t* n);

/* ------------------------------------------- host timetable construction */
/* Host-side timetable builder (not on the hot path): the synthetic
 * generator and nigiri's finalize() derivations (footpaths_in,
 * location_routes, route traffic days, lower-bound graphs, importance),
 * src/loader/init_finish.cc:64-198, build_lb_graph.h:11-99. */
typedef struct b2r_host_timetable b2r_host_timetable;

/* Synthetic timetable for workload `config` (1..5) with the given seed. */
int b2r_tt_generate(uint32_t config, uint64_t seed, b2r_host_timetable** out);
/* Build from base arrays (locations + routes); derived arrays are
 * computed here.  route_stop_times must already be in nigiri's layout. */
typedef struct b2r_tt_base {
  uint32_t n_locations;
  int32_t date_range_from;
  int32_t date_range_to;
  const uint8_t* transfer_time;
  const uint32_t* parent; /* or NULL */
  const uint8_t* location_type;
  const uint32_t* footpaths_out_index;
  const uint32_t* footpaths_out;
  uint32_t n_routes;
  const uint32_t* route_stop_index;
  const uint32_t* route_stops;
  const uint8_t* route_clasz; /* [n_routes] or NULL (all bus) */
  const uint32_t* route_n_transports;
  const uint16_t* route_stop_times; /* concatenated per route */
  const uint32_t* transport_bitfield; /* [n_transports] */
  uint32_t n_bitfields;
  const uint64_t* bitfields;
  const uint8_t* route_flags;         /* [n_routes] or NULL (no flags) */
  const uint8_t* route_section_flags; /* [route_stop_index[n_routes]] or NULL */
  /* footpaths of profiles 1..4 at index p - 1, CSR like footpaths_out, or
   * NULL (none); the builder derives their inbound lists and lower-bound
   * graphs as build_lb_graph (build_lb_graph.h:11-99) does per profile */
  const uint32_t* profile_footpaths_out_index[B2R_N_PROFILES - 1];
  const uint32_t* profile_footpaths_out[B2R_N_PROFILES - 1];
} b2r_tt_base;
int b2r_tt_build(const b2r_tt_base* base, b2r_host_timetable** out);
int b2r_tt_save(const b2r_host_timetable* t, const char* path);
int b2r_tt_load(const char* path, b2r_host_timetable** out);
int b2r_tt_desc(const b2r_host_timetable* t, b2r_timetable_desc* out);
int b2r_tt_destroy(b2r_host_timetable* t);

/* GTFS feeds (nigiri's loader::gtfs::load_timetable, the parts its routing
 * tests exercise): agency (the first agency's time zone for every trip,
 * noon_offsets.cc), stops with parent stations, routes (route_type ->
 * transport class), trips with blocks and bike / car / reservation flags,
 * stop times with pickup and drop-off restrictions, calendar,
 * calendar_dates, transfers.txt type 2.  Not read: frequencies, flex,
 * shapes, fares, stay-seated transfers, footpaths from stop proximity.
 * Time zones come from TZif files (tzdata_dir, default /usr/share/zoneinfo).
 * Mirrors loader_config (loader_interface.h:17-24). */
typedef struct b2r_gtfs_config {
  int32_t date_range_from, date_range_to; /* timetable::date_range_, days since the epoch */
  uint32_t default_transfer_time;         /* minutes (2) */
  uint16_t bikes_allowed_default;         /* bit c: trips of class c carry bikes unless trips.txt says */
  uint16_t cars_allowed_default;
  uint16_t reservation_not_required_default;
  uint16_t link_stop_distance;            /* metres: stops this close are linked by footpaths (100) */
  const char* default_tz;                 /* used when agency.txt names none */
  const char* tzdata_dir;                 /* NULL: /usr/share/zoneinfo */
} b2r_gtfs_config;
void b2r_gtfs_config_init(b2r_gtfs_config* c);
/* path: a directory with the feed's .txt files, or (is_text != 0) the feed
 * as one text of "# <file>.txt" sections (the mem_dir format of nigiri's
 * tests). */
int b2r_tt_load_gtfs(const char* path, int is_text, const b2r_gtfs_config* cfg,
                     b2r_host_timetable** out);
/* Feed identifiers of a loaded timetable: the stop_id of location l (special
 * stations: START, END, VIA0..VIA6), the route short name of transport x.
 * The strings live as long as the timetable. */
int b2r_tt_location_id(const b2r_host_timetable* t, uint32_t l, const char** id);
int b2r_tt_transport_name(const b2r_host_timetable* t, uint32_t x, const char** name);

/* Seeded synthetic query stream of a workload (configs 1..5). */
typedef struct b2r_query_set b2r_query_set;
int b2r_queries_generate(const b2r_host_timetable* t, uint32_t config,
                         uint64_t seed, uint32_t n, b2r_query_set** out);
uint32_t b2r_queries_count(const b2r_query_set* s);
const b2r_query* b2r_queries_get(const b2r_query_set* s, uint32_t i);
int b2r_queries_destroy(b2r_query_set* s);

#ifdef __cplusplus
}
#endif

#endif /* B2R_H_ */
