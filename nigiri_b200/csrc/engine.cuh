// Device-side data layout and helpers of the B200 RAPTOR engine.
//
// Round state is slot-minor: arrays are [round][location][slot] (and
// [location][slot] for best / tmp / lower bounds), so the 32 lanes of a warp
// working on one route for 32 resident queries read 32 consecutive words.
// Labels are 32-bit words  (tag:16 | key:16):
//   key  = direction-normalised time: t (forward) or ~t (backward), so that
//          "better" is always "smaller" and atomicMin serves both directions;
//          stored biased (key ^ 0x8000) to compare as unsigned.
//   tag  = 0xFFFF - generation.  round_times use the query generation of the
//          slot, best / tmp the start-time generation, so resetting a slot's
//          labels (raptor::reset_arrivals / next_start_time, raptor.h:174-188)
//          is a counter increment instead of a sweep.  A word whose tag is not
//          the current one reads as invalid (kInvalidDelta).
#pragma once

#include <cstdint>

#include "b2r.h"

namespace b2r::dev {

constexpr int kK = B2R_K;
constexpr int kKeyInv = 32767;
constexpr uint32_t kFull = 0xFFFFFFFFu;
constexpr int kMaxLegs = 40;
constexpr int kMaxTimeline = 128;

// slot states
enum : uint8_t {
  S_IDLE = 0,
  S_START = 1,     // admitted, first start-time group not yet seeded
  S_RUN = 2,       // running rounds
  S_COLLECT = 3,   // rounds of the current group finished
  S_DONE = 4,      // phase finished, host reads results
  S_ERROR = 5
};

// ------------------------------------------------------- timetable image
struct dtt {
  uint32_t n_loc, n_routes, n_transports, n_groups_unused;
  int32_t internal_from_days;
  uint8_t const* transfer_time;
  uint32_t const* parent;
  uint8_t const* loc_type;
  uint32_t const* children_idx;
  uint32_t const* children;
  uint32_t const* importance;
  uint32_t max_importance;
  uint32_t const* fp_out_idx;
  uint32_t const* fp_out;
  uint32_t const* fp_in_idx;
  uint32_t const* fp_in;
  // footpaths of profiles 1..4 (footpaths_out_[p] / footpaths_in_[p]):
  // fp_tab[4 (p - 1) + 0..3] = out index, out, in index, in; a profile
  // without footpaths points at an all-zero index
  uint32_t const* const* fp_tab;
  uint32_t const* route_stop_idx;
  uint32_t const* route_stops;
  uint32_t const* route_tr_from;
  uint32_t const* route_tr_to;
  uint32_t const* route_st_from;
  uint16_t const* st;  // route_stop_times (packed delta)
  uint32_t const* route_bf;
  uint32_t const* transport_bf;
  uint32_t const* transport_route;
  uint64_t const* bf;
  uint32_t const* loc_routes_idx;
  uint32_t const* loc_routes;
  uint8_t const* route_sorted;  // 1: every event column is ordered by mam
  // bit 0: the route's trips (transport, service day) compare the same way
  // at every event of the route, equal at all or strictly ordered at all;
  // bit 1: and (service day, transport offset) orders them as their times
  // do (columns ordered by minute, every first departure on its service day,
  // fewer than 16384 transports)
  uint8_t const* route_fifo;
  // lower-bound graphs (build_lb_graph.h), packed footpath words
  uint32_t const* lbg_fwd_idx;
  uint32_t const* lbg_fwd;
  uint32_t const* lbg_bwd_idx;
  uint32_t const* lbg_bwd;
  uint32_t const* with_children;  // locations that have children, ascending
  uint32_t n_with_children;
  // location -> (route, stop position) pairs in the order reconstruction
  // visits them: routes of location_routes_, then stop positions ascending
  uint32_t const* lrs_idx;
  uint32_t const* lrs_route;
  uint16_t const* lrs_stop;
  // route filters: per route, bits 0-3 transport class, 4-7 the flags set on
  // all sections, 8-11 the flags set on some sections (route_clasz_ and
  // route_flags_, timetable.h:348-355); per route stop index s of route r
  // the flags of the section s -> s + 1 (route_flags_per_section_)
  uint16_t const* route_filter;
  uint8_t const* route_sec;
  // real-time overlay (an engine bound to one; n_rt = 0 otherwise): rt
  // transports with their stop words, unix event times (transport x's
  // event at stop i: rt_times[2 (rt_stop_idx[x] - x) + 2 i - is_arr]),
  // filter words like route_filter and per-stop section flags; the static
  // trip each runs for; location -> rt transports (route marking) and
  // location -> (rt transport, stop position) pairs (reconstruction)
  uint32_t n_rt;
  uint32_t const* rt_stop_idx;
  uint32_t const* rt_stops;
  int32_t const* rt_times;
  uint16_t const* rt_filter;
  uint8_t const* rt_sec;
  uint32_t const* rt_static;
  uint16_t const* rt_static_day;
  uint32_t const* loc_rt_idx;
  uint32_t const* loc_rt;
  uint32_t const* lrs_rt_idx;
  uint32_t const* lrs_rt;
  uint16_t const* lrs_rt_stop;
};

// --------------------------------------------------------- per-slot data
struct tts_t {
  uint8_t is_default;
  int16_t min_transfer_time;
  int16_t additional_time;
  float factor;
};

struct journey_rec {  // routing::journey header
  int32_t start_time;
  int32_t dest_time;
  uint32_t dest;
  uint8_t transfers;
  uint8_t error;
  uint8_t reconstructed;
  uint8_t pad;
  uint16_t n_legs;
  uint16_t block;  // leg block of this journey
};

struct slot_t {
  // set at admission
  uint8_t state;
  uint8_t fwd;
  uint8_t one_to_all;
  uint8_t end_k;
  uint8_t intermodal_dest;
  uint8_t ontrip;
  uint8_t start_mode;
  uint8_t dest_mode;
  uint16_t base;  // day index of the base day
  uint16_t gen_query;
  int32_t base_days;
  int32_t iv_from, iv_to;
  int16_t fastest_direct;
  int16_t max_travel_time;
  uint32_t min_connection_count;
  uint8_t extend_earlier, extend_later, need_sweep, early_term;
  uint16_t allowed_claszes;  // bit c: transport class c allowed
  uint8_t req_flags;         // bit f: route flag f required
  uint8_t blast;             // bounds_last_k_ of a pong phase (raptor.h:172); 0: unbounded
  uint8_t recon_mode;        // 0: new journeys of the interval, 1: only the journey
                             // (recon_transfers, recon_start), 2: none
  uint8_t recon_transfers;
  uint8_t no_lb;             // lower bounds read as 0 (a pong phase)
  uint8_t prf;               // footpath profile (query::prf_idx_)
  int16_t span;              // worst time at destination = group start + dir(span)
  int32_t recon_start;
  tts_t tts;
  uint32_t starts_off, n_starts;  // start pool
  uint32_t dest_off, n_dest;      // dest pool (loc, dist)
  uint32_t soff_off, n_soff;      // start offsets (for reconstruction)
  uint32_t doff_off, n_doff;      // destination offsets
  // dynamic
  uint8_t k;
  uint8_t recon_defer;  // set at admission: journeys are rebuilt when the slot is done, off the
                        // rounds' path (a single start-time group: no later round changes them)
  uint16_t gen_group;
  uint32_t next_start;   // index of the next start label (group cursor)
  int32_t cur_start_time;
  uint32_t n_journeys;
  int32_t error;
  int16_t tad[kK];  // time_at_dest_ keys
  uint64_t n_rounds, n_groups_run;
};

// compact per-super-step view of a slot read by every lane (one 16-byte
// load)
struct __align__(16) lane_t {
  int16_t tad_k;
  uint16_t gtag;
  uint16_t qtag;
  uint16_t base;
  uint8_t fwd;
  uint8_t k;
  uint8_t run;
  uint8_t mode;  // bit0 intermodal dest, bit1 has dests, bit2 tts default, bit3 no lower
                 // bounds, bits 4-6 footpath profile, bit7 round times kept for a later
                 // start-time group (the writes set their touched bits)
  uint16_t claszes;  // allowed transport classes
  uint8_t req;       // required route flags
  uint8_t blast;     // pong bounds: last round (0: none)
};

struct start_rec {
  int32_t time_at_start;
  int32_t time_at_stop;
  uint32_t stop;
};

struct dest_rec {
  uint32_t loc;
  uint32_t dist;  // intermodal egress minutes
};

struct tl_entry {  // time_at_dest timeline of one phase
  uint32_t pos_hi, pos_lo;
  int32_t tad;
};

// what the host reads of every slot after a super-step chunk
struct slot_summary {
  uint8_t state, pad[3];
  uint32_t n_journeys;
};

// engine state: every device array in one POD passed by value
struct state {
  dtt tt;
  uint32_t S;        // slots (multiple of 32)
  uint32_t G;        // slot groups of 32
  uint32_t max_j;    // journeys per slot
  slot_t* slots;
  lane_t* lanes;
  uint32_t* rt;     // [K][n_loc][S]
  uint32_t* touched;  // [K][G][n_loc]: bit b of (k, g, l) is set by every round-time write
                      // at (k, l) of slot g * 32 + b while that slot may run a later
                      // start-time group (lane mode bit 7); the sweep reads only the set bits
  uint32_t* best;   // [n_loc][S]
  uint32_t* tmp;    // [n_loc][S]
  uint16_t* lb;     // [n_loc][S]
  uint32_t* X;      // station marks  [n_loc][G]
  uint32_t* Y;      // route-reached marks [n_loc][G]
  uint32_t* R;      // route marks [n_routes][G]
  uint32_t* RT_R;   // rt transport marks [n_rt][G] (an overlay is bound)
  uint32_t* rtlist; // frontier list of (rt transport * G + g)
  uint32_t* D;      // is-destination bits [n_loc][G]
  uint32_t* xlist;  // frontier lists of (loc * G + g)
  uint32_t* ylist;
  uint32_t* rlist;
  uint32_t* counters;  // [0] xlist, [1] ylist, [2] rlist, [3] recon count, [4] x2 ...
  uint32_t* run_mask;  // [G]
  uint32_t* sweep_mask;  // [G]
  uint32_t* any_mask;  // [G]
  start_rec* start_pool;
  dest_rec* dest_pool;
  b2r_offset* off_pool;
  journey_rec* journeys;  // [S][max_j]
  b2r_leg* legs;          // [S][max_j][kMaxLegs]
  uint32_t* blocks_used;  // [S][max_j / 32]
  uint32_t* recon_list;   // (slot << 16 | journey index)
  tl_entry* timeline;     // [S][kMaxTimeline]
  uint32_t* timeline_n;   // [S]
  int16_t* tad_phase;     // [S] tad[k] at the start of the phase
  uint32_t* status_word;  // [0] device error flags
  unsigned long long* prof;  // route-scan work counters (profiling engines)
  uint32_t profile;
  // lower bounds computed on the device: tagged distances, frontier bits
  // and lists (double-buffered), slots waiting for their bounds
  uint32_t* dist;        // [n_loc][S]
  uint32_t* F[2];        // [n_loc][G]
  uint32_t* flist[2];
  uint32_t* lb_mask;     // [G]
  // all-pairs lower-bound tables (forward / backward search), or null
  uint16_t const* lb_table_fwd;
  uint16_t const* lb_table_bwd;
  uint32_t lb_stride;  // table row length (n_loc rounded up to 8)
  // pong bounds (raptor_state::bounds_storage_): rows of the ping's round
  // times folded over the rounds, as keys of the bounded (pong) search
  int16_t* bounds;  // [K][n_loc][S]
  slot_summary* summary;  // [S]
};

// ------------------------------------------------------------- helpers
__device__ __forceinline__ uint16_t tagcode(uint16_t gen) { return static_cast<uint16_t>(0xFFFFu - gen); }

__device__ __forceinline__ uint32_t enc(uint16_t tag, int key) {
  return (static_cast<uint32_t>(tag) << 16) |
         (static_cast<uint32_t>(static_cast<uint16_t>(static_cast<int16_t>(key))) ^ 0x8000u);
}

__device__ __forceinline__ int dec(uint32_t w, uint16_t tag) {
  return (w >> 16) == tag ? static_cast<int>(static_cast<int16_t>((w & 0xFFFFu) ^ 0x8000u))
                          : kKeyInv;
}

__device__ __forceinline__ int clamp16(int v) { return v < -32768 ? -32768 : (v > 32767 ? 32767 : v); }

// delta_t <-> key
__device__ __forceinline__ int to_key(bool fwd, int t) { return fwd ? t : ~t; }
__device__ __forceinline__ int from_key(bool fwd, int k) { return fwd ? k : ~k; }

// clamp(t + dir(x)) in key space == clamp(key + x) (both directions)
__device__ __forceinline__ int key_add(int key, int x) { return clamp16(key + x); }

__device__ __forceinline__ bool bf_test(dtt const& T, uint32_t bf, uint32_t i) {
  return i < B2R_MAX_DAYS && ((__ldg(T.bf + 8ull * bf + (i >> 6)) >> (i & 63u)) & 1ull);
}

// The route filters of loop_routes (raptor.h:499-545) and of get_transport
// (reconstruct.cc:456-498): false if route r's class is not allowed or a
// required flag is on none of its sections; `sec` receives the required
// flags that are on some but not all sections, which the walk along the
// route checks section by section (raptor.h:1194-1217).
__device__ __forceinline__ bool route_allowed(dtt const& T, uint32_t r, uint32_t claszes, uint32_t req,
                                              uint32_t& sec) {
  auto const f = static_cast<uint32_t>(T.route_filter[r]);
  auto const need = req & ~(f >> 4);  // required, not on all sections
  sec = need;
  return ((claszes >> (f & 15u)) & 1u) != 0u && (need & ~(f >> 8) & 15u) == 0u;
}

// the same for a filter word of that layout (rt transports: the class of
// the first section, raptor.h:583-588)
__device__ __forceinline__ bool filter_allowed(uint16_t fw, uint32_t claszes, uint32_t req, uint32_t& sec) {
  auto const f = static_cast<uint32_t>(fw);
  auto const need = req & ~(f >> 4);
  sec = need;
  return ((claszes >> (f & 15u)) & 1u) != 0u && (need & ~(f >> 8) & 15u) == 0u;
}

// whether section s of route r (from its stop s to s + 1) carries every
// flag of `sec`
__device__ __forceinline__ bool section_ok(dtt const& T, uint32_t r_stop_base, uint32_t s, uint32_t sec) {
  return (static_cast<uint32_t>(T.route_sec[r_stop_base + s]) & sec) == sec;
}

// footpaths_out_[prf] (out) or footpaths_in_[prf] (timetable.h:97-98):
// the CSR index and the footpath words
__device__ __forceinline__ uint32_t const* fp_index(dtt const& T, uint32_t prf, bool out) {
  if (prf == 0u) return out ? T.fp_out_idx : T.fp_in_idx;
  return T.fp_tab[4u * (prf - 1u) + (out ? 0u : 2u)];
}
__device__ __forceinline__ uint32_t const* fp_words(dtt const& T, uint32_t prf, bool out) {
  if (prf == 0u) return out ? T.fp_out : T.fp_in;
  return T.fp_tab[4u * (prf - 1u) + (out ? 1u : 3u)];
}

// stop::in_allowed / out_allowed of the stop word, the wheelchair bits when
// wc (stop.h:51-67 can_start / can_finish with is_wheelchair)
__device__ __forceinline__ uint32_t stop_in_bit(uint32_t w, uint32_t wc) { return (w >> (28u + 2u * wc)) & 1u; }
__device__ __forceinline__ uint32_t stop_out_bit(uint32_t w, uint32_t wc) { return (w >> (29u + 2u * wc)) & 1u; }

__device__ __forceinline__ int delta_count(uint16_t d) {  // delta::count()
  return static_cast<int16_t>(static_cast<uint32_t>(d & 0x1Fu) * 1440u + (d >> 5));
}

// adjusted_transfer_time<T> for an int duration (float product truncated)
template <typename T>
__device__ __forceinline__ T adjusted(tts_t const& s, T d) {
  if (s.is_default) return d;
  auto const prod = static_cast<T>(__float2int_rz(__fmul_rn(static_cast<float>(d), s.factor)));
  auto const mn = static_cast<T>(s.min_transfer_time);
  return static_cast<T>(static_cast<T>(s.additional_time) + (prod > mn ? prod : mn));
}

// within_bounds, raptor.h:458-489 (no vias): a label `key` at l in round k
// of a bounded search may not be better than the bounding search's row
// (blast - k) at l plus l's transfer time.
__device__ __forceinline__ bool within_bounds(state const& st, uint32_t s, uint32_t blast, uint32_t k,
                                              uint32_t l, int key) {
  if (blast == 0u) return true;
  auto const row = static_cast<int>(st.bounds[(static_cast<size_t>(blast - k) * st.tt.n_loc + l) * st.S + s]);
  return key <= row + adjusted<int>(st.slots[s].tts, static_cast<int>(st.tt.transfer_time[l]));
}

// to_delta(day, mam) of raptor.h:1467-1469, as a key
__device__ __forceinline__ int to_delta_key(bool fwd, uint16_t day, uint16_t base, int mam) {
  return to_key(fwd, clamp16((static_cast<int>(day) - static_cast<int>(base)) * 1440 + mam));
}

}  // namespace b2r::dev
