// Per-round kernels of the batched RAPTOR super-step.  One super-step runs
// one RAPTOR round (raptor::execute's loop body, raptor.h:218-387) for every
// resident query whose current start-time group is still running, then
// collects, reconstructs and seeds the next start-time group of queries
// whose rounds ended (search.h:436-475).
#pragma once

#include "engine.cuh"
#include "et_search.cuh"
#include "reconstruct.cuh"

namespace b2r::dev {

enum : uint32_t { C_X = 0, C_Y = 1, C_R = 2, C_RECON = 3, C_ERR = 4, C_F0 = 5, C_F1 = 6, C_RT = 7 };

__device__ __forceinline__ size_t li(state const& st, uint32_t l, uint32_t s) {
  return static_cast<size_t>(l) * st.S + s;
}
__device__ __forceinline__ size_t rti(state const& st, uint32_t k, uint32_t l, uint32_t s) {
  return (static_cast<size_t>(k) * st.tt.n_loc + l) * st.S + s;
}

__device__ __forceinline__ void mark(state const& st, uint32_t* M, uint32_t* list, uint32_t counter,
                                     uint32_t e, uint32_t bits) {
  auto const old = atomicOr(&M[e], bits);
  if (old == 0u) list[atomicAdd(&st.counters[counter], 1u)] = e;
}

// warp-aggregated mark: lanes with `want` OR their bit into M[e(lane)];
// lanes sharing the same word combine into one atomic.
__device__ __forceinline__ void mark_warp(state const& st, uint32_t* M, uint32_t* list,
                                          uint32_t counter, bool want, uint32_t e, uint32_t lane) {
  auto const key = want ? e : 0xFFFFFFFFu;
  auto const peers = __match_any_sync(kFull, key);
  if (want && lane == static_cast<uint32_t>(__ffs(peers) - 1)) mark(st, M, list, counter, e, peers);
}

// Visits the (entry, query) pairs of a frontier list: a warp takes 32 list
// entries (a location or route with a group of 32 queries), and its lanes
// take their set query bits, one pair per lane per pass.  Resident queries
// are unrelated, so an entry holds few of its 32 queries; a lane per query of
// one entry would leave most lanes idle.  word(e) returns the entry's query
// bits; f(e, b) runs for every set bit b.  f must not synchronise the warp.
template <typename Word, typename F>
__device__ __forceinline__ void for_each_pair(uint32_t const* list, uint32_t n, Word&& word, F&& f) {
  auto const lane = threadIdx.x & 31u;
  auto const warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  auto const n_warps = (gridDim.x * blockDim.x) >> 5;
  for (auto w0 = warp * 32u; w0 < n; w0 += n_warps * 32u) {
    auto const w = w0 + lane;
    uint32_t e = 0, mask = 0;
    if (w < n) {
      e = list[w];
      mask = word(e);
    }
    auto const cnt = static_cast<uint32_t>(__popc(mask));
    auto end = cnt;  // inclusive prefix sum of the pair counts
    for (auto o = 1u; o < 32u; o <<= 1) {
      auto const v = __shfl_up_sync(kFull, end, o);
      if (lane >= o) end += v;
    }
    auto const total = __shfl_sync(kFull, end, 31);
    for (auto p0 = 0u; p0 < total; p0 += 32u) {
      auto const p = p0 + lane;
      uint32_t owner = 0;  // first lane whose prefix end exceeds p
      for (auto b = 16u; b > 0u; b >>= 1) {
        if (__shfl_sync(kFull, end, static_cast<int>(owner + b - 1u)) <= p) owner += b;
      }
      auto const o_e = __shfl_sync(kFull, e, static_cast<int>(owner));
      auto o_mask = __shfl_sync(kFull, mask, static_cast<int>(owner));
      auto const o_first = __shfl_sync(kFull, end, static_cast<int>(owner)) -
                           __shfl_sync(kFull, cnt, static_cast<int>(owner));
      if (p < total) {
        for (auto x = p - o_first; x != 0u; --x) o_mask &= o_mask - 1u;
        f(o_e, static_cast<uint32_t>(__ffs(o_mask) - 1));
      }
    }
  }
}

// A slot keeps its round times for a later start-time group unless it runs
// one group and nothing after it: a one-to-one query at one start time whose
// journeys are collected as usual, or a one-to-all query at one start time.
// Range queries, interval extension, pong phases and step-driven searches
// keep them (raptor.h:174-177: only reset_arrivals clears them).
__device__ __forceinline__ bool keeps_round_times(slot_t const& sl) {
  if (sl.ontrip && sl.one_to_all) return false;
  return !(sl.ontrip && sl.recon_mode == 0);
}

// the touched bit of a round-time write (k, l) of slot s
__device__ __forceinline__ void touch(state const& st, lane_t const& ln, uint32_t k, uint32_t l, uint32_t s) {
  if (!(ln.mode & 128u)) return;
  auto* w = st.touched + (static_cast<size_t>(k) * st.G + (s >> 5)) * st.tt.n_loc + l;
  auto const bit = 1u << (s & 31u);
  if ((*w & bit) == 0u) atomicOr(w, bit);
}

__device__ __forceinline__ void update_tad(slot_t& sl, uint32_t k, int key) {  // raptor.h:1479-1486
  if (sl.one_to_all) return;
  for (auto i = k; i < kK; ++i) {
    if (key < sl.tad[i]) sl.tad[i] = static_cast<int16_t>(key);
  }
}

// ----------------------------------------------------------- control
// Start of a super-step: the route-reached marks of the last one cleared
// (all threads), and per slot (threads < S, a warp per slot group) the lane
// view and the group's run / sweep masks, written whole from ballots.  The
// reached-list counter is reset by k_ctl_dest, after every thread here has
// read it.
__global__ void k_ctl_begin(state st) {
  auto const tid = blockIdx.x * blockDim.x + threadIdx.x;
  auto const ny = st.counters[C_Y];
  for (auto i = tid; i < ny; i += gridDim.x * blockDim.x) st.Y[st.ylist[i]] = 0u;
  if (tid == 0) {
    st.counters[C_R] = 0u;
    st.counters[C_RECON] = 0u;
    st.counters[C_RT] = 0u;
  }
  if ((tid & ~31u) >= st.S) return;  // whole warps: S is a multiple of 32
  auto const s = tid;
  auto& sl = st.slots[s];
  lane_t ln{};
  auto const run = sl.state == S_RUN;
  auto const run_bits = __ballot_sync(kFull, run);
  auto const sweep_bits = __ballot_sync(kFull, run && sl.need_sweep);
  if ((s & 31u) == 0u) {
    st.run_mask[s >> 5] = run_bits;
    st.sweep_mask[s >> 5] = sweep_bits;
    st.any_mask[s >> 5] = 0u;
  }
  if (run) {
    ln.run = 1;
    ln.fwd = sl.fwd;
    ln.k = sl.k;
    ln.base = sl.base;
    ln.gtag = tagcode(sl.gen_group);
    ln.qtag = tagcode(sl.gen_query);
    ln.mode = (sl.intermodal_dest ? 1u : 0u) |
              ((!sl.intermodal_dest && !sl.one_to_all && sl.n_dest != 0) ? 2u : 0u) |
              (sl.tts.is_default ? 4u : 0u) | (sl.no_lb ? 8u : 0u) | (static_cast<uint32_t>(sl.prf) << 4) |
              (keeps_round_times(sl) ? 128u : 0u);
    ln.tad_k = sl.tad[sl.k];
    ln.claszes = sl.allowed_claszes;
    ln.req = sl.req_flags;
    ln.blast = sl.blast;
    ++sl.n_rounds;
  }
  st.lanes[s] = ln;
}

// best <- min(best, round_times[k]) over all locations (raptor.h:219-223)
// for the slots whose earlier start-time groups left round times behind
// (range queries).  Only locations whose touched word of (round, slot group)
// has the slot's bit can hold such a round time, so a warp reads the words
// of 32 locations at once (one coalesced load) and spreads their set bits,
// the (location, slot) pairs, over its lanes: every lane loads one round
// time and best label, independent of the others.  Bits whose entry belongs
// to an earlier query of the slot (its tag no longer matches) are cleared
// here; any later write sets them again.  Slots of one group at different
// rounds are taken one round at a time.
__global__ void k_sweep(state st) {
  auto const lane = threadIdx.x & 31u;
  auto const warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  auto const n_warps = (gridDim.x * blockDim.x) >> 5;
  auto const n_loc = st.tt.n_loc;
  auto const n_chunks = (n_loc + 31u) / 32u;
  for (auto g = 0u; g != st.G; ++g) {
    auto const m = st.sweep_mask[g];
    if (m == 0u) continue;
    auto const ln = st.lanes[g * 32u + lane];
    auto const mine = ((m >> lane) & 1u) != 0u;
    auto pending = m;
    while (pending != 0u) {
      auto const k = __shfl_sync(kFull, static_cast<uint32_t>(ln.k), __ffs(pending) - 1);
      auto const same = __ballot_sync(kFull, mine && static_cast<uint32_t>(ln.k) == k);
      pending &= ~same;
      auto* tw = st.touched + (static_cast<size_t>(k) * st.G + g) * n_loc;
      for (auto c = warp; c < n_chunks; c += n_warps) {
        auto const l = c * 32u + lane;
        auto const word = l < n_loc ? (tw[l] & same) : 0u;
        if (__ballot_sync(kFull, word != 0u) == 0u) continue;
        auto const cnt = static_cast<uint32_t>(__popc(word));
        auto end = cnt;  // inclusive prefix sum of the pair counts
        for (auto o = 1u; o < 32u; o <<= 1) {
          auto const y = __shfl_up_sync(kFull, end, o);
          if (lane >= o) end += y;
        }
        auto const total = __shfl_sync(kFull, end, 31);
        for (auto p0 = 0u; p0 < total; p0 += 32u) {
          auto const p = p0 + lane;
          uint32_t owner = 0;  // first lane whose prefix end exceeds p
          for (auto b = 16u; b > 0u; b >>= 1) {
            if (__shfl_sync(kFull, end, static_cast<int>(owner + b - 1u)) <= p) owner += b;
          }
          auto o_word = __shfl_sync(kFull, word, static_cast<int>(owner));
          auto const o_first = __shfl_sync(kFull, end, static_cast<int>(owner)) -
                               __shfl_sync(kFull, cnt, static_cast<int>(owner));
          uint32_t b = 0u;
          if (p < total) {
            for (auto x = p - o_first; x != 0u; --x) o_word &= o_word - 1u;
            b = static_cast<uint32_t>(__ffs(o_word) - 1);
          }
          auto const qtag = __shfl_sync(kFull, static_cast<uint32_t>(ln.qtag), static_cast<int>(b));
          auto const gtag = __shfl_sync(kFull, static_cast<uint32_t>(ln.gtag), static_cast<int>(b));
          if (p < total) {
            auto const at = c * 32u + owner;
            auto const s = g * 32u + b;
            auto const r = dec(st.rt[rti(st, k, at, s)], static_cast<uint16_t>(qtag));
            if (r == kKeyInv) {
              atomicAnd(tw + at, ~(1u << b));
            } else {
              auto& bw = st.best[li(st, at, s)];
              if (r < dec(bw, static_cast<uint16_t>(gtag))) bw = enc(static_cast<uint16_t>(gtag), r);
            }
          }
        }
      }
    }
  }
}

// destination times into time_at_dest (raptor.h:224-226)
__global__ void k_ctl_dest(state st) {
  auto const s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s == 0) st.counters[C_Y] = 0u;  // k_ctl_begin has cleared the listed words
  if (s >= st.S) return;
  auto& sl = st.slots[s];
  if (sl.state != S_RUN || sl.one_to_all) return;
  auto const gtag = tagcode(sl.gen_group);
  if (sl.intermodal_dest) {
    update_tad(sl, sl.k, dec(st.best[li(st, B2R_SPECIAL_END, s)], gtag));
  } else {
    for (auto i = 0u; i != sl.n_dest; ++i) {
      update_tad(sl, sl.k, dec(st.best[li(st, st.dest_pool[sl.dest_off + i].loc, s)], gtag));
    }
  }
  st.lanes[s].tad_k = sl.tad[sl.k];
}

// station marks -> route marks (raptor.h:228-241)
// A warp takes 32 marked (location, group) words and spreads their
// (word, route) pairs over its lanes, so that hub stations with many routes
// do not hold one lane.  The per-group "any route marked" word is read
// before its atomicOr: it only gains bits during the kernel, so a read that
// shows the bits set makes the atomic redundant, and same-address atomics
// would queue in L2.
__global__ void k_mark_routes(state st) {
  auto const nx = st.counters[C_X];
  auto const lane = threadIdx.x & 31u;
  auto const warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  auto const n_warps = (gridDim.x * blockDim.x) >> 5;
  for (auto w0 = warp * 32u; w0 < nx; w0 += n_warps * 32u) {
    auto const i = w0 + lane;
    uint32_t g = 0, w = 0, rb = 0, cnt = 0;
    if (i < nx) {
      auto const e = st.xlist[i];
      g = e % st.G;
      auto const l = e / st.G;
      w = st.X[e] & st.run_mask[g];
      if (w != 0u) {
        rb = __ldg(st.tt.loc_routes_idx + l);
        cnt = __ldg(st.tt.loc_routes_idx + l + 1) - rb;
        if (cnt != 0u && (st.any_mask[g] & w) != w) atomicOr(&st.any_mask[g], w);
      }
    }
    auto end = cnt;  // inclusive prefix sum of the route counts
    for (auto o = 1u; o < 32u; o <<= 1) {
      auto const v = __shfl_up_sync(kFull, end, o);
      if (lane >= o) end += v;
    }
    auto const total = __shfl_sync(kFull, end, 31);
    for (auto p0 = 0u; p0 < total; p0 += 32u) {
      auto const p = p0 + lane;
      uint32_t owner = 0;  // first lane whose prefix end exceeds p
      for (auto b = 16u; b > 0u; b >>= 1) {
        if (__shfl_sync(kFull, end, static_cast<int>(owner + b - 1u)) <= p) owner += b;
      }
      auto const o_first = __shfl_sync(kFull, end, static_cast<int>(owner)) -
                           __shfl_sync(kFull, cnt, static_cast<int>(owner));
      auto const o_rb = __shfl_sync(kFull, rb, static_cast<int>(owner));
      auto const o_g = __shfl_sync(kFull, g, static_cast<int>(owner));
      auto const o_w = __shfl_sync(kFull, w, static_cast<int>(owner));
      if (p < total) {
        auto const r = __ldg(st.tt.loc_routes + o_rb + (p - o_first));
        atomicOr(&st.R[r * st.G + o_g], o_w);  // listed by k_list_routes
      }
    }
  }
}

// The indices of the non-zero words of W[0, n) appended to `list` (in no
// particular order).  Each thread reads 4 words with one 16-byte load
// (W comes from cudaMalloc and i is a multiple of 4), the block scans the
// counts and reserves its range with one atomicAdd per 4 * blockDim words.
__device__ __forceinline__ void list_nonzero(state const& st, uint32_t const* W, uint32_t n,
                                             uint32_t* list, uint32_t counter) {
  __shared__ uint32_t warp_off[32];
  __shared__ uint32_t base;
  auto const lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, n_warps = blockDim.x >> 5;
  auto const per_block = blockDim.x * 4u;
  for (auto b0 = blockIdx.x * per_block; b0 < n; b0 += gridDim.x * per_block) {
    auto const i = b0 + threadIdx.x * 4u;
    uint32_t w[4] = {0u, 0u, 0u, 0u};
    if (i + 3u < n) {
      auto const v = *reinterpret_cast<uint4 const*>(W + i);
      w[0] = v.x;
      w[1] = v.y;
      w[2] = v.z;
      w[3] = v.w;
    } else {
      for (auto j = 0u; j != 4u; ++j) w[j] = i + j < n ? W[i + j] : 0u;
    }
    auto const cnt = static_cast<uint32_t>(w[0] != 0u) + static_cast<uint32_t>(w[1] != 0u) +
                     static_cast<uint32_t>(w[2] != 0u) + static_cast<uint32_t>(w[3] != 0u);
    auto incl = cnt;  // inclusive scan over the warp
    for (auto d = 1u; d < 32u; d <<= 1) {
      auto const y = __shfl_up_sync(kFull, incl, d);
      if (lane >= d) incl += y;
    }
    if (lane == 31u) warp_off[warp] = incl;
    __syncthreads();
    if (warp == 0u) {  // scan of the warp totals, then the block's reservation
      auto const ws = lane < n_warps ? warp_off[lane] : 0u;
      auto x = ws;
      for (auto d = 1u; d < 32u; d <<= 1) {
        auto const y = __shfl_up_sync(kFull, x, d);
        if (lane >= d) x += y;
      }
      if (lane < n_warps) warp_off[lane] = x - ws;
      if (lane == 31u) base = x != 0u ? atomicAdd(&st.counters[counter], x) : 0u;
    }
    __syncthreads();
    auto at = base + warp_off[warp] + (incl - cnt);
    for (auto j = 0u; j != 4u; ++j) {
      if (w[j] != 0u) list[at++] = i + j;
    }
    __syncthreads();  // warp_off and base are reused by the next pass
  }
}

// marked (route, group) entries of this round
__global__ void k_list_routes(state st) { list_nonzero(st, st.R, st.tt.n_routes * st.G, st.rlist, C_R); }

// ------------------------------------------------ real-time transports
// station marks -> rt transport marks (raptor.h:234-240), a thread per
// marked (location, group) word; a marked rt transport also keeps its
// queries in the round (any_marked)
__global__ void k_mark_rt(state st) {
  auto const nx = st.counters[C_X];
  auto const& T = st.tt;
  for (auto i = blockIdx.x * blockDim.x + threadIdx.x; i < nx; i += gridDim.x * blockDim.x) {
    auto const e = st.xlist[i];
    auto const g = e % st.G, l = e / st.G;
    auto const w = st.X[e] & st.run_mask[g];
    if (w == 0u) continue;
    auto const b = T.loc_rt_idx[l], n = T.loc_rt_idx[l + 1] - b;
    if (n == 0u) continue;
    if ((st.any_mask[g] & w) != w) atomicOr(&st.any_mask[g], w);
    for (auto j = 0u; j != n; ++j) atomicOr(&st.RT_R[T.loc_rt[b + j] * st.G + g], w);  // listed by k_list_rt
  }
}

// marked (rt transport, group) entries of this round
__global__ void k_list_rt(state st) { list_nonzero(st, st.RT_R, st.tt.n_rt * st.G, st.rtlist, C_RT); }

__global__ void k_ctl_marked(state st) {
  auto const s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= st.S) return;
  auto& sl = st.slots[s];
  if (sl.state != S_RUN) return;
  if (!((st.any_mask[s >> 5] >> (s & 31)) & 1u)) {  // raptor.h:243-246
    sl.state = S_COLLECT;
    st.lanes[s].run = 0;
  }
}

// ------------------------------------------------------------ route scan
// update_route, raptor.h:1177-1349 (no vias), for every (route, query) pair
// marked this round.
//
// The reference walks a route's stops in order, carrying the trip it rides
// (et).  At a stop marked last round it looks up the earliest trip
// boardable there (get_earliest_transport) and switches to it when that
// trip is at least as good at this stop as the current one; at every stop
// it improves the arrival label with the current trip.  Walked like that,
// one (route, query) pair is a chain of dependent loads as long as the
// route.
//
// Here a warp takes one pair and its lanes take the stops, 32 at a time:
// * every boardable stop looks up its own earliest trip at once (the
//   lookup depends only on that stop's labels);
// * on a route whose trips keep one order at every event
//   (b2r_timetable: route_fifo), "switch when at least as good at this
//   stop" is "keep the best trip so far, the later stop on ties", whatever
//   stop compares them, so a warp prefix-minimum over the lanes gives the
//   trip each stop is reached by;
// * every stop then reads its arrival event of that trip.
// The result equals the sequential walk's; routes without that order and
// queries with per-section filters take the sequential walk
// (k_route_scan_seq).
// Labels are combined with atomicMin and marks with atomicOr, so the order
// of the pairs does not matter.

struct scan_ctr {
  uint32_t stops, ev, days, writes, warp_steps;
};

// the stop word at position i of route (sb, n) in search direction; for the
// wheelchair profile with its wheelchair bits in place of the in / out bits
// (can_start / can_finish, raptor.h:1252, 1304)
__device__ __forceinline__ uint32_t scan_stop_word(dtt const& T, uint32_t sb, uint32_t n, bool fwd, uint32_t i,
                                                   uint32_t sec) {
  auto const w = __ldg(T.route_stops + sb + (fwd ? i : n - 1u - i));
  return (sec & 0x100u) != 0u ? (w & 0xCFFFFFFFu) | ((w >> 2) & 0x30000000u) : w;
}

// the arrival-side label update of one stop (raptor.h:1242-1302)
template <bool Prof>
__device__ __forceinline__ void scan_arrive(state const& st, lane_t const& ln, uint32_t s, uint32_t g, uint32_t bit,
                                            uint32_t l, uint16_t lbv, int by, scan_ctr& pc) {
  if (by <= ln.tad_k && lbv != 0xFFFFu && by + static_cast<int>(lbv) <= ln.tad_k &&
      (ln.blast == 0u || within_bounds(st, s, ln.blast, ln.k, l, by))) {
    auto const word = enc(ln.gtag, by);
    auto* tp = &st.tmp[li(st, l, s)];
    if constexpr (Prof) {
      if (word < atomicMin(tp, word)) ++pc.writes;
    } else {
      atomicMin(tp, word);  // result unused: no round trip
    }
    atomicOr(&st.Y[l * st.G + g], bit);  // listed by k_list_reached
  }
}

// The reference's sequential walk of one (route, query) pair.
__device__ __forceinline__ void scan_walk_seq(state const& st, lane_t const& ln, uint32_t r, uint32_t g,
                                              uint32_t b, uint32_t sec, scan_ctr& pc) {
  auto const& T = st.tt;
  auto const s = g * 32u + b;
  auto const bit = 1u << b;
  auto const fwd = ln.fwd != 0;
  auto const k = static_cast<uint32_t>(ln.k);
  auto const sb = T.route_stop_idx[r];
  auto const n = T.route_stop_idx[r + 1] - sb;
  auto const n_t = T.route_tr_to[r] - T.route_tr_from[r];
  auto const* colbase = T.st + T.route_st_from[r];
  auto const lb_off = (ln.mode & 8u) != 0u;
  bool et_valid = false;
  uint32_t et_off = 0;
  uint16_t et_day = 0;
  for (auto i = 0u; i < n; ++i) {
    ++pc.stops;
    ++pc.warp_steps;
    auto const stp = scan_stop_word(T, sb, n, fwd, i, sec);
    auto const si = fwd ? i : n - 1u - i;
    auto const l = B2R_STOP_LOC(stp);
    auto const lbv = lb_off ? uint16_t{0} : st.lb[li(st, l, s)];
    auto const can_finish = fwd ? B2R_STOP_OUT(stp) : B2R_STOP_IN(stp);
    auto const can_start = fwd ? B2R_STOP_IN(stp) : B2R_STOP_OUT(stp);
    if ((sec & 15u) != 0u && i != 0u && !section_ok(T, sb, fwd ? i - 1u : si, sec & 15u)) {
      et_valid = false;  // raptor.h:1194-1217: the section ridden lacks a flag
    }
    bool arrival_ran = false;
    if (et_valid && can_finish) {
      arrival_ran = true;
      auto const ev = colbase[n_t * (si * 2u - (fwd ? 1u : 0u)) + et_off];
      scan_arrive<true>(st, ln, s, g, bit, l, lbv, to_delta_key(fwd, et_day, ln.base, delta_count(ev)), pc);
    }
    if (i + 1u == n || !can_start || !(st.X[l * st.G + g] & bit)) continue;
    if (lbv == 0xFFFFu) break;  // raptor.h:1309-1311: no later stop of this query
    auto const board_col = n_t * (si * 2u - (fwd ? 0u : 1u));
    auto const et_time =
        et_valid ? to_delta_key(fwd, et_day, ln.base, delta_count(colbase[board_col + et_off])) : kKeyInv;
    auto const prt = dec(st.rt[rti(st, k - 1u, l, s)], ln.qtag);
    if (prt == kKeyInv || prt > et_time) continue;
    auto const minutes = static_cast<int>(ln.base) * 1440 + from_key(fwd, prt);
    uint32_t nt = 0;
    uint16_t nd = 0;
    if (!et_search(T, fwd, r, si, static_cast<uint16_t>(minutes / 1440), minutes % 1440, static_cast<int>(lbv),
                   ln.tad_k, ln.base, nt, nd, pc.ev, pc.days)) {
      continue;
    }
    // current_best (raptor.h:1328-1329) is valid whenever the arrival part
    // ran or the station carries a label of this start time
    auto const cb_valid = arrival_ran || dec(st.best[li(st, l, s)], ln.gtag) != kKeyInv ||
                          dec(st.tmp[li(st, l, s)], ln.gtag) != kKeyInv;
    if (!cb_valid || to_delta_key(fwd, nd, ln.base, delta_count(colbase[board_col + nt])) <= et_time) {
      et_valid = true;
      et_off = nt;
      et_day = nd;
    }
  }
}

// The filters of a (route, query) pair: false if the route is filtered
// out; sec receives the flags checked per section (bits 0-3) and bit 8 for
// the wheelchair profile's stop bits.
__device__ __forceinline__ bool scan_filters(dtt const& T, lane_t const& ln, uint32_t r, uint32_t& sec) {
  sec = 0u;
  if ((ln.claszes != 0xFFFFu || ln.req != 0u) && !route_allowed(T, r, ln.claszes, ln.req, sec)) return false;
  if ((ln.mode & 0x70u) == (B2R_PROFILE_WHEELCHAIR << 4)) sec |= 0x100u;
  return true;
}

// The pairs the parallel scan leaves to the sequential walk: routes without
// one trip order at every event, queries with per-section filters.  A
// thread per marked (route, group) entry, before k_route_scan (which clears
// the route marks).
__global__ void __launch_bounds__(256) k_route_scan_seq(const __grid_constant__ state st) {
  auto const& T = st.tt;
  auto const nr = st.counters[C_R];
  scan_ctr pc{0u, 0u, 0u, 0u, 0u};
  for (auto w = blockIdx.x * blockDim.x + threadIdx.x; w < nr; w += gridDim.x * blockDim.x) {
    auto const e = st.rlist[w];
    auto const g = e % st.G, r = e / st.G;
    auto const fifo = __ldg(T.route_fifo + r) != 0u;
    for (auto mask = st.R[e]; mask != 0u; mask &= mask - 1u) {
      auto const b = static_cast<uint32_t>(__ffs(mask) - 1);
      auto const ln = st.lanes[g * 32u + b];
      uint32_t sec = 0u;
      if (!ln.run || !scan_filters(T, ln, r, sec)) continue;
      if ((sec & 15u) == 0u && fifo) continue;  // k_route_scan's
      scan_walk_seq(st, ln, r, g, b, sec, pc);
    }
  }
  if (st.profile && (pc.stops | pc.ev | pc.days | pc.writes) != 0u) {
    atomicAdd(&st.prof[0], static_cast<unsigned long long>(pc.stops));
    atomicAdd(&st.prof[1], static_cast<unsigned long long>(pc.ev));
    atomicAdd(&st.prof[2], static_cast<unsigned long long>(pc.days));
    atomicAdd(&st.prof[3], static_cast<unsigned long long>(pc.writes));
    atomicAdd(&st.prof[5], static_cast<unsigned long long>(pc.warp_steps));
  }
}

// One (route, query) pair, the warp's lanes over its stops.  Prof: count
// the work for the roofline (profiling engines only).
template <bool Prof>
__device__ __forceinline__ void scan_pair(state const& st, lane_t const& ln, uint32_t r, uint32_t g, uint32_t b,
                                          uint32_t lane, scan_ctr& pc) {
  auto const& T = st.tt;
  auto const s = g * 32u + b;
  uint32_t sec = 0u;
  if (!scan_filters(T, ln, r, sec)) return;
  auto const order = static_cast<uint32_t>(__ldg(T.route_fifo + r));
  if ((sec & 15u) != 0u || order == 0u) return;  // k_route_scan_seq's
  auto const bit = 1u << b;
  auto const fwd = ln.fwd != 0;
  auto const k = static_cast<uint32_t>(ln.k);
  auto const sb = __ldg(T.route_stop_idx + r);
  auto const n = __ldg(T.route_stop_idx + r + 1) - sb;
  auto const n_t = __ldg(T.route_tr_to + r) - __ldg(T.route_tr_from + r);
  auto const* colbase = T.st + __ldg(T.route_st_from + r);
  auto const lb_off = (ln.mode & 8u) != 0u;
  // The trips' order key, below 2^21, smaller is better: with route_fifo
  // bit 1 (service day - base + 64) * n_t + transport offset (the service
  // day lies within 64 days of the base day, n_t < 2^14), else the time at
  // the route's first departure event (|t| < 2^20 minutes) + 2^20; both
  // mirrored backward, where later is better.
  // The trip carried over from the earlier chunks: key, offset, day.
  bool c_valid = false;
  uint32_t c_key = 0;
  uint32_t c_off = 0;
  uint16_t c_day = 0;
  for (auto i0 = 0u; i0 < n; i0 += 32u) {
    auto const i = i0 + lane;
    auto const act = i < n;
    auto const si = fwd ? i : n - 1u - i;
    uint32_t stp = 0, l = 0;
    bool marked = false;
    uint16_t lbv = 0;
    if (act) {
      stp = scan_stop_word(T, sb, n, fwd, i, sec);
      l = B2R_STOP_LOC(stp);
      marked = (st.X[l * st.G + g] & bit) != 0u;
      if (!lb_off) lbv = st.lb[li(st, l, s)];
    }
    auto const can_finish = act && (fwd ? B2R_STOP_OUT(stp) : B2R_STOP_IN(stp)) != 0u;
    auto const boardable = act && i + 1u != n && (fwd ? B2R_STOP_IN(stp) : B2R_STOP_OUT(stp)) != 0u && marked;
    // raptor.h:1309-1311: the walk ends at the first boardable stop the
    // query cannot reach, after that stop's arrival
    auto const brk = __ballot_sync(kFull, boardable && lbv == 0xFFFFu);
    auto const fb = brk != 0u ? static_cast<uint32_t>(__ffs(brk) - 1) : 32u;
    // this stop's earliest boardable trip (raptor.h:1313-1327)
    bool cand = false, cb_bad = false;
    uint32_t nt = 0;
    uint16_t nd = 0;
    uint32_t key = 0;
    if (boardable && lane < fb) {
      auto const prt = dec(st.rt[rti(st, k - 1u, l, s)], ln.qtag);
      if (prt != kKeyInv) {
        auto const minutes = static_cast<int>(ln.base) * 1440 + from_key(fwd, prt);
        uint32_t n_ev = 0, n_days = 0;
        auto const found = et_search(T, fwd, r, si, static_cast<uint16_t>(minutes / 1440), minutes % 1440,
                                     static_cast<int>(lbv), ln.tad_k, ln.base, nt, nd, n_ev, n_days);
        if constexpr (Prof) {
          pc.ev += n_ev;
          pc.days += n_days;
        }
        if (found) {
          cand = true;
          cb_bad = dec(st.best[li(st, l, s)], ln.gtag) == kKeyInv && dec(st.tmp[li(st, l, s)], ln.gtag) == kKeyInv;
          if ((order & 2u) != 0u) {
            auto const x = static_cast<uint32_t>(static_cast<int>(nd) - static_cast<int>(ln.base) + 64) * n_t + nt;
            key = fwd ? x : (1u << 21) - 1u - x;
          } else {
            auto const t = (static_cast<int>(nd) - static_cast<int>(ln.base)) * 1440 + delta_count(__ldg(colbase + nt));
            key = static_cast<uint32_t>((fwd ? t : -t) + (1 << 20));
          }
        }
      }
    }
    // a marked station always carries a best label of its start time
    // (marks come with best updates), so the boarding rule never meets an
    // invalid current_best; were it to, the query is failed loudly
    if (cb_bad) atomicOr(&st.counters[C_ERR], 4u);
    if constexpr (Prof) {
      if (lane == 0u) {
        pc.stops += min(n - i0, min(fb + 1u, 32u));
        ++pc.warp_steps;
      }
    }
    // prefix minimum of (key, later stop first) over the lanes: the key's
    // 21 bits above 5 for the lane
    auto v = cand ? (key << 5) | (31u - lane) : 0xFFFFFFFFu;
    for (auto o = 1u; o < 32u; o <<= 1) {
      auto const y = __shfl_up_sync(kFull, v, o);
      if (lane >= o) v = min(v, y);
    }
    auto ex = __shfl_up_sync(kFull, v, 1);  // best candidate before this stop
    if (lane == 0u) ex = 0xFFFFFFFFu;
    auto const tot = __shfl_sync(kFull, v, 31);
    auto const src = static_cast<int>(31u - (ex & 31u));
    auto const x_off = __shfl_sync(kFull, nt, src);
    auto const x_day = static_cast<uint16_t>(__shfl_sync(kFull, static_cast<uint32_t>(nd), src));
    // the carried trip loses ties to the later stops of this chunk
    auto const use_x = ex != 0xFFFFFFFFu && (!c_valid || (ex >> 5) <= c_key);
    auto const et_valid = use_x || c_valid;
    if (act && lane <= fb && et_valid && can_finish) {
      auto const et_off = use_x ? x_off : c_off;
      auto const et_day = use_x ? x_day : c_day;
      auto const ev = __ldg(colbase + n_t * (si * 2u - (fwd ? 1u : 0u)) + et_off);
      scan_arrive<Prof>(st, ln, s, g, bit, l, lbv, to_delta_key(fwd, et_day, ln.base, delta_count(ev)), pc);
    }
    if (fb != 32u) return;
    if (tot != 0xFFFFFFFFu) {
      auto const t_src = static_cast<int>(31u - (tot & 31u));
      auto const t_off = __shfl_sync(kFull, nt, t_src);
      auto const t_day = static_cast<uint16_t>(__shfl_sync(kFull, static_cast<uint32_t>(nd), t_src));
      auto const t_key = tot >> 5;
      if (!c_valid || t_key <= c_key) {
        c_valid = true;
        c_key = t_key;
        c_off = t_off;
        c_day = t_day;
      }
    }
  }
}

// A warp per marked (route, group of 32 queries) entry, one pair of the
// entry after the other.  Builds with four, five or six blocks of 256
// threads resident per SM (the launch shape picks one), and with work
// counters for profiling engines.
template <int MinBlocks, bool Prof>
__global__ void __launch_bounds__(256, MinBlocks) k_route_scan(const __grid_constant__ state st) {
  auto const lane = threadIdx.x & 31u;
  auto const warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  auto const n_warps = (gridDim.x * blockDim.x) >> 5;
  auto const nr = st.counters[C_R];
  scan_ctr pc{0u, 0u, 0u, 0u, 0u};
  for (auto w = warp; w < nr; w += n_warps) {
    auto const e = st.rlist[w];
    auto mask = st.R[e];
    __syncwarp();
    if (lane == 0u) st.R[e] = 0u;
    auto const g = e % st.G, r = e / st.G;
    while (mask != 0u) {
      auto const b = static_cast<uint32_t>(__ffs(mask) - 1);
      mask &= mask - 1u;
      auto const ln = st.lanes[g * 32u + b];
      if (!ln.run) continue;
      scan_pair<Prof>(st, ln, r, g, b, lane, pc);
      __syncwarp();
    }
  }
  if constexpr (Prof) {  // work counters for the roofline (warp-reduced)
    __syncwarp();
    for (auto o = 16; o > 0; o >>= 1) {
      pc.stops += __shfl_xor_sync(kFull, pc.stops, o);
      pc.ev += __shfl_xor_sync(kFull, pc.ev, o);
      pc.days += __shfl_xor_sync(kFull, pc.days, o);
      pc.writes += __shfl_xor_sync(kFull, pc.writes, o);
      pc.warp_steps += __shfl_xor_sync(kFull, pc.warp_steps, o);
    }
    if (lane == 0) {
      atomicAdd(&st.prof[0], static_cast<unsigned long long>(pc.stops));
      atomicAdd(&st.prof[1], static_cast<unsigned long long>(pc.ev));
      atomicAdd(&st.prof[2], static_cast<unsigned long long>(pc.days));
      atomicAdd(&st.prof[3], static_cast<unsigned long long>(pc.writes));
      atomicAdd(&st.prof[5], static_cast<unsigned long long>(pc.warp_steps));  // warp stop steps
    }
  }
}
// update_rt_transport, raptor.h:1068-1175 (no vias), a lane per marked
// (rt transport, query) pair walking the run in search direction: et is
// whether the query rides the run when it passes the stop.  The filters are
// loop_rt_routes' (raptor.h:583-626): the class of the first section and
// the route flags, section by section where set on some sections only.
__global__ void k_rt_scan(state st) {
  auto const& T = st.tt;
  for_each_pair(
      st.rtlist, st.counters[C_RT],
      [&](uint32_t e) {
        auto const m = st.RT_R[e];
        st.RT_R[e] = 0u;
        return m;
      },
      [&](uint32_t e, uint32_t b) {
        auto const g = e % st.G, x = e / st.G;
        auto const s = g * 32u + b;
        auto const ln = st.lanes[s];
        if (!ln.run) return;
        uint32_t sec = 0u;
        if ((ln.claszes != 0xFFFFu || ln.req != 0u) && !filter_allowed(T.rt_filter[x], ln.claszes, ln.req, sec)) {
          return;
        }
        if ((ln.mode & 0x70u) == (B2R_PROFILE_WHEELCHAIR << 4)) sec |= 0x100u;
        auto const bit = 1u << b;
        auto const fwd = ln.fwd != 0;
        auto const k = static_cast<uint32_t>(ln.k);
        auto const sb = T.rt_stop_idx[x];
        auto const n = T.rt_stop_idx[x + 1] - sb;
        auto const* tm = T.rt_times + 2ull * (sb - x);
        auto const base_min = (T.internal_from_days + static_cast<int32_t>(ln.base)) * 1440;
        auto const lb_off = (ln.mode & 8u) != 0u;
        scan_ctr pc{};
        bool et = false;
        for (auto i = 0u; i != n; ++i) {
          auto const si = fwd ? i : n - 1u - i;
          auto w = T.rt_stops[sb + si];
          if ((sec & 0x100u) != 0u) w = (w & 0xCFFFFFFFu) | ((w >> 2) & 0x30000000u);
          auto const l = B2R_STOP_LOC(w);
          if ((sec & 15u) != 0u && i != 0u &&
              (static_cast<uint32_t>(T.rt_sec[sb + (fwd ? si - 1u : si)]) & (sec & 15u)) != (sec & 15u)) {
            et = false;
          }
          auto const lbv = lb_off ? uint16_t{0} : st.lb[li(st, l, s)];
          if (et && (fwd ? si != 0u : si + 1u != n) && (fwd ? B2R_STOP_OUT(w) : B2R_STOP_IN(w))) {
            auto const by = to_key(fwd, clamp16(tm[2u * si - (fwd ? 1u : 0u)] - base_min));
            scan_arrive<false>(st, ln, s, g, bit, l, lbv, by, pc);
          }
          if (lbv == 0xFFFFu) break;  // raptor.h:1156-1158: before the boarding test
          if (i + 1u == n || !(fwd ? B2R_STOP_IN(w) : B2R_STOP_OUT(w)) || !(st.X[l * st.G + g] & bit)) continue;
          auto const by = to_key(fwd, clamp16(tm[2u * si - (fwd ? 0u : 1u)] - base_min));
          if (dec(st.rt[rti(st, k - 1u, l, s)], ln.qtag) <= by) et = true;
        }
      });
}

// frontier list of the stations marked this round (transfers, footpaths,
// start labels): every nonzero station-mark word (location, group)
__global__ void k_list_marked(state st) { list_nonzero(st, st.X, st.tt.n_loc * st.G, st.xlist, C_X); }

// frontier list of the stations reached by the route scan: every nonzero
// route-reached word (location, group)
__global__ void k_list_reached(state st) { list_nonzero(st, st.Y, st.tt.n_loc * st.G, st.ylist, C_Y); }

__global__ void k_clear_x(state st) {
  auto const tid = blockIdx.x * blockDim.x + threadIdx.x;
  auto const nx = st.counters[C_X];
  for (auto i = tid; i < nx; i += gridDim.x * blockDim.x) st.X[st.xlist[i]] = 0u;
}


// ---------------------------------------------------- transfer phase
// Destination stations of station-to-station queries first, in location
// order, so that the time_at_dest updates they make (raptor.h:737-739) are
// seen by later stations exactly as in the sequential loop; the timeline of
// those updates is kept per query.
__global__ void k_transfers_pre(state st) {
  auto const s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s == 0) st.counters[C_X] = 0u;  // k_clear_x has cleared the listed marks
  if (s >= st.S) return;
  auto& sl = st.slots[s];
  auto const ln = st.lanes[s];
  st.timeline_n[s] = 0u;
  if (!ln.run) return;
  st.tad_phase[s] = sl.tad[ln.k];
  if (!(ln.mode & 2u)) return;
  auto const k = ln.k;
  auto const g = s >> 5;
  auto const bit = 1u << (s & 31);
  uint32_t tl_n = 0;
  for (auto i = 0u; i != sl.n_dest; ++i) {
    auto const d = st.dest_pool[sl.dest_off + i].loc;
    if (!(st.Y[d * st.G + g] & bit)) continue;
    auto const tk = dec(st.tmp[li(st, d, s)], ln.gtag);
    if (tk == kKeyInv) continue;
    auto const fp = key_add(tk, 0);
    auto const bk = dec(st.best[li(st, d, s)], ln.gtag);
    auto& rtw = st.rt[rti(st, k, d, s)];
    if (ln.blast == 0u && fp < bk && fp < dec(rtw, ln.qtag)) {
      rtw = enc(ln.qtag, fp);
      touch(st, ln, k, d, s);
    }
    auto const tad = static_cast<int>(sl.tad[k]);
    if (fp < bk && fp <= tad) {
      auto const lbv = (ln.mode & 8u) ? uint16_t{0} : st.lb[li(st, d, s)];
      if (lbv == 0xFFFFu || fp + static_cast<int>(lbv) > tad) continue;
      if (!within_bounds(st, s, ln.blast, k, d, fp)) continue;
      rtw = enc(ln.qtag, fp);
      touch(st, ln, k, d, s);
      st.best[li(st, d, s)] = enc(ln.gtag, fp);
      atomicOr(&st.X[d * st.G + g], bit);  // listed by k_list_marked
      if (fp < tad && tl_n < kMaxTimeline) {
        st.timeline[s * kMaxTimeline + tl_n++] = {d, 0u, fp};
      } else if (fp < tad) {
        atomicOr(&st.counters[C_ERR], 1u);
      }
      update_tad(sl, k, fp);
    }
  }
  st.timeline_n[s] = tl_n;
}

// tad in effect at position (hi, lo) of the phase's processing order
__device__ __forceinline__ int tad_at(state const& st, uint32_t s, uint32_t hi, uint32_t lo) {
  auto const n = st.timeline_n[s];
  int tad = st.tad_phase[s];
  for (auto i = 0u; i != n; ++i) {
    auto const& e = st.timeline[s * kMaxTimeline + i];
    if (e.pos_hi < hi || (e.pos_hi == hi && e.pos_lo < lo)) tad = e.tad;
    else break;
  }
  return tad;
}

// update_transfers, raptor.h:680-743: lane per reached (station, query)
__global__ void k_transfers(state st) {
  for_each_pair(
      st.ylist, st.counters[C_Y], [&](uint32_t e) { return st.Y[e]; },
      [&](uint32_t e, uint32_t b) {
        auto const g = e % st.G, l = e / st.G;
        auto const s = g * 32u + b;
        auto const ln = st.lanes[s];
        if (!ln.run || ((ln.mode & 2u) && ((st.D[e] >> b) & 1u))) return;
        auto const tk = dec(st.tmp[li(st, l, s)], ln.gtag);
        if (tk == kKeyInv) return;
        auto const slp = &st.slots[s];
        auto const tt = static_cast<int>(adjusted<int>(slp->tts, static_cast<int>(st.tt.transfer_time[l])));
        auto const fp = key_add(tk, tt);
        auto const bk = dec(st.best[li(st, l, s)], ln.gtag);
        auto& rtw = st.rt[rti(st, ln.k, l, s)];
        if (ln.blast == 0u && fp < bk && fp < dec(rtw, ln.qtag)) {
          rtw = enc(ln.qtag, fp);
          touch(st, ln, ln.k, l, s);
        }
        auto const tad = (ln.mode & 2u) ? tad_at(st, s, l, 0u) : static_cast<int>(st.tad_phase[s]);
        if (fp < bk && fp <= tad) {
          auto const lbv = (ln.mode & 8u) ? uint16_t{0} : st.lb[li(st, l, s)];
          if (lbv != 0xFFFFu && fp + static_cast<int>(lbv) <= tad &&
              within_bounds(st, s, ln.blast, ln.k, l, fp)) {
            rtw = enc(ln.qtag, fp);
            touch(st, ln, ln.k, l, s);
            st.best[li(st, l, s)] = enc(ln.gtag, fp);
            atomicOr(&st.X[e], 1u << b);  // listed by k_list_marked
          }
        }
      });
}

// update_intermodal_footpaths, raptor.h:954-1026: per query, its egress
// stations in location order
__device__ void intermodal_slot(state const& st, uint32_t s) {
  auto const ln = st.lanes[s];
  if (!ln.run || !(ln.mode & 1u)) return;
  auto& sl = st.slots[s];
  auto const g = s >> 5;
  auto const bit = 1u << (s & 31);
  for (auto i = 0u; i != sl.n_dest; ++i) {
    auto const dr = st.dest_pool[sl.dest_off + i];
    if (!(st.Y[dr.loc * st.G + g] & bit)) continue;
    auto const tk = dec(st.tmp[li(st, dr.loc, s)], ln.gtag);
    if (tk == kKeyInv) continue;
    auto const end_time = key_add(tk, static_cast<int>(dr.dist));
    if (end_time <= sl.tad[ln.k]) {
      st.rt[rti(st, ln.k, B2R_SPECIAL_END, s)] = enc(ln.qtag, end_time);
      touch(st, ln, ln.k, B2R_SPECIAL_END, s);
      st.best[li(st, B2R_SPECIAL_END, s)] = enc(ln.gtag, end_time);
      update_tad(sl, ln.k, end_time);
    }
  }
}

// ---------------------------------------------------- footpath phase
struct fp_cand {
  uint32_t src, pos, dest;
  int key;
};

// footpaths into destination stations, in the reference's processing order
// (source location, then position in the source's footpath list)
__device__ void footpaths_pre_slot(state const& st, uint32_t s) {
  auto& sl = st.slots[s];
  auto const ln = st.lanes[s];
  st.timeline_n[s] = 0u;
  if (!ln.run) return;
  st.tad_phase[s] = sl.tad[ln.k];
  if (!(ln.mode & 2u)) return;
  auto const fwd = ln.fwd != 0;
  auto const k = ln.k;
  auto const g = s >> 5;
  auto const bit = 1u << (s & 31);
  auto const& T = st.tt;
  constexpr int kMaxC = 64;
  fp_cand c[kMaxC];
  int nc = 0;
  for (auto i = 0u; i != sl.n_dest; ++i) {
    auto const d = st.dest_pool[sl.dest_off + i].loc;
    auto const prf = (static_cast<uint32_t>(ln.mode) >> 4) & 7u;
    auto const* iidx = fp_index(T, prf, !fwd);
    auto const* idat = fp_words(T, prf, !fwd);
    for (auto x = iidx[d]; x != iidx[d + 1]; ++x) {
      auto const src = B2R_FP_TARGET(idat[x]);
      if (!(st.Y[src * st.G + g] & bit)) continue;
      auto const tk = dec(st.tmp[li(st, src, s)], ln.gtag);
      if (tk == kKeyInv) continue;
      auto const* oidx = fp_index(T, prf, fwd);
      auto const* odat = fp_words(T, prf, fwd);
      for (auto y = oidx[src]; y != oidx[src + 1]; ++y) {
        if (B2R_FP_TARGET(odat[y]) != d) continue;
        if (nc == kMaxC) {
          atomicOr(&st.counters[C_ERR], 2u);
          break;
        }
        auto const dur = adjusted<int>(sl.tts, static_cast<int>(B2R_FP_DURATION(odat[y])));
        c[nc++] = {src, y - oidx[src], d, key_add(tk, dur)};
        break;
      }
    }
  }
  for (int a = 1; a < nc; ++a) {  // insertion sort by (src, pos)
    auto const x = c[a];
    int b = a - 1;
    while (b >= 0 && (c[b].src > x.src || (c[b].src == x.src && c[b].pos > x.pos))) {
      c[b + 1] = c[b];
      --b;
    }
    c[b + 1] = x;
  }
  uint32_t tl_n = 0;
  for (int a = 0; a < nc; ++a) {
    auto const d = c[a].dest;
    auto const fp = c[a].key;
    auto const bk = dec(st.best[li(st, d, s)], ln.gtag);
    auto& rtw = st.rt[rti(st, k, d, s)];
    if (ln.blast == 0u && fp < bk && fp < dec(rtw, ln.qtag)) {
      rtw = enc(ln.qtag, fp);
      touch(st, ln, k, d, s);
    }
    auto const tad = static_cast<int>(sl.tad[k]);
    if (fp < bk && fp <= tad) {
      auto const lbv = (ln.mode & 8u) ? uint16_t{0} : st.lb[li(st, d, s)];
      if (lbv == 0xFFFFu || fp + static_cast<int>(lbv) > tad) continue;
      if (!within_bounds(st, s, ln.blast, k, d, fp)) continue;
      rtw = enc(ln.qtag, fp);
      touch(st, ln, k, d, s);
      st.best[li(st, d, s)] = enc(ln.gtag, fp);
      atomicOr(&st.X[d * st.G + g], bit);  // listed by k_list_marked
      if (fp < tad && tl_n < kMaxTimeline) {
        st.timeline[s * kMaxTimeline + tl_n++] = {c[a].src, c[a].pos, fp};
      } else if (fp < tad) {
        atomicOr(&st.counters[C_ERR], 1u);
      }
      update_tad(sl, k, fp);
    }
  }
  st.timeline_n[s] = tl_n;
}

// update_intermodal_footpaths, then the footpaths into destination
// stations, per slot (the order of raptor.h:376-378)
__global__ void k_intermodal_fp_pre(state st) {
  auto const s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= st.S) return;
  intermodal_slot(st, s);
  footpaths_pre_slot(st, s);
}

// update_footpaths, raptor.h:745-845: lane per reached (station, query),
// walking the station's footpaths; labels of footpath targets are combined
// with atomicMin (the phase's final labels and marks do not depend on the
// processing order).
__global__ void k_footpaths(state st) {
  auto const& T = st.tt;
  for_each_pair(
      st.ylist, st.counters[C_Y], [&](uint32_t e) { return st.Y[e]; },
      [&](uint32_t e, uint32_t b) {
        auto const g = e % st.G, src = e / st.G;
        auto const s = g * 32u + b;
        auto const ln = st.lanes[s];
        if (!ln.run) return;
        auto const tk = dec(st.tmp[li(st, src, s)], ln.gtag);
        if (tk == kKeyInv) return;
        auto const fwd = ln.fwd != 0;
        auto const prf = (static_cast<uint32_t>(ln.mode) >> 4) & 7u;
        auto const* idx = fp_index(T, prf, fwd);
        auto const* dat = fp_words(T, prf, fwd);
        auto const fb = idx[src], n = idx[src + 1] - fb;
        slot_t const* slp = &st.slots[s];
        auto const tad_flat = (ln.mode & 2u) ? 0 : static_cast<int>(slp->tad[ln.k]);
        for (auto j = 0u; j != n; ++j) {
          auto const fp = dat[fb + j];
          auto const tgt = B2R_FP_TARGET(fp);
          if ((ln.mode & 2u) && ((st.D[tgt * st.G + g] >> b) & 1u)) continue;
          auto const key = key_add(tk, adjusted<int>(slp->tts, static_cast<int>(B2R_FP_DURATION(fp))));
          auto const bk = dec(st.best[li(st, tgt, s)], ln.gtag);
          if (key >= bk) continue;
          // the reference writes round_times ahead of its pruning only when
          // unbounded (raptor.h:790-794)
          if (ln.blast == 0u) {
            atomicMin(&st.rt[rti(st, ln.k, tgt, s)], enc(ln.qtag, key));
            touch(st, ln, ln.k, tgt, s);
          }
          auto const tad = (ln.mode & 2u) ? tad_at(st, s, src, j) : tad_flat;
          if (key > tad) continue;
          auto const lbv = (ln.mode & 8u) ? uint16_t{0} : st.lb[li(st, tgt, s)];
          if (lbv != 0xFFFFu && key + static_cast<int>(lbv) <= tad) {
            if (ln.blast != 0u) {
              if (!within_bounds(st, s, ln.blast, ln.k, tgt, key)) continue;
              atomicMin(&st.rt[rti(st, ln.k, tgt, s)], enc(ln.qtag, key));
              touch(st, ln, ln.k, tgt, s);
            }
            atomicMin(&st.best[li(st, tgt, s)], enc(ln.gtag, key));
            atomicOr(&st.X[tgt * st.G + g], 1u << b);  // listed by k_list_marked
          }
        }
      });
}

// ------------------------------------------------- round end / results
__device__ void ctl_end_slot(state const& st, uint32_t s) {
  auto& sl = st.slots[s];
  if (sl.state != S_RUN) return;
  sl.k = static_cast<uint8_t>(sl.k + 1);
  if (sl.k >= sl.end_k) sl.state = S_COLLECT;
}

__host__ __device__ inline bool dominates(journey_rec const& a, journey_rec const& b) {  // journey.h:84-92
  if (a.start_time <= a.dest_time) {
    return a.transfers <= b.transfers && a.start_time >= b.start_time && a.dest_time <= b.dest_time;
  }
  return a.transfers <= b.transfers && a.start_time <= b.start_time && a.dest_time >= b.dest_time;
}

__device__ int alloc_block(state const& st, uint32_t s) {
  auto const words = (st.max_j + 31u) / 32u;
  for (auto w = 0u; w != words; ++w) {
    auto& u = st.blocks_used[s * words + w];
    auto const free_bits = ~u;
    if (free_bits != 0u) {
      auto const b = __ffs(free_bits) - 1;
      if (w * 32u + b >= st.max_j) break;
      u |= 1u << b;
      return static_cast<int>(w * 32u + b);
    }
  }
  return -1;
}

__device__ void free_block(state const& st, uint32_t s, uint16_t blk) {
  auto const words = (st.max_j + 31u) / 32u;
  st.blocks_used[s * words + blk / 32u] &= ~(1u << (blk % 32u));
}

// pareto_set::add, pareto_set.h:21-37
__device__ bool pareto_add(state const& st, uint32_t s, slot_t& sl, journey_rec el) {
  auto* els = st.journeys + static_cast<size_t>(s) * st.max_j;
  uint32_t n_removed = 0;
  for (auto i = 0u; i < sl.n_journeys; ++i) {
    if (dominates(els[i], el)) return true;
    if (dominates(el, els[i])) {
      free_block(st, s, els[i].block);
      ++n_removed;
      continue;
    }
    els[i - n_removed] = els[i];
  }
  sl.n_journeys -= n_removed;
  auto const blk = alloc_block(st, s);
  if (blk < 0 || sl.n_journeys >= st.max_j) return false;
  el.block = static_cast<uint16_t>(blk);
  els[sl.n_journeys++] = el;
  return true;
}

// whether journey j of the slot is to be reconstructed now (search.h:457-475;
// a pong phase rebuilds only the journey of its ping result, pong.cc:322-339)
__device__ __forceinline__ bool recon_wanted(slot_t const& sl, journey_rec const& j) {
  if (j.reconstructed || j.error) return false;
  auto const tt = j.dest_time > j.start_time ? j.dest_time - j.start_time : j.start_time - j.dest_time;
  return sl.recon_mode == 0 ? ((sl.ontrip || (sl.iv_from <= j.start_time && j.start_time < sl.iv_to)) &&
                               tt < sl.fastest_direct)
         : sl.recon_mode == 1 ? (j.transfers == sl.recon_transfers && j.start_time == sl.recon_start)
                              : false;
}

// result collection (raptor.h:393-413) and the reconstruction worklist
// (search.h:457-475)
__device__ void collect_slot(state const& st, uint32_t s) {
  auto& sl = st.slots[s];
  if (sl.state != S_COLLECT || sl.one_to_all) return;
  auto const qtag = tagcode(sl.gen_query);
  auto const fwd = sl.fwd != 0;
  auto const n_d = sl.intermodal_dest ? 1u : sl.n_dest;
  for (auto i = 0u; i != n_d; ++i) {
    auto const d = sl.intermodal_dest ? B2R_SPECIAL_END : st.dest_pool[sl.dest_off + i].loc;
    for (auto k = 1u; k < sl.end_k; ++k) {
      auto const key = dec(st.rt[rti(st, k, d, s)], qtag);
      if (key == kKeyInv) continue;
      journey_rec j{};
      j.start_time = sl.cur_start_time;
      j.dest_time = sl.base_days * 1440 + from_key(fwd, key);
      j.dest = d;
      j.transfers = static_cast<uint8_t>(k - 1);
      if (!pareto_add(st, s, sl, j)) {
        sl.error = B2R_ERR_CAPACITY;
        sl.state = S_ERROR;
        return;
      }
    }
  }
  if (sl.recon_defer) return;  // rebuilt when the slot is done (k_reconstruct_done)
  auto* els = st.journeys + static_cast<size_t>(s) * st.max_j;
  for (auto i = 0u; i != sl.n_journeys; ++i) {
    if (recon_wanted(sl, els[i])) st.recon_list[atomicAdd(&st.counters[C_RECON], 1u)] = (s << 16) | i;
  }
}

// end of the round, then result collection when the group's rounds are done
__global__ void k_end_collect(state st) {
  auto const s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= st.S) return;
  ctl_end_slot(st, s);
  collect_slot(st, s);
}

// One journey (slot s, index ji) rebuilt by the calling warp.
__device__ __forceinline__ void reconstruct_one(state const& st, uint32_t s, uint32_t ji, uint32_t lane) {
  {
    uint64_t t_begin = 0;
    if (st.profile) asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_begin));
    auto& sl = st.slots[s];
    auto& j = st.journeys[static_cast<size_t>(s) * st.max_j + ji];
    recon_ctx c;
    c.st = &st;
    c.T = &st.tt;
    c.sl = &sl;
    c.s = s;
    c.fwd = sl.fwd != 0;
    c.qtag = tagcode(sl.gen_query);
    c.base_days = sl.base_days;
    c.base = sl.base;
    c.ontrip = sl.ontrip != 0;
    c.j = &j;
    c.lane = lane;
    c.legs = st.legs + (static_cast<size_t>(s) * st.max_j + j.block) * kMaxLegs;
    c.run();
    __syncwarp();
    if (lane == 0) {
      if (c.failed) {
        j.error = 1;
      } else {
        j.reconstructed = 1;
        j.n_legs = static_cast<uint16_t>(c.n_legs);
      }
      if (st.profile) {  // longest single reconstruction (ns), journeys
        uint64_t t_end = 0;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_end));
        atomicMax(&st.prof[6], static_cast<unsigned long long>(t_end - t_begin));
        atomicAdd(&st.prof[7], 1ull);
      }
    }
  }
}

// the journeys collected in this super-step (queries with several
// start-time groups: their next group changes the round times)
__global__ void k_reconstruct(state st) {
  auto const lane = threadIdx.x & 31u;
  auto const warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  auto const n_warps = (gridDim.x * blockDim.x) >> 5;
  auto const n = st.counters[C_RECON];
  for (auto i = warp; i < n; i += n_warps) {
    auto const e = st.recon_list[i];
    reconstruct_one(st, e >> 16, e & 0xFFFFu, lane);
  }
}

// One given journey of slot s (index ji), one warp: the Algo interface's
// reconstruct.
__global__ void k_reconstruct_one(state st, uint32_t s, uint32_t ji) {
  reconstruct_one(st, s, ji, threadIdx.x & 31u);
}

// The journeys of finished slots whose reconstruction was deferred, listed
// by the host as (slot << 16 | journey index): launched on the export stream
// while the next super-steps run.  A finished slot is left alone by the
// super-step kernels, so its round times are stable.
__global__ void k_reconstruct_done(state st, uint32_t const* list, uint32_t n) {
  auto const lane = threadIdx.x & 31u;
  auto const warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  auto const n_warps = (gridDim.x * blockDim.x) >> 5;
  for (auto i = warp; i < n; i += n_warps) {
    auto const e = list[i];
    auto const s = e >> 16, ji = e & 0xFFFFu;
    auto const& sl = st.slots[s];
    if (!sl.recon_defer || ji >= sl.n_journeys) continue;
    if (!recon_wanted(sl, st.journeys[static_cast<size_t>(s) * st.max_j + ji])) continue;
    reconstruct_one(st, s, ji, lane);
  }
}

// early termination (search.h:477-492) and seeding of the next start-time
// group: next_start_time + add_start (raptor.h:179-203) + the
// time_at_dest bound of execute (raptor.h:211-214)
__device__ void next_slot(state const& st, uint32_t s) {
  auto& sl = st.slots[s];
  if (sl.state != S_COLLECT && sl.state != S_START) return;
  auto const fwd = sl.fwd != 0;
  if (sl.state == S_COLLECT && sl.min_connection_count > 0 && !sl.one_to_all) {
    uint32_t n_in = 0;
    auto* els = st.journeys + static_cast<size_t>(s) * st.max_j;
    for (auto i = 0u; i != sl.n_journeys; ++i) {
      n_in += sl.ontrip ? 1u : ((sl.iv_from <= els[i].start_time && els[i].start_time < sl.iv_to) ? 1u : 0u);
    }
    if (n_in >= sl.min_connection_count &&
        ((fwd && sl.extend_earlier && !sl.extend_later) || (!fwd && !sl.extend_earlier && sl.extend_later))) {
      sl.early_term = 1;
      if (fwd) sl.iv_from = sl.cur_start_time;
      else sl.iv_to = sl.cur_start_time + 1;
    }
  }
  if (sl.state == S_COLLECT) sl.need_sweep = 1;
  auto const* starts = st.start_pool + sl.starts_off;
  if (sl.early_term || sl.next_start >= sl.n_starts) {
    sl.state = S_DONE;
    return;
  }
  // next start-time group
  auto const g0 = sl.next_start;
  auto const tas = starts[g0].time_at_start;
  auto g1 = g0 + 1;
  while (g1 < sl.n_starts && starts[g1].time_at_start == tas) ++g1;
  if (sl.gen_group >= 0xFFFEu) {  // tag space exhausted: clear this slot's labels
    for (auto l = 0u; l != st.tt.n_loc; ++l) {
      st.best[li(st, l, s)] = 0xFFFFFFFFu;
      st.tmp[li(st, l, s)] = 0xFFFFFFFFu;
    }
    sl.gen_group = 0;
  }
  ++sl.gen_group;
  auto const gtag = tagcode(sl.gen_group), qtag = tagcode(sl.gen_query);
  auto const g = s >> 5;
  auto const bit = 1u << (s & 31);
  for (auto i = g0; i != g1; ++i) {
    auto const l = starts[i].stop;
    auto const key = to_key(fwd, clamp16(starts[i].time_at_stop - sl.base_days * 1440));
    auto& bw = st.best[li(st, l, s)];
    if (key < dec(bw, gtag)) bw = enc(gtag, key);
    auto& rw = st.rt[rti(st, 0, l, s)];
    if (key < dec(rw, qtag)) rw = enc(qtag, key);
    atomicOr(&st.X[l * st.G + g], bit);  // listed by k_list_marked
  }
  auto const worst = tas + (fwd ? static_cast<int>(sl.span) : -static_cast<int>(sl.span));
  auto const d_worst = to_key(fwd, clamp16(worst - sl.base_days * 1440));
  for (auto i = 0; i != kK; ++i) {
    if (d_worst < sl.tad[i]) sl.tad[i] = static_cast<int16_t>(d_worst);
  }
  sl.cur_start_time = tas;
  sl.next_start = g1;
  sl.k = 1;
  sl.state = S_RUN;
  ++sl.n_groups_run;
}

// the next start-time group, then the slot's state for the host
__global__ void k_next_summary(state st) {
  auto const s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= st.S) return;
  next_slot(st, s);
  auto const& sl = st.slots[s];
  st.summary[s] = {sl.state, {0, 0, 0}, sl.n_journeys};
}

// ------------------------------------------------------- lower bounds
// Dijkstra from the destinations over the lower-bound graph (dijkstra.cc:
// 18-67, dial.h), computed for all newly admitted queries at once as a
// frontier-driven Bellman-Ford: distances are shortest-path lengths capped
// below kMaxTravelTime + 1 = 7201 (the dial's bucket count), which no
// processing order changes (all weights are non-negative).
constexpr uint32_t kLbBuckets = B2R_MAX_TRAVEL_TIME_MIN + 1;

__global__ void k_lb_relax(state st, uint32_t p) {
  auto const lane = threadIdx.x & 31u;
  auto const warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  auto const n_warps = (gridDim.x * blockDim.x) >> 5;
  auto const n = st.counters[C_F0 + p];
  auto const& T = st.tt;
  for (auto w = warp; w < n; w += n_warps) {
    auto const e = st.flist[p][w];
    auto const g = e % st.G, l = e / st.G;
    auto const m = st.F[p][e];
    auto const s = g * 32u + lane;
    auto const& sl = st.slots[s];
    bool act = (m >> lane) & 1u;
    auto const qtag = tagcode(sl.gen_query);
    int d = kKeyInv;
    if (act) {
      d = dec(st.dist[li(st, l, s)], qtag);
      act = d != kKeyInv;
    }
    auto const fwd = sl.fwd != 0;
    auto const* gi = fwd ? T.lbg_fwd_idx : T.lbg_bwd_idx;
    auto const* gd = fwd ? T.lbg_fwd : T.lbg_bwd;
    auto const b = act ? gi[l] : 0u;
    auto const cnt = act ? gi[l + 1] - b : 0u;
    auto n_max = cnt;
    for (auto o = 16; o > 0; o >>= 1) n_max = max(n_max, __shfl_xor_sync(kFull, n_max, o));
    for (auto j = 0u; j != n_max; ++j) {
      bool improved = false;
      uint32_t tgt = 0;
      if (j < cnt) {
        auto const edge = gd[b + j];
        tgt = B2R_FP_TARGET(edge);
        auto const nd = static_cast<uint32_t>(d) + B2R_FP_DURATION(edge);
        if (nd < kLbBuckets) {
          auto const word = enc(qtag, static_cast<int>(nd));
          auto* dp = &st.dist[li(st, tgt, s)];
          if (word < *dp) improved = word < atomicMin(dp, word);
          if (improved && st.profile) atomicAdd(&st.prof[4], 1ull);
        }
      }
      mark_warp(st, st.F[1 - p], st.flist[1 - p], C_F0 + (1 - p), improved, tgt * st.G + g, lane);
    }
  }
}

__global__ void k_lb_clear(state st, uint32_t p) {
  auto const n = st.counters[C_F0 + p];
  for (auto i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    st.F[p][st.flist[p][i]] = 0u;
  }
}

__global__ void k_lb_reset(state st, uint32_t p) {
  if (blockIdx.x == 0 && threadIdx.x == 0) st.counters[C_F0 + p] = 0u;
}

// children inherit their parent's bound (dijkstra.cc:60-65), in location
// order per query
__global__ void k_lb_children(state st) {
  auto const s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= st.S || !((st.lb_mask[s >> 5] >> (s & 31)) & 1u)) return;
  auto const qtag = tagcode(st.slots[s].gen_query);
  auto const& T = st.tt;
  for (auto x = 0u; x != T.n_with_children; ++x) {
    auto const i = T.with_children[x];
    auto const lbw = st.dist[li(st, i, s)];
    for (auto c = T.children_idx[i]; c != T.children_idx[i + 1]; ++c) {
      auto* cw = &st.dist[li(st, T.children[c], s)];
      if (dec(lbw, qtag) < dec(*cw, qtag)) *cw = lbw;
    }
  }
}

// tagged distances -> the u16 lower-bound column (unreachable = 0xFFFF)
__global__ void k_lb_finish(state st) {
  auto const n = static_cast<size_t>(st.tt.n_loc) * st.S;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    auto const s = static_cast<uint32_t>(i % st.S);
    if (!((st.lb_mask[s >> 5] >> (s & 31)) & 1u)) continue;
    auto const d = dec(st.dist[i], tagcode(st.slots[s].gen_query));
    st.lb[i] = d == kKeyInv ? uint16_t{0xFFFFu} : static_cast<uint16_t>(d);
  }
}

}  // namespace b2r::dev
