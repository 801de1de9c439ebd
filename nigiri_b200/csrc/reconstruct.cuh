// Device-side journey reconstruction: one warp per journey walks the round
// times of its query backwards (src/routing/raptor/reconstruct.cc:22-877 for
// Vias = 0 and no real-time overlay) and then applies the footpath
// optimisations of src/routing/raptor/optimize_footpaths.cc.  The search for
// the transport that produced a label is split across the lanes (one
// (route, stop position) candidate per lane); a ballot keeps the first
// success in the reference's iteration order.  The sequential parts run
// redundantly on all lanes; lane 0 owns the journey's leg block.
#pragma once

#include "engine.cuh"

namespace b2r::dev {

struct recon_ctx {
  state const* st;
  dtt const* T;
  slot_t const* sl;
  uint32_t s;          // slot
  bool fwd;
  uint16_t qtag;
  int32_t base_days;
  uint16_t base;
  bool ontrip;
  journey_rec* j;
  b2r_leg* legs;       // kMaxLegs, written by lane 0
  int n_legs;
  bool failed;
  uint32_t lane;
  b2r_leg last;        // last pushed leg (all lanes)

  // ------------------------------------------------------------- access
  __device__ int rt_t(unsigned k, uint32_t l) const {  // delta_t of round_times[k][l]
    auto const key = dec(st->rt[(static_cast<size_t>(k) * T->n_loc + l) * st->S + s], qtag);
    return from_key(fwd, key);
  }
  __device__ int inv() const { return fwd ? 32767 : -32768; }
  __device__ bool beq(int a, int b) const { return fwd ? a <= b : a >= b; }
  __device__ int dir(int a) const { return fwd ? a : -a; }
  __device__ uint32_t n_stops(uint32_t r) const { return T->route_stop_idx[r + 1] - T->route_stop_idx[r]; }
  __device__ uint32_t stopw(uint32_t r, uint32_t i) const { return T->route_stops[T->route_stop_idx[r] + i]; }
  __device__ uint16_t ev(uint32_t t, uint32_t s_idx, bool arr) const {
    auto const r = T->transport_route[t];
    auto const n_t = T->route_tr_to[r] - T->route_tr_from[r];
    return T->st[T->route_st_from[r] + n_t * (s_idx * 2u - (arr ? 1u : 0u)) + (t - T->route_tr_from[r])];
  }
  __device__ int32_t ev_time(uint32_t t, uint16_t day, uint32_t s_idx, bool arr) const {
    auto const e = ev(t, s_idx, arr);
    return (T->internal_from_days + static_cast<int32_t>(day)) * 1440 + (e & 31) * 1440 + (e >> 5);
  }
  __device__ int unix_to_delta(int32_t t) const { return clamp16(t - base_days * 1440); }
  __device__ int32_t delta_to_unix(int d) const { return base_days * 1440 + d; }
  __device__ b2r_offset const* start_offs() const { return st->off_pool + sl->soff_off; }
  __device__ b2r_offset const* dest_offs() const { return st->off_pool + sl->doff_off; }

  __device__ uint32_t root(uint32_t idx) const {
    if (T->parent == nullptr) return idx;
    auto l = idx;
    for (int i = 0;; ++i) {
      auto const p = T->parent[l];
      if (p == B2R_INVALID_IDX) break;
      if (p == idx || i > 20) {
        l = T->parent[idx];
        break;
      }
      l = p;
    }
    return l;
  }
  // matches(tt, mode, a, b), for_each_meta.h:47-70 (no equivalence lists)
  __device__ bool matches(uint8_t mode, uint32_t a, uint32_t b) const {
    if (a == b) return true;
    if (mode == B2R_MATCH_EXACT || T->children_idx == nullptr) {
      if (mode == B2R_MATCH_EQUIVALENT) return root(a) == b;
      return false;
    }
    if (mode == B2R_MATCH_INTERMODAL) {
      for (auto i = T->children_idx[a]; i != T->children_idx[a + 1]; ++i) {
        auto const c = T->children[i];
        if (T->loc_type != nullptr && T->loc_type[c] == B2R_LOC_GENERATED_TRACK && c == b) return true;
      }
      return false;
    }
    auto const r = mode == B2R_MATCH_EQUIVALENT ? root(a) : a;
    if (r == b) return true;
    for (auto i = T->children_idx[r]; i != T->children_idx[r + 1]; ++i) {
      auto const c = T->children[i];
      if (c == b) return true;
      for (auto j = T->children_idx[c]; j != T->children_idx[c + 1]; ++j) {
        if (T->children[j] == b) return true;
      }
    }
    return false;
  }
  __device__ bool is_journey_start(uint32_t l) const {
    auto const* o = start_offs();
    for (auto i = 0U; i != sl->n_soff; ++i) {
      if (matches(sl->start_mode, o[i].target, l)) return true;
    }
    return false;
  }

  // -------------------------------------------------------------- legs
  __device__ b2r_leg make_leg(uint32_t a, uint32_t b, int32_t ta, int32_t tb) const {
    b2r_leg l{};
    l.rt_transport = B2R_INVALID_IDX;
    l.from = fwd ? a : b;
    l.to = fwd ? b : a;
    l.dep_time = fwd ? ta : tb;
    l.arr_time = fwd ? tb : ta;
    return l;
  }
  __device__ static void set_run(b2r_leg& l, uint32_t t, uint16_t day, uint32_t a, uint32_t b) {
    l.kind = B2R_LEG_TRANSPORT;
    l.transport = t;
    l.day = day;
    l.stop_from = static_cast<uint16_t>(a < b ? a : b);
    l.stop_to = static_cast<uint16_t>((a < b ? b : a) + 1u);
  }
  __device__ static void set_fp(b2r_leg& l, uint32_t target, int dur) {
    l.kind = B2R_LEG_FOOTPATH;
    l.transport = target;
    l.duration = static_cast<int16_t>(dur > 511 ? 511 : dur);
    l.transport_mode_id = 0;
  }
  __device__ static void set_off(b2r_leg& l, b2r_offset const& o) {
    l.kind = B2R_LEG_OFFSET;
    l.transport = o.target;
    l.duration = o.duration;
    l.transport_mode_id = o.transport_mode_id;
  }
  __device__ void push(b2r_leg const& l) {
    if (n_legs >= kMaxLegs) {
      failed = true;
      return;
    }
    if (lane == 0) legs[n_legs] = l;
    ++n_legs;
    last = l;
  }

  __device__ static b2r_leg shfl_leg(b2r_leg const& l, int src) {
    static_assert(sizeof(b2r_leg) % 4 == 0, "leg size");
    constexpr int kW = sizeof(b2r_leg) / 4;
    uint32_t w[kW];
    memcpy(w, &l, sizeof(b2r_leg));
#pragma unroll
    for (int i = 0; i < kW; ++i) w[i] = __shfl_sync(kFull, w[i], src);
    b2r_leg out;
    memcpy(&out, w, sizeof(b2r_leg));
    return out;
  }

  // reconstruct.cc:180-280 (single pass: no vias).  The stops before the
  // exit stop are split across the lanes; the ballot keeps the first one in
  // the reference's order.  A section lacking one of the flags `sec` ends
  // the ride (reconstruct.cc:239-250): stops at or past the first such
  // section do not count.  Called by the whole warp with equal arguments.
  __device__ bool find_start_in_prev_round(unsigned k, uint32_t t, uint16_t day, uint32_t finish,
                                           uint32_t sec, b2r_leg& out) const {
    auto const r = T->transport_route[t];
    auto const size = n_stops(r);
    auto const n = fwd ? finish + 1u : size - finish;
    for (auto i0 = 1u; i0 < n; i0 += 32u) {
      auto const i = i0 + lane;
      bool ok = false, cut = false;
      uint32_t si = 0, l = 0;
      int event_time = 0;
      if (i < n) {
        si = fwd ? finish - i : finish + i;
        auto const w = stopw(r, si);
        l = B2R_STOP_LOC(w);
        // departure section forward, arrival section backward
        cut = sec != 0u && !section_ok(*T, T->route_stop_idx[r], fwd ? si : si - 1u, sec);
        // plain in / out bits for every profile: reconstruct.cc:252-253
        // passes the bool is_wheelchair as a profile index (0 or 1)
        if (!cut && !((fwd && !B2R_STOP_IN(w)) || (!fwd && !B2R_STOP_OUT(w)))) {
          event_time = unix_to_delta(ev_time(t, day, si, !fwd));
          auto const round_time = rt_t(k - 1, l);
          ok = beq(round_time, event_time) ||
               (k == 1 && sl->start_mode == B2R_MATCH_EQUIVALENT && is_journey_start(l) &&
                (ontrip ? beq(round_time, event_time) : round_time == event_time));
        }
      }
      auto m = __ballot_sync(kFull, ok);
      auto const cuts = __ballot_sync(kFull, cut);
      if (cuts != 0u) m &= (1u << (__ffs(cuts) - 1)) - 1u;  // lanes before the first cut
      if (m != 0u) {
        auto const src = __ffs(m) - 1;
        si = __shfl_sync(kFull, si, src);
        l = __shfl_sync(kFull, l, src);
        event_time = __shfl_sync(kFull, event_time, src);
        out = make_leg(l, B2R_STOP_LOC(stopw(r, finish)), delta_to_unix(event_time),
                       ev_time(t, day, finish, fwd));
        set_run(out, t, day, si, finish);
        return true;
      }
      if (cuts != 0u) return false;
    }
    return false;
  }

  // find_start_in_prev_round on a real-time run (rt::frun::from_rt): the
  // run's own stops and event times, as above.
  __device__ bool find_start_in_prev_round_rt(unsigned k, uint32_t x, uint32_t finish, uint32_t sec,
                                              b2r_leg& out) const {
    auto const sb = T->rt_stop_idx[x];
    auto const size = T->rt_stop_idx[x + 1] - sb;
    auto const* tm = T->rt_times + 2ull * (sb - x);
    auto const n = fwd ? finish + 1u : size - finish;
    for (auto i0 = 1u; i0 < n; i0 += 32u) {
      auto const i = i0 + lane;
      bool ok = false, cut = false;
      uint32_t si = 0, l = 0;
      int event_time = 0;
      if (i < n) {
        si = fwd ? finish - i : finish + i;
        auto const w = T->rt_stops[sb + si];
        l = B2R_STOP_LOC(w);
        cut = sec != 0u && (static_cast<uint32_t>(T->rt_sec[sb + (fwd ? si : si - 1u)]) & sec) != sec;
        if (!cut && !((fwd && !B2R_STOP_IN(w)) || (!fwd && !B2R_STOP_OUT(w)))) {
          event_time = unix_to_delta(tm[2u * si - (fwd ? 0u : 1u)]);
          auto const round_time = rt_t(k - 1, l);
          ok = beq(round_time, event_time) ||
               (k == 1 && sl->start_mode == B2R_MATCH_EQUIVALENT && is_journey_start(l) &&
                (ontrip ? beq(round_time, event_time) : round_time == event_time));
        }
      }
      auto m = __ballot_sync(kFull, ok);
      auto const cuts = __ballot_sync(kFull, cut);
      if (cuts != 0u) m &= (1u << (__ffs(cuts) - 1)) - 1u;
      if (m != 0u) {
        auto const src = __ffs(m) - 1;
        si = __shfl_sync(kFull, si, src);
        l = __shfl_sync(kFull, l, src);
        event_time = __shfl_sync(kFull, event_time, src);
        out = make_leg(l, B2R_STOP_LOC(T->rt_stops[sb + finish]), delta_to_unix(event_time),
                       tm[2u * finish - (fwd ? 1u : 0u)]);
        set_run(out, T->rt_static[x], T->rt_static_day[x], si, finish);
        out.rt_transport = x;
        return true;
      }
      if (cuts != 0u) return false;
    }
    return false;
  }

  // The transports of route r whose event at stop si has the minutes after
  // midnight of `time` (reconstruct.cc:292-373), one at a time from
  // `cursor`: columns are ordered by minutes after midnight, so they form
  // one run found by binary search and visited in index order.
  __device__ uint32_t first_cursor(int time, uint32_t r, uint32_t si) const {
    if (!T->route_sorted[r]) return 0u;
    auto const mam = static_cast<int16_t>((static_cast<int>(base) * 1440 + time) % 1440);
    auto const n_t = T->route_tr_to[r] - T->route_tr_from[r];
    auto const* col = T->st + T->route_st_from[r] + n_t * (si * 2u - (fwd ? 1u : 0u));
    uint32_t lo = 0, hi = n_t;
    while (lo < hi) {
      auto const mid = (lo + hi) >> 1;
      if ((col[mid] >> 5) < static_cast<uint16_t>(mam < 0 ? 0 : mam)) lo = mid + 1;
      else hi = mid;
    }
    return lo;
  }
  __device__ bool next_transport(int time, uint32_t r, uint32_t si, uint32_t& cursor, uint32_t& t,
                                 uint16_t& tday) const {
    auto const minutes = static_cast<int>(base) * 1440 + time;
    auto const day = static_cast<uint16_t>(minutes / 1440);
    auto const mam = static_cast<int16_t>(minutes % 1440);
    auto const t0 = T->route_tr_from[r], n_t = T->route_tr_to[r] - t0;
    auto const* col = T->st + T->route_st_from[r] + n_t * (si * 2u - (fwd ? 1u : 0u));
    for (auto x = cursor; x < n_t; ++x) {
      auto const cnt = delta_count(col[x]);
      auto const m = static_cast<int16_t>(cnt % 1440);
      if (m != mam) {
        if (T->route_sorted[r] && m > mam) break;
        continue;
      }
      auto const td = static_cast<uint16_t>(static_cast<int>(day) - cnt / 1440);
      if (!bf_test(*T, T->transport_bf[t0 + x], td)) continue;
      cursor = x + 1u;
      t = t0 + x;
      tday = td;
      return true;
    }
    cursor = n_t;
    return false;
  }

  // get_transport (reconstruct.cc:375-545) for a list of footpath
  // candidates, tried in order: candidate f reaches location `target(f)` at
  // `time(f)`; its real-time (run, stop position) pairs and then its (route,
  // stop position) pairs are visited in the reference's order
  // (reconstruct.cc:381-452 first).  All pairs of all candidates form one
  // sequence that the lanes take 32 at a time; the first success in
  // sequence order wins.
  // get(f, target, time) describes candidate f (lane-local); returns the
  // winning candidate or -1.
  template <typename Get>
  __device__ int get_transport(unsigned k, uint32_t n_cand, Get&& get, b2r_leg& out) const {
    for (auto f0 = 0u; f0 < n_cand; f0 += 32u) {
      // lane f: candidate f0 + f, its pair range and the inclusive prefix sum
      auto const f = f0 + lane;
      uint32_t tg = 0, pb = 0, cnt = 0, rb = 0, rcnt = 0;
      int tm = 0;
      if (f < n_cand) {
        get(f, tg, tm);
        pb = T->lrs_idx[tg];
        rb = T->lrs_rt_idx[tg];
        rcnt = T->lrs_rt_idx[tg + 1] - rb;
        cnt = rcnt + (T->lrs_idx[tg + 1] - pb);
      }
      auto end = cnt;
      for (auto o = 1u; o < 32u; o <<= 1) {
        auto const v = __shfl_up_sync(kFull, end, o);
        if (lane >= o) end += v;
      }
      auto const total = __shfl_sync(kFull, end, 31);
      for (auto p0 = 0u; p0 < total; p0 += 32u) {
        auto const p = p0 + lane;
        // owner candidate of pair p: the first lane whose prefix end > p
        uint32_t owner = 0;
        for (auto b = 16u; b > 0u; b >>= 1) {
          auto const probe = owner + b - 1u;
          auto const e = __shfl_sync(kFull, end, static_cast<int>(probe));
          if (e <= p) owner += b;
        }
        auto const o_tm = __shfl_sync(kFull, tm, static_cast<int>(owner));
        auto const o_pb = __shfl_sync(kFull, pb, static_cast<int>(owner));
        auto const o_end = __shfl_sync(kFull, end, static_cast<int>(owner));
        auto const o_cnt = __shfl_sync(kFull, cnt, static_cast<int>(owner));
        auto const o_rb = __shfl_sync(kFull, rb, static_cast<int>(owner));
        auto const o_rcnt = __shfl_sync(kFull, rcnt, static_cast<int>(owner));
        bool has = false, is_rt = false;
        uint32_t r = 0, i = 0, cursor = 0, t = 0, sec = 0;
        uint16_t tday = 0;
        if (p < total && p - (o_end - o_cnt) < o_rcnt) {  // a real-time run at the stop
          auto const x = o_rb + (p - (o_end - o_cnt));
          is_rt = true;
          r = T->lrs_rt[x];
          i = static_cast<uint32_t>(T->lrs_rt_stop[x]);
          auto const sb = T->rt_stop_idx[r];
          auto const n = T->rt_stop_idx[r + 1] - sb;
          auto const w = T->rt_stops[sb + i];
          auto const allowed = (sl->allowed_claszes == 0xFFFFu && sl->req_flags == 0u) ||
                               filter_allowed(T->rt_filter[r], sl->allowed_claszes, sl->req_flags, sec);
          // an earlier arrival than the label is accepted (reconstruct.cc:437-440)
          has = allowed &&
                !((fwd && (i == 0u || !B2R_STOP_OUT(w))) || (!fwd && (i + 1u == n || !B2R_STOP_IN(w)))) &&
                beq(T->rt_times[2ull * (sb - r) + 2u * i - (fwd ? 1u : 0u)], delta_to_unix(o_tm));
        } else if (p < total) {
          auto const x = o_pb + (p - (o_end - o_cnt) - o_rcnt);
          r = T->lrs_route[x];
          i = static_cast<uint32_t>(T->lrs_stop[x]);
          auto const w = stopw(r, i);
          auto const n = n_stops(r);
          auto const allowed = (sl->allowed_claszes == 0xFFFFu && sl->req_flags == 0u) ||
                               route_allowed(*T, r, sl->allowed_claszes, sl->req_flags, sec);
          if (allowed &&
              !((fwd && (i == 0u || !B2R_STOP_OUT(w))) || (!fwd && (i + 1u == n || !B2R_STOP_IN(w))))) {
            cursor = first_cursor(o_tm, r, i);
            has = next_transport(o_tm, r, i, cursor, t, tday);
          }
        }
        for (auto m = __ballot_sync(kFull, has); m != 0u; m = __ballot_sync(kFull, has)) {
          auto const src = static_cast<int>(__ffs(m) - 1);
          auto const bt = __shfl_sync(kFull, t, src);
          auto const bday = static_cast<uint16_t>(__shfl_sync(kFull, static_cast<uint32_t>(tday), src));
          auto const bi = __shfl_sync(kFull, i, src);
          auto const bsec = __shfl_sync(kFull, sec, src);
          auto const brt = __shfl_sync(kFull, is_rt ? 1u : 0u, src) != 0u;
          auto const bx = __shfl_sync(kFull, r, src);
          if (brt ? find_start_in_prev_round_rt(k, bx, bi, bsec, out)
                  : find_start_in_prev_round(k, bt, bday, bi, bsec, out)) {
            return static_cast<int>(f0 + __shfl_sync(kFull, owner, src));
          }
          if (static_cast<int>(lane) == src) has = !is_rt && next_transport(o_tm, r, i, cursor, t, tday);
        }
      }
    }
    return -1;
  }

  // check_fp (reconstruct.cc:547-666, no vias) for one footpath
  __device__ bool check_fp(unsigned k, uint32_t l, int curr_time, uint32_t target, int dur_raw,
                           bool adjust, b2r_leg& fp_leg, b2r_leg& tr_leg) const {
    auto const d = adjust ? static_cast<int>(adjusted<int16_t>(sl->tts, static_cast<int16_t>(dur_raw)))
                          : static_cast<int>(static_cast<int16_t>(dur_raw));
    auto const fp_start = static_cast<int>(static_cast<int16_t>(curr_time - dir(d)));
    auto const one = [&](uint32_t, uint32_t& tg, int& tm) {
      tg = target;
      tm = fp_start;
    };
    if (get_transport(k, 1u, one, tr_leg) < 0) return false;
    fp_leg = make_leg(target, l, delta_to_unix(fp_start), delta_to_unix(fp_start + dir(d)));
    set_fp(fp_leg, target, dur_raw);
    return true;
  }

  // reconstruct.cc:700-790
  __device__ bool get_legs(unsigned k, uint32_t l, b2r_leg& fp_leg, b2r_leg& tr_leg) const {
    auto const curr = rt_t(k, l);
    if (sl->dest_mode == B2R_MATCH_INTERMODAL && k == j->transfers + 1u) {
      auto const* o = dest_offs();
      for (auto i = 0u; i != sl->n_doff; ++i) {
        if (o[i].duration >= 511) continue;
        auto found = false;
        // for_each_meta(kIntermodal): the location and its generated tracks;
        // the last matching meta wins (reconstruct.cc:680-696)
        auto const try_eq = [&](uint32_t eq) {
          b2r_leg f, t;
          if (check_fp(k, l, curr, eq, o[i].duration, false, f, t)) {
            b2r_offset oo = o[i];
            oo.target = eq;
            set_off(f, oo);
            fp_leg = f;
            tr_leg = t;
            found = true;
          }
        };
        try_eq(o[i].target);
        if (T->children_idx != nullptr) {
          for (auto c = T->children_idx[o[i].target]; c != T->children_idx[o[i].target + 1]; ++c) {
            auto const ch = T->children[c];
            if (T->loc_type != nullptr && T->loc_type[ch] == B2R_LOC_GENERATED_TRACK) try_eq(ch);
          }
        }
        if (found) return true;
      }
      return false;
    }
    // candidate 0: staying at l (transfer time, or none at the destination);
    // candidates 1..: the footpaths into l, in order
    auto const same = (k == j->transfers + 1u)
                          ? 0
                          : static_cast<int>(adjusted<uint8_t>(sl->tts, T->transfer_time[l]));
    auto const* idx = fp_index(*T, sl->prf, !fwd);  // the query's profile (reconstruct.cc:81, 761)
    auto const* fps = fp_words(*T, sl->prf, !fwd);
    auto const fb = idx[l];
    auto const raw = [&](uint32_t f, uint32_t& tg, int& dur) {
      if (f == 0u) {
        tg = l;
        dur = same;
      } else {
        auto const w = fps[fb + f - 1u];
        tg = B2R_FP_TARGET(w);
        dur = static_cast<int>(B2R_FP_DURATION(w));
      }
    };
    auto const eff = [&](uint32_t f, int dur) {
      return f == 0u ? static_cast<int>(static_cast<int16_t>(dur))
                     : static_cast<int>(adjusted<int16_t>(sl->tts, static_cast<int16_t>(dur)));
    };
    auto const get = [&](uint32_t f, uint32_t& tg, int& tm) {
      int dur = 0;
      raw(f, tg, dur);
      tm = static_cast<int>(static_cast<int16_t>(curr - dir(eff(f, dur))));
    };
    auto const f = get_transport(k, 1u + (idx[l + 1] - fb), get, tr_leg);
    if (f < 0) return false;
    uint32_t tg = 0;
    int dur = 0;
    raw(static_cast<uint32_t>(f), tg, dur);
    auto const d = eff(static_cast<uint32_t>(f), dur);
    auto const fp_start = static_cast<int>(static_cast<int16_t>(curr - dir(d)));
    fp_leg = make_leg(tg, l, delta_to_unix(fp_start), delta_to_unix(fp_start + dir(d)));
    set_fp(fp_leg, tg, dur);
    return true;
  }

  // reconstruct.cc:30-160 (no vias)
  __device__ bool find_start_footpath(b2r_leg& out, bool& has) const {
    has = false;
    auto const& back = last;
    auto const lsl = fwd ? back.from : back.to;
    auto const lst = fwd ? back.dep_time : back.arr_time;
    if (sl->start_mode != B2R_MATCH_INTERMODAL && is_journey_start(lsl) && beq(j->start_time, lst)) {
      return true;
    }
    auto const* o = start_offs();
    if (sl->start_mode == B2R_MATCH_INTERMODAL) {
      for (auto i = 0u; i != sl->n_soff; ++i) {
        if (matches(sl->start_mode, o[i].target, lsl) && beq(j->start_time, lst - dir(o[i].duration))) {
          out = make_leg(B2R_SPECIAL_START, lsl, lst - dir(o[i].duration), lst);
          set_off(out, o[i]);
          has = true;
          return true;
        }
      }
      return false;
    }
    auto const jst = unix_to_delta(j->start_time);
    auto const fp_target_time = rt_t(0, lsl);
    auto const* idx = fp_index(*T, sl->prf, !fwd);  // the query's profile (reconstruct.cc:81, 761)
    auto const* fps = fp_words(*T, sl->prf, !fwd);
    for (auto i = idx[lsl]; i != idx[lsl + 1]; ++i) {
      auto const tgt = B2R_FP_TARGET(fps[i]);
      auto const d = static_cast<int>(adjusted<int16_t>(sl->tts, static_cast<int16_t>(B2R_FP_DURATION(fps[i]))));
      auto const lhs = jst + static_cast<int16_t>(dir(d));
      if (is_journey_start(tgt) && fp_target_time != inv() &&
          (ontrip ? beq(lhs, fp_target_time) : lhs == fp_target_time)) {
        out = make_leg(tgt, lsl, j->start_time, delta_to_unix(fp_target_time));
        set_fp(out, tgt, d);
        has = true;
        return true;
      }
    }
    return false;
  }

  // ---------------------------------------------- optimize_footpaths.cc
  // the stops and event times of a leg's run (rt::frun): a real-time run's
  // own, else the static trip's
  __device__ uint32_t r_of(b2r_leg const& l) const { return T->transport_route[l.transport]; }
  __device__ uint32_t word_at(b2r_leg const& l, uint32_t si) const {
    if (l.rt_transport != B2R_INVALID_IDX) return T->rt_stops[T->rt_stop_idx[l.rt_transport] + si];
    return stopw(r_of(l), si);
  }
  __device__ uint32_t loc_at(b2r_leg const& l, uint32_t si) const { return B2R_STOP_LOC(word_at(l, si)); }
  __device__ int32_t time_at(b2r_leg const& l, uint32_t si, bool arr) const {
    if (l.rt_transport != B2R_INVALID_IDX) {
      auto const x = l.rt_transport;
      return T->rt_times[2ull * (T->rt_stop_idx[x] - x) + 2u * si - (arr ? 1u : 0u)];
    }
    return ev_time(l.transport, l.day, si, arr);
  }
  __device__ uint32_t run_size(b2r_leg const& l) const {
    if (l.rt_transport != B2R_INVALID_IDX) return T->rt_stop_idx[l.rt_transport + 1] - T->rt_stop_idx[l.rt_transport];
    return n_stops(r_of(l));
  }

  // optimize_footpaths.cc:15-60; `offs` = start offsets of the journey query
  __device__ void opt_initial_departure(b2r_offset const* offs, uint32_t n_offs) {
    if (n_legs <= 1 || legs[0].kind != B2R_LEG_OFFSET || legs[1].kind != B2R_LEG_TRANSPORT) return;
    auto& ol = legs[0];
    auto& tl = legs[1];
    auto best = static_cast<int>(ol.duration);
    auto const end = static_cast<uint32_t>(tl.stop_to - 1u);
    for (auto si = 0u; si < end; ++si) {
      if (!B2R_STOP_IN(word_at(tl, si))) continue;
      for (auto i = 0u; i != n_offs; ++i) {
        auto const& o = offs[i];
        if (best <= o.duration || o.target != loc_at(tl, si)) continue;
        auto const dep = time_at(tl, si, false);
        auto const o_start = dep - o.duration;
        if (ol.dep_time <= o_start) {
          ol.to = loc_at(tl, si);
          ol.dep_time = o_start;
          ol.arr_time = dep;
          set_off(ol, o);
          tl.from = loc_at(tl, si);
          tl.dep_time = dep;
          tl.stop_from = static_cast<uint16_t>(si);
          best = o.duration;
        }
      }
    }
  }

  __device__ void opt_initial_start_footpath() {  // :62-120
    if (n_legs <= 1 || legs[0].kind != B2R_LEG_FOOTPATH || legs[1].kind != B2R_LEG_TRANSPORT) return;
    auto& fl = legs[0];
    auto& tl = legs[1];
    auto const start_loc = fl.from;
    auto best = static_cast<int>(adjusted<int16_t>(sl->tts, fl.duration));
    auto const end = static_cast<uint32_t>(tl.stop_to - 1u);
    for (auto si = 0u; si < end; ++si) {
      if (!B2R_STOP_IN(word_at(tl, si))) continue;
      auto const* oidx = fp_index(*T, sl->prf, true);  // optimize_footpaths.cc:91
      auto const* ofp = fp_words(*T, sl->prf, true);
      for (auto i = oidx[start_loc]; i != oidx[start_loc + 1]; ++i) {
        auto const fp = ofp[i];
        if (B2R_FP_TARGET(fp) != loc_at(tl, si)) continue;
        auto const d = static_cast<int>(adjusted<int16_t>(sl->tts, static_cast<int16_t>(B2R_FP_DURATION(fp))));
        if (d < best) {
          auto const dep = time_at(tl, si, false);
          auto const fp_start = dep - d;
          if (fl.dep_time <= fp_start) {
            fl.to = loc_at(tl, si);
            fl.dep_time = fp_start;
            fl.arr_time = dep;
            set_fp(fl, loc_at(tl, si), d);
            tl.from = loc_at(tl, si);
            tl.dep_time = dep;
            tl.stop_from = static_cast<uint16_t>(si);
            best = d;
          }
        }
        break;
      }
    }
  }

  __device__ void opt_last_arrival(b2r_offset const* offs, uint32_t n_offs) {  // :122-187
    if (n_legs <= 1 || legs[n_legs - 1].kind != B2R_LEG_OFFSET || legs[n_legs - 2].kind != B2R_LEG_TRANSPORT) {
      return;
    }
    auto& ol = legs[n_legs - 1];
    auto& tl = legs[n_legs - 2];
    auto best = static_cast<int>(ol.duration);
    auto const from = static_cast<uint32_t>(tl.stop_from + 1u);
    auto const size = run_size(tl);
    for (auto si = from; si < size; ++si) {
      if (!B2R_STOP_OUT(word_at(tl, si))) continue;
      for (auto i = 0u; i != n_offs; ++i) {
        auto const& o = offs[i];
        if (best <= o.duration || o.target != loc_at(tl, si)) continue;
        auto const arr = time_at(tl, si, true);
        auto const o_end = arr + o.duration;
        if (o_end <= ol.arr_time) {
          ol.from = loc_at(tl, si);
          ol.dep_time = arr;
          ol.arr_time = o_end;
          set_off(ol, o);
          tl.to = loc_at(tl, si);
          tl.arr_time = arr;
          tl.stop_to = static_cast<uint16_t>(si + 1u);
          best = o.duration;
        }
      }
    }
  }

  __device__ void opt_final_egress_footpath() {  // :189-257
    if (n_legs <= 1 || legs[n_legs - 1].kind != B2R_LEG_FOOTPATH || legs[n_legs - 2].kind != B2R_LEG_TRANSPORT) {
      return;
    }
    auto& fl = legs[n_legs - 1];
    auto& tl = legs[n_legs - 2];
    auto const dest_loc = fl.to;
    auto best = static_cast<int>(adjusted<int16_t>(sl->tts, fl.duration));
    auto const from = static_cast<uint32_t>(tl.stop_from + 1u);
    auto const size = run_size(tl);
    for (auto si = from; si < size; ++si) {
      if (!B2R_STOP_OUT(word_at(tl, si))) continue;
      auto const* iidx = fp_index(*T, sl->prf, false);  // optimize_footpaths.cc:215
      auto const* ifp = fp_words(*T, sl->prf, false);
      for (auto i = iidx[dest_loc]; i != iidx[dest_loc + 1]; ++i) {
        auto const fp = ifp[i];
        if (B2R_FP_TARGET(fp) != loc_at(tl, si)) continue;
        auto const d = static_cast<int>(adjusted<int16_t>(sl->tts, static_cast<int16_t>(B2R_FP_DURATION(fp))));
        if (d < best) {
          auto const arr = time_at(tl, si, true);
          auto const fp_end = arr + d;
          if (fp_end <= fl.arr_time) {
            fl.from = loc_at(tl, si);
            fl.dep_time = arr;
            fl.arr_time = fp_end;
            set_fp(fl, dest_loc, d);
            tl.to = loc_at(tl, si);
            tl.arr_time = arr;
            tl.stop_to = static_cast<uint16_t>(si + 1u);
            best = d;
          }
        }
        break;
      }
    }
  }

  // get_penalty, optimize_footpaths.cc:259-283, with IEEE double operations
  // spelled out (no contraction) so the result equals the host's.
  __device__ double penalty(int duration, int buffer, uint32_t from, uint32_t to) const {
    auto w = static_cast<double>(duration);
    if (matches(B2R_MATCH_EQUIVALENT, from, to)) {
      auto const x = root(from);
      auto const imp = T->importance == nullptr ? 0u : T->importance[x];
      auto const q = __ddiv_rn(static_cast<double>(imp), static_cast<double>(T->max_importance));
      w = __dsub_rn(w, __dmul_rn(q, 3.0));
    }
    auto const b = buffer < 0 ? 0 : (buffer > 15 ? 15 : buffer);
    return __dsub_rn(w, __dmul_rn(0.2, static_cast<double>(b)));
  }

  // optimize_footpaths.cc:285-450 (no vias).  For each transport-footpath-
  // transport triple the (exit stop, entry stop) pairs are split across the
  // lanes; pairs do not depend on each other except through the running best
  // penalty, so the sequential loop keeps the first pair (in its order) with
  // the smallest penalty below the initial one, which is what the warp
  // reduction over (penalty, pair index) selects.  Called by the whole warp;
  // lane 0 writes the legs.
  __device__ void opt_transfers() {
    for (auto i = 0; i + 2 < n_legs; ++i) {
      __syncwarp();
      auto const lf = legs[i];
      auto const lp = legs[i + 1];
      auto const lt = legs[i + 2];
      if (lf.kind != B2R_LEG_TRANSPORT || lp.kind != B2R_LEG_FOOTPATH || lt.kind != B2R_LEG_TRANSPORT) continue;
      auto const from_start = static_cast<uint32_t>(lf.stop_from + 1u);
      auto const from_size = run_size(lf);
      auto const to_end = static_cast<uint32_t>(lt.stop_to - 1u);
      auto const pbest0 = penalty(lp.duration, lt.dep_time - lp.arr_time, lf.from, lt.to);
      auto const n_sf = from_size > from_start ? from_size - from_start : 0u;
      auto const n_pairs = n_sf * to_end;
      double best = pbest0;
      uint32_t best_idx = 0xFFFFFFFFu, best_fp = 0;
      int32_t best_arr = 0, best_dep = 0, best_d = 0;
      for (auto x = lane; x < n_pairs; x += 32u) {
        auto const sf = from_start + x / to_end, s2 = x % to_end;
        if (!B2R_STOP_OUT(word_at(lf, sf)) || !B2R_STOP_IN(word_at(lt, s2))) continue;
        auto const a = loc_at(lf, sf), b = loc_at(lt, s2);
        auto const* oidx = fp_index(*T, sl->prf, true);  // optimize_footpaths.cc:405
        auto const* ofp = fp_words(*T, sl->prf, true);
        for (auto y = oidx[a]; y != oidx[a + 1]; ++y) {
          auto const fp = ofp[y];
          if (B2R_FP_TARGET(fp) != b) continue;
          auto const d = static_cast<int>(adjusted<int16_t>(sl->tts, static_cast<int16_t>(B2R_FP_DURATION(fp))));
          auto const arr = time_at(lf, sf, true);
          auto const dep = time_at(lt, s2, false);
          auto const arr_fp = arr + d;
          if (arr_fp <= dep) {
            auto const pen = penalty(d, dep - arr_fp, a, b);
            if (pen < best) {  // lanes visit their pairs in increasing order
              best = pen;
              best_idx = x;
              best_fp = fp;
              best_arr = arr;
              best_dep = dep;
              best_d = d;
            }
          }
          break;
        }
      }
      // (penalty, pair index) minimum over the warp
      auto win_pen = best;
      auto win_idx = best_idx;
      for (auto o = 16; o > 0; o >>= 1) {
        auto const op = __shfl_xor_sync(kFull, win_pen, o);
        auto const oi = __shfl_xor_sync(kFull, win_idx, o);
        if (op < win_pen || (op == win_pen && oi < win_idx)) {
          win_pen = op;
          win_idx = oi;
        }
      }
      if (win_idx == 0xFFFFFFFFu) continue;  // no pair below the initial penalty
      auto const owner = static_cast<int>(win_idx % 32u);
      auto const w_fp = __shfl_sync(kFull, best_fp, owner);
      auto const w_arr = __shfl_sync(kFull, best_arr, owner);
      auto const w_dep = __shfl_sync(kFull, best_dep, owner);
      auto const w_d = __shfl_sync(kFull, best_d, owner);
      if (lane == 0) {
        auto const sf = from_start + win_idx / to_end, s2 = win_idx % to_end;
        auto const a = loc_at(lf, sf), b = loc_at(lt, s2);
        auto& wf = legs[i];
        auto& wp = legs[i + 1];
        auto& wt = legs[i + 2];
        wf.to = a;
        wf.arr_time = w_arr;
        wf.stop_to = static_cast<uint16_t>(sf + 1u);
        wt.from = b;
        wt.dep_time = w_dep;
        wt.stop_from = static_cast<uint16_t>(s2);
        wp.from = a;
        wp.to = b;
        wp.dep_time = w_arr;
        wp.arr_time = w_arr + w_d;
        set_fp(wp, B2R_FP_TARGET(w_fp), static_cast<int>(B2R_FP_DURATION(w_fp)));
      }
    }
    __syncwarp();
  }

  // reconstruct.cc:792-877 + optimize_footpaths(journey_q)
  __device__ void run() {
    n_legs = 0;
    failed = false;
    auto l = j->dest;
    for (auto i = 0u; i <= j->transfers && !failed; ++i) {
      auto const k = j->transfers + 1u - i;
      b2r_leg fp_leg, tr_leg;
      if (!get_legs(k, l, fp_leg, tr_leg)) {
        failed = true;
        break;
      }
      l = fwd ? tr_leg.from : tr_leg.to;
      if (i != 0 || fp_leg.from != fp_leg.to || fp_leg.dep_time != fp_leg.arr_time) push(fp_leg);
      push(tr_leg);
    }
    if (!failed) {
      b2r_leg init;
      bool has = false;
      if (!find_start_footpath(init, has)) failed = true;
      else if (has) push(init);
    }
    if (failed) return;
    if (lane == 0) {
      if (fwd) {
        for (auto a = 0, b = n_legs - 1; a < b; ++a, --b) {
          auto const x = legs[a];
          legs[a] = legs[b];
          legs[b] = x;
        }
      } else {
        for (auto i = 1; i < n_legs; ++i) {
          if (legs[i].kind != B2R_LEG_FOOTPATH) continue;
          auto const diff = legs[i].dep_time - legs[i - 1].arr_time;
          legs[i].dep_time -= diff;
          legs[i].arr_time -= diff;
        }
      }
      // optimize_footpaths on the journey query (flipped for backward search)
      auto const* jq_start = fwd ? start_offs() : dest_offs();
      auto const n_jq_start = fwd ? sl->n_soff : sl->n_doff;
      auto const* jq_dest = fwd ? dest_offs() : start_offs();
      auto const n_jq_dest = fwd ? sl->n_doff : sl->n_soff;
      opt_initial_departure(jq_start, n_jq_start);
      opt_initial_start_footpath();
      opt_last_arrival(jq_dest, n_jq_dest);
      opt_final_egress_footpath();
    }
    opt_transfers();
  }
};

}  // namespace b2r::dev
