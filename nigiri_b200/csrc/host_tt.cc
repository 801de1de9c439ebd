// Timetable finalisation: the derived arrays nigiri computes once after
// loading.  Each function cites the reference code whose output it
// reproduces (paths relative to the nigiri source tree).
#include "host_tt.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <unordered_map>

namespace b2r {

namespace {

constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr uint32_t kFpMaxDuration = 511u;  // footpath.h:17-19

uint32_t pack_fp(uint32_t target, uint32_t duration) {
  // footpath(location_idx_t, duration_t) clamps the duration to kMaxDuration
  // (footpath.h:26-31).
  if (duration > kFpMaxDuration) duration = kFpMaxDuration;
  return (target & 0x7FFFFFu) | (duration << 23);
}

int delta_minutes(uint16_t d) { return B2R_DELTA_DAYS(d) * 1440 + B2R_DELTA_MAM(d); }

uint32_t root_idx(host_timetable const& t, uint32_t idx) {
  // timetable::locations::get_root_idx, timetable.h:62-76
  if (t.parent.empty()) return idx;
  auto l = idx;
  auto i = 0;
  for (auto p = t.parent[l]; p != kInvalid; p = t.parent[l]) {
    if (p == idx || i > 20) {
      l = t.parent[idx];
      break;
    }
    l = p;
    ++i;
  }
  return l;
}

uint16_t event(host_timetable const& t, uint32_t r, uint32_t tr, uint32_t s,
               bool arr) {
  auto const n_t = t.route_transport_to[r] - t.route_transport_from[r];
  auto const slot = s * 2U - (arr ? 1U : 0U);
  return t.route_stop_times[t.route_stop_time_from[r] + n_t * slot +
                            (tr - t.route_transport_from[r])];
}

// Insertion-ordered min-map (the reference uses ankerl::unordered_dense,
// whose iteration order is insertion order).
struct ordered_min_map {
  std::vector<std::pair<uint32_t, uint32_t>> v;
  std::unordered_map<uint32_t, size_t> pos;
  void update(uint32_t k, uint32_t d) {
    auto it = pos.find(k);
    if (it == pos.end()) {
      pos.emplace(k, v.size());
      v.emplace_back(k, d);
    } else {
      v[it->second].second = std::min(v[it->second].second, d);
    }
  }
  void clear() {
    v.clear();
    pos.clear();
  }
};

// loader/build_lb_graph.h:11-99 for one profile: its footpaths (in-lists
// forward, out-lists backward) and the routes, without those that do not
// carry cars (car profile) or bikes (bike profile) on any section
void build_lb_graph(host_timetable& t, bool fwd, uint32_t prf, std::vector<uint32_t> const& fi,
                    std::vector<uint32_t> const& fd, std::vector<uint32_t>& index,
                    std::vector<uint32_t>& data) {
  index.assign(1, 0U);
  data.clear();
  ordered_min_map weights;
  auto const flag_set = [&](uint32_t f, uint32_t r) {  // timetable::is_flag_set
    return !t.route_flags.empty() && ((t.route_flags[r] >> (2U * f)) & 3U) != 0U;
  };
  auto const add_edges = [&](uint32_t l) {
    auto const parent_l = root_idx(t, l);
    for (auto i = fi[l]; i != fi[l + 1]; ++i) {
      auto const target = root_idx(t, B2R_FP_TARGET(fd[i]));
      if (target != parent_l) weights.update(target, B2R_FP_DURATION(fd[i]));
    }
    for (auto ri = t.location_routes_index[l];
         ri != t.location_routes_index[l + 1]; ++ri) {
      auto const r = t.location_routes[ri];
      if ((prf == B2R_PROFILE_CAR && !flag_set(B2R_FLAG_CARS, r)) ||
          (prf == B2R_PROFILE_BIKE && !flag_set(B2R_FLAG_BIKES, r))) {
        continue;
      }
      auto const s0 = t.route_stop_index[r];
      auto const n = t.route_stop_index[r + 1] - s0;
      for (auto from = 0U; from + 1U < n; ++from) {
        auto const to = from + 1U;
        auto const from_l = B2R_STOP_LOC(t.route_stops[s0 + from]);
        auto const to_l = B2R_STOP_LOC(t.route_stops[s0 + to]);
        if ((fwd ? to_l : from_l) != l) continue;
        auto const target = root_idx(t, fwd ? from_l : to_l);
        if (target == parent_l) continue;
        auto mn = 32767;  // duration_t max
        for (auto tr = t.route_transport_from[r]; tr != t.route_transport_to[r];
             ++tr) {
          auto const a = event(t, r, tr, to, true);
          auto const b = event(t, r, tr, from, false);
          // delta operator- re-encodes the minute difference as a delta
          // (types.h:592-595); as_duration() reads it back.
          auto const diff = static_cast<uint16_t>(
              (B2R_DELTA_DAYS(a) - B2R_DELTA_DAYS(b)) * 1440 +
              (B2R_DELTA_MAM(a) - B2R_DELTA_MAM(b)));
          auto const enc_days = (diff / 1440U) & 0x1Fu;
          auto const enc_mam = (diff % 1440U) & 0x7FFu;
          auto const dur = static_cast<int>(enc_days * 1440U + enc_mam);
          mn = std::min(mn, dur);
        }
        weights.update(target, static_cast<uint32_t>(mn));
      }
    }
  };
  for (auto i = 0U; i != t.n_locations; ++i) {
    if (!t.parent.empty() && t.parent[i] != kInvalid) {
      index.push_back(static_cast<uint32_t>(data.size()));
      continue;
    }
    if (!t.children_index.empty()) {
      for (auto ci = t.children_index[i]; ci != t.children_index[i + 1]; ++ci) {
        auto const c = t.children[ci];
        add_edges(c);
        for (auto cci = t.children_index[c]; cci != t.children_index[c + 1];
             ++cci) {
          add_edges(t.children[cci]);
        }
      }
    }
    add_edges(i);
    for (auto const& [target, d] : weights.v) data.push_back(pack_fp(target, d));
    index.push_back(static_cast<uint32_t>(data.size()));
    weights.clear();
  }
}

}  // namespace

b2r_timetable_desc host_timetable::desc() const {
  b2r_timetable_desc d{};
  d.n_locations = n_locations;
  d.n_routes = n_routes;
  d.n_transports = n_transports;
  d.n_bitfields = n_bitfields();
  d.date_range_from = date_range_from;
  d.date_range_to = date_range_to;
  d.transfer_time = transfer_time.data();
  d.parent = parent.empty() ? nullptr : parent.data();
  d.location_type = location_type.empty() ? nullptr : location_type.data();
  d.children_index = children_index.empty() ? nullptr : children_index.data();
  d.children = children.data();
  d.importance = importance.data();
  d.max_importance = max_importance;
  d.footpaths_out_index = fp_out_index.data();
  d.footpaths_out = fp_out.data();
  d.footpaths_in_index = fp_in_index.data();
  d.footpaths_in = fp_in.data();
  d.route_stop_index = route_stop_index.data();
  d.route_stops = route_stops.data();
  d.route_transport_from = route_transport_from.data();
  d.route_transport_to = route_transport_to.data();
  d.route_stop_time_from = route_stop_time_from.data();
  d.route_stop_times = route_stop_times.data();
  d.n_route_stop_times = route_stop_times.size();
  d.route_traffic_days = route_traffic_days.data();
  d.transport_traffic_days = transport_traffic_days.data();
  d.transport_route = transport_route.data();
  d.bitfields = bitfields.data();
  d.location_routes_index = location_routes_index.data();
  d.location_routes = location_routes.data();
  d.lb_fwd_index = lb_fwd_index.data();
  d.lb_fwd = lb_fwd.data();
  d.lb_bwd_index = lb_bwd_index.data();
  d.lb_bwd = lb_bwd.data();
  d.route_clasz = route_clasz.empty() ? nullptr : route_clasz.data();
  d.route_flags = route_flags.empty() ? nullptr : route_flags.data();
  d.route_section_flags =
      route_section_flags.empty() ? nullptr : route_section_flags.data();
  auto const ptr = [](std::vector<uint32_t> const& v) { return v.empty() ? nullptr : v.data(); };
  for (auto p = 0U; p != B2R_N_PROFILES - 1U; ++p) {
    auto const& x = profiles[p];
    if (x.fp_out_index.empty()) continue;
    d.profile_footpaths_out_index[p] = x.fp_out_index.data();
    d.profile_footpaths_out[p] = x.fp_out.data();
    d.profile_footpaths_in_index[p] = x.fp_in_index.data();
    d.profile_footpaths_in[p] = x.fp_in.data();
    d.profile_lb_fwd_index[p] = ptr(x.lb_fwd_index);
    d.profile_lb_fwd[p] = x.lb_fwd.data();
    d.profile_lb_bwd_index[p] = ptr(x.lb_bwd_index);
    d.profile_lb_bwd[p] = x.lb_bwd.data();
  }
  return d;
}

void finalize(host_timetable& t) {
  // transports: contiguous per route, in route order (timetable.cc
  // register_route / finish_route).
  t.n_transports = t.transport_traffic_days.size();
  t.transport_route.assign(t.n_transports, 0U);
  for (auto r = 0U; r != t.n_routes; ++r) {
    for (auto tr = t.route_transport_from[r]; tr != t.route_transport_to[r];
         ++tr) {
      t.transport_route[tr] = r;
    }
  }

  if (t.parent.empty()) t.parent.assign(t.n_locations, kInvalid);
  if (t.location_type.empty()) t.location_type.assign(t.n_locations, 0U);
  if (t.children_index.empty()) {
    // children_ of each parent in location order, as the loaders append
    // them while reading stops (gtfs/stop.cc, hrd/stamm/meta_stations)
    std::vector<uint32_t> n_children(t.n_locations, 0U);
    for (auto l = 0U; l != t.n_locations; ++l) {
      if (t.parent[l] != kInvalid) ++n_children[t.parent[l]];
    }
    t.children_index.assign(t.n_locations + 1U, 0U);
    for (auto l = 0U; l != t.n_locations; ++l) t.children_index[l + 1] = t.children_index[l] + n_children[l];
    t.children.assign(t.children_index[t.n_locations], 0U);
    auto fill = std::vector<uint32_t>(t.children_index.begin(), t.children_index.end() - 1);
    for (auto l = 0U; l != t.n_locations; ++l) {
      if (t.parent[l] != kInvalid) t.children[fill[t.parent[l]]++] = l;
    }
  }

  // footpaths_in from footpaths_out, then sorted by duration
  // (build_footpaths.cc:404-415 sorts both lists by duration); the same for
  // every profile that has footpaths
  auto const derive_in = [&](std::vector<uint32_t> const& oi, std::vector<uint32_t> const& od,
                             std::vector<uint32_t>& ii, std::vector<uint32_t>& id) {
    std::vector<std::vector<uint32_t>> in(t.n_locations);
    for (auto l = 0U; l != t.n_locations; ++l) {
      for (auto i = oi[l]; i != oi[l + 1]; ++i) {
        in[B2R_FP_TARGET(od[i])].push_back(pack_fp(l, B2R_FP_DURATION(od[i])));
      }
    }
    ii.assign(1, 0U);
    id.clear();
    for (auto& v : in) {
      std::stable_sort(v.begin(), v.end(), [](uint32_t a, uint32_t b) {
        return B2R_FP_DURATION(a) < B2R_FP_DURATION(b);
      });
      id.insert(id.end(), v.begin(), v.end());
      ii.push_back(static_cast<uint32_t>(id.size()));
    }
  };
  derive_in(t.fp_out_index, t.fp_out, t.fp_in_index, t.fp_in);
  for (auto& x : t.profiles) {
    if (!x.fp_out_index.empty()) derive_in(x.fp_out_index, x.fp_out, x.fp_in_index, x.fp_in);
  }

  // location_routes: routes in registration order, no duplicates
  // (gtfs/load_timetable.cc:410-415).
  {
    std::vector<std::vector<uint32_t>> lr(t.n_locations);
    for (auto r = 0U; r != t.n_routes; ++r) {
      for (auto i = t.route_stop_index[r]; i != t.route_stop_index[r + 1];
           ++i) {
        auto& v = lr[B2R_STOP_LOC(t.route_stops[i])];
        if (v.empty() || v.back() != r) v.push_back(r);
      }
    }
    t.location_routes_index.assign(1, 0U);
    t.location_routes.clear();
    for (auto& v : lr) {
      t.location_routes.insert(t.location_routes.end(), v.begin(), v.end());
      t.location_routes_index.push_back(
          static_cast<uint32_t>(t.location_routes.size()));
    }
  }

  // route traffic days, loader/init_finish.cc:168-198
  t.route_traffic_days.assign(t.n_routes, 0U);
  for (auto r = 0U; r != t.n_routes; ++r) {
    uint64_t combined[8] = {};
    auto const n_stops = t.route_stop_index[r + 1] - t.route_stop_index[r];
    for (auto tr = t.route_transport_from[r]; tr != t.route_transport_to[r];
         ++tr) {
      auto max_delta = 0;
      for (auto s = 0U; s != n_stops; ++s) {
        if (s != 0U) {
          max_delta = std::max(max_delta, B2R_DELTA_DAYS(event(t, r, tr, s, true)));
        }
        if (s + 1U != n_stops) {
          max_delta = std::max(max_delta, B2R_DELTA_DAYS(event(t, r, tr, s, false)));
        }
      }
      auto const* bf = &t.bitfields[8U * t.transport_traffic_days[tr]];
      for (auto d = 0; d <= max_delta; ++d) {
        // combined |= (bf << d) over the 512-bit set
        for (auto w = 7; w >= 0; --w) {
          uint64_t v = 0;
          auto const word_shift = d / 64, bit_shift = d % 64;
          auto const src = w - word_shift;
          if (src >= 0) {
            v = bf[src] << bit_shift;
            if (bit_shift != 0 && src - 1 >= 0) v |= bf[src - 1] >> (64 - bit_shift);
          }
          combined[w] |= v;
        }
      }
    }
    t.route_traffic_days[r] = t.n_bitfields();
    t.bitfields.insert(t.bitfields.end(), combined, combined + 8);
  }

  build_lb_graph(t, true, B2R_PROFILE_DEFAULT, t.fp_in_index, t.fp_in, t.lb_fwd_index, t.lb_fwd);
  build_lb_graph(t, false, B2R_PROFILE_DEFAULT, t.fp_out_index, t.fp_out, t.lb_bwd_index, t.lb_bwd);

  // route flags: absent means no route carries any flag.  From per-section
  // flags, a route's flag f is "on all sections" when every section of the
  // route has it and "on some" when at least one has it
  // (timetable::register_route, timetable.cc:136-156).
  if (!t.route_section_flags.empty() && t.route_flags.empty()) {
    t.route_flags.assign(t.n_routes, 0U);
    for (auto r = 0U; r != t.n_routes; ++r) {
      auto const b = t.route_stop_index[r], n_sections = t.route_stop_index[r + 1] - b - 1U;
      for (auto f = 0U; f != 4U; ++f) {
        auto count = 0U;
        for (auto s = 0U; s != n_sections; ++s) count += (t.route_section_flags[b + s] >> f) & 1U;
        if (count == n_sections && n_sections != 0U) t.route_flags[r] |= static_cast<uint8_t>(1U << (2U * f));
        if (count != 0U) t.route_flags[r] |= static_cast<uint8_t>(1U << (2U * f + 1U));
      }
    }
  }
  if (!t.route_flags.empty() && t.route_section_flags.empty()) {
    // whole-route flags only: every section carries the "all sections" bits
    t.route_section_flags.assign(t.route_stop_index[t.n_routes], 0U);
    for (auto r = 0U; r != t.n_routes; ++r) {
      uint8_t all = 0U;
      for (auto f = 0U; f != 4U; ++f) {
        if (t.route_flags[r] & (1U << (2U * f))) all |= static_cast<uint8_t>(1U << f);
      }
      for (auto i = t.route_stop_index[r]; i != t.route_stop_index[r + 1]; ++i) {
        t.route_section_flags[i] = all;
      }
    }
  }

  // lower-bound graphs of the profiles that have footpaths (with the route
  // flags, which the car and bike profiles filter on)
  for (auto p = 0U; p != B2R_N_PROFILES - 1U; ++p) {
    auto& x = t.profiles[p];
    if (x.fp_out_index.empty()) continue;
    build_lb_graph(t, true, p + 1U, x.fp_in_index, x.fp_in, x.lb_fwd_index, x.lb_fwd);
    build_lb_graph(t, false, p + 1U, x.fp_out_index, x.fp_out, x.lb_bwd_index, x.lb_bwd);
  }

  // importance, loader/init_finish.cc:64-102 (float accumulation into a
  // uint32; class priorities of the reference table, zero past kOther's
  // slot 12 as its 16-entry array leaves them)
  {
    static constexpr float kPrio[16] = {20, 20, 20, 20, 20, 16, 15, 10,
                                        10, 3,  2,  10, 1,  0,  0,  0};
    if (t.route_clasz.empty()) t.route_clasz.assign(t.n_routes, 10U);  // bus
    t.importance.assign(t.n_locations, 0U);
    t.max_importance = 0U;
    for (auto l = 0U; l != t.n_locations; ++l) {
      unsigned counts[16] = {};
      for (auto ri = t.location_routes_index[l];
           ri != t.location_routes_index[l + 1]; ++ri) {
        auto const r = t.location_routes[ri];
        for (auto tr = t.route_transport_from[r]; tr != t.route_transport_to[r];
             ++tr) {
          auto const* bf = &t.bitfields[8U * t.transport_traffic_days[tr]];
          unsigned c = 0;
          for (auto w = 0; w != 8; ++w) c += __builtin_popcountll(bf[w]);
          counts[t.route_clasz[r]] += c;
        }
      }
      auto const p = t.parent[l];
      auto& x = t.importance[p == kInvalid ? l : p];
      for (auto c = 0; c != 16; ++c) {
        x += kPrio[c] * static_cast<float>(counts[c]);
      }
      t.max_importance = std::max(t.max_importance, x);
    }
  }
}

// ------------------------------------------------------------ persistence
namespace {
constexpr uint64_t kMagic = 0x3332424d49544232ull;  // "2BTIMB23"

template <typename T>
void put_vec(std::FILE* f, std::vector<T> const& v) {
  uint64_t n = v.size();
  std::fwrite(&n, sizeof(n), 1, f);
  if (n) std::fwrite(v.data(), sizeof(T), n, f);
}
template <typename T>
bool get_vec(std::FILE* f, std::vector<T>& v) {
  uint64_t n = 0;
  if (std::fread(&n, sizeof(n), 1, f) != 1) return false;
  v.resize(n);
  return n == 0 || std::fread(v.data(), sizeof(T), n, f) == n;
}
}  // namespace

#define B2R_TT_FIELDS(X)                                                       \
  X(transfer_time) X(parent) X(location_type) X(children_index) X(children)    \
  X(importance) X(fp_out_index) X(fp_out) X(fp_in_index) X(fp_in)              \
  X(route_stop_index) X(route_stops) X(route_clasz) X(route_transport_from)    \
  X(route_transport_to) X(route_stop_time_from) X(route_stop_times)            \
  X(route_traffic_days) X(transport_traffic_days) X(transport_route)           \
  X(bitfields) X(location_routes_index) X(location_routes) X(lb_fwd_index)     \
  X(lb_fwd) X(lb_bwd_index) X(lb_bwd) X(x) X(y) X(route_flags)                \
  X(route_section_flags)
#define B2R_TT_PROFILE_FIELDS(X)                                               \
  X(fp_out_index) X(fp_out) X(fp_in_index) X(fp_in) X(lb_fwd_index) X(lb_fwd)  \
  X(lb_bwd_index) X(lb_bwd)

bool save(host_timetable const& t, std::string const& path) {
  auto* f = std::fopen(path.c_str(), "wb");
  if (f == nullptr) return false;
  std::fwrite(&kMagic, sizeof(kMagic), 1, f);
  uint32_t hdr[6] = {t.n_locations, t.n_routes, t.n_transports,
                     static_cast<uint32_t>(t.date_range_from),
                     static_cast<uint32_t>(t.date_range_to), t.max_importance};
  std::fwrite(hdr, sizeof(hdr), 1, f);
#define X(name) put_vec(f, t.name);
  B2R_TT_FIELDS(X)
#undef X
  for (auto const& x : t.profiles) {
#define X(name) put_vec(f, x.name);
    B2R_TT_PROFILE_FIELDS(X)
#undef X
  }
  return std::fclose(f) == 0;
}

bool load(std::string const& path, host_timetable& t) {
  auto* f = std::fopen(path.c_str(), "rb");
  if (f == nullptr) return false;
  uint64_t magic = 0;
  uint32_t hdr[6];
  auto ok = std::fread(&magic, sizeof(magic), 1, f) == 1 && magic == kMagic &&
            std::fread(hdr, sizeof(hdr), 1, f) == 1;
  if (ok) {
    t.n_locations = hdr[0];
    t.n_routes = hdr[1];
    t.n_transports = hdr[2];
    t.date_range_from = static_cast<int32_t>(hdr[3]);
    t.date_range_to = static_cast<int32_t>(hdr[4]);
    t.max_importance = hdr[5];
#define X(name) ok = ok && get_vec(f, t.name);
    B2R_TT_FIELDS(X)
#undef X
    for (auto& x : t.profiles) {
#define X(name) ok = ok && get_vec(f, x.name);
      B2R_TT_PROFILE_FIELDS(X)
#undef X
    }
  }
  std::fclose(f);
  return ok;
}

}  // namespace b2r
