// GTFS feeds -> host timetable: the part of nigiri's GTFS loader
// (src/loader/gtfs/load_timetable.cc and the files it calls) that the
// reference's routing tests exercise.  Agencies (one time zone per feed),
// stops with parents, routes (route_type -> transport class), trips with
// blocks and bike / car / reservation flags, stop times with pickup and
// drop-off restrictions, calendar and calendar_dates, and transfers.txt
// (minimum transfer times, footpaths, stay-seated transfers joining trips
// into one transport), footpaths between nearby and same-named stops, and
// the footpath closure that finalize() builds.  Not restated: frequencies,
// flex, shapes, fares, translations, location equivalences and the merging
// of duplicate trips.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <limits>
#include <optional>
#include <queue>
#include <set>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "b2r.h"
#include "errors.h"
#include "host_tt.h"

namespace b2r {
namespace {

constexpr uint32_t kNoParent = 0xFFFFFFFFu;
constexpr uint32_t kSpecial = 9;  // special stations (special_stations.h:7-19)

// geo::approx_squared_distance with approx_distance_lng_degrees (the geo
// library, motis-project/geo at commit 7c78f91a, which the reference tree
// does not carry): an equirectangular approximation, squared metres, the
// longitude difference scaled at the first point's latitude.  Restated on a
// sphere of radius 6,371 km.
constexpr double kPi = 3.14159265358979323846;
constexpr double kMetersPerDegree = kPi * 6371000.0 / 180.0;
double approx_squared_distance(std::pair<double, double> const& a, std::pair<double, double> const& b) {
  auto const y = (a.first - b.first) * kMetersPerDegree;
  auto const x = (a.second - b.second) * kMetersPerDegree * std::cos(a.first * kPi / 180.0);
  return x * x + y * y;
}

// ------------------------------------------------------------------ CSV
struct csv {
  std::vector<std::string> header;
  std::vector<std::vector<std::string>> rows;
  int col(char const* name) const {
    for (auto i = 0U; i != header.size(); ++i) {
      if (header[i] == name) return static_cast<int>(i);
    }
    return -1;
  }
  std::string const& get(size_t r, int c) const {
    static std::string const empty;
    return (c < 0 || static_cast<size_t>(c) >= rows[r].size()) ? empty : rows[r][c];
  }
};

std::string trim(std::string s) {
  auto const b = s.find_first_not_of(" \t\r\n");
  if (b == std::string::npos) return {};
  auto const e = s.find_last_not_of(" \t\r\n");
  return s.substr(b, e - b + 1);
}

std::vector<std::string> split_line(std::string const& line) {  // RFC 4180 fields
  std::vector<std::string> out;
  std::string cur;
  auto quoted = false;
  for (auto i = size_t{0}; i < line.size(); ++i) {
    auto const c = line[i];
    if (quoted) {
      if (c == '"' && i + 1 < line.size() && line[i + 1] == '"') {
        cur += '"';
        ++i;
      } else if (c == '"') {
        quoted = false;
      } else {
        cur += c;
      }
    } else if (c == '"') {
      quoted = true;
    } else if (c == ',') {
      out.push_back(trim(cur));
      cur.clear();
    } else {
      cur += c;
    }
  }
  out.push_back(trim(cur));
  return out;
}

csv parse_csv(std::string const& text) {
  csv t;
  std::istringstream in{text};
  std::string line;
  auto first = true;
  while (std::getline(in, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (trim(line).empty()) continue;
    if (first) {
      if (line.size() >= 3 && static_cast<unsigned char>(line[0]) == 0xEF) line = line.substr(3);  // BOM
      t.header = split_line(line);
      first = false;
    } else {
      t.rows.push_back(split_line(line));
    }
  }
  return t;
}

// nigiri's mem_dir::read text: "# <file name>" lines start each file
std::map<std::string, std::string> split_mem_dir(std::string const& text) {
  std::map<std::string, std::string> files;
  std::istringstream in{text};
  std::string line, name;
  while (std::getline(in, line)) {
    if (line.rfind("# ", 0) == 0) {
      name = trim(line.substr(2));
      files[name];
    } else if (!name.empty()) {
      files[name] += line + "\n";
    }
  }
  return files;
}

// ------------------------------------------------------------------ dates
int64_t days_from_civil(int64_t y, unsigned m, unsigned d) {  // proleptic Gregorian
  y -= m <= 2;
  auto const era = (y >= 0 ? y : y - 399) / 400;
  auto const yoe = static_cast<unsigned>(y - era * 400);
  auto const doy = (153 * (m + (m > 2 ? -3 : 9)) + 2) / 5 + d - 1;
  auto const doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
  return era * 146097 + static_cast<int64_t>(doe) - 719468;
}

int32_t parse_yyyymmdd(std::string const& s) {
  if (s.size() < 8) throw std::runtime_error("bad date: " + s);
  auto const v = std::stoul(s.substr(0, 8));
  return static_cast<int32_t>(days_from_civil(v / 10000, (v / 100) % 100, v % 100));
}

// hhmm_to_min, parse_time.cc:9-25 (seconds ignored); -1 when empty
int parse_hhmm(std::string const& s) {
  if (s.empty()) return -1;
  auto const c = s.find(':');
  if (c == std::string::npos) return -1;
  auto const c2 = s.find(':', c + 1);
  return std::stoi(s.substr(0, c)) * 60 + std::stoi(s.substr(c + 1, c2 == std::string::npos ? std::string::npos : c2 - c - 1));
}

// ------------------------------------------------------------ time zones
// The UTC offset in effect at a local time, from the zone's TZif file
// (RFC 8536, version 2+ 64-bit data).
struct time_zone {
  std::vector<int64_t> transitions;  // UTC seconds
  std::vector<uint8_t> idx;
  std::vector<int32_t> utoff;  // per local time type
  int32_t initial{0};

  int32_t offset_at_utc(int64_t t) const {
    if (transitions.empty() || t < transitions.front()) return initial;
    auto const it = std::upper_bound(transitions.begin(), transitions.end(), t);
    return utoff[idx[static_cast<size_t>(it - transitions.begin()) - 1]];
  }
  // offset of the local time `local` (seconds since the epoch, local clock)
  int32_t offset_at_local(int64_t local) const {
    auto off = offset_at_utc(local);
    off = offset_at_utc(local - off);
    return offset_at_utc(local - off);
  }
};

int64_t be(uint8_t const* p, int n) {
  int64_t v = 0;
  for (auto i = 0; i != n; ++i) v = (v << 8) | p[i];
  if (n == 4) v = static_cast<int32_t>(static_cast<uint32_t>(v));
  return v;
}

time_zone load_zone(std::string const& dir, std::string const& name) {
  std::ifstream f{dir + "/" + name, std::ios::binary};
  if (!f) throw std::runtime_error("time zone not found: " + name);
  std::vector<uint8_t> b{std::istreambuf_iterator<char>{f}, {}};
  auto const header = [&](size_t at, uint32_t* cnt) {
    if (b.size() < at + 44 || std::memcmp(b.data() + at, "TZif", 4) != 0) {
      throw std::runtime_error("not a TZif file: " + name);
    }
    for (auto i = 0; i != 6; ++i) cnt[i] = static_cast<uint32_t>(be(b.data() + at + 20 + 4 * i, 4));
  };
  uint32_t c[6];  // isutcnt, isstdcnt, leapcnt, timecnt, typecnt, charcnt
  header(0, c);
  auto const version = b[4];
  size_t at = 44;
  auto tsize = 4;
  if (version >= '2') {  // skip the 32-bit block, read the 64-bit one
    at += c[3] * 5 + c[4] * 6 + c[5] + c[2] * 8 + c[1] + c[0];
    header(at, c);
    at += 44;
    tsize = 8;
  }
  time_zone z;
  for (auto i = 0U; i != c[3]; ++i) z.transitions.push_back(be(b.data() + at + i * tsize, tsize));
  at += c[3] * tsize;
  for (auto i = 0U; i != c[3]; ++i) z.idx.push_back(b[at + i]);
  at += c[3];
  for (auto i = 0U; i != c[4]; ++i) z.utoff.push_back(static_cast<int32_t>(be(b.data() + at + i * 6, 4)));
  if (z.utoff.empty()) throw std::runtime_error("empty TZif: " + name);
  z.initial = z.utoff.front();
  return z;
}

// --------------------------------------------------------- transport class
// to_clasz, src/loader/gtfs/route.cc:18-141 (GTFS and extended route types)
uint8_t to_clasz(int t) {
  enum : uint8_t { kAir, kHighSpeed, kLongDistance, kCoach, kNight, kRideSharing, kRegional, kSuburban,
                   kSubway, kTram, kBus, kShip, kODM, kFunicular, kAerialLift, kOther };
  switch (t) {
    case 0: return kTram;
    case 1: return kSubway;
    case 2: return kRegional;
    case 3: return kBus;
    case 4: return kShip;
    case 5: return kFunicular;
    case 6: return kAerialLift;
    case 7: return kFunicular;
    case 11: return kBus;
    case 12: return kOther;
    case 100: return kRegional;
    case 101: return kHighSpeed;
    case 102: return kLongDistance;
    case 103: return kRegional;
    case 104: return kLongDistance;
    case 105: return kNight;
    case 106: return kRegional;
    case 107: return kRegional;
    case 108: return kRegional;
    case 109: return kSuburban;
    case 110: return kRegional;
    case 111: return kRegional;
    case 112: return kRegional;
    case 113: return kRegional;
    case 114: return kLongDistance;
    case 115: return kRegional;
    case 116: return kFunicular;
    case 117: return kRegional;
    default: break;
  }
  if (t >= 200 && t < 300) {
    switch (t) {
      case 202: case 207: case 209: return kCoach;
      case 204: case 208: return kBus;
      default: return kCoach;
    }
  }
  if (t >= 400 && t < 500) {
    switch (t) {
      case 400: case 401: case 402: case 403: return kSubway;
      case 404: return kSuburban;
      case 405: return kOther;
      default: return kSubway;
    }
  }
  if (t >= 700 && t < 800) return t == 715 ? kODM : kBus;
  if (t == 800) return kBus;
  if (t >= 900 && t < 1000) return kTram;
  if (t >= 1000 && t < 1100) return kShip;
  if (t >= 1100 && t < 1200) return kAir;
  if (t >= 1200 && t < 1300) return kShip;
  if (t >= 1300 && t < 1400) return (t == 1303 || t == 1305) ? kOther : kAerialLift;
  if (t == 1400) return kFunicular;
  if (t >= 1500 && t < 1600) return t == 1551 ? kRideSharing : kODM;
  return kOther;
}

// ------------------------------------------------------------------ model
struct bits512 {
  std::array<uint64_t, 8> w{};
  void set(uint32_t i, bool v = true) {
    if (i >= 512U) return;
    if (v) w[i / 64] |= 1ULL << (i % 64);
    else w[i / 64] &= ~(1ULL << (i % 64));
  }
  bool test(uint32_t i) const { return i < 512U && ((w[i / 64] >> (i % 64)) & 1ULL) != 0ULL; }
  bool any() const {
    for (auto x : w)
      if (x != 0ULL) return true;
    return false;
  }
  bits512 operator&(bits512 const& o) const {
    bits512 r;
    for (auto i = 0; i != 8; ++i) r.w[i] = w[i] & o.w[i];
    return r;
  }
  bits512 operator~() const {
    bits512 r;
    for (auto i = 0; i != 8; ++i) r.w[i] = ~w[i];
    return r;
  }
  bool operator<(bits512 const& o) const { return w < o.w; }
  // std::bitset shift: bit i moves to bit i + n (to i - |n| for n < 0)
  bits512 shifted(int n) const {
    bits512 r;
    for (auto i = 0; i != 512; ++i) {
      if (test(static_cast<uint32_t>(i)) && i + n >= 0 && i + n < 512) r.set(static_cast<uint32_t>(i + n));
    }
    return r;
  }
};

struct event {
  int arr, dep;  // minutes after the service day's local midnight
};

struct trip {
  std::string id, block;
  uint32_t route{0};
  bits512 service;
  bool has_service{false};
  std::array<bool, 4> flags{};           // bikes, cars, wheelchair, no reservation
  std::vector<uint32_t> stops;           // stop words (location | in | out | in_wc | out_wc)
  std::vector<std::pair<uint32_t, event>> times;  // (stop_sequence, event)
  std::vector<event> events;
  bool bad{false};
};

uint32_t stop_word(uint32_t loc, bool in, bool out, bool in_wc, bool out_wc) {
  return (loc & 0x0FFFFFFFu) | (in ? 1u << 28 : 0u) | (out ? 1u << 29 : 0u) | (in_wc ? 1u << 30 : 0u) |
         (out_wc ? 1u << 31 : 0u);
}

// one transport of the timetable: a trip or a block chain on the UTC
// traffic days of one (day offset, time zone offset) key
struct utc_trip {
  std::vector<uint32_t> trips;
  std::vector<uint32_t> stop_seq;
  std::vector<uint8_t> sections;  // per section: flag f at bit f
  uint8_t clasz{0};
  std::vector<int> times;  // dep(0), arr(1), dep(1), ... in UTC minutes of its first day
  bits512 days;
};

struct route_key {
  std::vector<uint32_t> stops;
  uint8_t clasz;
  std::vector<uint8_t> sections;
  bool operator<(route_key const& o) const {
    return std::tie(stops, clasz, sections) < std::tie(o.stops, o.clasz, o.sections);
  }
};

}  // namespace

bool load_gtfs(std::map<std::string, std::string> const& files, b2r_gtfs_config const& cfg,
               b2r_host_timetable*& out, std::string& err) {
  auto const file = [&](char const* n) {
    auto const it = files.find(n);
    return it == files.end() ? csv{} : parse_csv(it->second);
  };
  // timetable::internal_interval_days: [date_range.from - 5, date_range.to + 1)
  auto const iv_from = cfg.date_range_from - B2R_TIMETABLE_OFFSET_DAYS;
  auto const iv_to = cfg.date_range_to + 1;
  auto const n_days = static_cast<uint32_t>(std::min(iv_to - iv_from, 512));

  // agency.txt: the feed's time zone is the first agency's (noon_offsets.cc:10-40)
  std::string tz_name = cfg.default_tz != nullptr ? cfg.default_tz : "";
  std::unordered_map<std::string, std::string> agency_tz;
  {
    auto const a = file("agency.txt");
    for (auto r = size_t{0}; r != a.rows.size(); ++r) {
      agency_tz[a.get(r, a.col("agency_id"))] = a.get(r, a.col("agency_timezone"));
      if (r == 0) tz_name = a.get(r, a.col("agency_timezone"));
    }
  }
  if (tz_name.empty()) {
    err = "no time zone: agency.txt is empty and no default_tz is set";
    return false;
  }
  auto const zone = load_zone(cfg.tzdata_dir != nullptr ? cfg.tzdata_dir : "/usr/share/zoneinfo", tz_name);
  // get_noon_offset, noon_offsets.cc:6-11: minutes at local noon of each day
  std::vector<int> noon(n_days);
  for (auto d = 0U; d != n_days; ++d) {
    auto const local_noon = (static_cast<int64_t>(iv_from) + d) * 86400 + 12 * 3600;
    noon[d] = zone.offset_at_local(local_noon) / 60;
  }

  // stops.txt (stop.cc:209-330): entrances and generic nodes dropped; file
  // order (the reference registers in its hash map's order)
  auto const st = file("stops.txt");
  std::unordered_map<std::string, uint32_t> loc_of;
  std::vector<std::string> ids, parent_ids, names;
  std::vector<bool> accessible;
  std::vector<std::pair<double, double>> coords;  // (lat, lng), clamped
  auto const coordinate = [](std::string const& x, double lim) {
    return std::clamp(x.empty() ? 0.0 : std::strtod(x.c_str(), nullptr), -lim, lim);
  };
  for (auto r = size_t{0}; r != st.rows.size(); ++r) {
    auto const lt = st.get(r, st.col("location_type"));
    if (lt == "2" || lt == "3") continue;
    auto const id = st.get(r, st.col("stop_id"));
    if (loc_of.contains(id)) continue;
    loc_of[id] = kSpecial + static_cast<uint32_t>(ids.size());
    ids.push_back(id);
    parent_ids.push_back(st.get(r, st.col("parent_station")));
    names.push_back(st.get(r, st.col("stop_name")));
    // wheelchair_boarding: unknown counts as accessible (stop.cc:266-268)
    accessible.push_back(st.get(r, st.col("wheelchair_boarding")) != "2");
    coords.emplace_back(coordinate(st.get(r, st.col("stop_lat")), 90.0),
                        coordinate(st.get(r, st.col("stop_lon")), 180.0));
  }
  for (auto const& p : parent_ids) {  // parents named only as parent_station
    if (!p.empty() && !loc_of.contains(p)) {
      loc_of[p] = kSpecial + static_cast<uint32_t>(ids.size());
      ids.push_back(p);
      parent_ids.emplace_back();
      names.emplace_back();
      accessible.push_back(true);
      coords.emplace_back(0.0, 0.0);
    }
  }
  auto const n_loc = kSpecial + static_cast<uint32_t>(ids.size());
  std::vector<uint32_t> parent(n_loc, kNoParent);
  std::vector<uint8_t> loc_type(n_loc, B2R_LOC_STATION);
  for (auto i = 0U; i != ids.size(); ++i) {
    if (!parent_ids[i].empty()) {
      parent[kSpecial + i] = loc_of[parent_ids[i]];
      loc_type[kSpecial + i] = B2R_LOC_TRACK;
    }
  }
  // transfers.txt (read_transfers, stop.cc:124-205): every row but types 3
  // (not possible) and 4 (stay seated, read with the trips) gives the
  // minimum transfer time of a stop with itself or a footpath between two
  // stops, in whole minutes; empty fields read as 0
  std::vector<std::optional<int>> transfer(n_loc);
  std::vector<std::vector<std::pair<uint32_t, int>>> fps(n_loc);
  auto const int_field = [](std::string const& x) { return x.empty() ? 0 : std::stoi(x); };
  {
    auto const tr = file("transfers.txt");
    for (auto r = size_t{0}; r != tr.rows.size(); ++r) {
      auto const type = int_field(tr.get(r, tr.col("transfer_type")));
      if (type == 3 || type == 4) continue;
      auto const a = loc_of.find(tr.get(r, tr.col("from_stop_id")));
      auto const b = loc_of.find(tr.get(r, tr.col("to_stop_id")));
      if (a == loc_of.end() || b == loc_of.end()) continue;
      auto const minutes = int_field(tr.get(r, tr.col("min_transfer_time"))) / 60;
      if (a->second == b->second) {
        auto& t = transfer[a->second];
        t = t.has_value() ? std::min(*t, minutes) : minutes;
      } else {
        auto& v = fps[a->second];
        if (std::none_of(v.begin(), v.end(), [&](auto const& x) { return x.first == b->second; })) {
          v.emplace_back(b->second, minutes);
        }
      }
    }
    // symmetric (stop.cc:368-378)
    for (auto l = 0U; l != n_loc; ++l) {
      for (auto const& [to, d] : std::vector<std::pair<uint32_t, int>>(fps[l])) {
        auto& back = fps[to];
        if (std::none_of(back.begin(), back.end(), [&](auto const& x) { return x.first == l; })) {
          back.emplace_back(l, d);
        }
      }
    }
  }

  // Footpaths between a stop and its "metas" (stop::get_metas and
  // read_stops, stop.cc:30-95, 380-402): itself, the stops of the same name,
  // and -- unless it lies within 2 degrees of (0, 0) -- the stops within
  // link_stop_distance; closed under parents and children; members farther
  // than 500 m (2000 m for its own parent or child) dropped; the children of
  // the rest added.  Each gets a walk of max(2, ceil(distance / 1.5 m/s))
  // minutes both ways, unless a footpath to that stop exists.
  {
    auto const n_stops = static_cast<uint32_t>(ids.size());
    auto const sq_dist = [&](uint32_t a, uint32_t b) { return approx_squared_distance(coords[a], coords[b]); };
    std::vector<std::vector<uint32_t>> children(n_stops);
    for (auto i = 0U; i != n_stops; ++i) {
      if (parent[kSpecial + i] != kNoParent) children[parent[kSpecial + i] - kSpecial].push_back(i);
    }
    auto const parent_of = [&](uint32_t i) {
      return parent[kSpecial + i] == kNoParent ? kNoParent : parent[kSpecial + i] - kSpecial;
    };
    std::unordered_map<std::string, std::vector<uint32_t>> same_name;
    for (auto i = 0U; i != n_stops; ++i) {
      if (!names[i].empty()) same_name[names[i]].push_back(i);
    }
    // stops by 0.002-degree cell, for the link_stop_distance radius search
    constexpr double kCell = 0.002;
    auto const cell = [&](double x) { return static_cast<int64_t>(std::floor(x / kCell)); };
    std::map<std::pair<int64_t, int64_t>, std::vector<uint32_t>> grid;
    for (auto i = 0U; i != n_stops; ++i) grid[{cell(coords[i].first), cell(coords[i].second)}].push_back(i);
    auto const link = static_cast<double>(cfg.link_stop_distance);
    auto const close = [&](uint32_t s, std::vector<uint32_t>& out) {
      auto const [lat, lng] = coords[s];
      if (cfg.link_stop_distance == 0U || (std::abs(lat) < 2.0 && std::abs(lng) < 2.0)) return;
      auto const dlat = static_cast<int64_t>(std::ceil(link / kMetersPerDegree / kCell)) + 1;
      auto const cosl = std::max(std::cos(lat * kPi / 180.0), 1e-3);
      auto const dlng = std::min<int64_t>(static_cast<int64_t>(std::ceil(link / (kMetersPerDegree * cosl) / kCell)) + 1,
                                          static_cast<int64_t>(360.0 / kCell));
      for (auto y = cell(lat) - dlat; y <= cell(lat) + dlat; ++y) {
        for (auto x = cell(lng) - dlng; x <= cell(lng) + dlng; ++x) {
          auto const it = grid.find({y, x});
          if (it == grid.end()) continue;
          for (auto const j : it->second) {
            if (sq_dist(s, j) <= link * link) out.push_back(j);
          }
        }
      }
    };
    auto const add_if_not_exists = [&](uint32_t from, uint32_t to, int d) {
      auto& v = fps[from];
      if (std::none_of(v.begin(), v.end(), [&](auto const& x) { return x.first == to; })) v.emplace_back(to, d);
    };
    for (auto s = 0U; s != n_stops; ++s) {
      std::vector<uint32_t> start{s};
      if (!names[s].empty()) {
        auto const& eq = same_name[names[s]];
        start.insert(start.end(), eq.begin(), eq.end());
      }
      close(s, start);
      std::set<uint32_t> todo(start.begin(), start.end()), done;
      while (!todo.empty()) {
        auto const next = *todo.begin();
        todo.erase(todo.begin());
        done.insert(next);
        if (auto const p = parent_of(next); p != kNoParent && !done.contains(p)) todo.insert(p);
        for (auto const c : children[next]) {
          if (!done.contains(c)) todo.insert(c);
        }
      }
      std::set<uint32_t> metas;
      for (auto const m : done) {
        auto const family = parent_of(s) == m || parent_of(m) == s;
        auto const d2 = sq_dist(s, m);
        if ((d2 > 500.0 * 500.0 && !family) || d2 > 2000.0 * 2000.0) continue;
        metas.insert(m);
      }
      for (auto const m : std::set<uint32_t>(metas)) metas.insert(children[m].begin(), children[m].end());
      for (auto const m : metas) {
        auto const dist = std::sqrt(sq_dist(s, m));
        auto const minutes = std::max(2, static_cast<int>(std::ceil((dist / 1.5) / 60.0)));
        if (minutes > 511) continue;  // footpath::kMaxDuration
        add_if_not_exists(kSpecial + s, kSpecial + m, minutes);
        add_if_not_exists(kSpecial + m, kSpecial + s, minutes);
      }
    }
  }

  // calendar.txt / calendar_dates.txt (services.cc): bit i = local date
  // iv_from + i
  std::unordered_map<std::string, bits512> services;
  {
    auto const c = file("calendar.txt");
    char const* wd[7] = {"sunday", "monday", "tuesday", "wednesday", "thursday", "friday", "saturday"};
    for (auto r = size_t{0}; r != c.rows.size(); ++r) {
      bits512 b;
      auto const from = std::max(parse_yyyymmdd(c.get(r, c.col("start_date"))), iv_from);
      auto const to = std::min(parse_yyyymmdd(c.get(r, c.col("end_date"))) + 1, iv_from + static_cast<int32_t>(n_days));
      for (auto d = from; d < to; ++d) {
        auto const weekday = static_cast<int>(((d % 7) + 11) % 7);  // 1970-01-01 was a Thursday (4)
        if (c.get(r, c.col(wd[weekday])) == "1") b.set(static_cast<uint32_t>(d - iv_from));
      }
      services[c.get(r, c.col("service_id"))] = b;
    }
    auto const cd = file("calendar_dates.txt");
    for (auto r = size_t{0}; r != cd.rows.size(); ++r) {
      auto const d = parse_yyyymmdd(cd.get(r, cd.col("date"))) - iv_from;
      auto& b = services[cd.get(r, cd.col("service_id"))];
      if (d >= 0 && d < 512) b.set(static_cast<uint32_t>(d), cd.get(r, cd.col("exception_type")) == "1");
    }
  }

  // routes.txt
  std::unordered_map<std::string, uint32_t> route_of;
  std::vector<uint8_t> route_clasz;
  std::vector<std::string> route_name;
  {
    auto const rt = file("routes.txt");
    for (auto r = size_t{0}; r != rt.rows.size(); ++r) {
      route_of[rt.get(r, rt.col("route_id"))] = static_cast<uint32_t>(route_clasz.size());
      auto const type = rt.get(r, rt.col("route_type"));
      route_clasz.push_back(to_clasz(type.empty() ? 3 : std::stoi(type)));
      route_name.push_back(rt.get(r, rt.col("route_short_name")));
    }
  }

  // trips.txt (trip.cc:290-330): flags from bikes_allowed, cars_allowed and
  // pickup_type over the per-class defaults
  std::vector<trip> trips;
  std::unordered_map<std::string, uint32_t> trip_of;
  {
    auto const tp = file("trips.txt");
    for (auto r = size_t{0}; r != tp.rows.size(); ++r) {
      trip t;
      t.id = tp.get(r, tp.col("trip_id"));
      t.block = tp.get(r, tp.col("block_id"));
      auto const ro = route_of.find(tp.get(r, tp.col("route_id")));
      if (ro == route_of.end()) continue;
      t.route = ro->second;
      auto const sv = services.find(tp.get(r, tp.col("service_id")));
      if (sv != services.end()) {
        t.service = sv->second;
        t.has_service = true;
      }
      auto const c = route_clasz[t.route];
      auto const v = [&](char const* n) {
        auto const s = tp.get(r, tp.col(n));
        return s.empty() ? 0 : std::stoi(s);
      };
      t.flags[0] = v("bikes_allowed") == 1 ? true : v("bikes_allowed") == 2 ? false : ((cfg.bikes_allowed_default >> c) & 1U) != 0U;
      t.flags[1] = v("cars_allowed") == 1 ? true : v("cars_allowed") == 2 ? false : ((cfg.cars_allowed_default >> c) & 1U) != 0U;
      t.flags[2] = v("wheelchair_accessible") == 1;
      t.flags[3] = (v("pickup_type") == 2 || v("pickup_type") > 3) ? false
                                                                      : ((cfg.reservation_not_required_default >> c) & 1U) != 0U;
      trip_of[t.id] = static_cast<uint32_t>(trips.size());
      trips.push_back(std::move(t));
    }
  }
  // stop_times.txt (stop_time.cc:111-130): ordered by stop_sequence
  {
    auto const sti = file("stop_times.txt");
    std::vector<std::vector<std::tuple<uint32_t, uint32_t, event, bool, bool>>> rows(trips.size());
    for (auto r = size_t{0}; r != sti.rows.size(); ++r) {
      auto const t = trip_of.find(sti.get(r, sti.col("trip_id")));
      auto const l = loc_of.find(sti.get(r, sti.col("stop_id")));
      if (t == trip_of.end() || l == loc_of.end()) continue;
      auto const seq = sti.get(r, sti.col("stop_sequence"));
      auto const pu = sti.get(r, sti.col("pickup_type")), dr = sti.get(r, sti.col("drop_off_type"));
      rows[t->second].emplace_back(static_cast<uint32_t>(seq.empty() ? r : std::stoul(seq)), l->second,
                                   event{parse_hhmm(sti.get(r, sti.col("arrival_time"))),
                                         parse_hhmm(sti.get(r, sti.col("departure_time")))},
                                   pu != "1", dr != "1");
    }
    for (auto i = 0U; i != trips.size(); ++i) {
      auto& v = rows[i];
      std::stable_sort(v.begin(), v.end(), [](auto const& a, auto const& b) { return std::get<0>(a) < std::get<0>(b); });
      for (auto const& [seq, l, ev, in, out] : v) {
        // the wheelchair bits: in / out at an accessible stop (stop_time.cc:119-124)
        auto const acc = accessible[l - kSpecial];
        trips[i].stops.push_back(stop_word(l, in, out, acc && in, acc && out));
        trips[i].events.push_back(ev);
        trips[i].bad = trips[i].bad || ev.arr < 0 || ev.dep < 0;  // needs interpolation: skipped
      }
      trips[i].bad = trips[i].bad || trips[i].events.size() < 2 || !trips[i].has_service;
    }
  }

  // transfers.txt, type 4 (stop.cc:156-165, load_timetable.cc:212-242):
  // stay-seated transfers from trip to trip, each pair once, in file order
  std::vector<std::vector<uint32_t>> seated_in(trips.size()), seated_out(trips.size());
  {
    auto const tr = file("transfers.txt");
    auto const push_unique = [](std::vector<uint32_t>& v, uint32_t x) {
      if (std::find(v.begin(), v.end(), x) == v.end()) v.push_back(x);
    };
    for (auto r = size_t{0}; r != tr.rows.size(); ++r) {
      if (int_field(tr.get(r, tr.col("transfer_type"))) != 4) continue;
      auto const a = trip_of.find(tr.get(r, tr.col("from_trip_id")));
      auto const b = trip_of.find(tr.get(r, tr.col("to_trip_id")));
      if (a == trip_of.end() || b == trip_of.end() || trips[a->second].bad || trips[b->second].bad) continue;
      push_unique(seated_in[b->second], a->second);
      push_unique(seated_out[a->second], b->second);
    }
  }
  auto const has_seated = [&](uint32_t i) { return !seated_in[i].empty() || !seated_out[i].empty(); };

  // block::rule_services, trip.cc:31-106: chains of a block's trips whose
  // first stop is the previous one's last stop, on the days all run.  Trips
  // with stay-seated transfers are joined by the seated pass below; a block
  // holding one builds its other trips alone (load_timetable.cc:335-360).
  struct combination {
    std::vector<uint32_t> trips;
    bits512 days;
  };
  std::vector<combination> combos;
  std::vector<std::string> block_order;
  std::unordered_map<std::string, std::vector<uint32_t>> blocks;
  for (auto i = 0U; i != trips.size(); ++i) {
    if (trips[i].bad) continue;
    if (trips[i].block.empty()) {
      // non-block trips first (load_timetable.cc:321-333)
      if (!has_seated(i)) combos.push_back({{i}, trips[i].service});
    } else {
      if (!blocks.contains(trips[i].block)) block_order.push_back(trips[i].block);
      blocks[trips[i].block].push_back(i);
    }
  }
  auto const loc_of_word = [](uint32_t w) { return w & 0x0FFFFFFFu; };
  for (auto const& b : block_order) {
    auto rule = blocks[b];
    if (std::any_of(rule.begin(), rule.end(), has_seated)) {
      for (auto const t : rule) {
        if (!has_seated(t)) combos.push_back({{t}, trips[t].service});
      }
      continue;
    }
    if (rule.size() == 1U) {
      combos.push_back({{rule.front()}, trips[rule.front()].service});
      continue;
    }
    std::stable_sort(rule.begin(), rule.end(), [&](uint32_t x, uint32_t y) {
      return trips[x].events.front().dep < trips[y].events.front().dep;
    });
    std::vector<bits512> days(rule.size());
    for (auto i = 0U; i != rule.size(); ++i) days[i] = trips[rule[i]].service;
    for (auto start = 0U; start != rule.size(); ++start) {
      struct entry {
        uint32_t cur;
        std::vector<uint32_t> collected;
        bits512 days;
      };
      std::vector<entry> stack{{start, {}, days[start]}};
      while (!stack.empty()) {
        auto next = stack.back();
        stack.pop_back();
        next.collected.push_back(next.cur);
        for (auto succ = next.cur + 1; succ < rule.size(); ++succ) {
          if (loc_of_word(trips[rule[next.cur]].stops.back()) != loc_of_word(trips[rule[succ]].stops.front())) {
            continue;
          }
          auto const both = next.days & days[succ];
          next.days = next.days & ~days[succ];
          if (both.any()) stack.push_back({succ, next.collected, both});
        }
        if (next.days.any()) {
          for (auto const x : next.collected) days[x] = days[x] & ~next.days;
          combination c;
          for (auto const x : next.collected) c.trips.push_back(rule[x]);
          c.days = next.days;
          combos.push_back(std::move(c));
        }
      }
    }
  }

  // expand_local_to_utc, local_to_utc.h:130-240, and get_stop_seq (:245-270)
  std::vector<utc_trip> utc;
  auto const expand = [&](combination const& c, std::vector<utc_trip>& out) {
    auto const& first = trips[c.trips.front()];
    auto const first_dep = first.events.front().dep;
    auto const last_arr = trips[c.trips.back()].events.back().arr;
    auto const first_day_off = first_dep / 1440, last_day_off = last_arr / 1440;
    std::vector<std::pair<std::pair<int, int>, bits512>> keys;  // (day offset, tz offset) -> days
    for (auto d = 0U; d != n_days; ++d) {
      auto const day = iv_from + static_cast<int32_t>(d);
      // the service's days must overlap timetable::date_range_
      if (day + last_day_off + 1 <= cfg.date_range_from || day + first_day_off >= cfg.date_range_to) continue;
      if (!c.days.test(d)) continue;
      auto const tz = noon[d];
      auto const utc_first = first_dep - tz;
      auto const day_off = static_cast<int>(std::floor(utc_first / 1440.0));
      auto const utc_day = static_cast<int>(d) + day_off;
      if (utc_day < 0 || utc_day >= 512) continue;
      auto const key = std::make_pair(day_off, tz);
      auto it = std::find_if(keys.begin(), keys.end(), [&](auto const& k) { return k.first == key; });
      if (it == keys.end()) {
        keys.emplace_back(key, bits512{});
        it = std::prev(keys.end());
      }
      it->second.set(static_cast<uint32_t>(utc_day));
    }
    for (auto const& [key, days] : keys) {
      utc_trip u;
      u.trips = c.trips;
      u.clasz = route_clasz[first.route];
      u.days = days;
      auto pred = 0;
      for (auto const ti : c.trips) {
        auto const& t = trips[ti];
        for (auto i = 0U; i + 1 < t.events.size(); ++i) {
          auto const dep = std::max(pred, t.events[i].dep - key.second - key.first * 1440);
          auto const arr = std::max(dep, t.events[i + 1].arr - key.second - key.first * 1440);
          u.times.push_back(dep);
          u.times.push_back(arr);
          pred = arr;
          uint8_t sec = 0;
          for (auto f = 0U; f != 4U; ++f) sec = static_cast<uint8_t>(sec | (t.flags[f] ? 1U << f : 0U));
          u.sections.push_back(sec);
        }
        if (u.stop_seq.empty()) {
          u.stop_seq = t.stops;
        } else {  // the joint stop: boarding of the next trip, alighting of the previous
          auto const prev = u.stop_seq.back(), cur = t.stops.front();
          u.stop_seq.back() = stop_word(loc_of_word(prev), ((cur >> 28) & 1U) != 0U, ((prev >> 29) & 1U) != 0U,
                                        ((cur >> 30) & 1U) != 0U, ((prev >> 31) & 1U) != 0U);
          u.stop_seq.insert(u.stop_seq.end(), t.stops.begin() + 1, t.stops.end());
        }
      }
      out.push_back(std::move(u));
    }
  };
  for (auto const& c : combos) expand(c, utc);

  // stay-seated transfers: expand_seated_trips (seated.h:29-66) and
  // build_seated_trips (seated.cc:14-290).  Every trip with a seated
  // transfer is expanded alone; then, repeatedly from the first expansion
  // that has traffic days left:
  //  1. the component: expansions linked by seated transfers (with a dwell
  //     under two hours), each with its day offset against the first, while
  //     the offset-aligned traffic days of all members still intersect;
  //  2. its entries: members with no incoming transfer inside it;
  //  3. depth-first from each entry along the outgoing transfers, appending
  //     the next trip's times (shifted by the day offsets) and its stops after
  //     the first -- the joint stop stays the arriving trip's last stop -- and
  //     emitting a transport wherever no transfer continues;
  //  4. the component's days are taken off its members.
  // The reference takes queued expansions in hash-map order; this reader
  // takes the lowest index first.
  {
    std::vector<int> rule_of(trips.size(), -1);
    std::vector<uint32_t> rule_trip;  // rule index -> trip
    for (auto i = 0U; i != trips.size(); ++i) {
      if (!trips[i].bad && has_seated(i)) {
        rule_of[i] = static_cast<int>(rule_trip.size());
        rule_trip.push_back(i);
      }
    }
    std::vector<utc_trip> rem;           // expansions
    std::vector<uint32_t> rem_rule;      // expansion -> rule index
    std::vector<std::vector<uint32_t>> rule_rems(rule_trip.size());
    for (auto r = 0U; r != rule_trip.size(); ++r) {
      std::vector<utc_trip> x;
      expand({{rule_trip[r]}, trips[rule_trip[r]].service}, x);
      for (auto& u : x) {
        rule_rems[r].push_back(static_cast<uint32_t>(rem.size()));
        rem_rule.push_back(r);
        rem.push_back(std::move(u));
      }
    }
    auto const rules = [&](std::vector<uint32_t> const& ts) {
      std::vector<uint32_t> out;
      for (auto const t : ts) out.push_back(static_cast<uint32_t>(rule_of[t]));
      return out;
    };
    std::vector<std::vector<uint32_t>> in_r(rule_trip.size()), out_r(rule_trip.size());
    for (auto r = 0U; r != rule_trip.size(); ++r) {
      in_r[r] = rules(seated_in[rule_trip[r]]);
      out_r[r] = rules(seated_out[rule_trip[r]]);
    }
    auto const first_dep = [&](uint32_t x) { return rem[x].times.front(); };
    auto const last_arr = [&](uint32_t x) { return rem[x].times.back(); };
    auto const day_change_offset = [&](uint32_t a, uint32_t b) {
      return (last_arr(a) / 1440 - first_dep(a) / 1440) + (last_arr(a) % 1440 > first_dep(b) ? 1 : 0);
    };
    auto const valid_dwell = [&](uint32_t a, uint32_t b) {
      auto diff = first_dep(b) - last_arr(a) % 1440;
      if (diff < 0) diff += 1440;
      return diff < 120;
    };
    std::vector<bool> has_bits(rem.size(), true);
    for (auto next = 0U; next < rem.size();) {
      if (!has_bits[next]) {
        ++next;
        continue;
      }
      // 1. the component (expansion -> day offset)
      std::map<uint32_t, int> component;
      auto comp_days = rem[next].days;
      std::map<uint32_t, int> q{{next, 0}};
      while (!q.empty()) {
        auto const [cur, offset] = *q.begin();
        q.erase(q.begin());
        auto const both = rem[cur].days.shifted(-offset) & comp_days;
        if (!both.any()) continue;
        comp_days = both;
        component.emplace(cur, offset);
        for (auto const o : out_r[rem_rule[cur]]) {
          for (auto const x : rule_rems[o]) {
            if (component.contains(x) || !valid_dwell(cur, x)) continue;
            q.emplace(x, offset + day_change_offset(cur, x));
          }
        }
        for (auto const i : in_r[rem_rule[cur]]) {
          for (auto const x : rule_rems[i]) {
            if (component.contains(x) || !valid_dwell(x, cur)) continue;
            q.emplace(x, offset - day_change_offset(x, cur));
          }
        }
      }
      auto const representative = [&](uint32_t rule) -> std::optional<std::pair<uint32_t, int>> {
        for (auto const& [x, off] : component) {
          if (rem_rule[x] == rule) return std::pair{x, off};
        }
        return std::nullopt;
      };
      // 2. entries
      struct item {
        utc_trip u;
        uint32_t rule;
        int transport_offset;
      };
      std::vector<item> stack;
      for (auto const& [x, off] : component) {
        auto const& ins = in_r[rem_rule[x]];
        if (std::any_of(ins.begin(), ins.end(), [&](uint32_t i) { return representative(i).has_value(); })) continue;
        auto start = rem[x];
        start.days = comp_days.shifted(off);
        stack.push_back({std::move(start), rem_rule[x], -off});
      }
      // 3. depth-first concatenation (a trip already in the chain ends it, so
      // that a cycle of transfers cannot loop)
      while (!stack.empty()) {
        auto cur = std::move(stack.back());
        stack.pop_back();
        auto has_next = false;
        for (auto const nx : out_r[cur.rule]) {
          auto const r = representative(nx);
          if (!r.has_value()) continue;
          auto const& nr = rem[r->first];
          if (std::find(cur.u.trips.begin(), cur.u.trips.end(), nr.trips.front()) != cur.u.trips.end()) continue;
          auto copy = cur.u;
          copy.trips.push_back(nr.trips.front());
          for (auto const t : nr.times) copy.times.push_back(t + (cur.transport_offset + r->second) * 1440);
          copy.stop_seq.insert(copy.stop_seq.end(), nr.stop_seq.begin() + 1, nr.stop_seq.end());
          copy.sections.insert(copy.sections.end(), nr.sections.begin(), nr.sections.end());
          stack.push_back({std::move(copy), rem_rule[r->first], cur.transport_offset});
          has_next = true;
        }
        if (!has_next) utc.push_back(std::move(cur.u));
      }
      // 4. the days used
      for (auto const& [x, off] : component) {
        rem[x].days = rem[x].days & ~comp_days.shifted(off);
        if (!rem[x].days.any()) has_bits[x] = false;
      }
    }
  }

  // routes: one key per (stop sequence, class, section flags), split by
  // the minutes-after-midnight order at every stop (get_index.h:8-29,
  // load_timetable.cc:277-309), in order of first appearance
  std::map<route_key, std::vector<std::vector<uint32_t>>> by_key;
  std::vector<route_key> key_order;
  auto const get_index = [&](std::vector<uint32_t> const& route, utc_trip const& s) -> int64_t {
    auto const key = s.times[0] % 1440;
    size_t index = 0;
    while (index < route.size() && utc[route[index]].times[0] % 1440 < key) ++index;
    for (auto i = 0U; i != s.times.size(); ++i) {
      auto const x = s.times[i] % 1440;
      if ((index > 0 && x < utc[route[index - 1]].times[i] % 1440) ||
          (index < route.size() && x > utc[route[index]].times[i] % 1440)) {
        return -1;
      }
    }
    return static_cast<int64_t>(index);
  };
  for (auto i = 0U; i != utc.size(); ++i) {
    // a flag's section list collapses to one entry for a single trip
    // (kSingleTripTransportationAllowed, load_timetable.cc:255-275) -- in
    // the route key only; the route's sections keep one entry per section
    auto ks = utc[i].sections;
    if (utc[i].trips.size() == 1U) ks.assign(1, ks.front());
    route_key k{utc[i].stop_seq, utc[i].clasz, ks};
    auto it = by_key.find(k);
    if (it == by_key.end()) {
      key_order.push_back(k);
      by_key[k].push_back({i});
      continue;
    }
    auto placed = false;
    for (auto& sub : it->second) {
      auto const idx = get_index(sub, utc[i]);
      if (idx >= 0) {
        sub.insert(sub.begin() + idx, i);
        placed = true;
        break;
      }
    }
    if (!placed) it->second.push_back({i});
  }

  // flattened arrays for b2r_tt_build
  std::vector<uint8_t> tt_(n_loc, 0);
  for (auto l = kSpecial; l != n_loc; ++l) {
    tt_[l] = static_cast<uint8_t>(transfer[l].value_or(static_cast<int>(cfg.default_transfer_time)));
  }
  // build_footpaths' connect_components (build_footpaths.cc:68-345) as
  // finalize() runs it by default (no walk-speed adjustment, no length
  // bound): self-walks dropped and one edge kept per target; then in every
  // connected component of the walk graph each member gets a walk to every
  // other member, the shortest over edges lengthened to both ends' transfer
  // times, itself at least both ends' transfer times (a component of two
  // keeps its edge so lengthened); sorted by duration (sort_footpaths).
  {
    constexpr uint32_t kNone = 0xFFFFFFFFu;
    std::vector<std::vector<std::pair<uint32_t, int>>> g(n_loc);
    for (auto l = 0U; l != n_loc; ++l) {
      for (auto const& [to, d] : fps[l]) {
        if (to == l || std::any_of(g[l].begin(), g[l].end(), [&](auto const& x) { return x.first == to; })) continue;
        g[l].emplace_back(to, std::min(d, 511));
      }
      std::stable_sort(g[l].begin(), g[l].end(), [](auto const& a, auto const& b) { return a.first < b.first; });
    }
    std::vector<uint32_t> comp(n_loc, kNone);  // find_components: first visitor's index
    for (auto i = 0U; i != n_loc; ++i) {
      if (comp[i] != kNone || g[i].empty()) continue;
      std::vector<uint32_t> stack{i};
      while (!stack.empty()) {
        auto const j = stack.back();
        stack.pop_back();
        if (comp[j] == i) continue;
        comp[j] = i;
        for (auto const& [to, d] : g[j]) {
          if (comp[to] != i) stack.push_back(to);
        }
      }
    }
    std::map<uint32_t, std::vector<uint32_t>> members;
    for (auto l = 0U; l != n_loc; ++l) {
      if (comp[l] != kNone) members[comp[l]].push_back(l);
    }
    auto const u8 = [](int m) { return std::min(m, 255); };  // u8_minutes
    std::vector<std::vector<std::pair<uint32_t, int>>> closed(n_loc);
    for (auto const& [c, ls] : members) {
      if (ls.size() == 2U) {  // process_2_node_component
        auto const a = ls[0], b = ls[1];
        if (!g[a].empty()) closed[a].emplace_back(b, std::max({u8(g[a].front().second), int{tt_[a]}, int{tt_[b]}}));
        if (!g[b].empty()) closed[b].emplace_back(a, std::max({u8(g[b].front().second), int{tt_[a]}, int{tt_[b]}}));
        continue;
      }
      auto const n = ls.size();
      auto const local = [&](uint32_t l) {
        return static_cast<size_t>(std::lower_bound(ls.begin(), ls.end(), l) - ls.begin());
      };
      std::vector<std::vector<std::pair<size_t, int>>> adj(n);  // build_component_graph
      for (auto i = size_t{0}; i != n; ++i) {
        for (auto const& [to, d] : g[ls[i]]) {
          auto const j = local(to);
          auto const w = std::max({int{tt_[ls[i]]}, int{tt_[to]}, u8(d)});
          adj[i].emplace_back(j, w);
          adj[j].emplace_back(i, w);
        }
      }
      std::vector<int> dist(n);
      for (auto i = size_t{0}; i != n; ++i) {  // dijkstra per member
        std::fill(dist.begin(), dist.end(), std::numeric_limits<int>::max());
        dist[i] = 0;
        std::priority_queue<std::pair<int, size_t>, std::vector<std::pair<int, size_t>>, std::greater<>> pq;
        pq.emplace(0, i);
        while (!pq.empty()) {
          auto const [d, u] = pq.top();
          pq.pop();
          if (d != dist[u]) continue;
          for (auto const& [v, w] : adj[u]) {
            if (d + w < dist[v]) {
              dist[v] = d + w;
              pq.emplace(dist[v], v);
            }
          }
        }
        for (auto j = size_t{0}; j != n; ++j) {
          if (j == i || dist[j] == std::numeric_limits<int>::max()) continue;
          closed[ls[i]].emplace_back(ls[j], std::max({u8(std::min(dist[j], 511)), int{tt_[ls[i]]}, int{tt_[ls[j]]}}));
        }
      }
    }
    fps = std::move(closed);
  }
  std::vector<uint32_t> fp_index(n_loc + 1, 0), fp_data;
  for (auto l = 0U; l != n_loc; ++l) {
    auto v = fps[l];
    std::stable_sort(v.begin(), v.end(), [](auto const& a, auto const& b) { return a.second < b.second; });
    for (auto const& [to, d] : v) fp_data.push_back((to & 0x7FFFFFu) | (static_cast<uint32_t>(std::min(d, 511)) << 23));
    fp_index[l + 1] = static_cast<uint32_t>(fp_data.size());
  }
  std::vector<uint32_t> rsi{0}, rstops, rnt, tbf;
  std::vector<uint16_t> stimes;
  std::vector<uint8_t> rclasz, rsec;
  std::vector<bits512> bfs;
  std::map<bits512, uint32_t> bf_of;
  std::vector<std::string> transport_names;
  auto const enc = [](int m) {
    return static_cast<uint16_t>((static_cast<uint32_t>(m / 1440) & 0x1Fu) | (static_cast<uint32_t>(m % 1440) << 5));
  };
  for (auto const& k : key_order) {
    for (auto const& sub : by_key[k]) {
      auto const& u0 = utc[sub.front()];
      rstops.insert(rstops.end(), u0.stop_seq.begin(), u0.stop_seq.end());
      rsi.push_back(static_cast<uint32_t>(rstops.size()));
      rclasz.push_back(u0.clasz);
      rsec.insert(rsec.end(), u0.sections.begin(), u0.sections.end());
      rsec.push_back(0U);
      rnt.push_back(static_cast<uint32_t>(sub.size()));
      for (auto const x : sub) {
        auto const it = bf_of.find(utc[x].days);
        if (it == bf_of.end()) {
          bf_of[utc[x].days] = static_cast<uint32_t>(bfs.size());
          tbf.push_back(static_cast<uint32_t>(bfs.size()));
          bfs.push_back(utc[x].days);
        } else {
          tbf.push_back(it->second);
        }
        transport_names.push_back(route_name[trips[utc[x].trips.front()].route]);
      }
      for (auto slot = 0U; slot != u0.times.size(); ++slot) {
        for (auto const x : sub) stimes.push_back(enc(utc[x].times[slot]));
      }
    }
  }
  std::vector<uint64_t> bf_words;
  for (auto const& b : bfs) bf_words.insert(bf_words.end(), b.w.begin(), b.w.end());
  if (bf_words.empty()) bf_words.assign(8, 0ULL);

  b2r_tt_base base{};
  base.n_locations = n_loc;
  base.date_range_from = cfg.date_range_from;
  base.date_range_to = cfg.date_range_to;
  base.transfer_time = tt_.data();
  base.parent = parent.data();
  base.location_type = loc_type.data();
  base.footpaths_out_index = fp_index.data();
  base.footpaths_out = fp_data.empty() ? fp_index.data() : fp_data.data();
  base.n_routes = static_cast<uint32_t>(rnt.size());
  base.route_stop_index = rsi.data();
  base.route_stops = rstops.empty() ? rsi.data() : rstops.data();
  base.route_clasz = rclasz.empty() ? nullptr : rclasz.data();
  base.route_n_transports = rnt.empty() ? rsi.data() : rnt.data();
  base.route_stop_times = stimes.empty() ? nullptr : stimes.data();
  base.transport_bitfield = tbf.empty() ? rsi.data() : tbf.data();
  base.n_bitfields = static_cast<uint32_t>(bf_words.size() / 8);
  base.bitfields = bf_words.data();
  base.route_section_flags = rsec.empty() ? nullptr : rsec.data();
  std::vector<uint16_t> no_times(1, 0);
  if (base.route_stop_times == nullptr) base.route_stop_times = no_times.data();
  b2r_host_timetable* h = nullptr;
  if (auto const rc = b2r_tt_build(&base, &h); rc != B2R_OK) {
    err = std::string{"b2r_tt_build: "} + b2r_last_error();
    return false;
  }
  h->t.location_ids.assign(kSpecial, std::string{});
  char const* special[kSpecial] = {"START", "END", "VIA0", "VIA1", "VIA2", "VIA3", "VIA4", "VIA5", "VIA6"};
  for (auto i = 0U; i != kSpecial; ++i) h->t.location_ids[i] = special[i];
  h->t.location_ids.insert(h->t.location_ids.end(), ids.begin(), ids.end());
  h->t.transport_names = std::move(transport_names);
  out = h;
  return true;
}

}  // namespace b2r

extern "C" {

void b2r_gtfs_config_init(b2r_gtfs_config* c) {
  std::memset(c, 0, sizeof(*c));
  c->default_transfer_time = 2;  // loader_config::default_transfer_time_
  c->link_stop_distance = 100;   // loader_config::link_stop_distance_ (loader_interface.h:18)
}

int b2r_tt_load_gtfs(const char* path, int is_text, const b2r_gtfs_config* cfg, b2r_host_timetable** out) {
  B2R_API_GUARD({
    if (path == nullptr || cfg == nullptr || out == nullptr) {
      return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "b2r_tt_load_gtfs: null argument");
    }
    if (cfg->date_range_to <= cfg->date_range_from || cfg->date_range_to - cfg->date_range_from > 500) {
      return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "b2r_tt_load_gtfs: date range empty or longer than 500 days");
    }
    std::map<std::string, std::string> files;
    if (is_text != 0) {
      files = b2r::split_mem_dir(path);
    } else {
      for (auto const* n : {"agency.txt", "stops.txt", "routes.txt", "trips.txt", "stop_times.txt",
                            "calendar.txt", "calendar_dates.txt", "transfers.txt"}) {
        std::ifstream f{std::string{path} + "/" + n, std::ios::binary};
        if (f) files[n] = std::string{std::istreambuf_iterator<char>{f}, {}};
      }
    }
    std::string err;
    try {
      if (!b2r::load_gtfs(files, *cfg, *out, err)) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, err);
    } catch (std::exception const& ex) {
      return b2r::fail(B2R_ERR_INVALID_ARGUMENT, std::string{"b2r_tt_load_gtfs: "} + ex.what());
    }
    return B2R_OK;
  });
}

int b2r_tt_location_id(const b2r_host_timetable* t, uint32_t l, const char** id) {
  if (t == nullptr || id == nullptr || l >= t->t.location_ids.size()) {
    return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "b2r_tt_location_id: no such location");
  }
  *id = t->t.location_ids[l].c_str();
  return B2R_OK;
}

int b2r_tt_transport_name(const b2r_host_timetable* t, uint32_t x, const char** name) {
  if (t == nullptr || name == nullptr || x >= t->t.transport_names.size()) {
    return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "b2r_tt_transport_name: no such transport");
  }
  *name = t->t.transport_names[x].c_str();
  return B2R_OK;
}

}  // extern "C"
