// Test helper: nigiri's search<Dir, Algo> (restated in b2r.hpp) with the
// engine's Algo, b2r_algo, callable through ctypes on a timetable image a
// test has uploaded.  The result has the b2r_result layout and stays valid
// until the next call (one call at a time).
#include <vector>

#include "b2r.hpp"

namespace r = b2r::routing;

namespace {
std::vector<b2r_journey> g_journeys;
std::vector<b2r_leg> g_legs;

b2r_leg c_leg(r::leg const& l) {
  b2r_leg x{};
  x.from = l.from_;
  x.to = l.to_;
  x.dep_time = l.dep_time_;
  x.arr_time = l.arr_time_;
  if (auto const* t = std::get_if<r::run_enter_exit>(&l.uses_)) {
    x.kind = B2R_LEG_TRANSPORT;
    x.transport = t->transport_;
    x.day = t->day_;
    x.stop_from = t->stop_from_;
    x.stop_to = t->stop_to_;
    x.rt_transport = t->rt_transport_;
  } else if (auto const* f = std::get_if<r::footpath>(&l.uses_)) {
    x.kind = B2R_LEG_FOOTPATH;
    x.transport = f->target_;
    x.duration = f->duration_;
    x.rt_transport = B2R_INVALID_IDX;
  } else {
    auto const& o = std::get<r::offset>(l.uses_);
    x.kind = B2R_LEG_OFFSET;
    x.transport = o.target_;
    x.duration = o.duration_;
    x.transport_mode_id = o.transport_mode_id_;
    x.rt_transport = B2R_INVALID_IDX;
  }
  return x;
}
}  // namespace

extern "C" int algo_search(b2r_timetable* uploaded, const b2r_timetable_desc* d, const b2r_query* c,
                           b2r_result* out) {
  try {
    b2r::timetable tt{uploaded, *d};
    auto const q = r::query_of(*c);
    r::b2r_algo_state state;
    auto const res =
        c->direction == B2R_FORWARD
            ? r::search<r::direction::kForward, r::b2r_algo<r::direction::kForward>>{tt, state, q}.execute()
            : r::search<r::direction::kBackward, r::b2r_algo<r::direction::kBackward>>{tt, state, q}.execute();
    g_journeys.clear();
    g_legs.clear();
    for (auto const& j : res.journeys_) {
      b2r_journey bj{j.start_time_, j.dest_time_, j.dest_, j.transfers_, static_cast<uint8_t>(j.error_ ? 1 : 0),
                     static_cast<uint16_t>(j.legs_.size()), static_cast<uint32_t>(g_legs.size())};
      for (auto const& l : j.legs_) g_legs.push_back(c_leg(l));
      g_journeys.push_back(bj);
    }
    *out = b2r_result{};
    out->status = res.status_;
    out->n_journeys = static_cast<uint32_t>(g_journeys.size());
    out->journeys = g_journeys.data();
    out->legs = g_legs.data();
    out->interval_from = res.interval_.from_;
    out->interval_to = res.interval_.to_;
    return B2R_OK;
  } catch (b2r::error const& e) {
    return e.status;
  }
}
