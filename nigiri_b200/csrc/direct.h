// Direct connections for pong's forward post-pass (host side).
#pragma once

#include <array>
#include <cstdint>

#include "b2r.h"
#include "prep.h"

namespace b2r {

// get_earliest_alternative (src/routing/raptor/pong.cc:35-61): the direct
// journey from `from` (reached at from_arr) to `to` that get_direct_journeys
// (src/routing/direct.cc:454-605) yields first for the exact-match query of
// make_alternative_query (src/routing/leg_alternatives.cc:27-45), if it
// arrives by to_dep: walk, transit, walk, the walk moved to start at
// from_arr.  Filters, footpath profile and transfer time settings are the
// query's.
bool earliest_alternative(host_view const& tt, tts_norm const& tts, uint32_t prf, uint32_t allowed_claszes,
                          uint8_t required_flags, uint32_t from, uint32_t to, int32_t from_arr,
                          int32_t to_dep, std::array<b2r_leg, 3>& out);

}  // namespace b2r
