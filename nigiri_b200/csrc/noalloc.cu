// One-to-all search of one query that allocates nothing
// (b2r_one_to_all_noalloc of include/b2r.h).
//
// routing::one_to_all (one_to_all.cc:25-92) for the static timetable: the
// starts of the query's offsets, then raptor::execute's rounds
// (raptor.h:218-387) without destinations and without lower bounds.  The
// whole search is ONE kernel on ONE thread-block cluster (8 CTAs of 1024
// threads); the phases of a round are separated by cluster barriers.  Its
// working state lives in g_noalloc_scratch, a fixed file-scope device array:
// the call issues no cudaMalloc / cudaFree and uses no engine, so callers
// whose device memory belongs to another allocator, or whose query path
// must not stall the device with cudaFree, can run one-to-all searches.
//
// The per-query rules are those of the batched engine's kernels (route
// scan, transfers, footpaths) for one query: labels are plain int keys
// (t forward, ~t backward, kKeyInv invalid) cleared at the start of every
// call, so the rows equal the rows b2r_search_batch returns.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>

#include "b2r.h"
#include "engine.cuh"
#include "errors.h"
#include "et_search.cuh"
#include "prep.h"
#include "timetable_image.h"

namespace b2r::noalloc {

constexpr uint32_t kCtas = 8;  // one cluster of the portable size
constexpr uint32_t kThreads = 1024;
constexpr uint32_t kAll = kCtas * kThreads;
constexpr uint32_t kRows = B2R_K;
constexpr uint32_t kMaxLoc = B2R_NOALLOC_MAX_LOCATIONS;
constexpr uint32_t kMaxRoutes = B2R_NOALLOC_MAX_ROUTES;
constexpr int kInv = dev::kKeyInv;

// scratch layout (byte offsets)
constexpr size_t kRtOff = 0;                                        // int [kRows][kMaxLoc]
constexpr size_t kBestOff = kRtOff + size_t{kRows} * kMaxLoc * 4;   // int [kMaxLoc]
constexpr size_t kTmpOff = kBestOff + size_t{kMaxLoc} * 4;          // int [kMaxLoc]
constexpr size_t kXOff = kTmpOff + size_t{kMaxLoc} * 4;             // station marks
constexpr size_t kYOff = kXOff + size_t{kMaxLoc} * 4;               // route-reached marks
constexpr size_t kXListOff = kYOff + size_t{kMaxLoc} * 4;
constexpr size_t kYListOff = kXListOff + size_t{kMaxLoc} * 4;
constexpr size_t kROff = kYListOff + size_t{kMaxLoc} * 4;           // route marks
constexpr size_t kRListOff = kROff + size_t{kMaxRoutes} * 4;
constexpr size_t kOutOff = kRListOff + size_t{kMaxRoutes} * 4;      // int16 [rows][n_loc]
constexpr size_t kCountOff = kOutOff + size_t{kRows} * kMaxLoc * 2; // list counters
constexpr size_t kBytes = kCountOff + 256;
static_assert(kBytes == B2R_NOALLOC_SCRATCH_BYTES, "scratch size and header disagree");

// list counters: station marks and route-reached marks per round parity
// (a round appends to its own parity while the previous round's list is
// still being read), route marks
enum : uint32_t { CX0 = 0, CY0 = 2, CR = 4, kCounters = 8 };

struct params {
  int32_t start_time;
  int32_t base_days;
  int32_t tad;  // worst time at destination (one_to_all.cc:44-46), as a key
  uint16_t base;
  uint8_t fwd;
  uint8_t mode;  // start match mode
  uint8_t end_k;
  uint32_t n_off;
  dev::tts_t tts;
  uint16_t claszes;  // allowed transport classes
  uint8_t req;       // required route flags
  uint8_t prf;       // footpath profile (query::prf_idx_)
  b2r_offset off[B2R_NOALLOC_MAX_OFFSETS];
};

}  // namespace b2r::noalloc

// The working state of every b2r_one_to_all_noalloc call on a device:
// round times, best / tmp labels, marks, frontier lists, the int16 result
// rows and the list counters.  Calls that overlap on the GPU share it.
static __device__ __align__(256) uint8_t g_noalloc_scratch[b2r::noalloc::kBytes];

namespace b2r::noalloc {
namespace {

namespace cg = cooperative_groups;
using dev::dtt;

// timetable::root (timetable.h:62-76) on the device image
__device__ uint32_t root_of(dtt const& T, uint32_t idx) {
  if (T.parent == nullptr) return idx;
  auto l = idx;
  for (auto i = 0;; ++i) {
    auto const par = T.parent[l];
    if (par == B2R_INVALID_IDX) break;
    if (par == idx || i > 20) {
      l = T.parent[idx];
      break;
    }
    l = par;
  }
  return l;
}

template <typename Fn>
__device__ void kids(dtt const& T, uint32_t l, Fn&& fn) {
  if (T.children_idx == nullptr) return;
  for (auto i = T.children_idx[l]; i != T.children_idx[l + 1]; ++i) fn(T.children[i]);
}

// for_each_meta (for_each_meta.h:8-45; the image has no equivalence lists)
template <typename Fn>
__device__ void metas(dtt const& T, uint8_t mode, uint32_t l, Fn&& fn) {
  switch (mode) {
    case B2R_MATCH_EXACT: fn(l); break;
    case B2R_MATCH_INTERMODAL:
      fn(l);
      kids(T, l, [&](uint32_t c) {
        if (T.loc_type != nullptr && T.loc_type[c] == B2R_LOC_GENERATED_TRACK) fn(c);
      });
      break;
    case B2R_MATCH_ONLY_CHILDREN:
      fn(l);
      kids(T, l, [&](uint32_t c) {
        fn(c);
        kids(T, c, fn);
      });
      break;
    default: {
      auto const r = root_of(T, l);
      fn(r);
      kids(T, r, [&](uint32_t c) {
        fn(c);
        kids(T, c, fn);
      });
    }
  }
}

// Labels and marks written by other CTAs of the cluster are read through L2.
__device__ __forceinline__ int ldk(int const* p) { return __ldcg(p); }
__device__ __forceinline__ uint32_t ldu(uint32_t const* p) { return __ldcg(p); }

__device__ __forceinline__ void mark(uint32_t* M, uint32_t* list, uint32_t* cnt, uint32_t e) {
  if (ldu(&M[e]) == 0u && atomicExch(&M[e], 1u) == 0u) list[atomicAdd(cnt, 1u)] = e;
}

__global__ void __cluster_dims__(kCtas, 1, 1) __launch_bounds__(kThreads, 1)
    k_one_to_all(dtt T, params P, uint8_t* scratch) {
  auto cluster = cg::this_cluster();
  auto const tid = static_cast<uint32_t>(cluster.block_rank()) * kThreads + threadIdx.x;
  auto* rt = reinterpret_cast<int*>(scratch + kRtOff);
  auto* best = reinterpret_cast<int*>(scratch + kBestOff);
  auto* tmp = reinterpret_cast<int*>(scratch + kTmpOff);
  auto* X = reinterpret_cast<uint32_t*>(scratch + kXOff);
  auto* Y = reinterpret_cast<uint32_t*>(scratch + kYOff);
  auto* xlist = reinterpret_cast<uint32_t*>(scratch + kXListOff);
  auto* ylist = reinterpret_cast<uint32_t*>(scratch + kYListOff);
  auto* R = reinterpret_cast<uint32_t*>(scratch + kROff);
  auto* rlist = reinterpret_cast<uint32_t*>(scratch + kRListOff);
  auto* out = reinterpret_cast<int16_t*>(scratch + kOutOff);
  auto* cnt = reinterpret_cast<uint32_t*>(scratch + kCountOff);
  auto const nl = T.n_loc, nr = T.n_routes;
  auto const fwd = P.fwd != 0;
  auto const tad = P.tad;
  auto const rows = static_cast<uint32_t>(P.end_k);
  // Every thread of the cluster reaches every barrier: the loops below are
  // uniform and the round loop's exit reads a count fixed before the barrier.
  auto const sync = [&]() {
    __threadfence();
    cluster.sync();
  };

  // labels start invalid, marks and counters at zero
  for (size_t i = tid; i < size_t{rows} * nl; i += kAll) rt[(i / nl) * kMaxLoc + i % nl] = kInv;
  for (auto i = tid; i < nl; i += kAll) {
    best[i] = kInv;
    tmp[i] = kInv;
    X[i] = 0u;
    Y[i] = 0u;
  }
  for (auto i = tid; i < nr; i += kAll) R[i] = 0u;
  if (tid < kCounters) cnt[tid] = 0u;
  sync();

  // starts in the order of the offsets (one_to_all.cc:30-39, add_start
  // raptor.h:190-203): round 0 and best, station marked
  if (tid == 0) {
    for (auto i = 0u; i != P.n_off; ++i) {
      auto const o = P.off[i];
      auto const t = fwd ? P.start_time + o.duration : P.start_time - o.duration;
      auto const key = dev::to_key(fwd, dev::clamp16(t - P.base_days * 1440));
      metas(T, P.mode, o.target, [&](uint32_t l) {
        if (key < ldk(&best[l])) best[l] = key;
        if (key < ldk(&rt[l])) rt[l] = key;
        if (ldu(&X[l]) == 0u) {
          X[l] = 1u;
          auto const at = ldu(&cnt[CX0]);
          xlist[at] = l;
          cnt[CX0] = at + 1u;
        }
      });
    }
  }
  sync();

  for (uint32_t k = 1; k < rows; ++k) {
    auto const px = (k - 1u) & 1u, cx = k & 1u;

    // route-reached marks of the previous round cleared; routes of the
    // stations marked in the previous round marked (raptor.h:228-241)
    {
      auto const ny = ldu(&cnt[CY0 + px]);
      for (auto i = tid; i < ny; i += kAll) Y[ldu(&ylist[i])] = 0u;
      auto const nx = ldu(&cnt[CX0 + px]);
      for (auto i = tid; i < nx; i += kAll) {
        auto const l = ldu(&xlist[i]);
        for (auto ri = T.loc_routes_idx[l]; ri != T.loc_routes_idx[l + 1]; ++ri) {
          mark(R, rlist, &cnt[CR], T.loc_routes[ri]);
        }
      }
    }
    sync();
    auto const n_marked = ldu(&cnt[CR]);
    if (n_marked == 0u) break;  // no station with a route marked (raptor.h:243-246)

    // update_route (raptor.h:1177-1349): one thread per marked route
    if (tid == 0) cnt[CY0 + px] = 0u;
    for (auto w = tid; w < n_marked; w += kAll) {
      auto const r = ldu(&rlist[w]);
      R[r] = 0u;
      uint32_t sec = 0u;  // required flags checked per section
      if ((P.claszes != 0xFFFFu || P.req != 0u) && !dev::route_allowed(T, r, P.claszes, P.req, sec)) continue;
      auto const sb = T.route_stop_idx[r];
      auto const n = T.route_stop_idx[r + 1] - sb;
      auto const n_t = T.route_tr_to[r] - T.route_tr_from[r];
      auto const* colbase = T.st + T.route_st_from[r];
      bool et_valid = false;
      uint32_t et_off = 0, n_ev = 0, n_days = 0;
      uint16_t et_day = 0;
      for (auto i = 0u; i != n; ++i) {
        auto const si = fwd ? i : n - 1u - i;
        auto const stp = T.route_stops[sb + si];
        auto const l = B2R_STOP_LOC(stp);
        auto const wc = P.prf == B2R_PROFILE_WHEELCHAIR ? 1u : 0u;  // one_to_all.cc:69
        auto const can_finish = fwd ? dev::stop_out_bit(stp, wc) : dev::stop_in_bit(stp, wc);
        auto const can_start = fwd ? dev::stop_in_bit(stp, wc) : dev::stop_out_bit(stp, wc);
        if (sec != 0u && i != 0u && !dev::section_ok(T, sb, fwd ? i - 1u : si, sec)) {
          et_valid = false;  // raptor.h:1194-1217
        }
        bool arrival_ran = false;
        if (et_valid && can_finish) {
          arrival_ran = true;
          auto const ev = colbase[n_t * (si * 2u - (fwd ? 1u : 0u)) + et_off];
          auto const by = dev::to_delta_key(fwd, et_day, P.base, dev::delta_count(ev));
          if (by <= tad) {
            if (by < ldk(&tmp[l])) atomicMin(&tmp[l], by);
            mark(Y, ylist, &cnt[CY0 + cx], l);
          }
        }
        if (i + 1u != n && can_start && ldu(&X[l]) != 0u) {
          auto const board_col = n_t * (si * 2u - (fwd ? 0u : 1u));
          auto const et_time =
              et_valid ? dev::to_delta_key(fwd, et_day, P.base, dev::delta_count(colbase[board_col + et_off]))
                       : kInv;
          auto const prt = ldk(&rt[(k - 1u) * kMaxLoc + l]);
          if (prt != kInv && prt <= et_time) {
            auto const minutes = static_cast<int>(P.base) * 1440 + dev::from_key(fwd, prt);
            auto const day = static_cast<uint16_t>(minutes / 1440);
            auto const mam = minutes % 1440;
            uint32_t nt = 0;
            uint16_t nd = 0;
            if (dev::et_search(T, fwd, r, si, day, mam, 0, tad, P.base, nt, nd, n_ev, n_days)) {
              // current_best (raptor.h:1328-1329) is valid whenever the
              // arrival part ran or the station carries a label
              auto const cb_valid = arrival_ran || ldk(&best[l]) != kInv || ldk(&tmp[l]) != kInv;
              auto const nt_time =
                  dev::to_delta_key(fwd, nd, P.base, dev::delta_count(colbase[board_col + nt]));
              if (!cb_valid || nt_time <= et_time) {
                et_valid = true;
                et_off = nt;
                et_day = nd;
              }
            }
          }
        }
      }
    }
    sync();

    // station marks of the previous round cleared
    {
      auto const nx = ldu(&cnt[CX0 + px]);
      for (auto i = tid; i < nx; i += kAll) X[ldu(&xlist[i])] = 0u;
      if (tid == 0) cnt[CR] = 0u;
    }
    sync();

    // update_transfers (raptor.h:680-743): one thread per reached station
    {
      if (tid == 0) cnt[CX0 + px] = 0u;
      auto const ny = ldu(&cnt[CY0 + cx]);
      for (auto i = tid; i < ny; i += kAll) {
        auto const l = ldu(&ylist[i]);
        auto const tk = ldk(&tmp[l]);
        if (tk == kInv) continue;
        auto const fp = dev::key_add(tk, dev::adjusted<int>(P.tts, static_cast<int>(T.transfer_time[l])));
        auto const bk = ldk(&best[l]);
        auto* rtw = &rt[k * kMaxLoc + l];
        if (fp < bk && fp < ldk(rtw)) *rtw = fp;
        if (fp < bk && fp <= tad) {
          *rtw = fp;
          best[l] = fp;
          mark(X, xlist, &cnt[CX0 + cx], l);
        }
      }
    }
    sync();

    // update_footpaths (raptor.h:745-845): one thread per reached station,
    // targets combined with atomicMin
    {
      auto const ny = ldu(&cnt[CY0 + cx]);
      auto const* idx = dev::fp_index(T, P.prf, fwd);
      auto const* dat = dev::fp_words(T, P.prf, fwd);
      for (auto i = tid; i < ny; i += kAll) {
        auto const src = ldu(&ylist[i]);
        auto const tk = ldk(&tmp[src]);
        if (tk == kInv) continue;
        for (auto j = idx[src]; j != idx[src + 1]; ++j) {
          auto const fpw = dat[j];
          auto const tgt = B2R_FP_TARGET(fpw);
          auto const key =
              dev::key_add(tk, dev::adjusted<int>(P.tts, static_cast<int>(B2R_FP_DURATION(fpw))));
          if (key < ldk(&best[tgt])) {
            atomicMin(&rt[k * kMaxLoc + tgt], key);
            if (key <= tad) {
              atomicMin(&best[tgt], key);
              mark(X, xlist, &cnt[CX0 + cx], tgt);
            }
          }
        }
      }
    }
    sync();
  }

  // rows as deltas (kInvalidDelta<Dir> where unreached)
  for (size_t i = tid; i < size_t{rows} * nl; i += kAll) {
    out[i] = static_cast<int16_t>(dev::from_key(fwd, ldk(&rt[(i / nl) * kMaxLoc + i % nl])));
  }
}

// scratch address per device, looked up once with the device current
constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch[kMaxDevices] = {};

int scratch_on(int device, void** out) {
  std::lock_guard<std::mutex> lock{g_setup_mutex};
  if (g_scratch[device] == nullptr) {
    void* p = nullptr;
    auto const e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      char msg[160];
      std::snprintf(msg, sizeof(msg), "b2r_one_to_all_noalloc: scratch address on device %d: %s",
                    device, cudaGetErrorString(e));
      return fail(B2R_ERR_CUDA, msg);
    }
    g_scratch[device] = p;
  }
  *out = g_scratch[device];
  return B2R_OK;
}

int run(b2r_timetable const* tt, b2r_query const* q, int16_t* round_times, uint64_t capacity,
        uint32_t* n_rows, int32_t* base_day, cudaStream_t stream) {
  char msg[192];
  if (tt == nullptr || q == nullptr || round_times == nullptr || n_rows == nullptr) {
    return fail(B2R_ERR_INVALID_ARGUMENT, "b2r_one_to_all_noalloc: null argument");
  }
  if (q->kind != B2R_ONE_TO_ALL || q->direction > B2R_BACKWARD ||
      q->start_match_mode > B2R_MATCH_INTERMODAL || (q->n_start != 0 && q->start == nullptr)) {
    return fail(B2R_ERR_INVALID_ARGUMENT,
                "b2r_one_to_all_noalloc: needs a one-to-all query with a valid direction, "
                "match mode and start offsets");
  }
  auto const nl = tt->d.n_loc, nr = tt->d.n_routes;
  if (nl > kMaxLoc || nr > kMaxRoutes) {
    std::snprintf(msg, sizeof(msg),
                  "b2r_one_to_all_noalloc: timetable has %u locations and %u routes; the "
                  "scratch array holds at most %u and %u",
                  nl, nr, kMaxLoc, kMaxRoutes);
    return fail(B2R_ERR_CAPACITY, msg);
  }
  if (q->n_start > B2R_NOALLOC_MAX_OFFSETS) {
    std::snprintf(msg, sizeof(msg),
                  "b2r_one_to_all_noalloc: query has %u start offsets; at most %u are supported",
                  q->n_start, B2R_NOALLOC_MAX_OFFSETS);
    return fail(B2R_ERR_CAPACITY, msg);
  }
  auto const end_k = static_cast<uint32_t>(std::min<int>(q->max_transfers, B2R_MAX_TRANSFERS) + 2);
  auto const need = static_cast<uint64_t>(end_k) * nl;
  if (capacity < need) {
    std::snprintf(msg, sizeof(msg),
                  "b2r_one_to_all_noalloc: round_times holds %llu values; %u rows of %u "
                  "locations need %llu",
                  static_cast<unsigned long long>(capacity), end_k, nl,
                  static_cast<unsigned long long>(need));
    return fail(B2R_ERR_CAPACITY, msg);
  }
  params P{};
  for (auto i = 0u; i != q->n_start; ++i) {
    if (q->start[i].target >= nl) {
      return fail(B2R_ERR_INVALID_ARGUMENT, "b2r_one_to_all_noalloc: start offset target out of range");
    }
    P.off[i] = q->start[i];
  }
  // one_to_all.cc:18-24 (make_base) and 44-46 (worst time at destination)
  auto const fwd = q->direction == B2R_FORWARD;
  P.n_off = q->n_start;
  P.fwd = fwd ? 1 : 0;
  P.mode = q->start_match_mode;
  P.end_k = static_cast<uint8_t>(end_k);
  P.start_time = q->start_time;
  P.base = static_cast<uint16_t>(round_to_days(q->start_time) - tt->d.internal_from_days);
  P.base_days = tt->d.internal_from_days + P.base;
  P.tts = {q->tts_default, q->tts_min_transfer_time, q->tts_additional_time, q->tts_factor};
  P.claszes = static_cast<uint16_t>(q->allowed_claszes & 0xFFFFu);
  if (q->prf_idx >= B2R_N_PROFILES) return fail(B2R_ERR_INVALID_ARGUMENT, "b2r_one_to_all_noalloc: prf_idx out of range");
  P.prf = q->prf_idx;
  P.req = static_cast<uint8_t>((q->require_bike_transport != 0 ? 1u << B2R_FLAG_BIKES : 0u) |
                               (q->require_car_transport != 0 ? 1u << B2R_FLAG_CARS : 0u) |
                               (q->prf_idx == B2R_PROFILE_WHEELCHAIR ? 1u << B2R_FLAG_WHEELCHAIR : 0u) |
                               (q->no_compulsory_reservation != 0 ? 1u << B2R_FLAG_RESERVATION_NOT_REQUIRED : 0u));
  auto const span = static_cast<int>(q->max_travel_time);
  auto const worst = std::clamp(q->start_time + (fwd ? span : -span) - P.base_days * 1440, -32768, 32767);
  P.tad = std::min(dev::kKeyInv, fwd ? worst : ~worst);

  int prev = 0;
  auto e = cudaGetDevice(&prev);
  if (e == cudaSuccess && prev != tt->device) e = cudaSetDevice(tt->device);
  if (e != cudaSuccess) {
    std::snprintf(msg, sizeof(msg), "b2r_one_to_all_noalloc: device %d: %s", tt->device,
                  cudaGetErrorString(e));
    return fail(B2R_ERR_CUDA, msg);
  }
  int status = B2R_OK;
  void* scratch = nullptr;
  if (tt->device < 0 || tt->device >= kMaxDevices) {
    status = fail(B2R_ERR_UNSUPPORTED, "b2r_one_to_all_noalloc: device index beyond 63");
  } else {
    status = scratch_on(tt->device, &scratch);
  }
  if (status == B2R_OK) {
    auto* base = static_cast<uint8_t*>(scratch);
    k_one_to_all<<<kCtas, kThreads, 0, stream>>>(tt->d, P, base);
    e = cudaGetLastError();
    if (e == cudaSuccess) {
      e = cudaMemcpyAsync(round_times, base + kOutOff, need * sizeof(int16_t), cudaMemcpyDeviceToHost,
                          stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
      std::snprintf(msg, sizeof(msg), "b2r_one_to_all_noalloc: %s", cudaGetErrorString(e));
      status = fail(B2R_ERR_CUDA, msg);
    } else {
      *n_rows = end_k;
      if (base_day != nullptr) *base_day = P.base_days;
    }
  }
  if (prev != tt->device) cudaSetDevice(prev);
  return status;
}

}  // namespace
}  // namespace b2r::noalloc

extern "C" int b2r_one_to_all_noalloc(const b2r_timetable* tt, const b2r_query* q, int16_t* round_times,
                                      uint64_t capacity, uint32_t* n_rows, int32_t* base_day,
                                      void* stream) {
  B2R_API_GUARD({
    return b2r::noalloc::run(tt, q, round_times, capacity, n_rows, base_day,
                             static_cast<cudaStream_t>(stream));
  });
}
