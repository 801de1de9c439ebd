// B200 RAPTOR engine: device timetable image, resident query slots, the
// batched super-step (captured as a CUDA graph), continuous admission and
// the C ABI of include/b2r.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "b2r.h"
#include "direct.h"
#include "engine.cuh"
#include "errors.h"
#include "kernels.cuh"
#include "prep.h"
#include "timetable_image.h"

namespace b2r {

namespace {

struct cuda_error : std::runtime_error {
  using std::runtime_error::runtime_error;
};

#define B2R_CUDA(call)                                                            \
  do {                                                                            \
    auto const e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                      \
      throw ::b2r::cuda_error(std::string{#call} + ": " + cudaGetErrorString(e_));       \
    }                                                                             \
  } while (0)

template <typename T>
T* dmalloc(size_t n, uint64_t& total) {
  T* p = nullptr;
  if (n == 0) n = 1;
  B2R_CUDA(cudaMalloc(&p, n * sizeof(T)));
  total += n * sizeof(T);
  return p;
}

template <typename T>
T* dupload(T const* src, size_t n, uint64_t& total) {
  auto* p = dmalloc<T>(n, total);
  if (src != nullptr && n != 0) B2R_CUDA(cudaMemcpy(p, src, n * sizeof(T), cudaMemcpyHostToDevice));
  return p;
}

int n_sms(int dev) {
  int n = 0;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 132;
}

}  // namespace
}  // namespace b2r

namespace b2r {
namespace {

template <typename T>
void host_copy(std::vector<T>& v, T const* p, size_t n) {
  if (p == nullptr) {
    v.clear();
    return;
  }
  v.assign(p, p + n);
}

}  // namespace
}  // namespace b2r

// ==================================================================== engine
// One-to-all rows of one result: page-locked host memory when the batch
// path copies the rows straight into it from the device, else ordinary
// heap memory (the serving loop, whose results live until b2r_release).
class row_buf {
 public:
  row_buf() = default;
  row_buf(row_buf const&) = delete;
  row_buf& operator=(row_buf const&) = delete;
  row_buf(row_buf&& o) noexcept { take(o); }
  row_buf& operator=(row_buf&& o) noexcept {
    if (this != &o) {
      free_mem();
      take(o);
    }
    return *this;
  }
  ~row_buf() { free_mem(); }
  // n values; a new block only if the current one is too small
  void resize(size_t n, bool pinned) {
    if (n > cap_ || pinned != pinned_) {
      free_mem();
      if (pinned) {
        void* q = nullptr;
        if (cudaMallocHost(&q, n * sizeof(int16_t)) != cudaSuccess) throw std::bad_alloc{};
        p_ = static_cast<int16_t*>(q);
      } else {
        p_ = static_cast<int16_t*>(::operator new(n * sizeof(int16_t)));
      }
      cap_ = n;
      pinned_ = pinned;
    }
    n_ = n;
  }
  void clear() { n_ = 0; }
  bool empty() const { return n_ == 0; }
  size_t size() const { return n_; }
  size_t capacity() const { return cap_; }
  bool pinned() const { return pinned_; }
  int16_t* data() { return p_; }
  int16_t const* data() const { return p_; }

 private:
  void take(row_buf& o) {
    p_ = o.p_;
    n_ = o.n_;
    cap_ = o.cap_;
    pinned_ = o.pinned_;
    o.p_ = nullptr;
    o.n_ = o.cap_ = 0;
  }
  void free_mem() {
    if (p_ != nullptr) {
      if (pinned_) cudaFreeHost(p_);
      else ::operator delete(p_);
    }
    p_ = nullptr;
    n_ = cap_ = 0;
  }
  int16_t* p_{nullptr};
  size_t n_{0}, cap_{0};
  bool pinned_{false};
};

struct b2r_engine {
  b2r_timetable* tt{nullptr};
  b2r_engine_config cfg{};
  b2r::host_view view{};      // the timetable's host view, with the bound overlay
  b2r_rt const* rt{nullptr};  // the bound real-time overlay, if any
  int lb_mode() const { return rt != nullptr ? 0 : static_cast<int>(cfg.use_lower_bounds); }
  uint32_t S{0}, G{0}, max_j{0}, max_starts{0}, max_dest{0}, max_off{0};
  uint64_t bytes_per_slot{0}, bytes{0};
  b2r::dev::state st{};
  cudaStream_t stream{nullptr};
  cudaGraphExec_t graph{nullptr};
  cudaStream_t stream2{nullptr};  // exports overlapping the super-steps
  b2r_launch_shape shape{8, 256, 8, 4, 4, 0};  // launch shape of the super-step
  cudaGraphExec_t lb_graph{nullptr};  // 4 x 2 Bellman-Ford iterations
  int sms{132};
  std::vector<void*> allocs;

  // host bookkeeping
  std::vector<uint16_t> gen_query;  // per slot
  std::vector<int64_t> slot_query;  // query index in the current batch, -1 free
  using summary_t = b2r::dev::slot_summary;
  summary_t* d_summary{nullptr};
  summary_t* h_summary{nullptr};  // pinned
  uint32_t* h_lbcount{nullptr};   // pinned
  uint64_t lb_chunks{0};
  double lb_ms{0};
  b2r::dev::journey_rec* d_keep{};  // journeys kept across interval-extension phases
  // host<->device bytes copied by the current batch call
  uint64_t h2d_bytes{0}, d2h_bytes{0};
  uint64_t aux_launches{0};  // kernels launched outside the super-steps (admission, export, ...)
  // host time of the current batch call: preparation (summed over the
  // workers), admission, export + finalisation, waiting for preparation
  std::atomic<uint64_t> prep_ns{0};
  double admit_ms{0}, export_ms{0}, idle_ms{0};
  // admission staging (pinned) and device mirror
  uint8_t* h_adm{nullptr};
  uint8_t* d_adm{nullptr};
  size_t adm_cap{0};
  // export staging
  uint8_t* h_exp{nullptr};
  uint8_t* d_exp{nullptr};
  size_t exp_cap{0};
  uint32_t* d_exp_list{nullptr};

  b2r_batch_stats last{};
  cudaEvent_t ev0{nullptr}, ev1{nullptr};
  // device busy time of a batch: the intervals (ms after ev_base) in which
  // super-step chunks (main stream) and finished-slot work (reconstruction
  // and export kernels, second stream) ran; their union is the batch's
  // device time
  cudaEvent_t ev_base{nullptr}, ev2a{nullptr}, ev2b{nullptr};
  cudaEvent_t ev_hdr{nullptr};  // an export's headers are on the host
  // timing engines (profile = 2): the route phase of every super-step,
  // bracketed inside the graph and read after each super-step
  cudaEvent_t ev_scan_a{nullptr}, ev_scan_b{nullptr};
  double scan_ms{0};
  uint64_t scan_launches{0};
  bool base_recorded{false};
  std::vector<std::pair<double, double>> busy;
  // profiling: event pairs bracketing each route-scan launch
  std::vector<cudaEvent_t> prof_ev;
  size_t prof_used{0};
  std::vector<cudaEvent_t> prof_rc_ev;  // around the reconstruction launches
  size_t prof_rc_used{0};
  // per route-scan launch: marked entries, cumulative stop visits
  static constexpr uint32_t kProfRows = 4096;
  unsigned long long* d_prof_rows{};
  std::chrono::steady_clock::time_point batch_t0;

  // results of the last batch / serving tickets
  struct result_store {
    std::vector<b2r_journey> journeys;
    std::vector<b2r_leg> legs;
    row_buf rt_rows;
    b2r_result view{};
  };
  std::vector<result_store> results;
  // page-locked one-to-all row buffers of results that the caller has given
  // up (the previous call's): the next batch copies rows straight into them
  std::vector<row_buf> row_pool;
  size_t row_pool_bytes{0};
  std::mutex row_mu;  // the pool: the serving loop takes, b2r_release gives back

  // serving (b2r_serve_start .. b2r_serve_stop): driver thread, preparation
  // pool and tickets; type-erased because the state is defined further down
  bool serving{false};
  std::shared_ptr<void> serve;

  ~b2r_engine();
};

namespace b2r {
namespace {

// admission flags: the previous phase's rounds 0..n-1 folded into pong
// bounds (raptor.h:117-170), round times and time_at_dest kept (a pong
// after the first of its iteration), destination bits of the previous
// phase cleared (the slot changes phase without retiring)
constexpr uint32_t kAdmFillRows = 0xFFu;  // rows folded by k_fill_bounds
constexpr uint32_t kAdmKeepRt = 1u << 8;
constexpr uint32_t kAdmRephase = 1u << 9;

struct adm_hdr {
  uint32_t slot;
  uint32_t n_starts, n_dest, n_off;
  uint32_t clear_rt;
  uint32_t lb_mode;  // 0 zeros, 1 column in payload, 2 solved on the device, 3 from the table,
                     // 4 kept (the column of the query's previous phase)
  uint32_t n_seeds;
  uint32_t flags;
  uint32_t n_keep, pad;
  uint64_t off_slot, off_starts, off_dest, off_off, off_lb, off_seeds, off_keep;
};

__global__ void k_admit(dev::state st, adm_hdr const* hdr, uint8_t const* payload, uint32_t n_adm,
                        uint32_t max_starts, uint32_t max_dest, uint32_t max_off) {
  auto const a = blockIdx.x;
  if (a >= n_adm) return;
  auto const h = hdr[a];
  auto const s = h.slot;
  auto const n_loc = st.tt.n_loc;
  __shared__ int16_t old_tad[dev::kK];
  if ((h.flags & (kAdmKeepRt | kAdmRephase)) != 0u) {  // the slot's previous phase, read before it is overwritten
    auto const& old = st.slots[s];
    if ((h.flags & kAdmKeepRt) != 0u && threadIdx.x < dev::kK) old_tad[threadIdx.x] = old.tad[threadIdx.x];
    if ((h.flags & kAdmRephase) != 0u && !old.intermodal_dest && !old.one_to_all) {
      for (auto i = threadIdx.x; i < old.n_dest; i += blockDim.x) {
        atomicAnd(&st.D[st.dest_pool[old.dest_off + i].loc * st.G + (s >> 5)], ~(1u << (s & 31)));
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    auto sl = *reinterpret_cast<dev::slot_t const*>(payload + h.off_slot);
    sl.gen_group = st.slots[s].gen_group;  // start-time generations persist
    if ((h.flags & kAdmKeepRt) != 0u) {
      for (auto i = 0; i != dev::kK; ++i) sl.tad[i] = old_tad[i];
    }
    sl.starts_off = s * max_starts;
    sl.dest_off = s * max_dest;
    sl.soff_off = s * max_off;
    sl.doff_off = s * max_off + sl.n_soff;
    st.slots[s] = sl;
  }
  auto const* starts = reinterpret_cast<dev::start_rec const*>(payload + h.off_starts);
  for (auto i = threadIdx.x; i < h.n_starts; i += blockDim.x) st.start_pool[s * max_starts + i] = starts[i];
  auto const* dests = reinterpret_cast<dev::dest_rec const*>(payload + h.off_dest);
  for (auto i = threadIdx.x; i < h.n_dest; i += blockDim.x) st.dest_pool[s * max_dest + i] = dests[i];
  auto const* offs = reinterpret_cast<b2r_offset const*>(payload + h.off_off);
  for (auto i = threadIdx.x; i < h.n_off; i += blockDim.x) st.off_pool[s * max_off + i] = offs[i];
  auto const* lbc = reinterpret_cast<uint16_t const*>(payload + h.off_lb);
  if (h.lb_mode < 2) {
    for (auto l = threadIdx.x; l < n_loc; l += blockDim.x) {
      st.lb[static_cast<size_t>(l) * st.S + s] = h.lb_mode ? lbc[l] : uint16_t{0};
    }
  }
  if (h.clear_rt) {  // query generations wrapped: no stale tag may survive
    for (size_t i = threadIdx.x; i < static_cast<size_t>(dev::kK) * n_loc; i += blockDim.x) {
      st.rt[i * st.S + s] = 0xFFFFFFFFu;
    }
    for (size_t i = threadIdx.x; i < n_loc; i += blockDim.x) st.dist[i * st.S + s] = 0xFFFFFFFFu;
  }
  auto const words = (st.max_j + 31u) / 32u;
  for (auto i = threadIdx.x; i < words; i += blockDim.x) st.blocks_used[s * words + i] = 0u;
  __syncthreads();
  if (h.n_keep != 0u && threadIdx.x == 0) {  // a pong's shared result set (pong.cc:322-326)
    auto const* keep = reinterpret_cast<dev::journey_rec const*>(payload + h.off_keep);
    auto* els = st.journeys + static_cast<size_t>(s) * st.max_j;
    for (auto i = 0u; i != h.n_keep; ++i) {
      els[i] = keep[i];
      st.blocks_used[s * words + keep[i].block / 32u] |= 1u << (keep[i].block % 32u);
    }
  }
  if (h.lb_mode == 2) {  // Dijkstra seeds into the device frontier
    auto const qtag = dev::tagcode(st.slots[s].gen_query);
    auto const* seeds = reinterpret_cast<uint32_t const*>(payload + h.off_seeds);
    for (auto i = threadIdx.x; i < h.n_seeds; i += blockDim.x) {
      auto const l = seeds[2 * i];
      atomicMin(&st.dist[static_cast<size_t>(l) * st.S + s], dev::enc(qtag, static_cast<int>(seeds[2 * i + 1])));
      dev::mark(st, st.F[0], st.flist[0], dev::C_F0, l * st.G + (s >> 5), 1u << (s & 31));
    }
    if (threadIdx.x == 0) atomicOr(&st.lb_mask[s >> 5], 1u << (s & 31));
  }
  if (h.lb_mode == 3) {  // k_lb_fill has written the column
    if (threadIdx.x == 0) {  // children inherit the parent's bound, in location order
      auto const& T = st.tt;
      for (auto w = 0u; w != T.n_with_children; ++w) {
        auto const i = T.with_children[w];
        auto const lbv = st.lb[static_cast<size_t>(i) * st.S + s];
        for (auto c = T.children_idx[i]; c != T.children_idx[i + 1]; ++c) {
          auto& cv = st.lb[static_cast<size_t>(T.children[c]) * st.S + s];
          if (lbv < cv) cv = lbv;
        }
      }
    }
  }
  // is-destination bits of station-to-station queries
  auto const& sl = st.slots[s];
  if (!sl.intermodal_dest && !sl.one_to_all) {
    for (auto i = threadIdx.x; i < h.n_dest; i += blockDim.x) {
      atomicOr(&st.D[dests[i].loc * st.G + (s >> 5)], 1u << (s & 31));
    }
  }
}

// Lower bounds from the all-pairs tables for the admissions in lower-bound
// mode 3: Dijkstra from the seeds (dijkstra.cc:18-67) as a minimum over
// table rows -- every path of length <= kMaxTravelTime only passes
// locations closer than that, so min(seed distance + row) is the capped
// multi-source distance.  blockIdx.y = slot group, blockIdx.x = a tile of
// 128 locations: the tile's values are computed with the threads over
// locations (table rows read in order) and written with a warp over the
// group's slots per location, 64 contiguous bytes of lb.
struct lb_group {
  uint32_t g, first, count, pad;
};
struct lb_entry {
  uint32_t lane, n_seeds, fwd, pad;
  uint64_t off_seeds;
};
constexpr uint32_t kLbTile = 128;

__global__ void k_lb_fill(dev::state st, lb_group const* groups, lb_entry const* entries,
                          uint8_t const* payload) {
  __shared__ uint16_t tile[32][kLbTile + 2];
  auto const grp = groups[blockIdx.y];
  auto const stride = st.lb_stride;  // table row length, a multiple of 8
  auto const x0 = blockIdx.x * kLbTile;
  // work items (entry, chunk of 8 locations): one 16-byte table load per
  // seed and chunk, eight running minima
  constexpr uint32_t kChunks = kLbTile / 8u;
  for (auto item = threadIdx.x; item < grp.count * kChunks; item += blockDim.x) {
    auto const e = item / kChunks, ch = item % kChunks;
    auto const xc = x0 + ch * 8u;
    uint32_t best[8];
    for (auto j = 0u; j != 8u; ++j) best[j] = 0xFFFFu;
    if (xc < stride) {  // the chunk lies inside the row (stride % 8 == 0)
      auto const en = entries[grp.first + e];
      auto const* seeds = reinterpret_cast<uint32_t const*>(payload + en.off_seeds);
      auto const* tab = en.fwd ? st.lb_table_fwd : st.lb_table_bwd;
      for (auto i = 0u; i != en.n_seeds; ++i) {
        auto const m = seeds[2 * i];
        auto const sd = seeds[2 * i + 1];
        auto const v = *reinterpret_cast<uint4 const*>(tab + static_cast<size_t>(m) * stride + xc);
        uint32_t const w[4] = {v.x, v.y, v.z, v.w};
        for (auto j = 0u; j != 8u; ++j) {
          auto const d = (w[j >> 1] >> (16u * (j & 1u))) & 0xFFFFu;
          if (d == 0xFFFFu) continue;
          auto const c = sd + d;
          if ((c <= B2R_MAX_TRAVEL_TIME_MIN || xc + j == m) && c < best[j]) best[j] = c;
        }
      }
    }
    for (auto j = 0u; j != 8u; ++j) tile[e][ch * 8u + j] = static_cast<uint16_t>(best[j]);
  }
  __syncthreads();
  auto const n_loc = st.tt.n_loc;
  for (auto i = threadIdx.x; i < kLbTile * 32u; i += blockDim.x) {
    auto const xi = i / 32u, e = i % 32u;
    auto const x = x0 + xi;
    if (e < grp.count && x < n_loc) {
      st.lb[static_cast<size_t>(x) * st.S + grp.g * 32u + entries[grp.first + e].lane] = tile[e][xi];
    }
  }
}

// fill_bounds (raptor.h:117-170) for the slots re-admitted to the first
// pong of an iteration, before k_admit overwrites them: row k = the best of
// rounds 0..k of the slot's ping, stored as a key of the flipped (pong)
// search.  blockIdx.y = item, threads over locations.
struct fill_item {
  uint32_t slot, rows;
};

__global__ void k_fill_bounds(dev::state st, fill_item const* items) {
  auto const it = items[blockIdx.y];
  auto const s = it.slot;
  auto const& sl = st.slots[s];
  auto const oq = dev::tagcode(sl.gen_query);
  auto const ofwd = sl.fwd != 0;
  auto const n_loc = st.tt.n_loc;
  for (auto l = blockIdx.x * blockDim.x + threadIdx.x; l < n_loc; l += gridDim.x * blockDim.x) {
    int best = dev::kKeyInv;
    for (auto k = 0u; k != it.rows; ++k) {
      auto const at = (static_cast<size_t>(k) * n_loc + l) * st.S + s;
      auto const key = dev::dec(st.rt[at], oq);
      if (key < best) best = key;
      st.bounds[at] = static_cast<int16_t>(dev::to_key(!ofwd, dev::from_key(ofwd, best)));
    }
  }
}

__global__ void k_retire(dev::state st, uint32_t const* slots, uint32_t n) {
  auto const a = blockIdx.x;
  if (a >= n) return;
  auto const s = slots[a];
  auto const& sl = st.slots[s];
  if (!sl.intermodal_dest && !sl.one_to_all) {
    for (auto i = threadIdx.x; i < sl.n_dest; i += blockDim.x) {
      atomicAnd(&st.D[st.dest_pool[sl.dest_off + i].loc * st.G + (s >> 5)], ~(1u << (s & 31)));
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) st.slots[s].state = dev::S_IDLE;
}


// profiling engines: the marked-entry count and cumulative stop visits after
// route-scan launch `idx`
__global__ void k_prof_row(dev::state st, unsigned long long* rows, uint32_t idx) {
  rows[2 * idx] = st.counters[dev::C_R];
  rows[2 * idx + 1] = st.prof[0];
}

// export: per listed slot, journey headers + leg blocks (+ one-to-all rows)
// legs exported with a slot's journeys
enum : uint32_t {
  kLegsAll = 0,    // kMaxLegs per journey
  kLegsMatch = 1,  // one journey: the first matching (recon_transfers, recon_start), the one a
                   // pong phase rebuilds; its index precedes the legs (UINT32_MAX: none)
  kLegsNone = 2,   // journey headers only (a ping phase rebuilds nothing)
};

struct exp_item {
  uint32_t slot;
  uint32_t n_j;
  uint32_t n_rows;  // one-to-all rows (0 otherwise)
  uint32_t legs_mode;
  uint64_t off_j, off_legs, off_rows, off_slot;
};

// blockIdx.x = item, blockIdx.y = share of the item's one-to-all rows
// (rows are n_rows x n_locations values: many blocks per item)
__global__ void k_export(dev::state st, exp_item const* items, uint32_t n_items, uint8_t* out) {
  if (blockIdx.x >= n_items) return;
  auto const it = items[blockIdx.x];
  auto const s = it.slot;
  auto const& sl = st.slots[s];
  if (blockIdx.y == 0) {
    if (threadIdx.x == 0) *reinterpret_cast<dev::slot_t*>(out + it.off_slot) = sl;
    auto* js = reinterpret_cast<dev::journey_rec*>(out + it.off_j);
    auto* legs = reinterpret_cast<b2r_leg*>(out + it.off_legs);
    for (auto i = threadIdx.x; i < it.n_j; i += blockDim.x) {
      js[i] = st.journeys[static_cast<size_t>(s) * st.max_j + i];
    }
    if (it.legs_mode == kLegsAll) {
      for (auto x = threadIdx.x; x < it.n_j * dev::kMaxLegs; x += blockDim.x) {
        auto const i = x / dev::kMaxLegs, k = x % dev::kMaxLegs;
        auto const blk = st.journeys[static_cast<size_t>(s) * st.max_j + i].block;
        legs[x] = st.legs[(static_cast<size_t>(s) * st.max_j + blk) * dev::kMaxLegs + k];
      }
    } else if (it.legs_mode == kLegsMatch) {
      __shared__ uint32_t match;
      if (threadIdx.x == 0) {
        match = UINT32_MAX;
        for (auto i = 0u; i != it.n_j; ++i) {
          auto const& j = st.journeys[static_cast<size_t>(s) * st.max_j + i];
          if (j.transfers == sl.recon_transfers && j.start_time == sl.recon_start) {
            match = i;
            break;
          }
        }
        *reinterpret_cast<uint32_t*>(out + it.off_legs) = match;
      }
      __syncthreads();
      if (match != UINT32_MAX) {
        auto* one = reinterpret_cast<b2r_leg*>(out + it.off_legs + 16);
        auto const blk = st.journeys[static_cast<size_t>(s) * st.max_j + match].block;
        for (auto k = threadIdx.x; k < static_cast<uint32_t>(dev::kMaxLegs); k += blockDim.x) {
          one[k] = st.legs[(static_cast<size_t>(s) * st.max_j + blk) * dev::kMaxLegs + k];
        }
      }
    }
  }
  if (it.n_rows != 0) {
    auto* rows = reinterpret_cast<int16_t*>(out + it.off_rows);
    auto const qtag = dev::tagcode(sl.gen_query);
    auto const n = static_cast<size_t>(it.n_rows) * st.tt.n_loc;
    for (size_t x = static_cast<size_t>(blockIdx.y) * blockDim.x + threadIdx.x; x < n;
         x += static_cast<size_t>(gridDim.y) * blockDim.x) {
      auto const k = static_cast<uint32_t>(x / st.tt.n_loc), l = static_cast<uint32_t>(x % st.tt.n_loc);
      auto const key = dev::dec(st.rt[(static_cast<size_t>(k) * st.tt.n_loc + l) * st.S + s], qtag);
      rows[x] = static_cast<int16_t>(dev::from_key(sl.fwd != 0, key));
    }
  }
}

// journeys rewritten by the host between interval-extension phases
__global__ void k_set_journeys(dev::state st, uint32_t s, dev::journey_rec const* js, uint32_t n) {
  auto* els = st.journeys + static_cast<size_t>(s) * st.max_j;
  auto const words = (st.max_j + 31u) / 32u;
  if (threadIdx.x == 0) {
    for (auto w = 0u; w != words; ++w) st.blocks_used[s * words + w] = 0u;
    for (auto i = 0u; i != n; ++i) {
      els[i] = js[i];
      st.blocks_used[s * words + js[i].block / 32u] |= 1u << (js[i].block % 32u);
    }
    st.slots[s].n_journeys = n;
  }
}

}  // namespace
}  // namespace b2r

b2r_engine::~b2r_engine() {
  for (auto ev : prof_ev) cudaEventDestroy(ev);
  for (auto ev : prof_rc_ev) cudaEventDestroy(ev);
  if (graph != nullptr) cudaGraphExecDestroy(graph);
  if (lb_graph != nullptr) cudaGraphExecDestroy(lb_graph);
  if (stream != nullptr) cudaStreamDestroy(stream);
  if (stream2 != nullptr) cudaStreamDestroy(stream2);
  if (ev0 != nullptr) cudaEventDestroy(ev0);
  if (ev1 != nullptr) cudaEventDestroy(ev1);
  if (ev_base != nullptr) cudaEventDestroy(ev_base);
  if (ev_scan_a != nullptr) cudaEventDestroy(ev_scan_a);
  if (ev_scan_b != nullptr) cudaEventDestroy(ev_scan_b);
  if (ev2a != nullptr) cudaEventDestroy(ev2a);
  if (ev2b != nullptr) cudaEventDestroy(ev2b);
  if (ev_hdr != nullptr) cudaEventDestroy(ev_hdr);
  if (h_summary != nullptr) cudaFreeHost(h_summary);
  if (h_lbcount != nullptr) cudaFreeHost(h_lbcount);
  if (h_adm != nullptr) cudaFreeHost(h_adm);
  if (h_exp != nullptr) cudaFreeHost(h_exp);
  for (auto* p : allocs) cudaFree(p);
  if (st.RT_R != nullptr) cudaFree(st.RT_R);
  if (st.rtlist != nullptr) cudaFree(st.rtlist);
}

namespace b2r {
namespace {

using dev::slot_t;

// An event record that becomes an event node of the graph when the stream
// is being captured (a plain record inside a capture only orders streams),
// so that its time can be read after every launch of the graph.
cudaError_t record_in_graph(cudaEvent_t ev, cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (auto const rc = cudaStreamIsCapturing(s, &cs); rc != cudaSuccess) return rc;
  return cs == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(ev, s, cudaEventRecordExternal)
                                             : cudaEventRecord(ev, s);
}

// ------------------------------------------------------------- super-step
void enqueue_superstep(b2r_engine& e, cudaStream_t s) {
  auto const& st = e.st;
  auto const slot_blocks = (e.S + 127) / 128;
  auto const list_blocks = e.sms * 8;
  dev::k_ctl_begin<<<list_blocks, 256, 0, s>>>(st);
  // a warp per 32-location chunk of the sweep: one pass over the locations
  auto const sweep_chunks = (st.tt.n_loc + 31U) / 32U;
  dev::k_sweep<<<std::min<uint32_t>(e.sms * 16U, std::max<uint32_t>(1U, (sweep_chunks + 7U) / 8U)), 256, 0, s>>>(st);
  dev::k_ctl_dest<<<slot_blocks, 128, 0, s>>>(st);
  auto const pair_blocks = e.sms * e.shape.pair_blocks_per_sm;
  dev::k_mark_routes<<<pair_blocks, 256, 0, s>>>(st);
  dev::k_list_routes<<<e.sms * 8, 256, 0, s>>>(st);
  if (st.tt.n_rt != 0U) {  // a real-time overlay is bound: its runs are marked too
    dev::k_mark_rt<<<list_blocks, 256, 0, s>>>(st);
    dev::k_list_rt<<<e.sms * 8, 256, 0, s>>>(st);
  }
  dev::k_ctl_marked<<<slot_blocks, 128, 0, s>>>(st);
  cudaEvent_t ev_a = nullptr, ev_b = nullptr;
  if (e.cfg.profile == 2U) {  // timing build: one event pair, captured in the super-step graph
    B2R_CUDA(record_in_graph(e.ev_scan_a, s));
  } else if (e.cfg.profile) {  // CUDA events on the launching stream around the scan
    while (e.prof_used + 2 > e.prof_ev.size()) {
      cudaEvent_t x;
      B2R_CUDA(cudaEventCreate(&x));
      e.prof_ev.push_back(x);
    }
    ev_a = e.prof_ev[e.prof_used++];
    ev_b = e.prof_ev[e.prof_used++];
    B2R_CUDA(cudaEventRecord(ev_a, s));
  }
  dev::k_route_scan_seq<<<list_blocks, 256, 0, s>>>(st);
  {
    auto const grid = e.sms * e.shape.scan_blocks_per_sm, block = e.shape.scan_threads;
    if (e.cfg.profile == 1U) {
      dev::k_route_scan<4, true><<<grid, block, 0, s>>>(st);
    } else if (e.shape.scan_occupancy == 2U) {
      dev::k_route_scan<6, false><<<grid, block, 0, s>>>(st);
    } else if (e.shape.scan_occupancy == 1U) {
      dev::k_route_scan<5, false><<<grid, block, 0, s>>>(st);
    } else {
      dev::k_route_scan<4, false><<<grid, block, 0, s>>>(st);
    }
  }
  if (e.cfg.profile == 2U) {
    B2R_CUDA(record_in_graph(e.ev_scan_b, s));
  } else if (e.cfg.profile) {
    B2R_CUDA(cudaEventRecord(ev_b, s));
    auto const idx = static_cast<uint32_t>(e.prof_used / 2 - 1);
    if (idx < b2r_engine::kProfRows) k_prof_row<<<1, 1, 0, s>>>(st, e.d_prof_rows, idx);
  }
  if (st.tt.n_rt != 0U) dev::k_rt_scan<<<pair_blocks, 256, 0, s>>>(st);
  dev::k_list_reached<<<e.sms * 8, 256, 0, s>>>(st);
  dev::k_clear_x<<<list_blocks, 256, 0, s>>>(st);
  dev::k_transfers_pre<<<slot_blocks, 128, 0, s>>>(st);
  dev::k_transfers<<<pair_blocks, 256, 0, s>>>(st);
  dev::k_intermodal_fp_pre<<<slot_blocks, 128, 0, s>>>(st);
  dev::k_footpaths<<<pair_blocks, 256, 0, s>>>(st);
  dev::k_end_collect<<<slot_blocks, 128, 0, s>>>(st);
  cudaEvent_t rc_a = nullptr, rc_b = nullptr;
  if (e.cfg.profile == 1U) {
    while (e.prof_rc_used + 2 > e.prof_rc_ev.size()) {
      cudaEvent_t x;
      B2R_CUDA(cudaEventCreate(&x));
      e.prof_rc_ev.push_back(x);
    }
    rc_a = e.prof_rc_ev[e.prof_rc_used++];
    rc_b = e.prof_rc_ev[e.prof_rc_used++];
    B2R_CUDA(cudaEventRecord(rc_a, s));
  }
  dev::k_reconstruct<<<e.sms * e.shape.recon_blocks_per_sm, 128, 0, s>>>(st);
  if (e.cfg.profile == 1U) B2R_CUDA(cudaEventRecord(rc_b, s));
  dev::k_next_summary<<<slot_blocks, 128, 0, s>>>(st);
  dev::k_list_marked<<<e.sms * 8, 256, 0, s>>>(st);
}
uint64_t launches_per_step(b2r_engine const& e) { return e.st.tt.n_rt != 0U ? 21U : 18U; }

// --------------------------------------------------------- admission
size_t admission_bytes(b2r_engine const& e, prepped_query const& p) {
  return sizeof(slot_t) + p.starts.size() * sizeof(dev::start_rec) +
         (p.dest_dist.size() + p.dest_locs.size()) * sizeof(dev::dest_rec) +
         (p.start_offsets.size() + p.dest_offsets.size()) * sizeof(b2r_offset) +
         (p.lb.empty() ? 0 : e.tt->d.n_loc * sizeof(uint16_t)) + 64;
}

int check_capacity(b2r_engine const& e, prepped_query const& p) {
  if (p.starts.size() > e.max_starts) return B2R_ERR_CAPACITY;
  if (p.dest_dist.size() + p.dest_locs.size() > e.max_dest) return B2R_ERR_CAPACITY;
  if (p.start_offsets.size() + p.dest_offsets.size() > e.max_off) return B2R_ERR_CAPACITY;
  return B2R_OK;
}

// new_gen: a new query generation (raptor::reset_arrivals); otherwise the
// round times of the slot's previous phase stay in effect
slot_t make_slot(b2r_engine& e, uint32_t s, prepped_query const& p, bool& clear_rt, bool new_gen = true) {
  slot_t sl{};
  sl.state = dev::S_START;
  sl.fwd = p.fwd ? 1 : 0;
  sl.one_to_all = p.one_to_all ? 1 : 0;
  sl.end_k = p.end_k;
  sl.intermodal_dest = p.intermodal_dest ? 1 : 0;
  sl.ontrip = p.ontrip ? 1 : 0;
  sl.start_mode = p.start_mode;
  sl.dest_mode = p.dest_mode;
  sl.base = p.base;
  clear_rt = false;
  if (new_gen) {
    if (e.gen_query[s] >= 0xFFFEu) {
      e.gen_query[s] = 0;
      clear_rt = true;
    }
    ++e.gen_query[s];
  }
  sl.gen_query = e.gen_query[s];
  sl.base_days = p.base_days;
  sl.iv_from = p.iv_from;
  sl.iv_to = p.iv_to;
  sl.fastest_direct = p.fastest_direct;
  sl.max_travel_time = p.max_travel_time;
  sl.min_connection_count = p.min_connection_count;
  sl.extend_earlier = p.extend_earlier ? 1 : 0;
  sl.extend_later = p.extend_later ? 1 : 0;
  sl.need_sweep = p.need_sweep ? 1 : 0;
  sl.early_term = 0;
  sl.tts = {p.tts.is_default, p.tts.min_transfer_time, p.tts.additional_time, p.tts.factor};
  sl.allowed_claszes = p.allowed_claszes;
  sl.req_flags = p.req_flags;
  sl.blast = p.blast;
  sl.recon_mode = p.recon_mode;
  // one start-time group and nothing after it: the journeys can wait until
  // the slot is done and be rebuilt while the next super-steps run
  sl.recon_defer = (p.ontrip && !p.one_to_all && p.recon_mode == 0) ? 1 : 0;
  sl.recon_transfers = p.recon_transfers;
  sl.no_lb = p.no_lb ? 1 : 0;
  sl.prf = p.prf;
  sl.recon_start = p.recon_start;
  sl.span = p.span;
  sl.n_starts = static_cast<uint32_t>(p.starts.size());
  sl.n_dest = static_cast<uint32_t>(p.intermodal_dest ? p.dest_dist.size() : p.dest_locs.size());
  sl.n_soff = static_cast<uint32_t>(p.start_offsets.size());
  sl.n_doff = static_cast<uint32_t>(p.dest_offsets.size());
  sl.k = 0;
  sl.next_start = 0;
  sl.n_journeys = 0;
  for (auto& x : sl.tad) x = dev::kKeyInv;
  return sl;
}

// Packs the admissions into pinned memory, copies them in one transfer and
// distributes them with one kernel.
void enqueue_lb_chunk(b2r_engine& e, cudaStream_t s) {
  for (auto it = 0; it != 4; ++it) {
    for (uint32_t p = 0; p != 2; ++p) {
      dev::k_lb_relax<<<e.sms * 8, 256, 0, s>>>(e.st, p);
      dev::k_lb_clear<<<e.sms * 4, 256, 0, s>>>(e.st, p);
      dev::k_lb_reset<<<1, 32, 0, s>>>(e.st, p);
    }
  }
}

// Runs the device Dijkstra of every query admitted in this wave to
// completion, then writes their lower-bound columns.
void solve_lower_bounds(b2r_engine& e, cudaStream_t s) {
  auto const t0 = std::chrono::steady_clock::now();
  uint32_t pending = 1;
  uint64_t chunks = 0;
  while (pending != 0) {
    e.aux_launches += 24;  // 4 x 2 iterations of 3 kernels
    if (e.lb_graph != nullptr) {
      B2R_CUDA(cudaGraphLaunch(e.lb_graph, s));
    } else {
      enqueue_lb_chunk(e, s);
    }
    ++chunks;
    e.d2h_bytes += sizeof(uint32_t);
    B2R_CUDA(cudaMemcpyAsync(e.h_lbcount, e.st.counters + dev::C_F0, sizeof(uint32_t),
                             cudaMemcpyDeviceToHost, s));
    B2R_CUDA(cudaStreamSynchronize(s));
    pending = *e.h_lbcount;
    if (chunks > 100000) throw std::runtime_error("lower-bound solver did not converge");
  }
  e.lb_chunks += chunks;
  e.aux_launches += e.tt->d.n_with_children != 0 ? 2 : 1;
  if (e.tt->d.n_with_children != 0) {
    dev::k_lb_children<<<(e.S + 127) / 128, 128, 0, s>>>(e.st);
  }
  dev::k_lb_finish<<<e.sms * 16, 256, 0, s>>>(e.st);
  B2R_CUDA(cudaMemsetAsync(e.st.lb_mask, 0, e.G * sizeof(uint32_t), s));
  B2R_CUDA(cudaGetLastError());
  B2R_CUDA(cudaStreamSynchronize(s));
  e.lb_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// The all-pairs lower-bound tables of a timetable: row s holds the
// Dijkstra distances from location s over the forward- / backward-search
// lower-bound graph.  Built on the host threads in row blocks and uploaded
// block by block; kept with the timetable for every later engine.
// Both tables and the stride are published together once both are built:
// an exception half way leaves the timetable without tables (lb_stride 0),
// never with one of them.
void ensure_lb_table(b2r_timetable& t, unsigned threads) {
  std::lock_guard<std::mutex> lock{t.lb_table_mutex};
  if (t.lb_stride != 0U) return;
  auto const n = static_cast<size_t>(t.d.n_loc);
  auto const stride = (n + 7U) / 8U * 8U;  // rows 16-byte aligned for vector loads, padding unreachable
  constexpr size_t kBlock = 1024;
  std::vector<uint16_t> buf(kBlock * stride, uint16_t{0xFFFFu});
  uint16_t* built[2] = {nullptr, nullptr};
  struct guard {  // frees what was built unless published
    uint16_t** p;
    ~guard() {
      for (auto i = 0; i != 2; ++i)
        if (p[i] != nullptr) cudaFree(p[i]);
    }
  } g{built};
  uint64_t bytes = 0;
  for (auto dir = 0; dir != 2; ++dir) {
    auto* dst = dmalloc<uint16_t>(n * stride, bytes);
    built[dir] = dst;
    for (size_t b = 0; b < n; b += kBlock) {
      auto const rows = std::min(kBlock, n - b);
      std::atomic<size_t> next{0};
      auto work = [&]() {
        for (auto r = next++; r < rows; r = next++) {
          lb_table_row(t.view, dir == 0, static_cast<uint32_t>(b + r), buf.data() + r * stride);
        }
      };
      std::vector<std::thread> pool;
      for (auto i = 1U; i < threads; ++i) pool.emplace_back(work);
      work();
      for (auto& th : pool) th.join();
      B2R_CUDA(cudaMemcpy(dst + b * stride, buf.data(), rows * stride * sizeof(uint16_t), cudaMemcpyHostToDevice));
    }
  }
  for (auto dir = 0; dir != 2; ++dir) {
    t.lb_table[dir] = built[dir];
    t.allocs.push_back(built[dir]);
    built[dir] = nullptr;
  }
  t.bytes += bytes;
  t.lb_stride = static_cast<uint32_t>(stride);
}

// one admission: a query (or the next phase of one) into slot `slot`
struct adm_req {
  uint32_t slot;
  prepped_query const* p;
  uint32_t flags{0};                                // kAdm*
  std::vector<dev::journey_rec> const* keep{nullptr};  // journeys the slot starts with
};

void admit(b2r_engine& e, std::vector<adm_req> const& adm, cudaStream_t s) {
  if (adm.empty()) return;
  bool any_device_lb = false;
  size_t need = adm.size() * (sizeof(adm_hdr) + sizeof(fill_item) + sizeof(lb_group) + sizeof(lb_entry)) + 256 + 64;
  for (auto const& r : adm) {
    need += admission_bytes(e, *r.p) + 64 + (r.keep ? r.keep->size() * sizeof(dev::journey_rec) + 16 : 0);
  }
  if (need > e.adm_cap) {
    B2R_CUDA(cudaStreamSynchronize(s));
    if (e.h_adm != nullptr) cudaFreeHost(e.h_adm);
    if (e.d_adm != nullptr) cudaFree(e.d_adm);
    e.adm_cap = need * 2;
    B2R_CUDA(cudaMallocHost(&e.h_adm, e.adm_cap));
    B2R_CUDA(cudaMalloc(&e.d_adm, e.adm_cap));
  } else {
    B2R_CUDA(cudaStreamSynchronize(s));  // staging buffer reuse
  }
  auto* hdr = reinterpret_cast<adm_hdr*>(e.h_adm);
  size_t off = (adm.size() * sizeof(adm_hdr) + 255) & ~size_t{255};
  auto const put = [&](void const* src, size_t n) {
    off = (off + 15) & ~size_t{15};
    auto const at = off;
    if (n != 0) std::memcpy(e.h_adm + off, src, n);
    off += n;
    return at;
  };
  for (auto i = 0U; i != adm.size(); ++i) {
    auto const s_idx = adm[i].slot;
    auto const& p = *adm[i].p;
    auto& h = hdr[i];
    h = {};
    h.slot = s_idx;
    h.flags = adm[i].flags;
    bool clear_rt = false;
    auto sl = make_slot(e, s_idx, p, clear_rt, (adm[i].flags & kAdmKeepRt) == 0u);
    h.clear_rt = clear_rt ? 1 : 0;
    if (adm[i].keep != nullptr) {
      if (adm[i].keep->size() > e.max_j) throw std::runtime_error("journey capacity exceeded");
      h.n_keep = static_cast<uint32_t>(adm[i].keep->size());
      sl.n_journeys = h.n_keep;
      h.off_keep = put(adm[i].keep->data(), adm[i].keep->size() * sizeof(dev::journey_rec));
    }
    h.off_slot = put(&sl, sizeof(sl));
    std::vector<dev::start_rec> starts(p.starts.size());
    for (auto j = 0U; j != p.starts.size(); ++j) {
      starts[j] = {p.starts[j].time_at_start, p.starts[j].time_at_stop, p.starts[j].stop};
    }
    h.n_starts = static_cast<uint32_t>(starts.size());
    h.off_starts = put(starts.data(), starts.size() * sizeof(dev::start_rec));
    std::vector<dev::dest_rec> dests;
    if (p.intermodal_dest) {
      for (auto const& [l, d] : p.dest_dist) dests.push_back({l, d});
    } else {
      for (auto l : p.dest_locs) dests.push_back({l, 0});
    }
    h.n_dest = static_cast<uint32_t>(dests.size());
    h.off_dest = put(dests.data(), dests.size() * sizeof(dev::dest_rec));
    std::vector<b2r_offset> offs = p.start_offsets;
    offs.insert(offs.end(), p.dest_offsets.begin(), p.dest_offsets.end());
    h.n_off = static_cast<uint32_t>(offs.size());
    h.off_off = put(offs.data(), offs.size() * sizeof(b2r_offset));
    h.lb_mode = p.keep_lb          ? 4
                : !p.lb.empty()      ? 1
                : p.one_to_all       ? 0
                : e.lb_mode() == 2 ? 2
                : e.lb_mode() == 3 ? 3
                                              : 0;
    h.off_lb = put(p.lb.data(), p.lb.size() * sizeof(uint16_t));
    std::vector<uint32_t> seeds;
    for (auto const& [l, d] : p.lb_seeds) {
      seeds.push_back(l);
      seeds.push_back(d);
    }
    h.n_seeds = static_cast<uint32_t>(p.lb_seeds.size());
    h.off_seeds = put(seeds.data(), seeds.size() * sizeof(uint32_t));
    any_device_lb = any_device_lb || h.lb_mode == 2;
  }
  std::vector<fill_item> fills;
  for (auto const& r : adm) {
    if ((r.flags & kAdmFillRows) != 0u) fills.push_back({r.slot, r.flags & kAdmFillRows});
  }
  auto const off_fills = put(fills.data(), fills.size() * sizeof(fill_item));
  // lower-bound mode 3 admissions by slot group
  std::vector<lb_entry> lb_entries;
  std::vector<lb_group> lb_groups;
  {
    std::vector<std::pair<uint32_t, uint32_t>> by_slot;  // (slot, admission)
    for (auto i = 0U; i != adm.size(); ++i) {
      if (hdr[i].lb_mode == 3) by_slot.emplace_back(adm[i].slot, i);
    }
    std::sort(by_slot.begin(), by_slot.end());
    for (auto const& [slot, i] : by_slot) {
      auto const g = slot / 32U;
      if (lb_groups.empty() || lb_groups.back().g != g) {
        lb_groups.push_back({g, static_cast<uint32_t>(lb_entries.size()), 0U, 0U});
      }
      ++lb_groups.back().count;
      lb_entries.push_back({slot % 32U, hdr[i].n_seeds, adm[i].p->fwd ? 1U : 0U, 0U, hdr[i].off_seeds});
    }
  }
  auto const off_lb_groups = put(lb_groups.data(), lb_groups.size() * sizeof(lb_group));
  auto const off_lb_entries = put(lb_entries.data(), lb_entries.size() * sizeof(lb_entry));
  e.h2d_bytes += off;
  B2R_CUDA(cudaMemcpyAsync(e.d_adm, e.h_adm, off, cudaMemcpyHostToDevice, s));
  if (!fills.empty()) {
    auto const bx = std::min<uint32_t>((e.tt->d.n_loc + 255u) / 256u, static_cast<uint32_t>(e.sms) * 2u);
    ++e.aux_launches;
    k_fill_bounds<<<dim3(bx, static_cast<unsigned>(fills.size())), 256, 0, s>>>(
        e.st, reinterpret_cast<fill_item const*>(e.d_adm + off_fills));
    B2R_CUDA(cudaGetLastError());
  }
  if (!lb_groups.empty()) {
    ++e.aux_launches;
    k_lb_fill<<<dim3((e.tt->d.n_loc + kLbTile - 1) / kLbTile, static_cast<unsigned>(lb_groups.size())), 256, 0,
                s>>>(e.st, reinterpret_cast<lb_group const*>(e.d_adm + off_lb_groups),
                     reinterpret_cast<lb_entry const*>(e.d_adm + off_lb_entries), e.d_adm);
    B2R_CUDA(cudaGetLastError());
  }
  ++e.aux_launches;
  k_admit<<<static_cast<unsigned>(adm.size()), 256, 0, s>>>(
      e.st, reinterpret_cast<adm_hdr const*>(e.d_adm), e.d_adm, static_cast<uint32_t>(adm.size()),
      e.max_starts, e.max_dest, e.max_off);
  B2R_CUDA(cudaGetLastError());
  if (any_device_lb) solve_lower_bounds(e, s);
}

void retire(b2r_engine& e, std::vector<uint32_t> const& slots, cudaStream_t s) {
  if (slots.empty()) return;
  uint32_t* d = nullptr;
  // reuse the export list buffer (sized for all slots)
  d = e.d_exp_list;
  e.h2d_bytes += slots.size() * sizeof(uint32_t);
  B2R_CUDA(cudaMemcpyAsync(d, slots.data(), slots.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  ++e.aux_launches;
  k_retire<<<static_cast<unsigned>(slots.size()), 128, 0, s>>>(e.st, d, static_cast<uint32_t>(slots.size()));
  B2R_CUDA(cudaGetLastError());
}

// a page-locked row buffer back into the pool (at most 512 buffers and
// 4 GiB; beyond that it is freed)
void give_rows(b2r_engine& e, row_buf&& r) {
  if (!r.pinned()) return;
  std::lock_guard<std::mutex> lock{e.row_mu};
  auto const bytes = r.capacity() * sizeof(int16_t);
  if (e.row_pool.size() >= 512 || e.row_pool_bytes + bytes > (size_t{4} << 30)) return;
  e.row_pool_bytes += bytes;
  e.row_pool.push_back(std::move(r));
}

// results of the previous call are no longer the caller's: their
// page-locked row buffers go back to the pool
void recycle_rows(b2r_engine& e) {
  for (auto& r : e.results) give_rows(e, std::move(r.rt_rows));
  e.results.clear();
}

// rows of a result: where export_slots puts them
enum class row_target {
  staging,  // ordinary memory, through the page-locked staging buffer
  pinned,   // a page-locked buffer: pooled, else newly allocated
};

// a page-locked row buffer of n values: the smallest pooled one that holds
// them, else a new one
row_buf take_rows(b2r_engine& e, size_t n) {
  row_buf v;
  {
    std::lock_guard<std::mutex> lock{e.row_mu};
    auto best = e.row_pool.end();
    for (auto it = e.row_pool.begin(); it != e.row_pool.end(); ++it) {
      if (it->capacity() >= n && (best == e.row_pool.end() || it->capacity() < best->capacity())) best = it;
    }
    if (best != e.row_pool.end()) {
      e.row_pool_bytes -= best->capacity() * sizeof(int16_t);
      v = std::move(*best);
      e.row_pool.erase(best);
    }
  }
  v.resize(n, true);
  return v;
}

// page-locked row buffers for up to `count` one-to-all results, allocated
// ahead (the serving loop takes from the pool and never allocates any)
void prewarm_rows(b2r_engine& e, uint32_t count, size_t max_bytes) {
  auto const n = static_cast<size_t>(dev::kK) * e.tt->d.n_loc;
  size_t have = 0;
  {
    std::lock_guard<std::mutex> lock{e.row_mu};
    for (auto const& r : e.row_pool) have += r.capacity() >= n ? 1U : 0U;
  }
  for (auto i = have; i < count && (i + 1) * n * sizeof(int16_t) <= max_bytes; ++i) {
    row_buf r;
    r.resize(n, true);
    give_rows(e, std::move(r));
  }
}

struct exported {
  slot_t sl;
  std::vector<dev::journey_rec> js;
  std::vector<b2r_leg> legs;  // kLegsAll: n_j * kMaxLegs; kLegsMatch: kMaxLegs of journey legs_of
  uint32_t legs_of{UINT32_MAX};
  row_buf rows;
};

void export_slots(b2r_engine& e, std::vector<uint32_t> const& slots,
                  std::vector<uint32_t> const& n_js, std::vector<uint32_t> const& n_rows,
                  std::vector<exported>& out, cudaStream_t s,
                  std::vector<uint8_t> const* legs_modes = nullptr, row_target rows_to = row_target::staging) {
  out.clear();
  out.resize(slots.size());
  if (slots.empty()) return;
  std::vector<exp_item> items(slots.size());
  // the journeys of slots whose reconstruction waits for the slot to finish
  // (k_reconstruct_done skips the others), uploaded after the items
  // (a deferred slot runs one start-time group of a one-to-one search, whose
  // legs are exported in full)
  std::vector<uint32_t> recon;
  for (auto i = 0U; i != slots.size(); ++i) {
    if (legs_modes != nullptr && (*legs_modes)[i] != kLegsAll) continue;
    for (auto ji = 0U; ji != n_js[i]; ++ji) recon.push_back((slots[i] << 16) | ji);
  }
  auto const recon_off = (slots.size() * sizeof(exp_item) + 15) & ~size_t{15};
  auto const header = recon_off + recon.size() * sizeof(uint32_t);
  size_t off = (header + 255) & ~size_t{255};
  for (auto i = 0U; i != slots.size(); ++i) {
    auto& it = items[i];
    it.slot = slots[i];
    it.n_j = n_js[i];
    it.n_rows = n_rows[i];
    it.legs_mode = legs_modes != nullptr ? (*legs_modes)[i] : kLegsAll;
    off = (off + 15) & ~size_t{15};
    it.off_slot = off;
    off += sizeof(slot_t);
    off = (off + 15) & ~size_t{15};
    it.off_j = off;
    off += it.n_j * sizeof(dev::journey_rec);
    off = (off + 15) & ~size_t{15};
    it.off_legs = off;
    off += it.legs_mode == kLegsAll     ? static_cast<size_t>(it.n_j) * dev::kMaxLegs * sizeof(b2r_leg)
           : it.legs_mode == kLegsMatch ? 16 + dev::kMaxLegs * sizeof(b2r_leg)
                                        : 0;
  }
  // the one-to-all rows after everything else: with page-locked result
  // buffers they go from here straight into them
  auto const rows_begin = (off + 255) & ~size_t{255};
  off = rows_begin;
  for (auto& it : items) {
    off = (off + 15) & ~size_t{15};
    it.off_rows = off;
    off += static_cast<size_t>(it.n_rows) * e.tt->d.n_loc * sizeof(int16_t);
  }
  if (off > e.exp_cap) {
    B2R_CUDA(cudaStreamSynchronize(s));
    if (e.h_exp != nullptr) cudaFreeHost(e.h_exp);
    if (e.d_exp != nullptr) cudaFree(e.d_exp);
    e.exp_cap = off * 2;
    B2R_CUDA(cudaMallocHost(&e.h_exp, e.exp_cap));
    B2R_CUDA(cudaMalloc(&e.d_exp, e.exp_cap));
  }
  std::memcpy(e.h_exp, items.data(), items.size() * sizeof(exp_item));
  if (!recon.empty()) std::memcpy(e.h_exp + recon_off, recon.data(), recon.size() * sizeof(uint32_t));
  e.h2d_bytes += header;
  B2R_CUDA(cudaMemcpyAsync(e.d_exp, e.h_exp, header, cudaMemcpyHostToDevice, s));
  if (e.base_recorded) B2R_CUDA(cudaEventRecord(e.ev2a, s));
  if (!recon.empty()) {
    ++e.aux_launches;
    dev::k_reconstruct_done<<<static_cast<unsigned>(std::min<size_t>(
                                  (recon.size() + 3) / 4, static_cast<size_t>(e.sms) * e.shape.recon_blocks_per_sm)),
                              128, 0, s>>>(e.st, reinterpret_cast<uint32_t const*>(e.d_exp + recon_off),
                                           static_cast<uint32_t>(recon.size()));
    B2R_CUDA(cudaGetLastError());
  }
  uint32_t row_blocks = 1;  // spread one-to-all rows over the SMs
  for (auto const r : n_rows) {
    if (r != 0) row_blocks = std::max<uint32_t>(row_blocks, static_cast<uint32_t>(e.sms) * 4u /
                                                                static_cast<uint32_t>(slots.size()) + 1u);
  }
  ++e.aux_launches;
  k_export<<<dim3(static_cast<unsigned>(slots.size()), row_blocks), 256, 0, s>>>(
      e.st, reinterpret_cast<exp_item const*>(e.d_exp), static_cast<uint32_t>(slots.size()), e.d_exp);
  B2R_CUDA(cudaGetLastError());
  if (e.base_recorded) B2R_CUDA(cudaEventRecord(e.ev2b, s));
  e.d2h_bytes += off;
  // headers, journeys and legs; the rows either into the page-locked
  // result buffers (left in flight: later work on this stream, and the end
  // of the batch, wait for them) or through the staging buffer
  B2R_CUDA(cudaMemcpyAsync(e.h_exp, e.d_exp, rows_begin, cudaMemcpyDeviceToHost, s));
  // rows for ordinary memory go through the staging buffer and are on the
  // host with the headers; rows for page-locked buffers go straight there
  // and are left in flight (later work on this stream, and the end of the
  // batch, wait for them)
  std::vector<uint8_t> direct(slots.size(), 0);
  for (auto i = 0U; i != slots.size(); ++i) {
    auto const& it = items[i];
    if (it.n_rows == 0) continue;
    auto const n = static_cast<size_t>(it.n_rows) * e.tt->d.n_loc;
    if (rows_to == row_target::staging) {
      out[i].rows.resize(n, false);
    } else {
      out[i].rows = take_rows(e, n);
    }
    direct[i] = out[i].rows.pinned() ? 1 : 0;
    if (!direct[i]) {
      B2R_CUDA(cudaMemcpyAsync(e.h_exp + it.off_rows, e.d_exp + it.off_rows, n * sizeof(int16_t),
                               cudaMemcpyDeviceToHost, s));
    }
  }
  B2R_CUDA(cudaEventRecord(e.ev_hdr, s));
  for (auto i = 0U; i != slots.size(); ++i) {
    if (!direct[i]) continue;
    B2R_CUDA(cudaMemcpyAsync(out[i].rows.data(), e.d_exp + items[i].off_rows, out[i].rows.size() * sizeof(int16_t),
                             cudaMemcpyDeviceToHost, s));
  }
  B2R_CUDA(cudaEventSynchronize(e.ev_hdr));
  if (e.base_recorded) {
    float a = 0, b = 0;
    B2R_CUDA(cudaEventElapsedTime(&a, e.ev_base, e.ev2a));
    B2R_CUDA(cudaEventElapsedTime(&b, e.ev_base, e.ev2b));
    e.busy.emplace_back(a, b);
  }
  for (auto i = 0U; i != slots.size(); ++i) {
    auto const& it = items[i];
    auto& o = out[i];
    std::memcpy(&o.sl, e.h_exp + it.off_slot, sizeof(slot_t));
    o.js.resize(it.n_j);
    std::memcpy(o.js.data(), e.h_exp + it.off_j, it.n_j * sizeof(dev::journey_rec));
    if (it.legs_mode == kLegsAll) {
      o.legs.resize(static_cast<size_t>(it.n_j) * dev::kMaxLegs);
      std::memcpy(o.legs.data(), e.h_exp + it.off_legs, o.legs.size() * sizeof(b2r_leg));
    } else if (it.legs_mode == kLegsMatch) {
      std::memcpy(&o.legs_of, e.h_exp + it.off_legs, sizeof(uint32_t));
      if (o.legs_of < it.n_j) {
        auto const n = o.js[o.legs_of].n_legs;
        o.legs.resize(n);
        std::memcpy(o.legs.data(), e.h_exp + it.off_legs + 16, n * sizeof(b2r_leg));
      }
    }
    if (it.n_rows != 0 && !direct[i]) {
      std::memcpy(o.rows.data(), e.h_exp + it.off_rows, o.rows.size() * sizeof(int16_t));
    }
  }
}

// ----------------------------------------------------- host finalisation
// Per query, what search::execute does between and after the Algo calls
// (search.h:237-336): interval extension and the final filtering.
// pong_search's sweep (pong.cc:236-361) between device phases
struct pong_run {
  int32_t start_time{0};
  std::vector<dev::journey_rec> results;  // the shared result set, pong frame
  // legs of the rebuilt results by their device leg block: a block keeps its
  // journey while that journey stays in the result set, and a journey is
  // rebuilt (and its legs exported) in the pong phase that matches it
  std::unordered_map<uint32_t, std::vector<b2r_leg>> legs_of_block;
  std::vector<dev::journey_rec> ping;     // this iteration's ping results
  size_t next{0};                         // ping result of the next pong
  bool in_ping{true};
  uint64_t n_rounds{0}, n_phases{0};
};

struct query_run {
  std::atomic<bool> ready{false};  // host preparation finished
  prepped_query p;
  int status{B2R_OK};
  bool finished{false};
  bool rearm{false};
  bool reset_arrivals{false};
  std::vector<dev::journey_rec> keep;  // journeys kept across a re-arm
  b2r_engine::result_store res;
  // pong: sweep state and the staged next phase of the query's slot
  std::unique_ptr<pong_run> pong;
  prepped_query phase;
  uint32_t adm_flags{0};
  std::vector<dev::journey_rec> upload;
  bool readmit{false};
};

void finish_result(b2r_engine& e, query_run& q, exported& x) {
  auto& p = q.p;
  auto& res = q.res;
  res.journeys.clear();
  res.legs.clear();
  res.rt_rows.clear();
  if (p.one_to_all) {
    res.rt_rows = std::move(x.rows);  // one-to-all rows can be large
    res.view.n_rows = p.end_k;
    res.view.base_day = p.base_days;
  } else {
    std::vector<size_t> order;
    for (auto i = 0U; i != x.js.size(); ++i) {
      auto const& j = x.js[i];
      auto const tt = std::abs(j.dest_time - j.start_time);
      if (!p.ontrip) {
        if (!(x.sl.iv_from <= j.start_time && j.start_time < x.sl.iv_to) || tt >= p.fastest_direct ||
            tt > p.max_travel_time) {
          continue;
        }
      }
      order.push_back(i);
    }
    if (!p.ontrip) {
      std::sort(order.begin(), order.end(), [&](size_t a, size_t b) {
        return std::tie(x.js[a].start_time, x.js[a].transfers) <
               std::tie(x.js[b].start_time, x.js[b].transfers);
      });
    }
    for (auto i : order) {
      auto const& j = x.js[i];
      if (!j.reconstructed) continue;
      b2r_journey bj{};
      bj.start_time = j.start_time;
      bj.dest_time = j.dest_time;
      bj.dest = j.dest;
      bj.transfers = j.transfers;
      bj.error = j.error;
      bj.n_legs = j.n_legs;
      bj.first_leg = static_cast<uint32_t>(res.legs.size());
      for (auto l = 0; l != j.n_legs; ++l) res.legs.push_back(x.legs[i * dev::kMaxLegs + l]);
      res.journeys.push_back(bj);
    }
  }
  res.view.status = q.status;
  res.view.interval_from = x.sl.iv_from;
  res.view.interval_to = x.sl.iv_to;
  res.view.n_rounds = x.sl.n_rounds;
  res.view.n_start_times = x.sl.n_groups_run;
  q.finished = true;
}

// decides between finishing and another interval-extension phase
void on_phase_done(b2r_engine& e, query_run& q, exported& x) {
  auto& p = q.p;
  if (x.sl.state == dev::S_ERROR) {
    q.status = x.sl.error != 0 ? x.sl.error : B2R_ERR_INTERNAL;
    finish_result(e, q, x);
    return;
  }
  auto const n_in = [&](int32_t f, int32_t t) {
    uint32_t c = 0;
    for (auto const& j : x.js) c += (!p.ontrip ? (f <= j.start_time && j.start_time < t) : true) ? 1u : 0u;
    return c;
  };
  if (p.one_to_all || x.js.empty() || p.ontrip || n_in(x.sl.iv_from, x.sl.iv_to) >= p.min_connection_count) {
    finish_result(e, q, x);
    return;
  }
  auto nf = x.sl.iv_from, nt = x.sl.iv_to;
  auto const& d = e.tt->host;
  if (!extend_interval(p, d.date_range_from * 1440, d.date_range_to * 1440,
                       p.min_connection_count - n_in(x.sl.iv_from, x.sl.iv_to), nf, nt)) {
    finish_result(e, q, x);
    return;
  }
  // search.h:283-316
  std::vector<start_label> starts;
  auto keep = x.js;
  q.reset_arrivals = false;
  auto const remove_outside = [&]() {
    std::vector<dev::journey_rec> k2;
    for (auto const& j : keep) {
      if (x.sl.iv_from <= j.start_time && j.start_time < x.sl.iv_to) k2.push_back(j);
    }
    keep = std::move(k2);
  };
  if (nf != x.sl.iv_from) {
    add_interval_starts(e.view, p, nf, x.sl.iv_from, !p.fwd, starts);
    if (!p.fwd) {
      q.reset_arrivals = true;
      remove_outside();
    }
  }
  if (nt != x.sl.iv_to) {
    add_interval_starts(e.view, p, x.sl.iv_to, nt, p.fwd, starts);
    if (p.fwd) {
      q.reset_arrivals = true;
      remove_outside();
    }
  }
  p.starts = std::move(starts);
  p.iv_from = nf;
  p.iv_to = nt;
  q.keep = std::move(keep);
  q.rearm = true;
}

// ------------------------------------------------------------------ pong
// pong.cc:363-472 after the sweep: unfinished, unvalidated, out-of-interval
// and too slow journeys dropped, start and destination time swapped back,
// the special stations of the first and last leg swapped, sorted by
// departure and transfers, and (forward) inner rides replaced by earlier
// direct alternatives.
void finish_pong(b2r_engine& e, query_run& q) {
  auto const& plan = *q.p.pong;
  auto& r = *q.pong;
  auto const fwd = plan.fwd;
  auto const better = [&](int32_t a, int32_t b) { return fwd ? a < b : a > b; };
  struct item {
    dev::journey_rec j;
    std::vector<b2r_leg> legs;
  };
  std::vector<item> out;
  for (auto i = 0U; i != r.results.size(); ++i) {
    auto const& j = r.results[i];
    auto const tt = std::abs(j.dest_time - j.start_time);
    auto const out_of_iv = fwd ? !plan.extend_later && j.dest_time >= plan.iv_to
                               : !plan.extend_earlier && j.dest_time < plan.iv_from;
    if (!j.reconstructed || !better(j.dest_time, r.start_time) || out_of_iv || tt >= plan.fastest_direct ||
        tt > plan.max_travel_time) {
      continue;
    }
    item it{j, {}};
    std::swap(it.j.start_time, it.j.dest_time);
    auto const lf = r.legs_of_block.find(j.block);
    if (lf == r.legs_of_block.end() || lf->second.size() != j.n_legs) {  // rebuilt, but its legs never came
      q.status = B2R_ERR_INTERNAL;
      continue;
    }
    it.legs = lf->second;
    auto const swap = [](uint32_t l) {
      return l == B2R_SPECIAL_START ? B2R_SPECIAL_END : l == B2R_SPECIAL_END ? B2R_SPECIAL_START : l;
    };
    if (!it.legs.empty()) {
      it.legs.front().from = swap(it.legs.front().from);
      it.legs.back().to = swap(it.legs.back().to);
    }
    out.push_back(std::move(it));
  }
  std::sort(out.begin(), out.end(), [](item const& a, item const& b) {
    return std::tie(a.j.start_time, a.j.transfers) < std::tie(b.j.start_time, b.j.transfers);
  });
  if (fwd) {
    auto const& v = e.tt->view;
    auto const& d = v.d;
    auto const loc = [&](b2r_leg const& l, uint32_t s) {
      auto const rr = d.transport_route[l.transport];
      return B2R_STOP_LOC(d.route_stops[d.route_stop_index[rr] + s]);
    };
    for (auto& it : out) {
      auto& l = it.legs;
      for (auto w = size_t{0}; w + 5U <= l.size(); ++w) {
        if (l[w].kind != B2R_LEG_TRANSPORT || l[w + 2].kind != B2R_LEG_TRANSPORT ||
            l[w + 4].kind != B2R_LEG_TRANSPORT) {
          continue;
        }
        std::array<b2r_leg, 3> alt;
        if (earliest_alternative(v, plan.ping.tts, plan.ping.prf, plan.ping.allowed_claszes, plan.ping.req_flags,
                                 loc(l[w], l[w].stop_to - 1U), loc(l[w + 4], l[w + 4].stop_from),
                                 l[w].arr_time, l[w + 4].dep_time, alt)) {
          l[w + 1] = alt[0];
          l[w + 2] = alt[1];
          l[w + 3] = alt[2];
        }
      }
    }
  }
  auto& res = q.res;
  res.journeys.clear();
  res.legs.clear();
  res.rt_rows.clear();
  for (auto const& it : out) {
    b2r_journey bj{};
    bj.start_time = it.j.start_time;
    bj.dest_time = it.j.dest_time;
    bj.dest = it.j.dest;
    bj.transfers = it.j.transfers;
    bj.error = it.j.error;
    bj.n_legs = static_cast<uint16_t>(it.legs.size());
    bj.first_leg = static_cast<uint32_t>(res.legs.size());
    res.legs.insert(res.legs.end(), it.legs.begin(), it.legs.end());
    res.journeys.push_back(bj);
  }
  res.view.status = q.status;
  res.view.interval_from = fwd ? plan.iv_from : r.start_time + 1;
  res.view.interval_to = fwd ? r.start_time : plan.iv_to;
  res.view.n_rounds = r.n_rounds;
  res.view.n_start_times = r.n_phases;
  q.finished = true;
}

// the sweep's loop condition, pong.cc:236-239
bool pong_continues(pong_plan const& plan, pong_run const& r) {
  auto const better = [&](int32_t a, int32_t b) { return plan.fwd ? a < b : a > b; };
  auto const end_time = plan.fwd ? plan.iv_to : plan.iv_from - 1;
  uint32_t n = 0;
  for (auto const& j : r.results) {
    if (!better(j.dest_time, r.start_time)) continue;
    auto const tt = std::abs(j.dest_time - j.start_time);
    n += 1U + ((tt < plan.fastest_direct && tt <= plan.max_travel_time) ? 1U : 0U);
  }
  return (better(r.start_time, end_time) || n < 2U * plan.min_connection_count) &&
         plan.ext_from <= r.start_time && r.start_time < plan.ext_to;
}

void stage_ping(b2r_engine& e, query_run& q) {
  auto& r = *q.pong;
  q.phase = q.p.pong->ping;
  q.phase.keep_lb = true;  // the lower bounds of the first ping stay in the slot
  phase_starts(e.view, q.phase, r.start_time, q.phase.starts);
  q.adm_flags = kAdmRephase;
  q.upload.clear();
  r.in_ping = true;
  q.readmit = true;
}

// the pong of ping result r.next (pong.cc:297-341): bounded by the ping's
// round times, starting at its arrival, no worse than its departure
void stage_pong(b2r_engine& e, query_run& q, bool first_of_iteration) {
  auto& r = *q.pong;
  auto const& pj = r.ping[r.next];
  q.phase = q.p.pong->pong;
  phase_starts(e.view, q.phase, pj.dest_time, q.phase.starts);
  q.phase.end_k = static_cast<uint8_t>(std::min<int>(pj.transfers, B2R_MAX_TRANSFERS) + 2);
  q.phase.blast = static_cast<uint8_t>(pj.transfers + 1U);
  q.phase.span = static_cast<int16_t>(std::abs(pj.dest_time - pj.start_time));
  q.phase.recon_transfers = pj.transfers;
  q.phase.recon_start = pj.dest_time;
  q.phase.need_sweep = !first_of_iteration;
  q.adm_flags = first_of_iteration ? (kAdmRephase | (r.ping.front().transfers + 1U)) : kAdmKeepRt;
  q.upload = r.results;
  r.in_ping = false;
  q.readmit = true;
}

// a phase of a pong query finished on the device: the next phase is staged
// (q.readmit) or the sweep ends (q.finished)
void pong_phase_done(b2r_engine& e, query_run& q, exported& x) {
  auto const& plan = *q.p.pong;
  if (!q.pong) {
    q.pong = std::make_unique<pong_run>();
    q.pong->start_time = plan.fwd ? plan.iv_from : plan.iv_to - 1;
  }
  auto& r = *q.pong;
  r.n_rounds += x.sl.n_rounds;
  ++r.n_phases;
  q.readmit = false;
  if (x.sl.state == dev::S_ERROR) {
    q.status = x.sl.error != 0 ? x.sl.error : B2R_ERR_INTERNAL;
    finish_pong(e, q);
    return;
  }
  auto const better = [&](int32_t a, int32_t b) { return plan.fwd ? a < b : a > b; };
  auto const dominated = [&](dev::journey_rec const& j) {
    for (auto const& o : r.results) {
      if (dev::dominates(o, j)) return true;
    }
    return false;
  };
  if (r.in_ping) {
    r.ping = x.js;
    std::erase_if(r.ping, dominated);
    if (r.ping.empty()) {  // no ping results, or all dominated (pong.cc:268-285)
      finish_pong(e, q);
      return;
    }
    std::sort(r.ping.begin(), r.ping.end(),
              [](dev::journey_rec const& a, dev::journey_rec const& b) { return a.transfers > b.transfers; });
    r.next = 0;
    stage_pong(e, q, true);
  } else {
    r.results = x.js;
    if (x.legs_of < x.js.size()) r.legs_of_block[x.js[x.legs_of].block] = std::move(x.legs);
    auto& pj = r.ping[r.next];
    auto const m = std::find_if(r.results.begin(), r.results.end(), [&](dev::journey_rec const& j) {
      return j.transfers == pj.transfers && j.start_time == pj.dest_time;
    });
    if (m == r.results.end()) {  // "no pong" (pong.cc:328-333)
      q.status = B2R_ERR_INTERNAL;
      finish_pong(e, q);
      return;
    }
    pj.start_time = m->dest_time;
    if (++r.next < r.ping.size()) {
      stage_pong(e, q, false);
    } else {
      auto const first = std::min_element(r.ping.begin(), r.ping.end(),
                                          [&](dev::journey_rec const& a, dev::journey_rec const& b) {
                                            return better(a.start_time, b.start_time);
                                          });
      auto const next = first->start_time + (plan.fwd ? 1 : -1);
      if (!better(r.start_time, next)) {  // "no pong progress" (pong.cc:348-351)
        q.status = B2R_ERR_INTERNAL;
        finish_pong(e, q);
        return;
      }
      r.start_time = next;
      if (!pong_continues(plan, r)) {
        finish_pong(e, q);
        return;
      }
      stage_ping(e, q);
    }
  }
  if (q.readmit && check_capacity(e, q.phase) != B2R_OK) {
    q.readmit = false;
    q.status = B2R_ERR_CAPACITY;
    finish_pong(e, q);
  }
}

// the legs the host reads after the phase running in a query's slot: none
// after a ping, the rebuilt journey's after a pong, all others' in full
uint8_t legs_mode(query_run const& q) {
  if (!q.p.pong) return kLegsAll;
  return (!q.pong || q.pong->in_ping) ? kLegsNone : kLegsMatch;
}

// after an exported phase: pong queries go on to their next phase, search
// queries to their next interval-extension phase or their result
void phase_done(b2r_engine& e, query_run& q, exported& x) {
  if (q.p.pong) {
    pong_phase_done(e, q, x);
  } else {
    on_phase_done(e, q, x);
  }
}

}  // namespace

// ------------------------------------------------------------- the loop
// Free slots for admission.  Range queries run several start-time groups and
// so sweep their round times every round (k_sweep); they take slots from the
// top of the pool, all other queries from the bottom, so that the sweeping
// slots share slot groups.
template <typename Free>
struct slot_picker {
  slot_picker(uint32_t n, Free f) : is_free{f}, n_slots{n}, hi{static_cast<int64_t>(n) - 1} {}
  int64_t take(bool top) {
    if (top) {
      while (hi >= 0 && !is_free(static_cast<uint32_t>(hi))) --hi;
      return hi < 0 ? -1 : hi--;
    }
    while (lo < n_slots && !is_free(static_cast<uint32_t>(lo))) ++lo;
    return lo >= n_slots ? -1 : lo++;
  }
  Free is_free;
  int64_t n_slots;
  int64_t lo{0}, hi;
};

bool sweeps(prepped_query const& p) { return !p.ontrip && !p.one_to_all; }

// one start-time group and nothing after it: the slot's journeys are final
// when it is done (the queries whose reconstruction waits for that)
bool single_group(prepped_query const& p) { return p.ontrip && !p.one_to_all && p.recon_mode == 0 && !p.pong; }

// a new interval-extension phase for the query in slot s (search.h:283-316)
void rearm(b2r_engine& e, uint32_t s, query_run& q, cudaStream_t st) {
  // new phase: upload the new starts (and journeys kept), keep the rt
  // generation unless reset_arrivals (raptor.h:174-177)
  auto const tad_keep = !q.reset_arrivals;
  slot_t cur{};
  e.d2h_bytes += sizeof(slot_t);
  B2R_CUDA(cudaMemcpyAsync(&cur, e.st.slots + s, sizeof(slot_t), cudaMemcpyDeviceToHost, st));
  B2R_CUDA(cudaStreamSynchronize(st));
  if (q.reset_arrivals) {
    if (e.gen_query[s] >= 0xFFFEu) throw std::runtime_error("query generation exhausted");
    cur.gen_query = ++e.gen_query[s];
    for (auto& x : cur.tad) x = dev::kKeyInv;
  }
  (void)tad_keep;
  cur.state = dev::S_START;
  cur.iv_from = q.p.iv_from;
  cur.iv_to = q.p.iv_to;
  cur.need_sweep = q.reset_arrivals ? 0 : 1;
  cur.early_term = 0;
  cur.next_start = 0;
  cur.n_starts = static_cast<uint32_t>(q.p.starts.size());
  if (cur.n_starts > e.max_starts) throw std::runtime_error("start capacity exceeded");
  std::vector<dev::start_rec> starts(q.p.starts.size());
  for (auto j = 0U; j != starts.size(); ++j) {
    starts[j] = {q.p.starts[j].time_at_start, q.p.starts[j].time_at_stop, q.p.starts[j].stop};
  }
  B2R_CUDA(cudaMemcpyAsync(e.st.start_pool + cur.starts_off, starts.data(),
                           starts.size() * sizeof(dev::start_rec), cudaMemcpyHostToDevice, st));
  if (q.keep.size() > e.max_j) throw std::runtime_error("journey capacity exceeded");
  auto* dj = e.d_keep;  // engine-owned, reused (this function synchronises)
  B2R_CUDA(cudaMemcpyAsync(dj, q.keep.data(), q.keep.size() * sizeof(dev::journey_rec),
                           cudaMemcpyHostToDevice, st));
  ++e.aux_launches;
  k_set_journeys<<<1, 32, 0, st>>>(e.st, s, dj, static_cast<uint32_t>(q.keep.size()));
  B2R_CUDA(cudaMemcpyAsync(e.st.slots + s, &cur, sizeof(slot_t), cudaMemcpyHostToDevice, st));
  B2R_CUDA(cudaStreamSynchronize(st));
  e.h2d_bytes += starts.size() * sizeof(dev::start_rec) + q.keep.size() * sizeof(dev::journey_rec) +
                 sizeof(slot_t);
  q.rearm = false;
}

// length of the union of [start, end) intervals
double busy_union_ms(std::vector<std::pair<double, double>> v) {
  std::sort(v.begin(), v.end());
  double total = 0, lo = 0, hi = -1;
  for (auto const& [a, b] : v) {
    if (a > hi) {
      if (hi > lo) total += hi - lo;
      lo = a;
      hi = b;
    } else {
      hi = std::max(hi, b);
    }
  }
  if (hi > lo) total += hi - lo;
  return total;
}

struct batch_runner {
  b2r_engine& e;
  std::vector<query_run>& runs;
  bool use_graph;
  uint64_t launches{0}, steps{0};
  double busy_ms{0};  // device time: union of the chunks' and the finished-slot work's intervals

  void run(uint32_t chunk) {
    auto const S = e.S;
    auto* st = e.stream;
    // row copies into result buffers may still be in flight when an error
    // unwinds the batch: they end before those buffers can be freed
    struct drain {
      cudaStream_t s;
      ~drain() { cudaStreamSynchronize(s); }
    } drain2{e.stream2};
    e.busy.clear();
    B2R_CUDA(cudaEventRecord(e.ev_base, st));
    e.base_recorded = true;
    struct unrecord {  // the serving loop exports without a base event
      b2r_engine& e;
      ~unrecord() { e.base_recorded = false; }
    } unrec{e};
    size_t next = 0;
    std::vector<int64_t>& slot_q = e.slot_query;
    std::fill(slot_q.begin(), slot_q.end(), -1);
    // slots whose query's next pong phase is staged: their summaries are
    // stale until the re-admission at the next admission point
    std::vector<uint8_t> waiting(S, 0);
    std::vector<uint32_t> pending;
    auto const admit_free = [&]() {
      std::vector<adm_req> adm;
      for (auto const s : pending) {
        auto& q = runs[static_cast<size_t>(slot_q[s])];
        adm.push_back({s, &q.phase, q.adm_flags, &q.upload});
        q.readmit = false;
        waiting[s] = 0;
      }
      pending.clear();
      slot_picker pick{S, [&](uint32_t s) { return slot_q[s] == -1; }};
      while (next < runs.size()) {
        while (next < runs.size()) {
          auto& q = runs[next];
          if (!q.ready.load(std::memory_order_acquire)) break;
          if (q.p.status != B2R_OK || q.p.empty_result) {
            q.status = q.p.status;
            q.res.view.status = q.p.status;
            q.res.view.interval_from = q.p.iv_from;
            q.res.view.interval_to = q.p.iv_to;
            q.finished = true;
            ++next;
            continue;
          }
          if (auto const c = check_capacity(e, q.p); c != B2R_OK) {
            q.status = c;
            q.res.view.status = c;
            q.finished = true;
            ++next;
            continue;
          }
          break;
        }
        if (next >= runs.size() || !runs[next].ready.load(std::memory_order_acquire)) break;
        auto const s = pick.take(sweeps(runs[next].p));
        if (s < 0) break;
        slot_q[s] = static_cast<int64_t>(next);
        adm.push_back({static_cast<uint32_t>(s), &runs[next].p});
        ++next;
      }
      auto const t0 = std::chrono::steady_clock::now();
      admit(e, adm, st);
      e.admit_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    };
    // Pipelined: right after the sync of chunk c the next chunk is
    // launched, and the slots that finished in chunk c are exported on a
    // second stream while it runs.  Finished slots are left alone by the
    // super-step kernels, so the export reads stable data.  Their
    // retirement is queued behind the chunk in flight, whose summary still
    // shows them finished: they stay "retiring" (not admissible, state
    // ignored) until that summary has been read.
    constexpr int64_t kRetiring = -2;
    std::vector<uint8_t> stale(S, 0);  // rearmed: the next summary predates it
    std::vector<uint8_t> held(S, 0);   // finished, export held back (below)
    std::vector<uint32_t> held_nj(S, 0), held_list;
    std::vector<b2r_engine::summary_t> sum(S);
    bool in_flight = false;
    auto const running = [&]() {
      for (auto x : slot_q)
        if (x >= 0) return true;
      return false;
    };
    auto const busy = [&]() { return next < runs.size() || running(); };
    auto const launch_chunk = [&](uint32_t n_steps) {
      B2R_CUDA(cudaEventRecord(e.ev0, st));
      for (uint32_t c = 0; c != n_steps; ++c) {
        if (use_graph) {
          B2R_CUDA(cudaGraphLaunch(e.graph, st));
        } else {
          enqueue_superstep(e, st);
          B2R_CUDA(cudaGetLastError());
        }
        launches += launches_per_step(e);
        ++steps;
      }
      B2R_CUDA(cudaEventRecord(e.ev1, st));
      e.d2h_bytes += S * sizeof(b2r_engine::summary_t);
      B2R_CUDA(cudaMemcpyAsync(e.h_summary, e.d_summary, S * sizeof(b2r_engine::summary_t),
                               cudaMemcpyDeviceToHost, st));
      in_flight = true;
    };
    // every start-time group ends within end_k super-steps; the cap turns a
    // logic error into a reported failure instead of an endless loop
    uint64_t max_steps = 10000;
    for (auto const& q : runs) {
      max_steps += 40ull * (q.p.starts.size() + 2) * (q.p.end_k + 2);
      if (q.p.pong) max_steps += 40ull * 4096 * (q.p.end_k + 2);  // a sweep of many phases
    }
    admit_free();
    while (busy()) {
      if (steps > max_steps) throw std::runtime_error("super-step cap exceeded");
      if (!in_flight) {
        if (!running()) {  // every resident query finished: wait for preparation
          for (auto& x : slot_q)
            if (x == kRetiring) x = -1;  // no summary in flight can predate it
          auto const t0 = std::chrono::steady_clock::now();
          std::this_thread::yield();
          e.idle_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
          admit_free();
          continue;
        }
        launch_chunk(chunk);
      }
      B2R_CUDA(cudaStreamSynchronize(st));
      in_flight = false;
      {
        float a = 0, b = 0;
        B2R_CUDA(cudaEventElapsedTime(&a, e.ev_base, e.ev0));
        B2R_CUDA(cudaEventElapsedTime(&b, e.ev_base, e.ev1));
        e.busy.emplace_back(a, b);
        if (e.cfg.profile == 2U) {  // one super-step per chunk: its route phase
          B2R_CUDA(cudaEventElapsedTime(&a, e.ev_scan_a, e.ev_scan_b));
          e.scan_ms += a;
          ++e.scan_launches;
        }
      }
      std::copy(e.h_summary, e.h_summary + S, sum.begin());
      for (auto& x : slot_q)
        if (x == kRetiring) x = -1;  // their retirement ran before this summary's chunk ended
      std::vector<uint32_t> done_slots, n_js, n_rows;
      for (uint32_t s = 0; s != S; ++s) {
        if (slot_q[s] < 0 || waiting[s] || held[s]) continue;
        if (stale[s]) {
          stale[s] = 0;
          continue;
        }
        auto const state = sum[s].state;
        if (state == dev::S_DONE || state == dev::S_ERROR) {
          done_slots.push_back(s);
          n_js.push_back(sum[s].n_journeys);
          auto const& q = runs[static_cast<size_t>(slot_q[s])];
          n_rows.push_back(q.p.one_to_all ? q.p.end_k : 0u);
        }
      }
      admit_free();  // into free slots, queued before the next chunk
      // next chunk in flight unless every resident query has just finished
      size_t n_active = 0;
      for (uint32_t s = 0; s != S; ++s) n_active += (slot_q[s] >= 0 && !waiting[s] && !held[s]) ? 1U : 0U;
      auto const others_run = done_slots.size() < n_active;
      // Finished queries of one start-time group and nothing after it wait
      // in their slots (held) while other slots run and no query waits for
      // a slot, and are exported together: a quarter of the slots at once,
      // or all of them when nothing else runs.  Each export's journey
      // rebuilding lasts as long as its longest journey, so fewer exports
      // rebuild the same journeys in less device time.
      {
        std::vector<uint32_t> d2, j2, r2;
        for (auto i = 0U; i != done_slots.size(); ++i) {
          auto const s = done_slots[i];
          if (others_run && next >= runs.size() && single_group(runs[static_cast<size_t>(slot_q[s])].p)) {
            held[s] = 1;
            held_nj[s] = n_js[i];
            held_list.push_back(s);
          } else {
            d2.push_back(s);
            j2.push_back(n_js[i]);
            r2.push_back(n_rows[i]);
          }
        }
        if (!held_list.empty() && (!others_run || next < runs.size() || held_list.size() >= S / 4U)) {
          for (auto const s : held_list) {
            held[s] = 0;
            d2.push_back(s);
            j2.push_back(held_nj[s]);
            r2.push_back(0u);
          }
          held_list.clear();
        }
        done_slots.swap(d2);
        n_js.swap(j2);
        n_rows.swap(r2);
      }
      // a finished pong phase is followed by the next phase of its sweep:
      // that phase is staged from the export, so the next chunk waits for
      // it instead of leaving the slot idle for a whole chunk
      auto phase_follows = false;
      for (auto const s : done_slots) phase_follows = phase_follows || runs[static_cast<size_t>(slot_q[s])].p.pong;
      if (!phase_follows && running() && others_run) launch_chunk(chunk);
      if (done_slots.empty()) continue;
      auto const t_exp = std::chrono::steady_clock::now();
      std::vector<exported> ex;
      std::vector<uint8_t> modes;
      for (auto const s : done_slots) modes.push_back(legs_mode(runs[static_cast<size_t>(slot_q[s])]));
      export_slots(e, done_slots, n_js, n_rows, ex, e.stream2, &modes, row_target::pinned);
      std::vector<uint32_t> retired;
      auto const now_ms = std::chrono::duration<double, std::milli>(
                              std::chrono::steady_clock::now() - e.batch_t0)
                              .count();
      for (auto i = 0U; i != done_slots.size(); ++i) {
        auto const s = done_slots[i];
        auto& q = runs[static_cast<size_t>(slot_q[s])];
        phase_done(e, q, ex[i]);
        q.res.view.latency_ms = now_ms;
        if (q.readmit) {
          pending.push_back(s);
          waiting[s] = 1;
        } else if (q.rearm) {
          rearm(e, s, q, st);
          stale[s] = in_flight ? 1 : 0;
        } else {
          retired.push_back(s);
          slot_q[s] = in_flight ? kRetiring : -1;
        }
      }
      retire(e, retired, st);
      e.export_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_exp).count();
      if (!in_flight) admit_free();
    }
    B2R_CUDA(cudaStreamSynchronize(st));
    B2R_CUDA(cudaStreamSynchronize(e.stream2));  // one-to-all rows still on their way
    busy_ms = busy_union_ms(e.busy);
  }
};

void capture_graph(b2r_engine& e) {
  cudaGraph_t g = nullptr;
  B2R_CUDA(cudaStreamBeginCapture(e.stream, cudaStreamCaptureModeThreadLocal));
  enqueue_superstep(e, e.stream);
  B2R_CUDA(cudaStreamEndCapture(e.stream, &g));
  B2R_CUDA(cudaGraphInstantiate(&e.graph, g, 0));
  cudaGraphDestroy(g);
}

// Host preparation on worker threads, in query order, overlapping the
// device work of the queries already admitted.
struct preparer {
  std::vector<std::thread> pool;
  std::atomic<uint32_t> next{0};
  void start(b2r_engine& e, b2r_query const* qs, uint32_t n, std::vector<query_run>& runs,
             bool inline_all) {
    auto const hw = std::max(1U, std::thread::hardware_concurrency());
    auto const n_threads = std::max(1U, std::min<uint32_t>(
        e.cfg.host_threads != 0 ? e.cfg.host_threads : (hw > 1 ? hw - 1 : 1), n));
    auto const lb_mode = e.lb_mode();
    auto work = [&e, qs, n, &runs, lb_mode, this]() {
      for (auto i = next++; i < n; i = next++) {
        auto const t0 = std::chrono::steady_clock::now();
        prepare(e.view, qs[i], lb_mode, runs[i].p);
        e.prep_ns += static_cast<uint64_t>(
            std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count());
        runs[i].ready.store(true, std::memory_order_release);
      }
    };
    if (inline_all) {
      work();
      return;
    }
    for (auto t = 0U; t < n_threads; ++t) pool.emplace_back(work);
  }
  void join() {
    for (auto& t : pool) t.join();
    pool.clear();
  }
  ~preparer() { join(); }
};

void fill_out(b2r_engine& e, std::vector<query_run>& runs, b2r_result* out) {
  e.results.resize(runs.size());
  for (auto i = 0U; i != runs.size(); ++i) {
    e.results[i] = std::move(runs[i].res);
    auto& r = e.results[i];
    r.view.n_journeys = static_cast<uint32_t>(r.journeys.size());
    r.view.journeys = r.journeys.data();
    r.view.legs = r.legs.data();
    r.view.round_times = r.rt_rows.empty() ? nullptr : r.rt_rows.data();
    out[i] = r.view;
  }
}

// ------------------------------------------------------------- serving
// Continuous batching: submitted queries are prepared on a host pool and
// admitted into free slots at super-step boundaries while the queries
// already resident keep running; finished slots are exported and retired
// after every chunk of super-steps.  One driver thread owns the device.
struct serve_item {
  uint64_t ticket{0};
  b2r_query q{};
  std::vector<b2r_offset> start, dest;  // the query's offsets (copied)
  std::chrono::steady_clock::time_point t_submit;
  query_run run;
  bool finished{false};
};

struct serve_state {
  explicit serve_state(b2r_engine& eng) : e{eng}, slot_item(eng.S, nullptr) {}
  b2r_engine& e;
  std::mutex mu;
  std::condition_variable cv_prep, cv_driver, cv_done;
  std::deque<serve_item*> to_prepare, ready;
  std::unordered_map<uint64_t, std::unique_ptr<serve_item>> items;
  std::vector<serve_item*> slot_item;
  std::vector<uint32_t> pending;  // slots whose pong query's next phase is staged
  uint64_t next_ticket{1};
  uint64_t unfinished{0};  // submitted, not finished
  bool stop{false};
  int failed_status{B2R_OK};
  std::string failed_msg;
  std::vector<std::thread> prep_pool;
  std::thread driver;
  // counters for b2r_serve_stats (nanoseconds of host time by step)
  std::atomic<uint64_t> n_steps{0}, n_launches{0}, admit_ns{0}, export_ns{0}, idle_ns{0}, prep_ns{0}, sync_ns{0};
  bool backlog{false};  // the last admission left prepared queries waiting for slots (driver thread)

  void finish(serve_item& it) {  // with mu held
    auto& r = it.run.res;
    r.view.n_journeys = static_cast<uint32_t>(r.journeys.size());
    r.view.journeys = r.journeys.data();
    r.view.legs = r.legs.data();
    r.view.round_times = r.rt_rows.empty() ? nullptr : r.rt_rows.data();
    r.view.latency_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - it.t_submit).count();
    it.finished = true;
    --unfinished;
  }

  void fail_item(serve_item& it, int status) {  // with mu held
    it.run.status = status;
    it.run.res.view.status = status;
    finish(it);
  }

  void prep_loop() {
    auto const lb_mode = e.lb_mode();
    std::unique_lock<std::mutex> lock{mu};
    while (true) {
      cv_prep.wait(lock, [&] { return stop || !to_prepare.empty(); });
      if (to_prepare.empty()) return;  // stopping and nothing left
      auto* it = to_prepare.front();
      to_prepare.pop_front();
      lock.unlock();
      auto status = B2R_OK;
      auto const t0 = std::chrono::steady_clock::now();
      try {
        prepare(e.view, it->q, lb_mode, it->run.p);
      } catch (...) {
        status = B2R_ERR_INTERNAL;
      }
      prep_ns += ns_since(t0);
      lock.lock();
      if (status != B2R_OK) {
        fail_item(*it, status);
        cv_done.notify_all();
        cv_driver.notify_one();  // it may be waiting for the last query to end
        continue;
      }
      ready.push_back(it);
      cv_driver.notify_one();
    }
  }

  // Free slots and staged pong phases admitted (queued on the main stream);
  // with nothing resident and nothing in flight it waits for prepared
  // queries.  Returns false when the loop is to end, else whether any slot
  // holds a query.
  bool admit_ready(std::vector<uint8_t>& retiring, std::vector<uint8_t>& waiting, bool in_flight, bool& busy) {
    std::vector<adm_req> adm;
    for (auto const s : pending) {  // pong phases staged by the last export
      auto& run = slot_item[s]->run;
      adm.push_back({s, &run.phase, run.adm_flags, &run.upload});
      run.readmit = false;
      waiting[s] = 0;
    }
    pending.clear();
    {
      std::unique_lock<std::mutex> lock{mu};
      auto const has_busy = [&] {
        for (auto* x : slot_item)
          if (x != nullptr) return true;
        return false;
      };
      if (!has_busy() && !in_flight && adm.empty()) {
        auto const t0 = std::chrono::steady_clock::now();
        cv_driver.wait(lock, [&] { return !ready.empty() || (stop && unfinished == 0); });
        idle_ns += ns_since(t0);
        if (ready.empty() && stop && unfinished == 0) return false;
      }
      slot_picker pick{e.S, [&](uint32_t s) { return slot_item[s] == nullptr && retiring[s] == 0; }};
      while (!ready.empty()) {
        while (!ready.empty()) {
          auto* it = ready.front();
          auto const& p = it->run.p;
          if (p.status != B2R_OK || p.empty_result) {
            ready.pop_front();
            it->run.res.view.interval_from = p.iv_from;
            it->run.res.view.interval_to = p.iv_to;
            fail_item(*it, p.status);
            cv_done.notify_all();
            continue;
          }
          if (auto const c = check_capacity(e, p); c != B2R_OK) {
            ready.pop_front();
            fail_item(*it, c);
            cv_done.notify_all();
            continue;
          }
          break;
        }
        if (ready.empty()) break;
        auto* it = ready.front();
        auto const s = pick.take(sweeps(it->run.p));
        if (s < 0) break;
        ready.pop_front();
        slot_item[s] = it;
        adm.push_back({static_cast<uint32_t>(s), &it->run.p});
      }
      busy = has_busy();
      backlog = !ready.empty();  // prepared queries wait for slots
    }
    auto const t0 = std::chrono::steady_clock::now();
    admit(e, adm, e.stream);
    admit_ns += ns_since(t0);
    return true;
  }
  static uint64_t ns_since(std::chrono::steady_clock::time_point t0) {
    return static_cast<uint64_t>(
        std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count());
  }

  // Pipelined like the batch loop: right after the sync of chunk c the
  // next chunk is launched, and the slots that finished in c are exported
  // on the second stream while it runs.  Retirements, re-arms and staged
  // pong phases are then queued behind that chunk, whose summary predates
  // them: such slots are skipped in it (retiring, stale, waiting) and only
  // then reused.
  void driver_loop() {
    auto* st = e.stream;
    auto const chunk = e.cfg.steps_per_sync != 0 ? e.cfg.steps_per_sync : std::min(2U, e.shape.steps_per_sync);
    auto const use_graph = e.cfg.use_graphs != 0 && e.graph != nullptr;
    try {
      B2R_CUDA(cudaSetDevice(e.tt->device));
      std::vector<uint8_t> retiring(e.S, 0), stale(e.S, 0), waiting(e.S, 0);
      std::vector<b2r_engine::summary_t> sum(e.S);
      bool in_flight = false;
      // 2 super-steps per check for short latencies; while queries wait for
      // slots, the batch loop's tuned chunk (as long as a batch, the loop
      // is throughput-bound then)
      auto const launch_chunk = [&]() {
        auto const n_steps = backlog ? std::max(chunk, e.shape.steps_per_sync) : chunk;
        this->n_steps += n_steps;
        n_launches += n_steps * launches_per_step(e);
        for (uint32_t c = 0; c != n_steps; ++c) {
          if (use_graph) {
            B2R_CUDA(cudaGraphLaunch(e.graph, st));
          } else {
            enqueue_superstep(e, st);
            B2R_CUDA(cudaGetLastError());
          }
        }
        B2R_CUDA(cudaMemcpyAsync(e.h_summary, e.d_summary, e.S * sizeof(b2r_engine::summary_t),
                                 cudaMemcpyDeviceToHost, st));
        in_flight = true;
      };
      while (true) {
        if (!in_flight) {
          std::fill(retiring.begin(), retiring.end(), 0);  // nothing in flight predates a retirement
          bool busy = false;
          if (!admit_ready(retiring, waiting, false, busy)) return;
          if (!busy) continue;
          launch_chunk();
        }
        auto const t_sync = std::chrono::steady_clock::now();
        B2R_CUDA(cudaStreamSynchronize(st));
        sync_ns += ns_since(t_sync);
        in_flight = false;
        std::copy(e.h_summary, e.h_summary + e.S, sum.begin());
        std::vector<uint32_t> done_slots, n_js, n_rows;
        for (uint32_t s = 0; s != e.S; ++s) {
          if (slot_item[s] == nullptr || waiting[s]) continue;
          if (stale[s]) {
            stale[s] = 0;
            continue;
          }
          auto const state = sum[s].state;
          if (state == dev::S_DONE || state == dev::S_ERROR) {
            done_slots.push_back(s);
            n_js.push_back(sum[s].n_journeys);
            n_rows.push_back(slot_item[s]->run.p.one_to_all ? slot_item[s]->run.p.end_k : 0u);
          }
        }
        std::fill(retiring.begin(), retiring.end(), 0);  // their retirement precedes what is queued next
        bool busy = false;
        if (!admit_ready(retiring, waiting, true, busy)) return;
        // a finished pong phase is followed by its next phase, staged from
        // the export: the next chunk waits for it
        auto phase_follows = false;
        for (auto const s : done_slots) phase_follows = phase_follows || slot_item[s]->run.p.pong;
        size_t n_active = 0;  // resident queries the next chunk would run, the finished ones included
        for (uint32_t s = 0; s != e.S; ++s) n_active += (slot_item[s] != nullptr && !waiting[s]) ? 1U : 0U;
        if (!phase_follows && busy && done_slots.size() < n_active) launch_chunk();
        if (done_slots.empty()) continue;
        auto const t_exp = std::chrono::steady_clock::now();
        std::vector<exported> ex;
        std::vector<uint8_t> modes;
        for (auto const s : done_slots) modes.push_back(legs_mode(slot_item[s]->run));
        export_slots(e, done_slots, n_js, n_rows, ex, e.stream2, &modes, row_target::pinned);
        B2R_CUDA(cudaStreamSynchronize(e.stream2));  // the rows, before any ticket shows finished
        std::vector<uint32_t> retired;
        for (auto i = 0U; i != done_slots.size(); ++i) {
          auto const s = done_slots[i];
          auto& it = *slot_item[s];
          phase_done(e, it.run, ex[i]);
          if (it.run.readmit) {
            pending.push_back(s);
            waiting[s] = 1;
            continue;
          }
          if (it.run.rearm) {
            rearm(e, s, it.run, st);
            stale[s] = in_flight ? 1 : 0;
            continue;
          }
          retired.push_back(s);
          retiring[s] = in_flight ? 1 : 0;
          std::lock_guard<std::mutex> lock{mu};
          slot_item[s] = nullptr;
          finish(it);
        }
        retire(e, retired, st);
        export_ns += ns_since(t_exp);
        cv_done.notify_all();
      }
    } catch (std::exception const& ex) {
      std::lock_guard<std::mutex> lock{mu};
      failed_status = B2R_ERR_CUDA;
      failed_msg = ex.what();
      for (auto& [t, it] : items) {
        if (!it->finished) fail_item(*it, B2R_ERR_CUDA);
      }
      for (auto& x : slot_item) x = nullptr;
      ready.clear();
      to_prepare.clear();
      cv_done.notify_all();
    }
  }
};

serve_state* serving_of(b2r_engine* e) { return static_cast<serve_state*>(e->serve.get()); }

}  // namespace b2r

// ===================================================================== C ABI
extern "C" {

int b2r_timetable_upload(const b2r_timetable_desc* d, int device, b2r_timetable** out) {
  B2R_API_GUARD({
    if (d == nullptr || out == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
    for (auto p = 0U; p != B2R_N_PROFILES - 1U; ++p) {  // a profile's lists come in (index, words) pairs
      uint32_t const* const lists[8] = {d->profile_footpaths_out_index[p], d->profile_footpaths_out[p],
                                        d->profile_footpaths_in_index[p],  d->profile_footpaths_in[p],
                                        d->profile_lb_fwd_index[p],        d->profile_lb_fwd[p],
                                        d->profile_lb_bwd_index[p],        d->profile_lb_bwd[p]};
      auto ok = (lists[0] == nullptr) == (lists[2] == nullptr);  // footpaths out and in together
      for (auto x = 0U; ok && x != 8U; x += 2U) {
        if (lists[x] == nullptr) continue;
        auto const n = lists[x][d->n_locations];
        ok = n == 0U || lists[x + 1U] != nullptr;
        for (auto i = 0U; ok && i != n; ++i) ok = B2R_FP_TARGET(lists[x + 1U][i]) < d->n_locations;
      }
      if (!ok) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "b2r_timetable_upload: malformed profile footpaths");
    }
    try {
      B2R_CUDA(cudaSetDevice(device));
      auto t = std::make_unique<b2r_timetable>();
      t->device = device;
      t->host = *d;
      auto& a = t->allocs;
      auto& by = t->bytes;
      auto const nl = d->n_locations, nr = d->n_routes, ntr = d->n_transports;
      auto up = [&](auto const* p, size_t n) {
        auto* x = b2r::dupload(p, n, by);
        a.push_back(x);
        return x;
      };
      // host copies for the query preparation
      b2r::host_copy(t->transfer_time, d->transfer_time, nl);
      b2r::host_copy(t->parent, d->parent, nl);
      b2r::host_copy(t->location_type, d->location_type, nl);
      if (d->children_index != nullptr) {
        b2r::host_copy(t->children_index, d->children_index, nl + 1);
        b2r::host_copy(t->children, d->children, d->children_index[nl]);
      }
      b2r::host_copy(t->fp_out_index, d->footpaths_out_index, nl + 1);
      b2r::host_copy(t->fp_out, d->footpaths_out, d->footpaths_out_index[nl]);
      b2r::host_copy(t->fp_in_index, d->footpaths_in_index, nl + 1);
      b2r::host_copy(t->fp_in, d->footpaths_in, d->footpaths_in_index[nl]);
      b2r::host_copy(t->route_stop_index, d->route_stop_index, nr + 1);
      b2r::host_copy(t->route_stops, d->route_stops, d->route_stop_index[nr]);
      b2r::host_copy(t->route_transport_from, d->route_transport_from, nr);
      b2r::host_copy(t->route_transport_to, d->route_transport_to, nr);
      b2r::host_copy(t->route_stop_time_from, d->route_stop_time_from, nr);
      b2r::host_copy(t->route_stop_times, d->route_stop_times, d->n_route_stop_times);
      b2r::host_copy(t->route_traffic_days, d->route_traffic_days, nr);
      b2r::host_copy(t->transport_traffic_days, d->transport_traffic_days, ntr);
      b2r::host_copy(t->transport_route, d->transport_route, ntr);
      b2r::host_copy(t->bitfields, d->bitfields, 8ull * d->n_bitfields);
      b2r::host_copy(t->location_routes_index, d->location_routes_index, nl + 1);
      b2r::host_copy(t->location_routes, d->location_routes, d->location_routes_index[nl]);
      b2r::host_copy(t->lb_fwd_index, d->lb_fwd_index, nl + 1);
      b2r::host_copy(t->lb_fwd, d->lb_fwd, d->lb_fwd_index[nl]);
      b2r::host_copy(t->lb_bwd_index, d->lb_bwd_index, nl + 1);
      b2r::host_copy(t->lb_bwd, d->lb_bwd, d->lb_bwd_index[nl]);
      auto& v = t->view.d;
      v = *d;
      v.transfer_time = t->transfer_time.data();
      v.parent = t->parent.empty() ? nullptr : t->parent.data();
      v.location_type = t->location_type.empty() ? nullptr : t->location_type.data();
      v.children_index = t->children_index.empty() ? nullptr : t->children_index.data();
      v.children = t->children.data();
      v.footpaths_out_index = t->fp_out_index.data();
      v.footpaths_out = t->fp_out.data();
      v.footpaths_in_index = t->fp_in_index.data();
      v.footpaths_in = t->fp_in.data();
      v.route_stop_index = t->route_stop_index.data();
      v.route_stops = t->route_stops.data();
      v.route_transport_from = t->route_transport_from.data();
      v.route_transport_to = t->route_transport_to.data();
      v.route_stop_time_from = t->route_stop_time_from.data();
      v.route_stop_times = t->route_stop_times.data();
      v.route_traffic_days = t->route_traffic_days.data();
      v.transport_traffic_days = t->transport_traffic_days.data();
      v.transport_route = t->transport_route.data();
      v.bitfields = t->bitfields.data();
      v.location_routes_index = t->location_routes_index.data();
      v.location_routes = t->location_routes.data();
      v.lb_fwd_index = t->lb_fwd_index.data();
      v.lb_fwd = t->lb_fwd.data();
      v.lb_bwd_index = t->lb_bwd_index.data();
      v.lb_bwd = t->lb_bwd.data();
      v.importance = nullptr;
      // footpath profiles 1..4: (index, words) of out, in, lb fwd, lb bwd
      for (auto p = 0U; p != B2R_N_PROFILES - 1U; ++p) {
        uint32_t const* const src[8] = {d->profile_footpaths_out_index[p], d->profile_footpaths_out[p],
                                        d->profile_footpaths_in_index[p],  d->profile_footpaths_in[p],
                                        d->profile_lb_fwd_index[p],        d->profile_lb_fwd[p],
                                        d->profile_lb_bwd_index[p],        d->profile_lb_bwd[p]};
        uint32_t const** const dst[8] = {&v.profile_footpaths_out_index[p], &v.profile_footpaths_out[p],
                                         &v.profile_footpaths_in_index[p],  &v.profile_footpaths_in[p],
                                         &v.profile_lb_fwd_index[p],        &v.profile_lb_fwd[p],
                                         &v.profile_lb_bwd_index[p],        &v.profile_lb_bwd[p]};
        auto& pc = t->profiles[p];
        for (auto x = 0U; x != 8U; x += 2U) {
          *dst[x] = nullptr;
          *dst[x + 1U] = nullptr;
          if (src[x] == nullptr) continue;
          b2r::host_copy(pc.lists[x], src[x], nl + 1);
          b2r::host_copy(pc.lists[x + 1U], src[x + 1U], src[x][nl]);
          *dst[x] = pc.lists[x].data();
          *dst[x + 1U] = pc.lists[x + 1U].data();
        }
      }
      // route filters on the host: pong's direct alternatives
      t->route_clasz.assign(nr, 10U);
      if (d->route_clasz != nullptr) t->route_clasz.assign(d->route_clasz, d->route_clasz + nr);
      t->route_flags.assign(nr, 0U);
      if (d->route_flags != nullptr) t->route_flags.assign(d->route_flags, d->route_flags + nr);
      t->route_section_flags.assign(d->route_stop_index[nr], 0U);
      if (d->route_section_flags != nullptr) {
        t->route_section_flags.assign(d->route_section_flags, d->route_section_flags + d->route_stop_index[nr]);
      }
      v.route_clasz = t->route_clasz.data();
      v.route_flags = t->route_flags.data();
      v.route_section_flags = t->route_section_flags.data();

      // route filter words: class | all-sections flags << 4 | some << 8
      std::vector<uint16_t> rfilter(nr, 10U);  // no classes given: bus
      for (auto r = 0U; r != nr; ++r) {
        auto const c = d->route_clasz != nullptr ? d->route_clasz[r] : 10U;
        if (c >= 16U) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "route_clasz out of range (0..15)");
        auto const fl = d->route_flags != nullptr ? d->route_flags[r] : 0U;
        uint32_t all = 0U, some = 0U;
        for (auto f = 0U; f != 4U; ++f) {
          all |= ((fl >> (2U * f)) & 1U) << f;
          some |= ((fl >> (2U * f + 1U)) & 1U) << f;
        }
        rfilter[r] = static_cast<uint16_t>(c | (all << 4) | (some << 8));
      }
      std::vector<uint8_t> rsec(d->route_stop_index[nr], 0U);
      if (d->route_section_flags != nullptr) {
        std::copy(d->route_section_flags, d->route_section_flags + rsec.size(), rsec.begin());
      }

      // column order check: get_earliest_transport's binary search needs
      // every event column ordered by minutes after midnight
      std::vector<uint8_t> sorted(nr, 1U);
      for (auto r = 0U; r != nr; ++r) {
        auto const n_t = d->route_transport_to[r] - d->route_transport_from[r];
        auto const n_s = d->route_stop_index[r + 1] - d->route_stop_index[r];
        auto const* c = d->route_stop_times + d->route_stop_time_from[r];
        for (auto slot = 0U; n_s > 1U && slot < 2U * (n_s - 1U) && sorted[r]; ++slot) {
          for (auto x = 1U; x < n_t; ++x) {
            if ((c[slot * n_t + x] >> 5) < (c[slot * n_t + x - 1] >> 5)) {
              sorted[r] = 0U;
              break;
            }
          }
        }
      }

      // trip order check for the route scan's parallel boarding: the trips
      // (transport, service day) of a route must compare the same way at
      // every event of the route, equal at all or strictly ordered at all.
      // A trip on day d is its transport's times shifted by d days, so with
      // the transports sorted by their first departure within its day, the
      // neighbours (and the last against the first one day later) cover
      // every pair: consistent neighbours order all trips consistently.
      std::vector<uint8_t> fifo(nr, 1U);
      {
        std::vector<uint32_t> ord;
        std::vector<int32_t> shift;
        for (auto r = 0U; r != nr; ++r) {
          auto const n_t = d->route_transport_to[r] - d->route_transport_from[r];
          auto const n_s = d->route_stop_index[r + 1] - d->route_stop_index[r];
          if (n_s < 2U || n_t == 0U) continue;
          auto const n_slots = 2U * (n_s - 1U);
          auto const* c = d->route_stop_times + d->route_stop_time_from[r];
          auto const count = [&](uint32_t slot, uint32_t x) {
            auto const w = c[slot * n_t + x];
            return static_cast<int32_t>(w & 31U) * 1440 + static_cast<int32_t>(w >> 5);
          };
          ord.resize(n_t);
          shift.resize(n_t);
          for (auto x = 0U; x != n_t; ++x) {
            ord[x] = x;
            auto const c0 = count(0U, x);
            shift[x] = (c0 >= 0 ? c0 / 1440 : -((-c0 + 1439) / 1440)) * 1440;
          }
          std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) {
            return count(0U, a) - shift[a] < count(0U, b) - shift[b];
          });
          for (auto q = 0U; q != n_t && fifo[r] != 0U; ++q) {
            auto const a = ord[q];
            auto const wrap = q + 1U == n_t;
            auto const b = wrap ? ord[0] : ord[q + 1U];
            auto const off = (wrap ? 1440 : 0) - shift[b] + shift[a];
            bool all_zero = true, all_pos = true;
            for (auto slot = 0U; slot != n_slots; ++slot) {
              auto const diff = count(slot, b) + off - count(slot, a);
              all_zero = all_zero && diff == 0;
              all_pos = all_pos && diff > 0;
            }
            if (!all_zero && !all_pos) fifo[r] = 0U;
          }
          // bit 1: on such a route whose columns are ordered by minute and
          // whose transports all leave the first stop on their service day,
          // (service day, transport offset) orders the trips as their times
          // do (the route scan's order key needs no event read then)
          bool first_day = true;
          for (auto x = 0U; x != n_t && first_day; ++x) first_day = (c[x] & 31U) == 0U;
          if (fifo[r] != 0U && sorted[r] != 0U && first_day && n_t < 16384U) fifo[r] |= 2U;
        }
      }

      auto& dd = t->d;
      dd.n_loc = nl;
      dd.n_routes = nr;
      dd.n_transports = ntr;
      dd.internal_from_days = d->date_range_from - B2R_TIMETABLE_OFFSET_DAYS;
      dd.transfer_time = up(d->transfer_time, nl);
      dd.parent = d->parent != nullptr ? up(d->parent, nl) : nullptr;
      dd.loc_type = d->location_type != nullptr ? up(d->location_type, nl) : nullptr;
      if (d->children_index != nullptr) {
        dd.children_idx = up(d->children_index, nl + 1);
        dd.children = up(d->children, d->children_index[nl]);
      }
      dd.importance = d->importance != nullptr ? up(d->importance, nl) : nullptr;
      dd.max_importance = d->max_importance;
      dd.fp_out_idx = up(d->footpaths_out_index, nl + 1);
      dd.fp_out = up(d->footpaths_out, d->footpaths_out_index[nl]);
      dd.fp_in_idx = up(d->footpaths_in_index, nl + 1);
      dd.fp_in = up(d->footpaths_in, d->footpaths_in_index[nl]);
      {  // footpath profiles 1..4 (a profile without footpaths: a zero index)
        std::vector<uint32_t> zero(nl + 1, 0U);
        auto* dz = up(zero.data(), zero.size());
        dd.n_rt = 0;  // no real-time runs until an engine binds an overlay
        dd.loc_rt_idx = dz;
        dd.lrs_rt_idx = dz;
        std::vector<uint32_t const*> tab(4U * (B2R_N_PROFILES - 1U), dz);
        for (auto p = 0U; p != B2R_N_PROFILES - 1U; ++p) {
          auto const& pc = t->profiles[p];
          for (auto x = 0U; x != 4U; x += 2U) {
            if (pc.lists[x].empty()) continue;
            tab[4U * p + x] = up(pc.lists[x].data(), nl + 1);
            if (!pc.lists[x + 1U].empty()) tab[4U * p + x + 1U] = up(pc.lists[x + 1U].data(), pc.lists[x + 1U].size());
          }
        }
        dd.fp_tab = up(tab.data(), tab.size());
      }
      dd.route_stop_idx = up(d->route_stop_index, nr + 1);
      dd.route_stops = up(d->route_stops, d->route_stop_index[nr]);
      dd.route_tr_from = up(d->route_transport_from, nr);
      dd.route_tr_to = up(d->route_transport_to, nr);
      dd.route_st_from = up(d->route_stop_time_from, nr);
      dd.st = up(d->route_stop_times, d->n_route_stop_times);
      dd.route_bf = up(d->route_traffic_days, nr);
      dd.transport_bf = up(d->transport_traffic_days, ntr);
      dd.transport_route = up(d->transport_route, ntr);
      dd.bf = up(d->bitfields, 8ull * d->n_bitfields);
      dd.loc_routes_idx = up(d->location_routes_index, nl + 1);
      dd.loc_routes = up(d->location_routes, d->location_routes_index[nl]);
      dd.route_sorted = up(sorted.data(), nr);
      dd.route_fifo = up(fifo.data(), nr);
      dd.route_filter = up(rfilter.data(), nr);
      dd.route_sec = up(rsec.data(), rsec.size());
      dd.lbg_fwd_idx = up(d->lb_fwd_index, nl + 1);
      dd.lbg_fwd = up(d->lb_fwd, d->lb_fwd_index[nl]);
      dd.lbg_bwd_idx = up(d->lb_bwd_index, nl + 1);
      dd.lbg_bwd = up(d->lb_bwd, d->lb_bwd_index[nl]);
      {
        std::vector<uint32_t> wc;
        if (d->children_index != nullptr) {
          for (auto l = 0U; l != nl; ++l) {
            if (d->children_index[l + 1] != d->children_index[l]) wc.push_back(l);
          }
        }
        dd.with_children = up(wc.data(), wc.size());
        dd.n_with_children = static_cast<uint32_t>(wc.size());
      }
      {  // location -> (route, stop position) pairs (reconstruct.cc:496-515 order)
        std::vector<uint32_t> idx(nl + 1, 0U), rr;
        std::vector<uint16_t> ss;
        for (auto l = 0U; l != nl; ++l) {
          for (auto ri = d->location_routes_index[l]; ri != d->location_routes_index[l + 1]; ++ri) {
            auto const r = d->location_routes[ri];
            for (auto i = d->route_stop_index[r]; i != d->route_stop_index[r + 1]; ++i) {
              if (B2R_STOP_LOC(d->route_stops[i]) == l) {
                rr.push_back(r);
                ss.push_back(static_cast<uint16_t>(i - d->route_stop_index[r]));
              }
            }
          }
          idx[l + 1] = static_cast<uint32_t>(rr.size());
        }
        dd.lrs_idx = up(idx.data(), idx.size());
        dd.lrs_route = up(rr.data(), rr.size());
        dd.lrs_stop = up(ss.data(), ss.size());
      }
      *out = t.release();
      return B2R_OK;
    } catch (b2r::cuda_error const& ex) {
      return b2r::fail(B2R_ERR_CUDA, ex.what());
    }
  });
}

int b2r_timetable_destroy(b2r_timetable* tt) {
  delete tt;
  return B2R_OK;
}

uint64_t b2r_timetable_device_bytes(const b2r_timetable* tt) { return tt == nullptr ? 0 : tt->bytes; }

int b2r_engine_create(b2r_timetable* tt, const b2r_engine_config* cfg_in, b2r_engine** out) {
  B2R_API_GUARD({
    if (tt == nullptr || out == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
    try {
      B2R_CUDA(cudaSetDevice(tt->device));
      auto e = std::make_unique<b2r_engine>();
      b2r_engine_config cfg;
      b2r_engine_config_init(&cfg);
      if (cfg_in != nullptr) cfg = *cfg_in;
      e->tt = tt;
      e->view = tt->view;
      e->cfg = cfg;
      e->sms = b2r::n_sms(tt->device);
      e->max_j = std::max(32U, std::min(4096U, (cfg.max_journeys + 31U) & ~31U));
      e->max_starts = cfg.max_starts != 0 ? cfg.max_starts : 4096U;
      if (cfg.profile == 1U) e->cfg.use_graphs = 0;
      if (cfg.steps_per_sync != 0) e->shape.steps_per_sync = cfg.steps_per_sync;
      e->max_dest = 512U;
      e->max_off = 128U;
      if (cfg.use_lower_bounds == 3) {  // the table when it fits, else no bounds
        auto const n = static_cast<uint64_t>(tt->d.n_loc);
        if (2 * n * n * sizeof(uint16_t) <= B2R_LB_TABLE_MAX_BYTES) {
          auto const hw = std::max(1U, std::thread::hardware_concurrency());
          b2r::ensure_lb_table(*tt, cfg.host_threads != 0 ? cfg.host_threads : hw);
        } else {
          e->cfg.use_lower_bounds = 0;
        }
      }
      auto const nl = tt->d.n_loc;
      e->bytes_per_slot = static_cast<uint64_t>(nl) * (b2r::dev::kK * (4 + 2) + 4 + 4 + 2 + 4) +
                          static_cast<uint64_t>(e->max_j) *
                              (sizeof(b2r::dev::journey_rec) + b2r::dev::kMaxLegs * sizeof(b2r_leg)) +
                          e->max_starts * sizeof(b2r::dev::start_rec) +
                          e->max_dest * sizeof(b2r::dev::dest_rec) + e->max_off * sizeof(b2r_offset) +
                          b2r::dev::kMaxTimeline * sizeof(b2r::dev::tl_entry) +
                          (static_cast<uint64_t>(nl) * (4 + b2r::dev::kK) + tt->d.n_routes) / 8 + 256;
      auto by_budget = cfg.hbm_budget / std::max<uint64_t>(1, e->bytes_per_slot);
      auto slots = std::min<uint64_t>(std::max(32U, cfg.max_slots), by_budget);
      slots &= ~uint64_t{31};
      if (slots == 0) {
        return b2r::fail(B2R_ERR_OUT_OF_MEMORY, "HBM budget too small for one slot group");
      }
      e->S = static_cast<uint32_t>(slots);
      e->G = e->S / 32;
      auto& st = e->st;
      st.tt = tt->d;
      st.S = e->S;
      st.G = e->G;
      st.max_j = e->max_j;
      auto& by = e->bytes;
      auto al = [&](auto*& p, size_t n) {
        using T = std::remove_reference_t<decltype(*p)>;
        p = b2r::dmalloc<std::remove_const_t<T>>(n, by);
        e->allocs.push_back(const_cast<void*>(static_cast<void const*>(p)));
      };
      auto const S = static_cast<size_t>(e->S), G = static_cast<size_t>(e->G);
      al(st.slots, S);
      al(st.lanes, S);
      al(st.rt, static_cast<size_t>(b2r::dev::kK) * nl * S);
      al(st.touched, static_cast<size_t>(b2r::dev::kK) * G * nl);
      al(st.bounds, static_cast<size_t>(b2r::dev::kK) * nl * S);
      al(st.best, static_cast<size_t>(nl) * S);
      al(st.tmp, static_cast<size_t>(nl) * S);
      al(st.lb, static_cast<size_t>(nl) * S);
      al(st.X, static_cast<size_t>(nl) * G);
      al(st.Y, static_cast<size_t>(nl) * G);
      al(st.R, static_cast<size_t>(tt->d.n_routes) * G);
      al(st.D, static_cast<size_t>(nl) * G);
      al(st.xlist, static_cast<size_t>(nl) * G);
      al(st.ylist, static_cast<size_t>(nl) * G);
      al(st.rlist, static_cast<size_t>(tt->d.n_routes) * G);
      al(st.counters, 16);
      al(st.run_mask, G);
      al(st.sweep_mask, G);
      al(st.any_mask, G);
      al(st.start_pool, S * e->max_starts);
      al(st.dest_pool, S * e->max_dest);
      al(st.off_pool, S * e->max_off);
      al(st.journeys, S * e->max_j);
      al(st.legs, S * e->max_j * b2r::dev::kMaxLegs);
      al(st.blocks_used, S * ((e->max_j + 31) / 32));
      al(st.recon_list, S * e->max_j);
      al(st.timeline, S * b2r::dev::kMaxTimeline);
      al(st.timeline_n, S);
      al(st.tad_phase, S);
      al(st.status_word, 4);
      al(e->d_summary, S);
      st.summary = e->d_summary;
      al(st.prof, 8);
      al(st.dist, static_cast<size_t>(nl) * S);
      al(st.F[0], static_cast<size_t>(nl) * G);
      al(st.F[1], static_cast<size_t>(nl) * G);
      al(st.flist[0], static_cast<size_t>(nl) * G);
      al(st.flist[1], static_cast<size_t>(nl) * G);
      al(st.lb_mask, G);
      st.lb_table_fwd = tt->lb_table[0];
      st.lb_table_bwd = tt->lb_table[1];
      st.lb_stride = tt->lb_stride;
      B2R_CUDA(cudaMemset(st.dist, 0xFF, static_cast<size_t>(nl) * S * 4));
      B2R_CUDA(cudaMemset(st.F[0], 0, static_cast<size_t>(nl) * G * 4));
      B2R_CUDA(cudaMemset(st.F[1], 0, static_cast<size_t>(nl) * G * 4));
      B2R_CUDA(cudaMemset(st.lb_mask, 0, G * 4));
      st.profile = cfg.profile == 1U ? 1u : 0u;  // device work counters
      B2R_CUDA(cudaMemset(st.prof, 0, 8 * sizeof(unsigned long long)));
      al(e->d_exp_list, S);
      al(e->d_keep, e->max_j);
      if (cfg.profile) al(e->d_prof_rows, 2 * b2r_engine::kProfRows);
      B2R_CUDA(cudaMemset(st.slots, 0, S * sizeof(b2r::dev::slot_t)));
      B2R_CUDA(cudaMemset(st.rt, 0xFF, static_cast<size_t>(b2r::dev::kK) * nl * S * 4));
      B2R_CUDA(cudaMemset(st.touched, 0, static_cast<size_t>(b2r::dev::kK) * G * nl * 4));
      B2R_CUDA(cudaMemset(st.best, 0xFF, static_cast<size_t>(nl) * S * 4));
      B2R_CUDA(cudaMemset(st.tmp, 0xFF, static_cast<size_t>(nl) * S * 4));
      B2R_CUDA(cudaMemset(st.X, 0, static_cast<size_t>(nl) * G * 4));
      B2R_CUDA(cudaMemset(st.Y, 0, static_cast<size_t>(nl) * G * 4));
      B2R_CUDA(cudaMemset(st.R, 0, static_cast<size_t>(tt->d.n_routes) * G * 4));
      B2R_CUDA(cudaMemset(st.D, 0, static_cast<size_t>(nl) * G * 4));
      B2R_CUDA(cudaMemset(st.counters, 0, 16 * 4));
      e->gen_query.assign(S, 0);
      e->slot_query.assign(S, -1);
      B2R_CUDA(cudaMallocHost(&e->h_summary, S * sizeof(b2r_engine::summary_t)));
      B2R_CUDA(cudaMallocHost(&e->h_lbcount, sizeof(uint32_t)));
      B2R_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
      B2R_CUDA(cudaStreamCreateWithFlags(&e->stream2, cudaStreamNonBlocking));
      B2R_CUDA(cudaEventCreate(&e->ev0));
      B2R_CUDA(cudaEventCreate(&e->ev1));
      B2R_CUDA(cudaEventCreate(&e->ev_base));
      B2R_CUDA(cudaEventCreate(&e->ev_scan_a));
      B2R_CUDA(cudaEventCreate(&e->ev_scan_b));
      B2R_CUDA(cudaEventCreate(&e->ev2a));
      B2R_CUDA(cudaEventCreate(&e->ev2b));
      B2R_CUDA(cudaEventCreateWithFlags(&e->ev_hdr, cudaEventDisableTiming));
      if (e->cfg.use_graphs) {
        b2r::capture_graph(*e);
        cudaGraph_t g = nullptr;
        B2R_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        b2r::enqueue_lb_chunk(*e, e->stream);
        B2R_CUDA(cudaStreamEndCapture(e->stream, &g));
        B2R_CUDA(cudaGraphInstantiate(&e->lb_graph, g, 0));
        cudaGraphDestroy(g);
      }
      B2R_CUDA(cudaDeviceSynchronize());
      *out = e.release();
      return B2R_OK;
    } catch (b2r::cuda_error const& ex) {
      return b2r::fail(B2R_ERR_CUDA, ex.what());
    }
  });
}

int b2r_engine_destroy(b2r_engine* e) {
  if (e != nullptr && e->serving) b2r_serve_stop(e);
  delete e;
  return B2R_OK;
}

uint64_t b2r_engine_bytes_per_slot(const b2r_engine* e) { return e == nullptr ? 0 : e->bytes_per_slot; }
uint32_t b2r_engine_slots(const b2r_engine* e) { return e == nullptr ? 0 : e->S; }

int b2r_search_batch(b2r_engine* e, const b2r_query* qs, uint32_t n, b2r_result* out) {
  B2R_API_GUARD({
    if (e == nullptr || (n != 0 && (qs == nullptr || out == nullptr))) {
      return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
    }
    if (e->serving) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "engine is serving");
    try {
      B2R_CUDA(cudaSetDevice(e->tt->device));
      b2r::recycle_rows(*e);
      std::vector<b2r::query_run> runs(n);
      auto const t0 = std::chrono::steady_clock::now();
      e->batch_t0 = t0;
      e->prof_used = 0;
      e->prof_rc_used = 0;
      e->lb_ms = 0;
      e->lb_chunks = 0;
      e->h2d_bytes = 0;
      e->d2h_bytes = 0;
      e->aux_launches = 0;
      e->prep_ns = 0;
      e->admit_ms = e->export_ms = e->idle_ms = 0;
      b2r::preparer prep;
      prep.start(*e, qs, n, runs, false);
      b2r::batch_runner br{*e, runs, e->cfg.use_graphs != 0 && e->graph != nullptr};
      if (e->cfg.profile) B2R_CUDA(cudaMemsetAsync(e->st.prof, 0, 8 * sizeof(unsigned long long), e->stream));
      e->scan_ms = 0;
      e->scan_launches = 0;
      br.run(e->cfg.profile == 2U ? 1U : e->shape.steps_per_sync);
      prep.join();
      auto const t1 = std::chrono::steady_clock::now();
      B2R_CUDA(cudaStreamSynchronize(e->stream));
      e->last = {};
      e->last.device_ms = br.busy_ms;
      e->last.host_prep_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();  // wall of the call
      e->last.kernel_launches = br.launches + e->aux_launches;
      e->last.super_steps = br.steps;
      e->last.lb_ms = e->lb_ms;
      e->last.lb_iterations = e->lb_chunks * 8;
      e->last.h2d_bytes = e->h2d_bytes;
      e->last.d2h_bytes = e->d2h_bytes;
      e->last.host_prep_cpu_ms = static_cast<double>(e->prep_ns.load()) / 1e6;
      e->last.host_admit_ms = e->admit_ms;
      e->last.host_export_ms = e->export_ms;
      e->last.host_idle_ms = e->idle_ms;
      if (e->cfg.profile == 2U) {
        e->last.route_scan_launches = e->scan_launches;
        e->last.route_scan_ms = e->scan_ms;
      } else if (e->cfg.profile) {
        double scan_ms = 0;
        for (size_t i = 0; i + 1 < e->prof_used; i += 2) {
          float x = 0;
          cudaEventElapsedTime(&x, e->prof_ev[i], e->prof_ev[i + 1]);
          scan_ms += x;
        }
        unsigned long long c[8] = {};
        B2R_CUDA(cudaMemcpy(c, e->st.prof, sizeof(c), cudaMemcpyDeviceToHost));
        e->last.route_scan_launches = e->prof_used / 2;
        e->last.route_scan_ms = scan_ms;
        e->last.route_stop_visits = c[0];
        e->last.et_events = c[1];
        e->last.et_days = c[2];
        e->last.label_writes = c[3];
        // byte model of the route phase: per scanned stop of a query the
        // stop word (4 B), its previous-round label (2 B) and one event time
        // (2 B); per trip search 2 B per examined event and 8 B per examined
        // service day; 2 B per label write
        e->last.route_scan_bytes = c[0] * 8ull + c[1] * 2ull + c[2] * 8ull + c[3] * 2ull;
        e->last.lb_relaxations = c[4];
        e->last.route_warp_steps = c[5];
        double rc_ms = 0;
        for (size_t i = 0; i + 1 < e->prof_rc_used; i += 2) {
          float x = 0;
          cudaEventElapsedTime(&x, e->prof_rc_ev[i], e->prof_rc_ev[i + 1]);
          rc_ms += x;
        }
        e->last.recon_ms = rc_ms;
        e->last.recon_max_journey_us = static_cast<double>(c[6]) / 1e3;
        e->last.recon_journeys = c[7];
      }
      uint32_t err = 0;
      B2R_CUDA(cudaMemcpy(&err, e->st.counters + b2r::dev::C_ERR, 4, cudaMemcpyDeviceToHost));
      if (err != 0) {
        B2R_CUDA(cudaMemset(e->st.counters + b2r::dev::C_ERR, 0, 4));
        for (auto& r : runs) {
          r.status = B2R_ERR_DEVICE_STATUS;
          r.res.view.status = B2R_ERR_DEVICE_STATUS;
        }
      }
      b2r::fill_out(*e, runs, out);
      return err != 0 ? b2r::fail(B2R_ERR_DEVICE_STATUS, "device status word set") : B2R_OK;
    } catch (b2r::cuda_error const& ex) {
      return b2r::fail(B2R_ERR_CUDA, ex.what());
    }
  });
}

int b2r_search_plain(b2r_engine* e, const b2r_query* q, b2r_result* out) {
  B2R_API_GUARD({
    if (e == nullptr || q == nullptr || out == nullptr) {
      return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
    }
    try {
      B2R_CUDA(cudaSetDevice(e->tt->device));
      b2r::recycle_rows(*e);
      std::vector<b2r::query_run> runs(1);
      e->aux_launches = 0;
      b2r::preparer prep;
      prep.start(*e, q, 1, runs, true);
      b2r::batch_runner br{*e, runs, false};
      br.run(1);
      e->last = {};
      e->last.kernel_launches = br.launches + e->aux_launches;
      e->last.super_steps = br.steps;
      b2r::fill_out(*e, runs, out);
      return B2R_OK;
    } catch (b2r::cuda_error const& ex) {
      return b2r::fail(B2R_ERR_CUDA, ex.what());
    }
  });
}

int b2r_engine_get_shape(const b2r_engine* e, b2r_launch_shape* out) {
  if (e == nullptr || out == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
  *out = e->shape;
  return B2R_OK;
}

int b2r_engine_set_shape(b2r_engine* e, const b2r_launch_shape* sh) {
  B2R_API_GUARD({
    if (e == nullptr || sh == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
    if (e->serving) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "engine is serving");
    auto const ok = sh->scan_blocks_per_sm >= 1 && sh->scan_blocks_per_sm <= 64 &&
                    sh->scan_threads >= 32 && sh->scan_threads <= 256 && sh->scan_threads % 32 == 0 &&
                    sh->pair_blocks_per_sm >= 1 && sh->pair_blocks_per_sm <= 64 &&
                    sh->recon_blocks_per_sm >= 1 && sh->recon_blocks_per_sm <= 64 &&
                    sh->steps_per_sync >= 1 && sh->steps_per_sync <= 64 && sh->scan_occupancy <= 2;
    if (!ok) {
      return b2r::fail(B2R_ERR_INVALID_ARGUMENT,
                       "launch shape out of range (blocks per SM 1..64, scan threads 32..256 in steps "
                       "of 32, steps per sync 1..64, scan occupancy 0..2)");
    }
    try {
      B2R_CUDA(cudaSetDevice(e->tt->device));
      e->shape = *sh;
      if (e->graph != nullptr) {  // the graph holds the old launch configuration
        B2R_CUDA(cudaStreamSynchronize(e->stream));
        cudaGraphExecDestroy(e->graph);
        e->graph = nullptr;
        b2r::capture_graph(*e);
      }
      return B2R_OK;
    } catch (b2r::cuda_error const& ex) {
      return b2r::fail(B2R_ERR_CUDA, ex.what());
    }
  });
}

int b2r_engine_autotune(b2r_engine* e, const b2r_query* sample, uint32_t n, b2r_tune_report* report) {
  B2R_API_GUARD({
    if (e == nullptr || sample == nullptr || n == 0) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
    if (e->serving) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "engine is serving");
    std::vector<b2r_result> out(n);
    // objective: wall time of the sample batch (best of three runs)
    auto const measure = [&](b2r_launch_shape const& sh) -> double {
      if (auto const rc = b2r_engine_set_shape(e, &sh); rc != B2R_OK) throw b2r::cuda_error(b2r_last_error());
      auto best = 1e300;
      for (auto rep = 0; rep != 3; ++rep) {
        if (b2r_search_batch(e, sample, n, out.data()) != B2R_OK) throw b2r::cuda_error(b2r_last_error());
        best = std::min(best, e->last.host_prep_ms);
      }
      return best;
    };
    try {
      b2r_tune_report rep{};
      auto cur = e->shape;
      rep.start = cur;
      if (b2r_search_batch(e, sample, n, out.data()) != B2R_OK) return B2R_ERR_INTERNAL;  // warm-up
      auto cur_ms = measure(cur);
      rep.start_ms = cur_ms;
      rep.n_tried = 1;
      // coordinate descent over the knobs, repeated until a pass changes
      // nothing (at most three passes)
      struct knob {
        uint32_t b2r_launch_shape::*field;
        std::vector<uint32_t> values;
      };
      std::vector<knob> const knobs = {{&b2r_launch_shape::scan_blocks_per_sm, {2, 4, 8, 16, 32}},
                                       {&b2r_launch_shape::scan_threads, {128, 256}},
                                       {&b2r_launch_shape::pair_blocks_per_sm, {2, 4, 8, 16}},
                                       {&b2r_launch_shape::recon_blocks_per_sm, {1, 2, 4, 8}},
                                       {&b2r_launch_shape::steps_per_sync, {1, 2, 4, 8}},
                                       {&b2r_launch_shape::scan_occupancy, {0, 1, 2}}};
      for (auto pass = 0; pass != 3; ++pass) {
        auto changed = false;
        for (auto const& k : knobs) {
          auto const at_start = cur.*(k.field);
          for (auto const v : k.values) {
            if (cur.*(k.field) == v) continue;
            auto trial = cur;
            trial.*(k.field) = v;
            auto const ms = measure(trial);
            ++rep.n_tried;
            if (ms < cur_ms) {
              cur = trial;
              cur_ms = ms;
            }
          }
          changed = changed || cur.*(k.field) != at_start;
        }
        if (!changed) break;
        cur_ms = measure(cur);  // re-measured: the first figure may have been a lucky one
      }
      // the start and the pick measured once more side by side, so that a
      // lucky early figure cannot leave a slower shape in place
      auto const start_again = measure(rep.start);
      auto const best_again = measure(cur);
      rep.n_tried += 2;
      rep.start_ms = start_again;
      if (start_again < best_again) {
        cur = rep.start;
        cur_ms = start_again;
      } else {
        cur_ms = best_again;
      }
      if (b2r_engine_set_shape(e, &cur) != B2R_OK) return B2R_ERR_CUDA;
      rep.best = cur;
      rep.best_ms = cur_ms;
      if (report != nullptr) *report = rep;
      return B2R_OK;
    } catch (b2r::cuda_error const& ex) {
      return b2r::fail(B2R_ERR_CUDA, ex.what());
    }
  });
}

int b2r_last_batch_scan_profile(const b2r_engine* e, double* scan_ms, uint64_t* entries,
                                uint64_t* stop_visits, uint32_t cap, uint32_t* n) {
  B2R_API_GUARD({
    if (e == nullptr || n == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
    if (e->cfg.profile != 1U) return b2r::fail(B2R_ERR_UNSUPPORTED, "engine was not created with profile = 1");
    auto const launches = static_cast<uint32_t>(std::min<size_t>(e->prof_used / 2, b2r_engine::kProfRows));
    *n = launches;
    auto const m = std::min(cap, launches);
    if (m == 0) return B2R_OK;
    if (scan_ms == nullptr || entries == nullptr || stop_visits == nullptr) {
      return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null output array");
    }
    std::vector<unsigned long long> rows(2 * m);
    if (cudaMemcpy(rows.data(), e->d_prof_rows, rows.size() * sizeof(unsigned long long),
                   cudaMemcpyDeviceToHost) != cudaSuccess) {
      return b2r::fail(B2R_ERR_CUDA, "reading the profile rows failed");
    }
    unsigned long long prev = 0;
    for (auto i = 0U; i != m; ++i) {
      float ms = 0;
      cudaEventElapsedTime(&ms, e->prof_ev[2 * i], e->prof_ev[2 * i + 1]);
      scan_ms[i] = ms;
      entries[i] = rows[2 * i];
      stop_visits[i] = rows[2 * i + 1] - prev;
      prev = rows[2 * i + 1];
    }
    return B2R_OK;
  });
}

int b2r_last_batch_stats(const b2r_engine* e, b2r_batch_stats* s) {
  if (e == nullptr || s == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
  *s = e->last;
  return B2R_OK;
}

// ------------------------------------------------------------------ serving
int b2r_serve_start(b2r_engine* e) {
  B2R_API_GUARD({
    if (e == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
    if (e->serving) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "engine is already serving");
    try {  // page-locked rows for the one-to-all results the loop exports
      B2R_CUDA(cudaSetDevice(e->tt->device));
      b2r::prewarm_rows(*e, 64, size_t{1} << 30);
    } catch (std::exception const& ex) {
      return b2r::fail(B2R_ERR_CUDA, ex.what());
    }
    auto ss = std::make_shared<b2r::serve_state>(*e);
    auto const hw = std::max(1U, std::thread::hardware_concurrency());
    auto const n_prep = e->cfg.host_threads != 0 ? e->cfg.host_threads : std::max(1U, std::min(8U, hw / 2));
    for (auto i = 0U; i != n_prep; ++i) ss->prep_pool.emplace_back([p = ss.get()] { p->prep_loop(); });
    ss->driver = std::thread([p = ss.get()] { p->driver_loop(); });
    e->serve = ss;
    e->serving = true;
    return B2R_OK;
  });
}

int b2r_serve_stop(b2r_engine* e) {
  B2R_API_GUARD({
    if (e == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
    if (!e->serving) return B2R_OK;
    auto* ss = b2r::serving_of(e);
    {
      std::lock_guard<std::mutex> lock{ss->mu};
      ss->stop = true;
    }
    ss->cv_prep.notify_all();
    ss->cv_driver.notify_all();
    for (auto& t : ss->prep_pool) t.join();
    ss->prep_pool.clear();
    {
      std::lock_guard<std::mutex> lock{ss->mu};  // nothing is prepared any more
      ss->cv_driver.notify_all();
    }
    if (ss->driver.joinable()) ss->driver.join();
    e->serving = false;  // finished results stay readable until released
    return ss->failed_status == B2R_OK ? B2R_OK : b2r::fail(ss->failed_status, ss->failed_msg);
  });
}

int b2r_submit(b2r_engine* e, const b2r_query* q, uint64_t* ticket) {
  B2R_API_GUARD({
    if (e == nullptr || q == nullptr || ticket == nullptr) {
      return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
    }
    if (!e->serving) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "engine is not serving (b2r_serve_start)");
    auto* ss = b2r::serving_of(e);
    auto it = std::make_unique<b2r::serve_item>();
    it->q = *q;
    it->start.assign(q->start, q->start + (q->start != nullptr ? q->n_start : 0U));
    it->dest.assign(q->destination, q->destination + (q->destination != nullptr ? q->n_destination : 0U));
    it->q.start = it->start.data();
    it->q.n_start = static_cast<uint32_t>(it->start.size());
    it->q.destination = it->dest.data();
    it->q.n_destination = static_cast<uint32_t>(it->dest.size());
    it->t_submit = std::chrono::steady_clock::now();
    std::lock_guard<std::mutex> lock{ss->mu};
    if (ss->stop) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "engine is stopping");
    if (ss->failed_status != B2R_OK) return b2r::fail(ss->failed_status, ss->failed_msg);
    it->ticket = ss->next_ticket++;
    *ticket = it->ticket;
    auto* raw = it.get();
    ss->items.emplace(it->ticket, std::move(it));
    ss->to_prepare.push_back(raw);
    ++ss->unfinished;
    ss->cv_prep.notify_one();
    return B2R_OK;
  });
}

namespace {
int serve_result(b2r_engine* e, uint64_t ticket, b2r_result* out, bool block) {
  B2R_API_GUARD({
    if (e == nullptr || out == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
    auto* ss = b2r::serving_of(e);
    if (ss == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "engine never served");
    std::unique_lock<std::mutex> lock{ss->mu};
    auto const found = ss->items.find(ticket);
    if (found == ss->items.end()) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "unknown ticket");
    auto& it = *found->second;
    if (block) ss->cv_done.wait(lock, [&] { return it.finished; });
    if (!it.finished) return B2R_ERR_NOT_READY;
    *out = it.run.res.view;
    return B2R_OK;
  });
}
}  // namespace

int b2r_poll(b2r_engine* e, uint64_t ticket, b2r_result* out) { return serve_result(e, ticket, out, false); }
int b2r_wait(b2r_engine* e, uint64_t ticket, b2r_result* out) { return serve_result(e, ticket, out, true); }

int b2r_release(b2r_engine* e, uint64_t ticket) {
  B2R_API_GUARD({
    if (e == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
    auto* ss = b2r::serving_of(e);
    if (ss == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "engine never served");
    std::lock_guard<std::mutex> lock{ss->mu};
    auto const found = ss->items.find(ticket);
    if (found == ss->items.end()) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "unknown ticket");
    if (!found->second->finished) return b2r::fail(B2R_ERR_NOT_READY, "ticket still running");
    b2r::give_rows(*e, std::move(found->second->run.res.rt_rows));
    ss->items.erase(found);
    return B2R_OK;
  });
}

int b2r_serve_stats(const b2r_engine* e, b2r_batch_stats* out) {
  B2R_API_GUARD({
    if (e == nullptr || out == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
    auto* ss = static_cast<b2r::serve_state const*>(e->serve.get());
    if (ss == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "engine never served");
    *out = b2r_batch_stats{};
    out->super_steps = ss->n_steps.load();
    out->kernel_launches = ss->n_launches.load();
    out->host_admit_ms = static_cast<double>(ss->admit_ns.load()) / 1e6;
    out->host_export_ms = static_cast<double>(ss->export_ns.load()) / 1e6;
    out->host_idle_ms = static_cast<double>(ss->idle_ns.load()) / 1e6;
    out->host_prep_cpu_ms = static_cast<double>(ss->prep_ns.load()) / 1e6;
    out->device_ms = static_cast<double>(ss->sync_ns.load()) / 1e6;
    return B2R_OK;
  });
}

}  // extern "C"

// ------------------------------------------------------------ the Algo concept
// routing::search<Dir, Algo>'s Algo over the engine: one query's raptor
// state in slot 0 of a 32-slot engine.  Each execute is one admission of a
// single start-time group (the start labels added since next_start_time);
// round times and time_at_dest carry over from the previous execute unless
// reset_arrivals came in between, as raptor_state's do.  Results come back
// as the slot's collected journeys; legs are rebuilt on request from the
// round times the last execute left.
struct b2r_search_plan_impl {
  b2r_search_plan view{};
  b2r::prepped_query p;  // the whole preparation (interval extension reads it)
  std::vector<b2r_start> starts;
  std::vector<uint32_t> dests;
  std::vector<uint16_t> dist, lb;
  void set_starts(std::vector<b2r::start_label> const& v) {
    starts.clear();
    for (auto const& s : v) starts.push_back({s.time_at_start, s.time_at_stop, s.stop});
    view.n_starts = static_cast<uint32_t>(starts.size());
    view.starts = starts.data();
  }
};

struct b2r_raptor {
  b2r_engine* e{nullptr};
  b2r::prepped_query tmpl;              // the constructor's arguments
  std::vector<b2r::start_label> starts;  // added since next_start_time
  bool fresh{true};                      // reset_arrivals since the last execute
  bool lb_sent{false};                   // the lower-bound column is on the device
  bool executed{false};
  b2r::dev::slot_t sl{};                 // slot 0 as the last execute left it
  uint64_t n_rounds{0};
  ~b2r_raptor() {
    if (e != nullptr) b2r_engine_destroy(e);
  }
};

namespace b2r {
namespace {

// super-steps until slot 0's phase is over; its summary
dev::slot_summary run_slot0(b2r_engine& e) {
  auto* st = e.stream;
  for (uint64_t step = 0;; ++step) {
    if (step > 100000) throw std::runtime_error("super-step cap exceeded");
    if (e.cfg.use_graphs != 0 && e.graph != nullptr) {
      B2R_CUDA(cudaGraphLaunch(e.graph, st));
    } else {
      enqueue_superstep(e, st);
      B2R_CUDA(cudaGetLastError());
    }
    B2R_CUDA(cudaMemcpyAsync(e.h_summary, e.d_summary, sizeof(b2r_engine::summary_t), cudaMemcpyDeviceToHost, st));
    B2R_CUDA(cudaStreamSynchronize(st));
    auto const state = e.h_summary[0].state;
    if (state == dev::S_DONE || state == dev::S_ERROR) return e.h_summary[0];
  }
}

}  // namespace
}  // namespace b2r

extern "C" {

int b2r_search_prepare(const b2r_timetable* tt, const b2r_query* q, b2r_search_plan** out) {
  B2R_API_GUARD({
    if (tt == nullptr || q == nullptr || out == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
    if (q->kind != B2R_ONE_TO_ONE || q->algorithm != B2R_ALGO_RAPTOR) {
      return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "b2r_search_prepare: one-to-one raptor queries only");
    }
    b2r::prepped_query p;
    b2r::prepare(tt->view, *q, 1, p);  // lower bounds by the reference's Dijkstra on the host
    auto x = std::make_unique<b2r_search_plan_impl>();
    auto& v = x->view;
    v.status = p.status;
    v.direction = q->direction;
    v.ontrip = p.ontrip ? 1 : 0;
    v.start_dest_overlap = p.empty_result ? 1 : 0;
    v.max_transfers = q->max_transfers;
    v.base_day = p.base_days;
    v.interval_from = p.iv_from;
    v.interval_to = p.iv_to;
    v.fastest_direct = p.fastest_direct;
    v.max_travel_time = p.max_travel_time;
    v.tts_default = p.tts.is_default;
    v.tts_min_transfer_time = p.tts.min_transfer_time;
    v.tts_additional_time = p.tts.additional_time;
    v.tts_factor = p.tts.factor;
    x->set_starts(p.starts);
    if (p.intermodal_dest) {
      x->dist.assign(tt->d.n_loc, uint16_t{0xFFFFu});
      for (auto const& [l, dd] : p.dest_dist) x->dist[l] = dd;
      x->dests.push_back(B2R_SPECIAL_END);
    } else {
      x->dests = p.dest_locs;
    }
    x->lb = p.lb;
    x->p = std::move(p);
    v.n_destinations = static_cast<uint32_t>(x->dests.size());
    v.destinations = x->dests.data();
    v.dist_to_dest = x->dist.empty() ? nullptr : x->dist.data();
    v.lower_bounds = x->lb.empty() ? nullptr : x->lb.data();
    *out = &x.release()->view;
    return B2R_OK;
  });
}

int b2r_search_extend(const b2r_timetable* tt, b2r_search_plan* plan, uint32_t n_missing, uint8_t* changed,
                      uint8_t* reset_arrivals) {
  B2R_API_GUARD({
    if (tt == nullptr || plan == nullptr || changed == nullptr || reset_arrivals == nullptr) {
      return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
    }
    auto* x = reinterpret_cast<b2r_search_plan_impl*>(plan);
    auto& p = x->p;
    *changed = 0;
    *reset_arrivals = 0;
    auto nf = p.iv_from, nt = p.iv_to;
    auto const& d = tt->host;
    if (!b2r::extend_interval(p, d.date_range_from * 1440, d.date_range_to * 1440, n_missing, nf, nt)) {
      return B2R_OK;
    }
    std::vector<b2r::start_label> starts;  // search.h:290-312
    if (nf != p.iv_from) {
      b2r::add_interval_starts(tt->view, p, nf, p.iv_from, !p.fwd, starts);
      if (!p.fwd) *reset_arrivals = 1;
    }
    if (nt != p.iv_to) {
      b2r::add_interval_starts(tt->view, p, p.iv_to, nt, p.fwd, starts);
      if (p.fwd) *reset_arrivals = 1;
    }
    p.iv_from = nf;
    p.iv_to = nt;
    x->view.interval_from = nf;
    x->view.interval_to = nt;
    x->set_starts(starts);
    *changed = 1;
    return B2R_OK;
  });
}

void b2r_search_plan_free(b2r_search_plan* p) {
  // the view is the first member of its owner
  delete reinterpret_cast<b2r_search_plan_impl*>(p);
}

int b2r_raptor_create(b2r_timetable* tt, const b2r_raptor_args* a, b2r_raptor** out) {
  B2R_API_GUARD({
    if (tt == nullptr || a == nullptr || out == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
    if (a->prf_idx >= B2R_N_PROFILES) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "profile index out of range");
    if (a->n_destinations != 0 && a->destinations == nullptr) {
      return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null destination array");
    }
    auto const nl = tt->d.n_loc;
    auto r = std::make_unique<b2r_raptor>();
    auto& p = r->tmpl;
    p.fwd = a->direction == B2R_FORWARD;
    p.ontrip = true;  // one start-time group per execute
    p.allowed_claszes = a->allowed_claszes;
    p.req_flags = static_cast<uint8_t>((a->require_bike_transport != 0 ? 1U << B2R_FLAG_BIKES : 0U) |
                                       (a->require_car_transport != 0 ? 1U << B2R_FLAG_CARS : 0U) |
                                       (a->prf_idx == B2R_PROFILE_WHEELCHAIR ? 1U << B2R_FLAG_WHEELCHAIR : 0U) |
                                       (a->no_compulsory_reservation != 0 ? 1U << B2R_FLAG_RESERVATION_NOT_REQUIRED : 0U));
    p.prf = a->prf_idx;
    p.tts = {a->tts_default, a->tts_min_transfer_time, a->tts_additional_time, a->tts_factor};
    p.tts_raw = p.tts;
    p.base_days = a->base_day;
    auto const base = a->base_day - tt->view.internal_from_days();
    if (base < 0 || base >= B2R_MAX_DAYS) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "base day outside the timetable");
    p.base = static_cast<uint16_t>(base);
    p.intermodal_dest = a->dist_to_dest != nullptr;
    if (p.intermodal_dest) {
      for (auto l = 0U; l != nl; ++l) {
        if (a->dist_to_dest[l] != 0xFFFFu) p.dest_dist.emplace_back(l, a->dist_to_dest[l]);
      }
    } else {
      for (auto i = 0U; i != a->n_destinations; ++i) {
        if (a->destinations[i] >= nl) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "destination out of range");
        p.dest_locs.push_back(a->destinations[i]);
      }
      std::sort(p.dest_locs.begin(), p.dest_locs.end());
      p.dest_locs.erase(std::unique(p.dest_locs.begin(), p.dest_locs.end()), p.dest_locs.end());
    }
    if (a->lower_bounds != nullptr) p.lb.assign(a->lower_bounds, a->lower_bounds + nl);
    p.recon_mode = 2;  // legs on request (b2r_raptor_reconstruct)
    p.fastest_direct = 32767;
    p.max_travel_time = B2R_MAX_TRAVEL_TIME_MIN;
    b2r_engine_config cfg;
    b2r_engine_config_init(&cfg);
    cfg.max_slots = 32;
    cfg.use_lower_bounds = 0;  // the column comes with the arguments
    if (auto const rc = b2r_engine_create(tt, &cfg, &r->e); rc != B2R_OK) return rc;
    if (b2r::check_capacity(*r->e, p) != B2R_OK) {
      return b2r::fail(B2R_ERR_CAPACITY, "b2r_raptor_create: more destinations than a slot holds");
    }
    *out = r.release();
    return B2R_OK;
  });
}

int b2r_raptor_destroy(b2r_raptor* r) {
  delete r;
  return B2R_OK;
}

int b2r_raptor_reset_arrivals(b2r_raptor* r) {
  if (r == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
  r->fresh = true;
  return B2R_OK;
}

int b2r_raptor_next_start_time(b2r_raptor* r) {
  if (r == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
  r->starts.clear();  // best, tmp and marks: the next group's generation
  return B2R_OK;
}

int b2r_raptor_add_start(b2r_raptor* r, uint32_t location, int32_t time) {
  if (r == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
  if (location >= r->e->tt->d.n_loc) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "start location out of range");
  if (r->starts.size() >= r->e->max_starts) return b2r::fail(B2R_ERR_CAPACITY, "too many start labels");
  r->starts.push_back({0, time, location});
  return B2R_OK;
}

int b2r_raptor_execute(b2r_raptor* r, int32_t start_time, uint8_t max_transfers, int32_t worst_time_at_dest,
                       b2r_journey* results, uint32_t capacity, uint32_t* n) {
  B2R_API_GUARD({
    if (r == nullptr || n == nullptr || (capacity != 0 && results == nullptr)) {
      return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
    }
    *n = 0;
    auto& e = *r->e;
    try {
      B2R_CUDA(cudaSetDevice(e.tt->device));
      auto p = r->tmpl;
      for (auto const& s : r->starts) p.starts.push_back({start_time, s.time_at_stop, s.stop});
      p.max_transfers = max_transfers;
      p.end_k = static_cast<uint8_t>(std::min<int>(max_transfers, B2R_MAX_TRANSFERS) + 2);
      auto const span = p.fwd ? static_cast<int64_t>(worst_time_at_dest) - start_time
                              : static_cast<int64_t>(start_time) - worst_time_at_dest;
      p.span = static_cast<int16_t>(std::clamp<int64_t>(span, -32768, 32767));
      p.iv_from = p.iv_to = start_time;
      p.need_sweep = !r->fresh;  // round times of earlier executes stay in effect
      p.keep_lb = r->lb_sent;
      uint32_t const flags = r->fresh ? 0U : b2r::kAdmKeepRt;
      b2r::admit(e, {{0U, &p, flags}}, e.stream);
      auto const sum = b2r::run_slot0(e);
      std::vector<b2r::exported> ex;
      std::vector<uint8_t> const no_legs{b2r::kLegsNone};  // legs on request (b2r_raptor_reconstruct)
      b2r::export_slots(e, {0U}, {sum.n_journeys}, {0U}, ex, e.stream2, &no_legs);
      r->sl = ex[0].sl;
      r->fresh = false;
      r->lb_sent = r->lb_sent || !p.lb.empty();
      r->executed = true;
      r->n_rounds = r->sl.n_rounds;
      if (r->sl.state == b2r::dev::S_ERROR) {
        return b2r::fail(r->sl.error != 0 ? r->sl.error : B2R_ERR_INTERNAL, "execute failed on the device");
      }
      *n = static_cast<uint32_t>(ex[0].js.size());
      if (ex[0].js.size() > capacity) return b2r::fail(B2R_ERR_CAPACITY, "result capacity exceeded");
      for (auto i = 0U; i != ex[0].js.size(); ++i) {
        auto const& j = ex[0].js[i];
        results[i] = b2r_journey{j.start_time, j.dest_time, j.dest, j.transfers, 0, 0, 0};
      }
      return B2R_OK;
    } catch (b2r::cuda_error const& ex) {
      return b2r::fail(B2R_ERR_CUDA, ex.what());
    }
  });
}

int b2r_raptor_reconstruct(b2r_raptor* r, const b2r_query* q, b2r_journey* j, b2r_leg* legs, uint32_t capacity) {
  B2R_API_GUARD({
    if (r == nullptr || q == nullptr || j == nullptr || legs == nullptr) {
      return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
    }
    if (!r->executed) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "b2r_raptor_reconstruct before execute");
    if (capacity < static_cast<uint32_t>(b2r::dev::kMaxLegs)) {
      return b2r::fail(B2R_ERR_CAPACITY, "leg capacity below the longest journey (40 legs)");
    }
    auto& e = *r->e;
    // the query's offsets in query::sanitize's order (query.cc:59-67)
    std::vector<b2r_offset> so(q->start, q->start + (q->start != nullptr ? q->n_start : 0U));
    std::vector<b2r_offset> dz(q->destination, q->destination + (q->destination != nullptr ? q->n_destination : 0U));
    auto const by_dur = [](b2r_offset const& a, b2r_offset const& b) { return a.duration < b.duration; };
    std::sort(so.begin(), so.end(), by_dur);
    std::sort(dz.begin(), dz.end(), by_dur);
    if (so.size() + dz.size() > e.max_off) return b2r::fail(B2R_ERR_CAPACITY, "too many offsets");
    try {
      B2R_CUDA(cudaSetDevice(e.tt->device));
      auto sl = r->sl;
      sl.start_mode = q->start_match_mode;
      sl.dest_mode = q->dest_match_mode;
      sl.ontrip = q->is_interval == 0 ? 1 : 0;
      sl.soff_off = 0;
      sl.n_soff = static_cast<uint32_t>(so.size());
      sl.doff_off = sl.n_soff;
      sl.n_doff = static_cast<uint32_t>(dz.size());
      so.insert(so.end(), dz.begin(), dz.end());
      b2r::dev::journey_rec jr{j->start_time, j->dest_time, j->dest, j->transfers, 0, 0, 0, 0, 0};
      auto* s = e.stream;
      if (!so.empty()) {
        B2R_CUDA(cudaMemcpyAsync(e.st.off_pool, so.data(), so.size() * sizeof(b2r_offset), cudaMemcpyHostToDevice, s));
      }
      B2R_CUDA(cudaMemcpyAsync(e.st.slots, &sl, sizeof(sl), cudaMemcpyHostToDevice, s));
      B2R_CUDA(cudaMemcpyAsync(e.st.journeys, &jr, sizeof(jr), cudaMemcpyHostToDevice, s));
      b2r::dev::k_reconstruct_one<<<1, 32, 0, s>>>(e.st, 0U, 0U);
      B2R_CUDA(cudaGetLastError());
      B2R_CUDA(cudaMemcpyAsync(&jr, e.st.journeys, sizeof(jr), cudaMemcpyDeviceToHost, s));
      B2R_CUDA(cudaMemcpyAsync(legs, e.st.legs, b2r::dev::kMaxLegs * sizeof(b2r_leg), cudaMemcpyDeviceToHost, s));
      B2R_CUDA(cudaStreamSynchronize(s));
      j->error = jr.error;
      j->n_legs = jr.error != 0 ? 0 : jr.n_legs;
      j->first_leg = 0;
      return B2R_OK;
    } catch (b2r::cuda_error const& ex) {
      return b2r::fail(B2R_ERR_CUDA, ex.what());
    }
  });
}

uint64_t b2r_raptor_rounds(const b2r_raptor* r) { return r == nullptr ? 0 : r->n_rounds; }

}  // extern "C"

// ------------------------------------------------------- real-time overlay
// The device arrays of an overlay: the timetable image with the overlay's
// traffic days (transport_bf repointed at appended bitfields) and its runs.
struct b2r_rt {
  b2r_timetable* tt{nullptr};
  b2r::rt_host host;
  b2r::dev::dtt d{};
  std::vector<void*> allocs;
  uint64_t bytes{0};
  ~b2r_rt() {
    for (auto* p : allocs) cudaFree(p);
  }
};

extern "C" {

int b2r_rt_upload(b2r_timetable* tt, const b2r_rt_desc* desc, b2r_rt** out) {
  B2R_API_GUARD({
    if (tt == nullptr || desc == nullptr || out == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
    auto r = std::make_unique<b2r_rt>();
    r->tt = tt;
    auto const nl = tt->d.n_loc, ntr = tt->d.n_transports;
    if (!r->host.init(*desc, nl, ntr)) {
      return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "b2r_rt_upload: malformed overlay");
    }
    auto const& h = r->host;
    try {
      B2R_CUDA(cudaSetDevice(tt->device));
      auto up = [&](auto const* p, size_t n) {
        auto* x = b2r::dupload(p, n, r->bytes);
        r->allocs.push_back(x);
        return x;
      };
      auto& d = r->d;
      d = tt->d;
      // traffic days: the changed transports point at bitfields appended to
      // the timetable's (rt_timetable::transport_traffic_days_ with
      // kRtBitfieldFlag)
      auto const n_bf = static_cast<uint32_t>(tt->host.n_bitfields);
      std::vector<uint32_t> tbf(tt->transport_traffic_days.begin(), tt->transport_traffic_days.end());
      std::vector<uint64_t> bf(tt->bitfields.begin(), tt->bitfields.end());
      bf.insert(bf.end(), h.changed_days.begin(), h.changed_days.end());
      for (auto i = 0U; i != h.changed_transport.size(); ++i) tbf[h.changed_transport[i]] = n_bf + i;
      d.transport_bf = up(tbf.data(), tbf.size());
      d.bf = up(bf.data(), bf.size());
      auto const n_rt = h.d.n_rt_transports;
      d.n_rt = n_rt;
      d.rt_stop_idx = up(h.stop_index.data(), h.stop_index.size());
      d.rt_stops = up(h.stops.data(), h.stops.size());
      d.rt_times = up(h.times.data(), h.times.size());
      std::vector<uint16_t> filt(n_rt);
      for (auto x = 0U; x != n_rt; ++x) {  // class | all-sections flags << 4 | some << 8, as route_filter
        uint32_t all = 0U, some = 0U;
        for (auto f = 0U; f != 4U; ++f) {
          all |= ((h.flags[x] >> (2U * f)) & 1U) << f;
          some |= ((h.flags[x] >> (2U * f + 1U)) & 1U) << f;
        }
        filt[x] = static_cast<uint16_t>(h.clasz[x] | (all << 4) | (some << 8));
      }
      d.rt_filter = up(filt.data(), filt.size());
      d.rt_sec = up(h.section_flags.data(), h.section_flags.size());
      d.rt_static = up(h.static_transport.data(), h.static_transport.size());
      d.rt_static_day = up(h.static_day.data(), h.static_day.size());
      d.loc_rt_idx = up(h.loc_idx.data(), h.loc_idx.size());
      d.loc_rt = up(h.loc_rt.data(), h.loc_rt.size());
      // location -> (run, stop position) in reconstruction's order: the
      // runs of location_rt_transports_, then stop positions ascending
      std::vector<uint32_t> idx(nl + 1U, 0U), xs;
      std::vector<uint16_t> ss;
      for (auto l = 0U; l != nl; ++l) {
        for (auto k = h.loc_idx[l]; k != h.loc_idx[l + 1]; ++k) {
          auto const x = h.loc_rt[k];
          for (auto i = 0U; i != h.n_stops(x); ++i) {
            if (B2R_STOP_LOC(h.stop(x, i)) == l) {
              xs.push_back(x);
              ss.push_back(static_cast<uint16_t>(i));
            }
          }
        }
        idx[l + 1U] = static_cast<uint32_t>(xs.size());
      }
      d.lrs_rt_idx = up(idx.data(), idx.size());
      d.lrs_rt = up(xs.data(), xs.size());
      d.lrs_rt_stop = up(ss.data(), ss.size());
      *out = r.release();
      return B2R_OK;
    } catch (b2r::cuda_error const& ex) {
      return b2r::fail(B2R_ERR_CUDA, ex.what());
    }
  });
}

int b2r_rt_destroy(b2r_rt* rt) {
  delete rt;
  return B2R_OK;
}

int b2r_engine_set_rt(b2r_engine* e, const b2r_rt* rt) {
  B2R_API_GUARD({
    if (e == nullptr) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "null argument");
    if (e->serving) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "engine is serving");
    if (rt != nullptr && rt->tt != e->tt) return b2r::fail(B2R_ERR_INVALID_ARGUMENT, "overlay of another timetable");
    try {
      B2R_CUDA(cudaSetDevice(e->tt->device));
      B2R_CUDA(cudaStreamSynchronize(e->stream));
      auto const n_rt = rt != nullptr ? rt->d.n_rt : 0U;
      if (e->st.RT_R != nullptr) cudaFree(e->st.RT_R);
      if (e->st.rtlist != nullptr) cudaFree(e->st.rtlist);
      e->st.RT_R = nullptr;
      e->st.rtlist = nullptr;
      if (n_rt != 0U) {
        auto const words = static_cast<size_t>(n_rt) * e->G;
        B2R_CUDA(cudaMalloc(&e->st.RT_R, words * sizeof(uint32_t)));
        B2R_CUDA(cudaMalloc(&e->st.rtlist, words * sizeof(uint32_t)));
        B2R_CUDA(cudaMemset(e->st.RT_R, 0, words * sizeof(uint32_t)));
      }
      e->rt = rt;
      e->st.tt = rt != nullptr ? rt->d : e->tt->d;
      e->view = e->tt->view;
      e->view.rt = rt != nullptr ? &rt->host : nullptr;
      if (e->graph != nullptr) {  // the graph holds the old image and kernels
        cudaGraphExecDestroy(e->graph);
        e->graph = nullptr;
        b2r::capture_graph(*e);
      }
      return B2R_OK;
    } catch (b2r::cuda_error const& ex) {
      return b2r::fail(B2R_ERR_CUDA, ex.what());
    }
  });
}

}  // extern "C"
