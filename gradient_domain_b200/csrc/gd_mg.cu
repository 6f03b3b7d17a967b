// Batched cell-centred MGPCG: hierarchy planning, launch sequencing and the
// C ABI of gd_poisson.h.
//
// One plan holds any number of instances (images x channels) of any sizes and
// boundary types.  Every kernel launch covers one step of the V-cycle or of
// the Krylov loop for all instances at once through a tile list, so a batch
// of uneven solves costs the same number of launches as one solve
// (poisson.py:137-145 and :216-242 loop over channels one at a time).
// Levels are aligned at the top: launch `down[l]` / `up[l]` holds level l of
// every instance whose hierarchy reaches below l, and one `bottom` launch
// finishes every instance's small levels.  One Krylov iteration is
//   down[0..D-1], bottom, up[D-1..0], pupdate, cgupdate, fold, resid
// with all scalars on the device, so the host only polls a counter of active
// instances every `check_every` iterations and the iteration can be captured
// once as a CUDA graph.

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "gd_coarse.cuh"
#include "gd_stream.cuh"
#include "gd_tile.cuh"

using namespace gd;

struct gd_plan_s {
  int n = 0;
  int sms = 148;  // SMs of the plan's device (tile launches below one CTA per SM run wider CTAs)
  gd_params prm{};
  bool fp64 = false;
  std::vector<InstInfo> inst;
  std::vector<LevelInfo> lv;
  std::vector<Tile> tiles;
  int fine_base = 0, fine_count = 0, depth = 0;
  std::vector<int> down_base, down_count, up_base, up_count;     // strip maps per level
  std::vector<int> tdown_base, tdown_count, tup_base, tup_count;  // tile maps per level
  std::vector<char> tsmall;  // per level: tiles of the small shape (fewer large tiles than SMs)
  // per strip level: some strip instance is masked (at the level or the next) or
  // too large for 32-bit row offsets, so the launch needs the general strips
  std::vector<char> strip_any;
  size_t arena_elems = 0, code_bytes = 0, dense_elems = 0, xs_elems = 0;
  int max_partials = 1;
  size_t o_lv = 0, o_inst = 0, o_st = 0, o_tiles = 0, o_arena = 0, o_codes = 0, o_dense = 0,
         o_xs = 0, o_p0 = 0, o_p1 = 0, o_cnt = 0, o_nact = 0, o_trip = 0, total = 0;
  size_t bottom_smem = 0;
  // persistent launch of the coarse levels (gd_coarse.cuh): used when the plan has
  // tile levels below its strips and the device takes cooperative launches
  bool persistent = false;
  bool dependent_launch = false;  // chain_launch: programmatic dependent launches
  int coarse_from = 0;   // first level index with no strip launch at or below it
  int coarse_grid = 0;   // CTAs of the persistent launch (at most one per SM)
  coarse::Phases phases{};
  char *ws = nullptr;
  bool prepared = false;
  std::vector<char> mask_set;
  cudaGraphExec_t gexec = nullptr;  // the whole solve: init, device-side while loop, mean
  cudaStream_t cap = nullptr;
  int cap_device = -1;
  long long solves = 0;  // completed solves; the graph is captured from the second on
  int *h_nact = nullptr;
  InstState *h_st = nullptr;
  size_t h_st_bytes = 0;
  InstInfo *h_inst = nullptr;  // pinned staging of the per-solve instance table
  size_t h_inst_bytes = 0;
  cudaEvent_t done_ev = nullptr;  // recorded after the states of an asynchronous solve
  bool pending = false;           // an asynchronous solve awaits gd_solve_finish
  // profiling: events around every launch (graphs are bypassed while enabled)
  bool profiling = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<int> ev_kind;
  std::vector<int> ev_level;
  std::vector<double> ev_cells;
  size_t ev_used = 0;
  double prof_ms[GD_KERNEL_KINDS] = {0};
  double prof_cells[GD_KERNEL_KINDS] = {0};
  long long prof_launches[GD_KERNEL_KINDS] = {0};
  gd_kernel_time prof_level[GD_KERNEL_KINDS * GD_PROFILE_LEVELS] = {};
  std::vector<double> launch_cells;  // fine cells covered by each launch map
  std::vector<double> tile_cells;    // cells covered by the tile maps of each level
  double fine_cells = 0;
};

namespace {

constexpr int kPitchAlign = 4;       // elements; rows start on 16-byte boundaries for FP32
constexpr size_t kArrayAlign = 256;  // bytes

// Process-wide recycling of the small pinned host blocks and capture streams
// that every plan needs.  Allocating and freeing page-locked memory
// synchronises the whole device, which would stall every other stream each
// time a served request brings a new plan shape; recycled blocks cost nothing.
struct HostPools {
  std::mutex mu;
  std::multimap<size_t, void *> pinned;         // size class -> free block
  std::multimap<int, cudaStream_t> streams;     // device -> free capture stream
};

HostPools &pools() {
  static HostPools *h = new HostPools();  // never destroyed: used until process exit
  return *h;
}

size_t pinned_class(size_t bytes) {
  size_t c = 256;
  while (c < bytes) c <<= 1;
  return c;
}

void *pinned_get(size_t bytes) {
  const size_t c = pinned_class(bytes);
  {
    std::lock_guard<std::mutex> g(pools().mu);
    auto it = pools().pinned.find(c);
    if (it != pools().pinned.end()) {
      void *b = it->second;
      pools().pinned.erase(it);
      return b;
    }
  }
  void *b = nullptr;
  return cudaMallocHost(&b, c) == cudaSuccess ? b : nullptr;
}

void pinned_put(void *b, size_t bytes) {
  if (!b) return;
  std::lock_guard<std::mutex> g(pools().mu);
  pools().pinned.emplace(pinned_class(bytes), b);
}

cudaError_t capture_stream_get(int device, cudaStream_t *out) {
  {
    std::lock_guard<std::mutex> g(pools().mu);
    auto it = pools().streams.find(device);
    if (it != pools().streams.end()) {
      *out = it->second;
      pools().streams.erase(it);
      return cudaSuccess;
    }
  }
  return cudaStreamCreateWithFlags(out, cudaStreamNonBlocking);
}

void capture_stream_put(int device, cudaStream_t s) {
  if (!s) return;
  std::lock_guard<std::mutex> g(pools().mu);
  pools().streams.emplace(device, s);
}

// Record an event before a launch of `kind` covering `cells` grid cells of
// multigrid level `level` (0 for launches not tied to one level).
void prof_begin(gd_plan p, int kind, double cells, cudaStream_t st, int level = 0) {
  if (!p->profiling) return;
  while (p->ev_pool.size() < p->ev_used + 2) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    p->ev_pool.push_back(e);
  }
  if (p->ev_kind.size() < p->ev_used + 2) {
    p->ev_kind.resize(p->ev_used + 2);
    p->ev_level.resize(p->ev_used + 2);
    p->ev_cells.resize(p->ev_used + 2);
  }
  p->ev_kind[p->ev_used] = kind;
  p->ev_level[p->ev_used] = std::min(std::max(level, 0), GD_PROFILE_LEVELS - 1);
  p->ev_cells[p->ev_used] = cells;
  cudaEventRecord(p->ev_pool[p->ev_used], st);
  p->ev_used += 1;
}

void prof_end(gd_plan p, cudaStream_t st) {
  if (!p->profiling) return;
  p->ev_kind[p->ev_used] = -1;
  cudaEventRecord(p->ev_pool[p->ev_used], st);
  p->ev_used += 1;
}

// After a synchronize: fold the recorded pairs into the per-kind totals.
void prof_collect(gd_plan p) {
  for (size_t k = 0; k + 1 < p->ev_used; k += 2) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, p->ev_pool[k], p->ev_pool[k + 1]);
    const int kind = p->ev_kind[k];
    p->prof_ms[kind] += ms;
    p->prof_cells[kind] += p->ev_cells[k];
    p->prof_launches[kind] += 1;
    gd_kernel_time &t = p->prof_level[kind * GD_PROFILE_LEVELS + p->ev_level[k]];
    t.milliseconds += ms;
    t.cells += p->ev_cells[k];
    t.launches += 1;
  }
  p->ev_used = 0;
}

// Launch of a kernel of the solve chain.  With the plan's dependent-launch
// flag the launch carries the programmatic-serialization attribute: the
// kernel may be scheduled while the one ahead of it is finishing and waits for
// it inside (dep_wait), so the launch gap and the kernel's table reads overlap
// the previous kernel's tail.  Errors are left for cudaGetLastError.
template <typename... KP, typename... AT>
void chain_launch(gd_plan p, void (*kernel)(KP...), int grid, int block, size_t smem,
                  cudaStream_t st, AT &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = p->dependent_launch ? 1 : 0;
  cudaLaunchKernelEx(&cfg, kernel, std::forward<AT>(args)...);
}

// Strip geometry of the down / up kernels for a plan's precision and sweeps.
template <typename T, int S>
struct StripCfg {
  static constexpr int down_ow = st::DownGeom<T, S>::H::OW;
  static constexpr int up_ow = st::UpGeom<T, S, S>::H::OW;
};

template <typename T>
struct Runner {
  template <int S>
  static void set_attrs() {
    cudaFuncSetAttribute(k_bottom<T, S, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kBottomSmem);
    cudaFuncSetAttribute(st::k_down_s<T, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)down_smem<S>(false));
    cudaFuncSetAttribute(st::k_up_s<T, S, S, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)up_smem<S, true>(false));
    cudaFuncSetAttribute(st::k_up_s<T, S, S, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)up_smem<S, false>(false));
    if constexpr (sizeof(T) == 4) {
      cudaFuncSetAttribute(st::k_down_s<T, S, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)down_smem<S>(true));
      cudaFuncSetAttribute(st::k_up_s<T, S, S, true, false>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)up_smem<S, true>(true));
      cudaFuncSetAttribute(st::k_up_s<T, S, S, false, false>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)up_smem<S, false>(true));
    }
    cudaFuncSetAttribute(tile::k_down_t<T, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)tile::DownT<T, S>::smem);
    cudaFuncSetAttribute(tile::k_up_t<T, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)tile::UpT<T, S>::smem);
    cudaFuncSetAttribute(small_down<S>(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)SmallDown<S>::smem);
    cudaFuncSetAttribute(small_up<S>(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)SmallUp<S>::smem);
    cudaFuncSetAttribute(st::k_pupdate_s<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)st::pupdate_smem<T>());
    cudaFuncSetAttribute(st::k_cgupdate_s<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)st::cgupdate_smem<T>());
    cudaFuncSetAttribute(st::k_refresh_s<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)st::refresh_smem<T>());
    cudaFuncSetAttribute(st::k_refresh_s<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)st::refresh_smem<T>());
    cudaFuncSetAttribute(coarse::k_coarse<T, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)coarse_smem_max<S>());
  }

  // Small-tile forms of the tile kernels (levels with fewer large tiles than SMs).
  template <int S>
  using SmallDown = tile::DownT<T, S, tile::kTYs, tile::kTXs>;
  template <int S>
  using SmallUp = tile::UpT<T, S, tile::kTYs, tile::kTXs>;
  template <int S>
  static constexpr auto small_down() {
    return tile::k_down_t<T, S, tile::kThreadsSmall, tile::kTYs, tile::kTXs>;
  }
  template <int S>
  static constexpr auto small_up() {
    return tile::k_up_t<T, S, tile::kThreadsSmall, tile::kTYs, tile::kTXs>;
  }

  // Shared memory of the persistent coarse launch (whose tile levels are all
  // small-tile levels): the larger of the bottom's (at most kBottomSmem) and a
  // small tile's.
  template <int S>
  static constexpr size_t coarse_smem_max() {
    return std::max<size_t>((size_t)kBottomSmem, std::max(SmallDown<S>::smem, SmallUp<S>::smem));
  }

  // The coarse levels and the bottom in one cooperative launch; false when the
  // launch was refused (the caller then runs them level by level, and the plan
  // stops using the persistent form).
  template <int S>
  static bool launch_coarse(gd_plan p, const Args<T> &a, cudaStream_t st) {
    const size_t smem = std::max(p->bottom_smem, std::max(SmallDown<S>::smem, SmallUp<S>::smem));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)p->coarse_grid);
    cfg.blockDim = dim3(kBThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    prof_begin(p, GD_K_COARSE, 0.0, st);
    const cudaError_t e = cudaLaunchKernelEx(&cfg, coarse::k_coarse<T, S>, a, p->phases);
    prof_end(p, st);
    if (e != cudaSuccess) {
      cudaGetLastError();
      p->persistent = false;
      return false;
    }
    return true;
  }

  static Args<T> args(gd_plan p) {
    Args<T> a;
    a.lv = reinterpret_cast<const LevelInfo *>(p->ws + p->o_lv);
    a.inst = reinterpret_cast<const InstInfo *>(p->ws + p->o_inst);
    a.st = reinterpret_cast<InstState *>(p->ws + p->o_st);
    a.arena = reinterpret_cast<T *>(p->ws + p->o_arena);
    a.xs = reinterpret_cast<double *>(p->ws + p->o_xs);
    a.codes = reinterpret_cast<const unsigned char *>(p->ws + p->o_codes);
    a.dense = reinterpret_cast<const double *>(p->ws + p->o_dense);
    a.part0 = reinterpret_cast<double *>(p->ws + p->o_p0);
    a.part1 = reinterpret_cast<double *>(p->ws + p->o_p1);
    a.counter = reinterpret_cast<unsigned *>(p->ws + p->o_cnt);
    a.n_active = reinterpret_cast<int *>(p->ws + p->o_nact);
    a.tiles = reinterpret_cast<const Tile *>(p->ws + p->o_tiles);
    a.ninst = p->n;
    a.tol2 = p->prm.tolerance * p->prm.tolerance;
    a.delta2 = p->fp64 ? 0.0 : p->prm.reliable_delta * p->prm.reliable_delta;
    a.max_iter = p->prm.max_iterations;
    a.zero_start = p->prm.zero_start != 0;
    return a;
  }

  static Args<T> at_tiles(Args<T> a, int base) {
    a.tiles += base;
    return a;
  }

  // Levels whose strip instances are all rectangles run the rectangle-only
  // strip kernels (FP32), which fit more CTAs per SM.
  static bool rect_only(gd_plan p, int l) { return sizeof(T) == 4 && !p->strip_any[l]; }

  // Dynamic shared memory of the strip kernels (rectangle-only forms or not).
  template <int S>
  static size_t down_smem(bool rect) {
    return rect ? st::strip_smem<T, S, false, false>() : st::strip_smem<T, S, false>();
  }
  template <int S, bool LEVEL0>
  static size_t up_smem(bool rect) {
    constexpr int NT = st::UpCta<LEVEL0>::NT;
    return rect ? st::strip_smem<T, S, true, false, NT>() : st::strip_smem<T, S, true, true, NT>();
  }

  template <int S>
  static void down_level(gd_plan p, const Args<T> &a, cudaStream_t st, int l) {
    if (p->down_count[l] > 0) {
      prof_begin(p, l == 0 ? GD_K_DOWN0 : GD_K_DOWN, p->launch_cells[2 * l], st, l);
      if (rect_only(p, l))
        chain_launch(p, st::k_down_s<T, S, false>, p->down_count[l], st::kSThreads,
                     down_smem<S>(true), st, at_tiles(a, p->down_base[l]));
      else
        chain_launch(p, st::k_down_s<T, S>, p->down_count[l], st::kSThreads,
                     down_smem<S>(false), st, at_tiles(a, p->down_base[l]));
      prof_end(p, st);
    }
    if (p->tdown_count[l] > 0) {
      prof_begin(p, GD_K_DOWN, p->tile_cells[l], st, l);
      if (p->tsmall[l])
        chain_launch(p, small_down<S>(), p->tdown_count[l], tile::kThreadsSmall,
                     SmallDown<S>::smem, st, at_tiles(a, p->tdown_base[l]));
      else
        chain_launch(p, tile::k_down_t<T, S>, p->tdown_count[l], tile::kThreads,
                     tile::DownT<T, S>::smem, st, at_tiles(a, p->tdown_base[l]));
      prof_end(p, st);
    }
  }

  template <int S>
  static void up_level(gd_plan p, const Args<T> &a, cudaStream_t st, int l) {
    if (p->tup_count[l] > 0) {
      prof_begin(p, GD_K_UP, p->tile_cells[l], st, l);
      if (p->tsmall[l])
        chain_launch(p, small_up<S>(), p->tup_count[l], tile::kThreadsSmall, SmallUp<S>::smem,
                     st, at_tiles(a, p->tup_base[l]));
      else
        chain_launch(p, tile::k_up_t<T, S>, p->tup_count[l], tile::kThreads,
                     tile::UpT<T, S>::smem, st, at_tiles(a, p->tup_base[l]));
      prof_end(p, st);
    }
    if (p->up_count[l] <= 0) return;
    prof_begin(p, l == 0 ? GD_K_UP0 : GD_K_UP, p->launch_cells[2 * l + 1], st, l);
    const Args<T> at = at_tiles(a, p->up_base[l]);
    const int n = p->up_count[l];
    constexpr int NT0 = st::UpCta<true>::NT, NT1 = st::UpCta<false>::NT;
    const bool rect = rect_only(p, l);
    if (rect && l == 0)
      chain_launch(p, st::k_up_s<T, S, S, true, false>, n, NT0, up_smem<S, true>(true), st, at);
    else if (rect)
      chain_launch(p, st::k_up_s<T, S, S, false, false>, n, NT1, up_smem<S, false>(true), st, at);
    else if (l == 0)
      chain_launch(p, st::k_up_s<T, S, S, true>, n, NT0, up_smem<S, true>(false), st, at);
    else
      chain_launch(p, st::k_up_s<T, S, S, false>, n, NT1, up_smem<S, false>(false), st, at);
    prof_end(p, st);
  }

  // Levels at and below coarse_from (no strips there) and the bottom go to the
  // persistent launch when the plan uses it, else one launch per level.
  template <int S>
  static void vcycle(gd_plan p, const Args<T> &a, cudaStream_t st) {
    const int top = p->persistent ? p->coarse_from : p->depth;
    for (int l = 0; l < top; ++l) down_level<S>(p, a, st, l);
    if (!(p->persistent && launch_coarse<S>(p, a, st))) {
      for (int l = top; l < p->depth; ++l) down_level<S>(p, a, st, l);
      prof_begin(p, GD_K_BOTTOM, 0.0, st, p->depth);
      chain_launch(p, k_bottom<T, S, S>, p->n, kBThreads, p->bottom_smem, st, a);
      prof_end(p, st);
      for (int l = p->depth - 1; l >= top; --l) up_level<S>(p, a, st, l);
    }
    for (int l = top - 1; l >= 0; --l) up_level<S>(p, a, st, l);
  }

  // One Krylov iteration; `refresh` false leaves out the FP64 refresh, which
  // the solve graph launches behind a conditional node instead.
  template <int S>
  static void iteration(gd_plan p, const Args<T> &a, cudaStream_t st, bool refresh) {
    vcycle<S>(p, a, st);
    const Args<T> f = at_tiles(a, p->fine_base);
    const double c = p->fine_cells;
    prof_begin(p, GD_K_PUPDATE, c, st);
    chain_launch(p, st::k_pupdate_s<T>, p->fine_count, st::kThreads, st::pupdate_smem<T>(), st,
                 f);
    prof_end(p, st);
    prof_begin(p, GD_K_CGUPDATE, c, st);
    chain_launch(p, st::k_cgupdate_s<T>, p->fine_count, st::kThreads, st::cgupdate_smem<T>(),
                 st, f);
    prof_end(p, st);
    if (refresh) launch_refresh(p, a, st);
  }

  static void launch_refresh(gd_plan p, const Args<T> &a, cudaStream_t st) {
    prof_begin(p, GD_K_RESID, p->fine_cells, st);
    chain_launch(p, st::k_refresh_s<T, false>, p->fine_count, st::kThreads,
                 st::refresh_smem<T>(), st, at_tiles(a, p->fine_base));
    prof_end(p, st);
  }

  static void dispatch_attrs(int s) {
    if (s == 1) set_attrs<1>();
    else if (s == 2) set_attrs<2>();
    else set_attrs<3>();
  }

  // What one wave of the strip kernels holds on the whole GPU: down warps,
  // level-0 up CTAs (of UpCta<true>::W warps) and coarse up warps; the
  // rectangle-only forms when `rect`.  Zero where the occupancy query failed.
  template <int S>
  static void strip_capacity(gd_plan p, bool rect, long long cap[3]) {
    auto occ = [&](const void *kernel, int threads, size_t smem) -> long long {
      int blocks = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, threads, smem) !=
          cudaSuccess) {
        cudaGetLastError();
        blocks = 0;
      }
      return (long long)blocks * p->sms;
    };
    constexpr int NT0 = st::UpCta<true>::NT, NT1 = st::UpCta<false>::NT;
    bool done = false;
    if constexpr (sizeof(T) == 4) {
      if (rect) {
        cap[0] = occ((const void *)st::k_down_s<T, S, false>, st::kSThreads, down_smem<S>(true));
        cap[1] = occ((const void *)st::k_up_s<T, S, S, true, false>, NT0, up_smem<S, true>(true));
        cap[2] = occ((const void *)st::k_up_s<T, S, S, false, false>, NT1,
                     up_smem<S, false>(true));
        done = true;
      }
    }
    if (!done) {
      cap[0] = occ((const void *)st::k_down_s<T, S>, st::kSThreads, down_smem<S>(false));
      cap[1] = occ((const void *)st::k_up_s<T, S, S, true>, NT0, up_smem<S, true>(false));
      cap[2] = occ((const void *)st::k_up_s<T, S, S, false>, NT1, up_smem<S, false>(false));
    }
    cap[0] *= st::kSWarps;
    cap[2] *= st::UpCta<false>::W;
  }
  static void dispatch_capacity(gd_plan p, bool rect, long long cap[3]) {
    const int s = p->prm.pre_sweeps;
    if (s == 1) strip_capacity<1>(p, rect, cap);
    else if (s == 2) strip_capacity<2>(p, rect, cap);
    else strip_capacity<3>(p, rect, cap);
  }
  static void dispatch_iteration(gd_plan p, const Args<T> &a, cudaStream_t st,
                                 bool refresh = true) {
    const int s = p->prm.pre_sweeps;
    if (s == 1) iteration<1>(p, a, st, refresh);
    else if (s == 2) iteration<2>(p, a, st, refresh);
    else iteration<3>(p, a, st, refresh);
  }
  static void dispatch_vcycle(gd_plan p, const Args<T> &a, cudaStream_t st) {
    const int s = p->prm.pre_sweeps;
    if (s == 1) vcycle<1>(p, a, st);
    else if (s == 2) vcycle<2>(p, a, st);
    else vcycle<3>(p, a, st);
  }
};

void strip_widths(gd_plan p, int *down_ow, int *up_ow) {
  const int s = p->prm.pre_sweeps;
  if (p->fp64) {
    if (s == 1) { *down_ow = StripCfg<double, 1>::down_ow; *up_ow = StripCfg<double, 1>::up_ow; }
    else if (s == 2) { *down_ow = StripCfg<double, 2>::down_ow; *up_ow = StripCfg<double, 2>::up_ow; }
    else { *down_ow = StripCfg<double, 3>::down_ow; *up_ow = StripCfg<double, 3>::up_ow; }
  } else {
    if (s == 1) { *down_ow = StripCfg<float, 1>::down_ow; *up_ow = StripCfg<float, 1>::up_ow; }
    else if (s == 2) { *down_ow = StripCfg<float, 2>::down_ow; *up_ow = StripCfg<float, 2>::up_ow; }
    else { *down_ow = StripCfg<float, 3>::down_ow; *up_ow = StripCfg<float, 3>::up_ow; }
  }
}

// Shared-memory layout of a bottom holding levels first..last (padded b, u and
// classes per level, then the dense solve's FP64 right-hand side); returns its
// size in bytes and, with `write`, records the offsets in the levels.
int bottom_layout(gd_plan p, int first, int last, size_t es, bool write) {
  size_t off = 0;
  auto a16 = [](size_t v) { return (v + 15) & ~(size_t)15; };
  for (int l = first; l <= last; ++l) {
    LevelInfo &L = p->lv[l];
    const size_t px = (size_t)L.nx + 3, cells = px * ((size_t)L.ny + 3);
    const size_t b = off;
    off = a16(off + cells * es);
    const size_t u = off;
    off = a16(off + cells * es);
    const size_t r = off;
    off = a16(off + cells * es);
    const size_t c = off;
    off = a16(off + cells);
    if (write) {
      L.sm_b = (int)b;
      L.sm_u = (int)u;
      L.sm_r = (int)r;
      L.sm_c = (int)c;
      L.sm_px = (int)px;
    }
  }
  // FP64 right-hand side of the dense solve, then the dense inverse
  const size_t d = off;
  off = a16(off + (size_t)kCoarsestCells * sizeof(double) +
            (size_t)kCoarsestCells * kCoarsestCells * sizeof(double));
  if (write) {
    p->lv[last].sm_d = (int)d;
    for (int l = first; l <= last; ++l) p->lv[l].sm_end = (int)off;
  }
  return off > (size_t)INT_MAX ? INT_MAX : (int)off;
}

// The bottom of one instance (levels level0 .. level0 + last): the first level
// with at most bottom_cells (default kBottomCells) cells whose levels fit
// kBottomSmem bytes and kBottomLevels levels, else the coarsest.
int choose_bottom(gd_plan p, int level0, int last, size_t es) {
  const long long max_cells = p->prm.bottom_cells > 0 ? p->prm.bottom_cells : kBottomCells;
  for (int l = 0; l <= last; ++l) {
    const LevelInfo &L = p->lv[level0 + l];
    if ((long long)L.ny * L.nx > max_cells) continue;
    if (last - l + 1 > kBottomLevels) continue;
    if (bottom_layout(p, level0 + l, level0 + last, es, false) <= kBottomSmem) return l;
  }
  return last;
}

// Level 0's default strip rule: warps per launch.
constexpr int kLevel0TargetWarps = 1800;

// Strip height (rows per warp, a multiple of st::kRzRows) of level l.
//
// target > 0: the tallest of 64, 32, 16, 8 rows that still gives `target` warps
// over the level-l strips of all instances (one launch), else 8.
//
// target == 0 (the default on coarse levels): the height that minimises the launch time modelled
// as waves x rows a warp walks, for the down and the up launch together.  A
// strip walks its rows plus its warm-up rows (4 S + 2 for down, 4 S for up);
// a wave is what the GPU holds at once (cap: down warps, level-0 up CTAs of
// UpCta<true>::W warps, coarse up warps; resident warps each walk their strip
// in parallel).  A launch that overflows a wave by a few strips pays a whole
// second wave, and a launch of few tall strips leaves each warp a long row
// chain; the model avoids both (e.g. 2048 x 2048 x 3: 68 rows and one wave
// instead of 64 rows and 1.03 waves).  `only` >= 0: that instance alone.
int strip_rows(const gd_plan p, const std::vector<int> &bottoms, int l, int down_ow, int up_ow,
               const long long cap[3], int target, int only = -1) {
  const long long tile_max = p->prm.tile_cells > 0 ? p->prm.tile_cells : kTileCells;
  auto strip_level = [&](int i) {
    if (only >= 0 && i != only) return false;
    if (l >= bottoms[i]) return false;
    const LevelInfo &L = p->lv[p->inst[i].level0 + l];
    return !(l >= 1 && (long long)L.ny * L.nx <= tile_max);  // else on the tile kernels
  };
  if (target > 0) {
    const int ow = std::min(down_ow, up_ow);
    for (int rb = 64; rb >= 8; rb >>= 1) {
      long long warps = 0;
      for (int i = 0; i < p->n; ++i) {
        if (!strip_level(i)) continue;
        const LevelInfo &L = p->lv[p->inst[i].level0 + l];
        warps += (long long)ceil_div(L.nx, ow) * ceil_div(L.ny, rb);
      }
      if (warps >= target) return rb;
    }
    return 8;
  }
  const int s = p->prm.pre_sweeps;
  const long long cd = cap[0] > 0 ? cap[0] : 12LL * p->sms;
  const int upw = l == 0 ? st::UpCta<true>::W : st::UpCta<false>::W;
  const long long cu = l == 0 ? (cap[1] > 0 ? cap[1] : 3LL * p->sms)
                              : (cap[2] > 0 ? cap[2] : 12LL * p->sms);
  long long best_cost = -1;
  int best = 8;
  for (int rb = 256; rb >= st::kRzRows; rb -= st::kRzRows) {
    long long sd = 0, su = 0;
    for (int i = 0; i < p->n; ++i) {
      if (!strip_level(i)) continue;
      const LevelInfo &L = p->lv[p->inst[i].level0 + l];
      sd += (long long)ceil_div(L.nx, down_ow) * ceil_div(L.ny, rb);
      su += (long long)ceil_div(L.nx, up_ow) * ceil_div(L.ny, upw * rb);
    }
    if (sd == 0) return 8;
    const long long cost = ((sd + cd - 1) / cd) * (rb + 4 * s + 2) + ((su + cu - 1) / cu) * (rb + 4 * s);
    if (best_cost < 0 || cost < best_cost) {  // ties keep the taller strips
      best_cost = cost;
      best = rb;
    }
  }
  return best;
}

template <typename T>
__global__ void k_load_r(T *r, int pitch, const double *src, int spitch, int ny, int nx) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ny * nx) return;
  const int y = k / nx, x = k - y * nx;
  r[(long long)y * pitch + x] = (T)src[(long long)y * spitch + x];
}

template <typename T>
__global__ void k_store_z(double *dst, int dpitch, const T *z, int pitch, int ny, int nx) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ny * nx) return;
  const int y = k / nx, x = k - y * nx;
  dst[(long long)y * dpitch + x] = (double)z[(long long)y * pitch + x];
}

size_t elem_size(const gd_plan p) { return p->fp64 ? sizeof(double) : sizeof(float); }

// Lay out hierarchy, arena, tile lists and workspace for the plan.
int build_plan(gd_plan p, const gd_grid_desc *grids) {
  const size_t es = elem_size(p);
  const size_t align_el = kArrayAlign / es;
  auto take = [&](size_t &cursor, size_t elems) {
    const size_t off = cursor;
    cursor = align_up(cursor + elems, align_el);
    return (long long)off;
  };
  size_t arena = 0, codes = 0, dense = 0, xs = 0;
  std::vector<int> bottoms(p->n);
  for (int i = 0; i < p->n; ++i) {
    const gd_grid_desc &g = grids[i];
    InstInfo I{};
    I.ny = g.height;
    I.nx = g.width;
    I.bc = g.boundary;
    I.zero_mean = (g.boundary == GD_NEUMANN && (g.flags & 1)) ? 1 : 0;
    I.pitch = (int)align_up((size_t)g.width, kPitchAlign);
    const size_t cells0 = (size_t)I.ny * I.pitch;
    I.r_off = take(arena, cells0);
    I.p_off = take(arena, cells0);
    I.d_off = take(arena, cells0);
    I.z_off = take(arena, cells0);
    I.q_off = take(arena, cells0);
    I.xs_off = (long long)xs;
    xs = align_up(xs + cells0, kArrayAlign / sizeof(double));
    I.level0 = (int)p->lv.size();
    int ny = I.ny, nx = I.nx, level = 0;
    int bottom = -1;
    while (true) {
      LevelInfo L{};
      L.ny = ny;
      L.nx = nx;
      L.pitch = level == 0 ? I.pitch : (int)align_up((size_t)nx, kPitchAlign);
      L.inst = i;
      L.bc = g.boundary;
      L.level = level;
      L.wall = g.boundary == GD_NEUMANN ? 0.0f : (level == 0 ? 1.0f : 2.0f);
      if (level == 0) {
        L.b_off = I.r_off;
        L.u_off = I.z_off;
      } else {
        L.b_off = take(arena, (size_t)ny * L.pitch);
        L.u_off = take(arena, (size_t)ny * L.pitch);
      }
      L.w_off = -1;
      L.code_off = -1;
      if (g.boundary == GD_MASKED) {
        L.code_off = (long long)codes;
        codes = align_up(codes + (size_t)ny * L.pitch, kArrayAlign);
      }
      L.inv_off = -1;
      const long long cells = (long long)ny * nx;
      L.is_bottom = 0;
      const bool coarsest = cells <= kCoarsestCells;
      // the coarse level is always the next table entry; the smoothing kernels read
      // it as lv[level + 1] together with the level's own entry
      L.coarse = coarsest ? -1 : (int)p->lv.size() + 1;
      if (coarsest) {
        L.inv_off = (long long)dense;
        dense += align_up((size_t)cells * cells, 32);
      }
      p->lv.push_back(L);
      if (coarsest) break;
      ny = (ny + 1) / 2;
      nx = (nx + 1) / 2;
      ++level;
    }
    I.nlevels = level + 1;
    bottom = choose_bottom(p, I.level0, level, es);
    p->lv[I.level0 + bottom].is_bottom = 1;
    I.bottom = I.level0 + bottom;
    I.coarsest = I.level0 + level;
    bottoms[i] = bottom;
    p->depth = std::max(p->depth, bottom);
    p->inst.push_back(I);
  }
  // tile lists
  for (int i = 0; i < p->n; ++i) {
    const InstInfo &I = p->inst[i];
    for (int l = 0; l < bottoms[i]; ++l) {
      LevelInfo &L = p->lv[I.level0 + l];
      L.w_off = take(arena, (size_t)L.ny * L.pitch);
    }
  }
  int down_ow = 0, up_ow = 0;
  strip_widths(p, &down_ow, &up_ow);
  const int target_warps = std::max(p->prm.strip_target_warps, 0);
  long long cap[3] = {0, 0, 0};
  {
    bool any_masked = false;
    for (int i = 0; i < p->n; ++i) any_masked = any_masked || p->inst[i].bc == BC_MASK;
    if (p->fp64) Runner<double>::dispatch_capacity(p, false, cap);
    else Runner<float>::dispatch_capacity(p, !any_masked, cap);
  }
  for (int i = 0; i < p->n; ++i) p->inst[i].rz_rows = st::kRzRows;
  for (int l = 0; l < p->depth; ++l) {
    // level 0 keeps the warps-per-launch rule by default: one wave of tall strips
    // was measured slower there (4096 x 4096 x 3: 256 rows, up0 170 -> 295 us per
    // launch) than several waves of 64-row strips
    const int target = (l == 0 && target_warps == 0) ? kLevel0TargetWarps : target_warps;
    const int rb = strip_rows(p, bottoms, l, down_ow, up_ow, cap, target);
    for (int i = 0; i < p->n; ++i) {
      if (l >= bottoms[i]) continue;
      p->lv[p->inst[i].level0 + l].rows_per_warp = rb;
      // r.z group height: level 0's height for the instance alone (the
      // warps-per-launch rule only gives taller strips to larger launches, and
      // its heights are powers of two, so rb is a multiple of it)
      if (l == 0) p->inst[i].rz_rows = strip_rows(p, bottoms, 0, down_ow, up_ow, cap, target, i);
    }
  }
  p->fine_base = (int)p->tiles.size();
  for (int i = 0; i < p->n; ++i) {
    InstInfo &I = p->inst[i];
    I.fine_begin = (int)p->tiles.size() - p->fine_base;
    for (int ty = 0; ty < ceil_div(I.ny, kFTY); ++ty)
      for (int tx = 0; tx < ceil_div(I.nx, kFTX); ++tx)
        p->tiles.push_back(Tile{I.level0, i, ty, tx});
    I.fine_end = (int)p->tiles.size() - p->fine_base;
  }
  p->fine_count = (int)p->tiles.size() - p->fine_base;
  p->down_base.assign(p->depth, 0);
  p->down_count.assign(p->depth, 0);
  p->up_base.assign(p->depth, 0);
  p->up_count.assign(p->depth, 0);
  p->tdown_base.assign(p->depth, 0);
  p->tdown_count.assign(p->depth, 0);
  p->tup_base.assign(p->depth, 0);
  p->tup_count.assign(p->depth, 0);
  p->tile_cells.assign(std::max(p->depth, 1), 0.0);
  // coarse levels up to tile_max cells run on the shared-memory tile kernels
  const long long tile_max = p->prm.tile_cells > 0 ? p->prm.tile_cells : kTileCells;
  auto on_tiles = [&](int i, int l) {
    const LevelInfo &F = p->lv[p->inst[i].level0 + l];
    return l >= 1 && (long long)F.ny * F.nx <= tile_max;
  };
  p->tsmall.assign(p->depth, 0);
  for (int l = 1; l < p->depth; ++l) {
    p->tdown_base[l] = (int)p->tiles.size();
    long long large = 0;  // large tiles the level would have
    for (int i = 0; i < p->n; ++i) {
      if (bottoms[i] <= l || !on_tiles(i, l)) continue;
      const LevelInfo &F = p->lv[p->inst[i].level0 + l];
      large += (long long)ceil_div(F.ny, tile::kTY) * ceil_div(F.nx, tile::kTX);
    }
    p->tsmall[l] = large > 0 && large < p->sms;
    const int ty_cells = p->tsmall[l] ? tile::kTYs : tile::kTY;
    const int tx_cells = p->tsmall[l] ? tile::kTXs : tile::kTX;
    for (int i = 0; i < p->n; ++i) {
      if (bottoms[i] <= l || !on_tiles(i, l)) continue;
      const LevelInfo &F = p->lv[p->inst[i].level0 + l];
      for (int ty = 0; ty < ceil_div(F.ny, ty_cells); ++ty)
        for (int tx = 0; tx < ceil_div(F.nx, tx_cells); ++tx)
          p->tiles.push_back(Tile{p->inst[i].level0 + l, i, ty, tx});
      p->tile_cells[l] += (double)F.ny * F.nx;
    }
    p->tdown_count[l] = (int)p->tiles.size() - p->tdown_base[l];
    p->tup_base[l] = p->tdown_base[l];  // the up kernel uses the same tiles
    p->tup_count[l] = p->tdown_count[l];
  }
  p->strip_any.assign(std::max(p->depth, 1), 0);
  for (int l = 0; l < p->depth; ++l)
    for (int i = 0; i < p->n; ++i) {
      if (bottoms[i] <= l || on_tiles(i, l)) continue;
      const LevelInfo &F = p->lv[p->inst[i].level0 + l];
      const LevelInfo &Fc = p->lv[p->inst[i].level0 + l + 1];
      if (F.code_off >= 0 || Fc.code_off >= 0 ||
          (long long)(F.ny + 16) * F.pitch >= (1LL << 31))
        p->strip_any[l] = 1;
    }
  for (int l = 0; l < p->depth; ++l) {
    p->down_base[l] = (int)p->tiles.size();
    for (int i = 0; i < p->n; ++i) {
      if (bottoms[i] <= l || on_tiles(i, l)) continue;
      const LevelInfo &F = p->lv[p->inst[i].level0 + l];
      const int rows = st::kSWarps * F.rows_per_warp;
      for (int ty = 0; ty < ceil_div(F.ny, rows); ++ty)
        for (int tx = 0; tx < ceil_div(F.nx, down_ow); ++tx)
          p->tiles.push_back(Tile{p->inst[i].level0 + l, i, ty, tx});
    }
    p->down_count[l] = (int)p->tiles.size() - p->down_base[l];
  }
  int rz_parts = 0;
  for (int l = 0; l < p->depth; ++l) {
    p->up_base[l] = (int)p->tiles.size();
    for (int i = 0; i < p->n; ++i) {
      InstInfo &I = p->inst[i];
      if (bottoms[i] <= l || on_tiles(i, l)) continue;
      const LevelInfo &F = p->lv[I.level0 + l];
      const int rows = (l == 0 ? st::UpCta<true>::W : st::UpCta<false>::W) * F.rows_per_warp;
      if (l == 0) {  // the instance's r.z group partials (st::RzGroups)
        I.up0_begin = rz_parts;
        rz_parts += ceil_div(F.ny, I.rz_rows) * ceil_div(F.nx, up_ow);
        I.up0_end = rz_parts;
      }
      for (int ty = 0; ty < ceil_div(F.ny, rows); ++ty)
        for (int tx = 0; tx < ceil_div(F.nx, up_ow); ++tx)
          p->tiles.push_back(Tile{I.level0 + l, i, ty, tx});
    }
    p->up_count[l] = (int)p->tiles.size() - p->up_base[l];
  }
  p->max_partials = std::max(1, std::max(p->fine_count, rz_parts));
  p->launch_cells.assign(2 * std::max(p->depth, 1), 0.0);
  p->fine_cells = 0;
  for (int i = 0; i < p->n; ++i) {
    const InstInfo &I = p->inst[i];
    p->fine_cells += (double)I.ny * I.nx;
    for (int l = 0; l < bottoms[i]; ++l) {
      if (on_tiles(i, l)) continue;
      const LevelInfo &F = p->lv[I.level0 + l];
      p->launch_cells[2 * l] += (double)F.ny * F.nx;
      p->launch_cells[2 * l + 1] += (double)F.ny * F.nx;
    }
  }
  // bottom shared memory
  size_t bsm = 0;
  for (int i = 0; i < p->n; ++i)
    bsm = std::max(bsm, (size_t)bottom_layout(p, p->inst[i].bottom, p->inst[i].coarsest, es,
                                              true));
  p->bottom_smem = bsm;
  // the persistent coarse launch: tile levels below the last strip level, the
  // bottom, and the tile levels again on the way up
  {
    // below the last strip level and the last level of large tiles: the
    // persistent launch holds only small-tile levels (large tile levels keep
    // their own launch of many CTAs)
    int top = 0;
    for (int l = 0; l < p->depth; ++l)
      if (p->down_count[l] > 0 || (p->tdown_count[l] > 0 && !p->tsmall[l])) top = l + 1;
    coarse::Phases ph{};
    auto add = [&](int kind, int base, int items) {
      ph.kind[ph.count] = kind;
      ph.base[ph.count] = base;
      ph.items[ph.count] = items;
      ++ph.count;
    };
    for (int l = top; l < p->depth; ++l)
      if (p->tdown_count[l] > 0) add(coarse::kPhaseDown, p->tdown_base[l], p->tdown_count[l]);
    add(coarse::kPhaseBottom, 0, p->n);
    for (int l = p->depth - 1; l >= top; --l)
      if (p->tup_count[l] > 0) add(coarse::kPhaseUp, p->tup_base[l], p->tup_count[l]);
    int items = 0;
    for (int q = 0; q < ph.count; ++q) items = std::max(items, ph.items[q]);
    p->coarse_from = top;
    p->phases = ph;
    p->coarse_grid = std::min(p->sms, items);
    // a single phase (the bottom alone) gains nothing from the persistent form
    p->persistent = p->persistent && ph.count > 1;
  }
  p->arena_elems = arena;
  p->code_bytes = std::max<size_t>(codes, kArrayAlign);
  p->dense_elems = std::max<size_t>(dense, 32);
  p->xs_elems = xs;
  // workspace
  size_t o = 0;
  auto sect = [&](size_t bytes) {
    const size_t at = o;
    o = align_up(o + bytes, kArrayAlign);
    return at;
  };
  p->o_lv = sect(p->lv.size() * sizeof(LevelInfo));
  p->o_inst = sect(p->inst.size() * sizeof(InstInfo));
  p->o_st = sect(p->n * sizeof(InstState));
  p->o_tiles = sect(p->tiles.size() * sizeof(Tile));
  p->o_arena = sect(p->arena_elems * es);
  p->o_codes = sect(p->code_bytes);
  p->o_dense = sect(p->dense_elems * sizeof(double));
  p->o_xs = sect(p->xs_elems * sizeof(double));
  p->o_p0 = sect(p->max_partials * sizeof(double));
  p->o_p1 = sect(p->max_partials * sizeof(double));
  p->o_cnt = sect(16 * sizeof(unsigned));
  p->o_nact = sect(sizeof(int));
  p->o_trip = sect(sizeof(int));
  p->total = o;
  return GD_OK;
}

}  // namespace

extern "C" int gd_plan_create(const gd_grid_desc *grids, int32_t n, const gd_params *params,
                              gd_plan *out) {
  GD_REQUIRE(grids && params && out && n > 0, GD_ERR_ARG, "gd_plan_create: bad arguments");
  *out = nullptr;
  GD_REQUIRE(params->pre_sweeps == params->post_sweeps && params->pre_sweeps >= 1 &&
                 params->pre_sweeps <= 3,
             GD_ERR_UNSUPPORTED, "gd_plan_create: pre_sweeps == post_sweeps in 1..3 required");
  GD_REQUIRE(params->precision == GD_MIXED || params->precision == GD_FP64, GD_ERR_ARG,
             "gd_plan_create: unknown precision %d", params->precision);
  GD_REQUIRE(params->bottom_cells >= 0 && params->tile_cells >= 0, GD_ERR_ARG,
             "gd_plan_create: negative bottom_cells / tile_cells");
  GD_REQUIRE(params->max_iterations >= 0 && params->tolerance >= 0.0, GD_ERR_ARG,
             "gd_plan_create: bad tolerance / iteration budget");
  GD_REQUIRE(params->persistent_coarse == 0 || params->persistent_coarse == 1, GD_ERR_ARG,
             "gd_plan_create: persistent_coarse must be 0 or 1");
  GD_REQUIRE(params->dependent_launch == 0 || params->dependent_launch == 1, GD_ERR_ARG,
             "gd_plan_create: dependent_launch must be 0 or 1");
  for (int i = 0; i < n; ++i) {
    GD_REQUIRE(grids[i].height > 0 && grids[i].width > 0, GD_ERR_ARG,
               "gd_plan_create: instance %d has an empty grid", i);
    GD_REQUIRE(grids[i].boundary >= 0 && grids[i].boundary <= 2, GD_ERR_ARG,
               "gd_plan_create: instance %d has unknown boundary %d", i, grids[i].boundary);
    GD_REQUIRE((long long)grids[i].height * grids[i].width < (1ll << 31), GD_ERR_ARG,
               "gd_plan_create: instance %d is too large", i);
  }
  gd_plan p = new gd_plan_s();
  p->n = n;
  p->prm = *params;
  if (p->prm.check_every <= 0) p->prm.check_every = 4;
  if (p->prm.reliable_delta <= 0.0) p->prm.reliable_delta = 1e-4;
  p->fp64 = params->precision == GD_FP64;
  p->dependent_launch = params->dependent_launch == 1;
  {
    int dev = 0, sms = 0, coop = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
        sms > 0)
      p->sms = sms;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess) coop = 0;
    cudaGetLastError();  // no device (CPU-only build checks): keep the defaults
    p->persistent = params->persistent_coarse == 1 && coop != 0;
  }
  p->mask_set.assign(n, 0);
  // kernel attributes first: the strip heights depend on the kernels' occupancy
  if (p->fp64) Runner<double>::dispatch_attrs(p->prm.pre_sweeps);
  else Runner<float>::dispatch_attrs(p->prm.pre_sweeps);
  build_plan(p, grids);
  // the limits above are constants every plan sets alike; a failure (no device in a
  // CPU-only check) must not stay behind as this thread's last error, where a later
  // launch check would report it as its own
  cudaGetLastError();
  p->h_st_bytes = sizeof(InstState) * n;
  p->h_nact = static_cast<int *>(pinned_get(2 * sizeof(int)));  // active count, error word
  p->h_st = static_cast<InstState *>(pinned_get(p->h_st_bytes));
  p->h_inst_bytes = sizeof(InstInfo) * n;
  p->h_inst = static_cast<InstInfo *>(pinned_get(p->h_inst_bytes));
  if (!p->h_nact || !p->h_st || !p->h_inst) {
    set_error("gd_plan_create: pinned host allocation failed");
    gd_plan_destroy(p);
    return GD_ERR_CUDA;
  }
  if (p->bottom_smem > (size_t)kBottomSmem) {
    set_error("gd_plan_create: bottom levels need %zu bytes of shared memory", p->bottom_smem);
    gd_plan_destroy(p);
    return GD_ERR_UNSUPPORTED;
  }
  *out = p;
  return GD_OK;
}

extern "C" void gd_plan_destroy(gd_plan p) {
  if (!p) return;
  for (cudaEvent_t e : p->ev_pool) cudaEventDestroy(e);
  if (p->gexec) cudaGraphExecDestroy(p->gexec);
  if (p->done_ev) cudaEventDestroy(p->done_ev);
  capture_stream_put(p->cap_device, p->cap);
  pinned_put(p->h_nact, 2 * sizeof(int));
  pinned_put(p->h_st, p->h_st_bytes);
  pinned_put(p->h_inst, p->h_inst_bytes);
  delete p;
}

extern "C" size_t gd_plan_workspace_bytes(gd_plan p) { return p ? p->total : 0; }

extern "C" int gd_plan_bind(gd_plan p, void *ws, size_t bytes, cudaStream_t st) {
  GD_REQUIRE(p && ws, GD_ERR_ARG, "gd_plan_bind: bad arguments");
  GD_REQUIRE(bytes >= p->total, GD_ERR_ARG, "gd_plan_bind: workspace %zu < %zu bytes", bytes,
             p->total);
  GD_REQUIRE(((uintptr_t)ws & (kArrayAlign - 1)) == 0, GD_ERR_ARG,
             "gd_plan_bind: workspace must be 256-byte aligned");
  if (p->gexec) {
    cudaGraphExecDestroy(p->gexec);
    p->gexec = nullptr;
  }
  p->ws = (char *)ws;
  p->prepared = false;
  GD_CHECK_CUDA(cudaMemsetAsync(ws, 0, p->total, st));
  GD_CHECK_CUDA(cudaMemcpyAsync(p->ws + p->o_lv, p->lv.data(), p->lv.size() * sizeof(LevelInfo),
                                cudaMemcpyHostToDevice, st));
  GD_CHECK_CUDA(cudaMemcpyAsync(p->ws + p->o_inst, p->inst.data(),
                                p->inst.size() * sizeof(InstInfo), cudaMemcpyHostToDevice, st));
  // pageable sources are staged before cudaMemcpyAsync returns: no sync needed
  GD_CHECK_CUDA(cudaMemcpyAsync(p->ws + p->o_tiles, p->tiles.data(),
                                p->tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice, st));
  return GD_OK;
}

extern "C" int gd_plan_set_mask(gd_plan p, int32_t i, const uint8_t *mask, int32_t mpitch,
                                cudaStream_t st) {
  GD_REQUIRE(p && p->ws && mask && i >= 0 && i < p->n, GD_ERR_ARG,
             "gd_plan_set_mask: bad arguments or unbound plan");
  const InstInfo &I = p->inst[i];
  GD_REQUIRE(I.bc == GD_MASKED, GD_ERR_ARG, "gd_plan_set_mask: instance %d is not masked", i);
  GD_REQUIRE(mpitch >= I.nx, GD_ERR_ARG, "gd_plan_set_mask: pitch %d < width %d", mpitch, I.nx);
  unsigned char *codes = (unsigned char *)(p->ws + p->o_codes);
  const LevelInfo &L0 = p->lv[I.level0];
  k_codes_fine<<<ceil_div(L0.ny * L0.nx, 256), 256, 0, st>>>(codes + L0.code_off, L0.pitch, mask,
                                                             mpitch, L0.ny, L0.nx);
  for (int l = I.level0 + 1; l <= I.coarsest; ++l) {
    const LevelInfo &F = p->lv[l - 1], &C = p->lv[l];
    k_codes_coarse_act<<<ceil_div(C.ny * C.nx, 256), 256, 0, st>>>(
        codes + C.code_off, C.pitch, C.ny, C.nx, codes + F.code_off, F.pitch, F.ny, F.nx);
    k_codes_classes<<<ceil_div(C.ny * C.nx, 256), 256, 0, st>>>(codes + C.code_off, C.pitch,
                                                                C.ny, C.nx);
  }
  GD_CHECK_LAUNCH();
  p->mask_set[i] = 1;
  p->prepared = false;
  return GD_OK;
}

extern "C" int gd_plan_prepare(gd_plan p, cudaStream_t st) {
  GD_REQUIRE(p && p->ws, GD_ERR_STATE, "gd_plan_prepare: plan is not bound");
  for (int i = 0; i < p->n; ++i)
    GD_REQUIRE(p->inst[i].bc != GD_MASKED || p->mask_set[i], GD_ERR_STATE,
               "gd_plan_prepare: masked instance %d has no mask", i);
  k_coarse_inverse<<<p->n, 256, 0, st>>>(
      reinterpret_cast<const LevelInfo *>(p->ws + p->o_lv),
      reinterpret_cast<const InstInfo *>(p->ws + p->o_inst),
      reinterpret_cast<const unsigned char *>(p->ws + p->o_codes),
      reinterpret_cast<double *>(p->ws + p->o_dense));
  GD_CHECK_LAUNCH();
  p->prepared = true;
  return GD_OK;
}

namespace {

// Condition of the solve graph's while loop: iterate while any instance is
// active, at most `cap` times.  `start` resets the trip counter.
__global__ void k_loop_gate(cudaGraphConditionalHandle h, const int *n_active, int *trips,
                            int start, int cap) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int t = start ? 0 : *trips + 1;
  *trips = t;
  cudaGraphSetConditional(h, (*n_active > 0 && t < cap) ? 1u : 0u);
}

// Condition of the refresh node in the loop body: some instance asked for an
// FP64 refresh (FLAG_RU).  Iterations without one launch no refresh kernel.
__global__ void k_refresh_gate(cudaGraphConditionalHandle h, const InstState *st, int n) {
  if (blockIdx.x != 0) return;
  bool any = false;
  for (int i = threadIdx.x; i < n; i += blockDim.x) any = any || (st[i].flags & FLAG_RU);
  any = __any_sync(0xffffffffu, any);
  if (threadIdx.x == 0) cudaGraphSetConditional(h, any ? 1u : 0u);
}

template <typename T>
void launch_init(gd_plan p, const Args<T> &fine, cudaStream_t st) {
  prof_begin(p, GD_K_INIT, p->fine_cells, st);
  chain_launch(p, k_fmean<T>, p->fine_count, kFThreads, 0, st, fine);
  chain_launch(p, st::k_refresh_s<T, true>, p->fine_count, st::kThreads, st::refresh_smem<T>(),
               st, fine);
  prof_end(p, st);
}

bool plan_any_mean(gd_plan p) {
  for (int i = 0; i < p->n; ++i)
    if (p->inst[i].zero_mean) return true;
  return false;
}

// After the loop: the mean of zero-mean instances, then the solution into the
// caller's buffer (mean subtracted; copied from the plan's copy where the last
// refresh left it there).  Every refresh that folds a correction leaves the
// mean of the new solution in the instance state, and a zero-start solve that
// never folds has mean zero, so only solves that start from the caller's x
// (which may converge on its initial residual) need the separate mean pass.
template <typename T>
void launch_finish(gd_plan p, const Args<T> &fine, cudaStream_t st) {
  prof_begin(p, GD_K_MEAN, p->fine_cells, st);
  if (plan_any_mean(p) && !p->prm.zero_start)
    chain_launch(p, k_mean<T>, p->fine_count, kFThreads, 0, st, fine);
  chain_launch(p, k_submean<T>, p->fine_count, kFThreads, 0, st, fine);
  prof_end(p, st);
}

int loop_cap(gd_plan p) {
  return (int)std::min<long long>((long long)p->prm.max_iterations + 8, 1ll << 30);
}

// One graph per plan for a whole solve: the initial residual, a conditional
// while node whose body is one Krylov iteration (V-cycle, p update, d / r
// update, then the FP64 refresh behind an if node, launched only when some
// instance asked for one) followed by k_loop_gate, and the zero-mean
// projection.  The device decides when to stop, so a solve is a single graph
// launch with no host round trip and no iteration past the last active
// instance.
template <typename T>
int build_solve_graph(gd_plan p, const Args<T> &a, const Args<T> &fine) {
  if (!p->cap) {
    GD_CHECK_CUDA(cudaGetDevice(&p->cap_device));
    GD_CHECK_CUDA(capture_stream_get(p->cap_device, &p->cap));
  }
  cudaStream_t cs = p->cap;
  int *trips = reinterpret_cast<int *>(p->ws + p->o_trip);
  const int cap = loop_cap(p);
  GD_CHECK_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaSuccess;
  cudaGraphConditionalHandle h{};
  cudaGraph_t body = nullptr;
  do {
    launch_init(p, fine, cs);
    cudaStreamCaptureStatus status;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    if ((e = cudaStreamGetCaptureInfo(cs, &status, nullptr, &cg, &deps, &nd)) != cudaSuccess) break;
    if ((e = cudaGraphConditionalHandleCreate(&h, cg, 0, cudaGraphCondAssignDefault)) !=
        cudaSuccess)
      break;
    k_loop_gate<<<1, 32, 0, cs>>>(h, a.n_active, trips, 1, cap);
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    if ((e = cudaStreamGetCaptureInfo(cs, &status, nullptr, &cg, &deps, &nd)) != cudaSuccess) break;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wn;
    if ((e = cudaGraphAddNode(&wn, cg, deps, nd, &cp)) != cudaSuccess) break;
    body = cp.conditional.phGraph_out[0];
    if ((e = cudaStreamUpdateCaptureDependencies(cs, &wn, 1, cudaStreamSetCaptureDependencies)) !=
        cudaSuccess)
      break;
    launch_finish(p, fine, cs);
    e = cudaGetLastError();
  } while (0);
  cudaGraph_t g = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(cs, &g);
  if (e == cudaSuccess) e = ee;
  // loop body: an iteration without the refresh, the refresh behind an if
  // node that k_refresh_gate sets, then the loop gate
  cudaGraph_t refresh_body = nullptr;
  if (e == cudaSuccess) {
    e = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      do {
        Runner<T>::dispatch_iteration(p, a, cs, false);
        cudaStreamCaptureStatus status;
        cudaGraph_t cg = nullptr;
        const cudaGraphNode_t *deps = nullptr;
        size_t nd = 0;
        cudaGraphConditionalHandle hr{};
        if ((e = cudaStreamGetCaptureInfo(cs, &status, nullptr, &cg, &deps, &nd)) != cudaSuccess)
          break;
        if ((e = cudaGraphConditionalHandleCreate(&hr, cg, 0, cudaGraphCondAssignDefault)) !=
            cudaSuccess)
          break;
        k_refresh_gate<<<1, 32, 0, cs>>>(hr, a.st, p->n);
        if ((e = cudaGetLastError()) != cudaSuccess) break;
        if ((e = cudaStreamGetCaptureInfo(cs, &status, nullptr, &cg, &deps, &nd)) != cudaSuccess)
          break;
        cudaGraphNodeParams ip = {};
        ip.type = cudaGraphNodeTypeConditional;
        ip.conditional.handle = hr;
        ip.conditional.type = cudaGraphCondTypeIf;
        ip.conditional.size = 1;
        cudaGraphNode_t in;
        if ((e = cudaGraphAddNode(&in, cg, deps, nd, &ip)) != cudaSuccess) break;
        refresh_body = ip.conditional.phGraph_out[0];
        if ((e = cudaStreamUpdateCaptureDependencies(cs, &in, 1,
                                                     cudaStreamSetCaptureDependencies)) !=
            cudaSuccess)
          break;
        k_loop_gate<<<1, 32, 0, cs>>>(h, a.n_active, trips, 0, cap);
        e = cudaGetLastError();
      } while (0);
      cudaGraph_t bg = nullptr;
      const cudaError_t eb = cudaStreamEndCapture(cs, &bg);
      if (e == cudaSuccess) e = eb;
    }
  }
  if (e == cudaSuccess) {
    e = cudaStreamBeginCaptureToGraph(cs, refresh_body, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      Runner<T>::launch_refresh(p, a, cs);
      e = cudaGetLastError();
      cudaGraph_t rg = nullptr;
      const cudaError_t er = cudaStreamEndCapture(cs, &rg);
      if (e == cudaSuccess) e = er;
    }
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&p->gexec, g, 0);
  if (g) cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    p->gexec = nullptr;
    set_error("solve graph: %s", cudaGetErrorString(e));
    return GD_ERR_CUDA;
  }
  return GD_OK;
}

// Enqueue one solve on `st`.  With the plan's graph the call returns at once
// (the states are copied to pinned host memory behind the graph and
// `done_ev` marks them); without it (first solve, profiling) it runs the
// host-polled loop and returns with the stream drained.
template <typename T>
int enqueue_solve(gd_plan p, cudaStream_t st) {
  const Args<T> a = Runner<T>::args(p);
  const Args<T> fine = Runner<T>::at_tiles(a, p->fine_base);
  // A plan solved once runs on direct launches with the host polling the
  // active count every `check_every` iterations; from its second solve on the
  // whole solve is one graph launch (capture and instantiation cost more than
  // they save in a single solve).
  const bool graph = p->prm.use_graph && !p->profiling && p->solves >= 1;
  if (graph) {
    if (!p->gexec) {
      int rc = build_solve_graph<T>(p, a, fine);
      if (rc != GD_OK && p->persistent) {
        // a graph that cannot hold the cooperative launch: levels one by one
        cudaGetLastError();
        p->persistent = false;
        rc = build_solve_graph<T>(p, a, fine);
      }
      if (rc != GD_OK) return rc;
    }
    GD_CHECK_CUDA(cudaGraphLaunch(p->gexec, st));
  } else {
    launch_init(p, fine, st);
    GD_CHECK_LAUNCH();
    GD_CHECK_CUDA(cudaMemcpyAsync(p->h_nact, p->ws + p->o_nact, sizeof(int),
                                  cudaMemcpyDeviceToHost, st));
    GD_CHECK_CUDA(cudaStreamSynchronize(st));
    // profiled solves poll every iteration, so that no launch is timed after
    // the last instance stopped (its kernels would return at once)
    const int chunk = p->profiling ? 1 : p->prm.check_every;
    const long long cap_iters = loop_cap(p);
    long long done = 0;
    while (*p->h_nact > 0 && done < cap_iters) {
      for (int c = 0; c < chunk; ++c) Runner<T>::dispatch_iteration(p, a, st);
      GD_CHECK_LAUNCH();
      done += chunk;
      GD_CHECK_CUDA(cudaMemcpyAsync(p->h_nact, p->ws + p->o_nact, sizeof(int),
                                    cudaMemcpyDeviceToHost, st));
      GD_CHECK_CUDA(cudaStreamSynchronize(st));
      prof_collect(p);
    }
    launch_finish(p, fine, st);
    GD_CHECK_LAUNCH();
  }
  GD_CHECK_CUDA(cudaMemcpyAsync(p->h_st, p->ws + p->o_st, sizeof(InstState) * p->n,
                                cudaMemcpyDeviceToHost, st));
  GD_CHECK_CUDA(cudaMemcpyAsync(p->h_nact + 1, p->ws + p->o_cnt + kErrWord * sizeof(unsigned),
                                sizeof(int), cudaMemcpyDeviceToHost, st));
  if (!p->done_ev) GD_CHECK_CUDA(cudaEventCreateWithFlags(&p->done_ev, cudaEventDisableTiming));
  GD_CHECK_CUDA(cudaEventRecord(p->done_ev, st));
  ++p->solves;
  p->pending = true;
  return GD_OK;
}

// Wait for the last enqueued solve and turn its device states into reports.
int collect_reports(gd_plan p, gd_report *reports) {
  GD_REQUIRE(p->pending, GD_ERR_STATE, "gd_solve_finish: no solve in flight");
  GD_CHECK_CUDA(cudaEventSynchronize(p->done_ev));
  p->pending = false;
  prof_collect(p);
  const unsigned err = (unsigned)p->h_nact[1];
  GD_REQUIRE(!(err & bulk::kErrWait), GD_ERR_CUDA,
             "solve: a kernel's bounded wait for its bulk copies gave up (error word %#x); "
             "the solution is not valid", err);
  GD_REQUIRE(!(err & coarse::kErrBarrier), GD_ERR_CUDA,
             "solve: a grid barrier of the persistent coarse launch gave up (error word %#x); "
             "the solution is not valid", err);
  GD_REQUIRE(!(err & st::kErrStrip), GD_ERR_CUDA,
             "solve: a rectangle-only strip kernel met a masked level (error word %#x); "
             "the solution is not valid", err);
  GD_REQUIRE(err == 0, GD_ERR_CUDA, "solve: device error word %#x; the solution is not valid",
             err);
  for (int i = 0; i < p->n; ++i) {
    const InstState &S = p->h_st[i];
    gd_report &R = reports[i];
    R.iterations = S.iters;
    R.status = S.status == GD_ACTIVE ? GD_MAX_ITERATIONS : S.status;
    R.initial_norm = std::sqrt(S.ff);
    R.relative_residual = S.ff > 0.0 ? std::sqrt(S.rr_true / S.ff) : 0.0;
    R.refreshes = S.refreshes;
    R.reserved = 0;
  }
  return GD_OK;
}

}  // namespace

namespace {
int bind_solve(gd_plan p, const double *const *f, double *const *x, const int32_t *pitch,
               const double *scale, cudaStream_t st) {
  GD_REQUIRE(p && f && x && pitch && scale, GD_ERR_ARG, "gd_solve: bad arguments");
  GD_REQUIRE(p->ws && p->prepared, GD_ERR_STATE, "gd_solve: plan not bound and prepared");
  GD_REQUIRE(!p->pending, GD_ERR_STATE, "gd_solve: the previous asynchronous solve of this "
                                        "plan has not been finished");
  for (int i = 0; i < p->n; ++i) {
    GD_REQUIRE(f[i] && x[i] && pitch[i] >= p->inst[i].nx, GD_ERR_ARG,
               "gd_solve: instance %d has a bad pointer or pitch", i);
    p->inst[i].f = f[i];
    p->inst[i].x = x[i];
    p->inst[i].upitch = pitch[i];
    p->inst[i].scale = scale[i];
  }
  // through pinned memory: a copy from pageable memory may wait for the work
  // already queued on the stream, which would serialise pipelined solves; the
  // staging buffer is not reused before this solve is finished
  std::memcpy(p->h_inst, p->inst.data(), p->h_inst_bytes);
  GD_CHECK_CUDA(cudaMemcpyAsync(p->ws + p->o_inst, p->h_inst, p->h_inst_bytes,
                                cudaMemcpyHostToDevice, st));
  return p->fp64 ? enqueue_solve<double>(p, st) : enqueue_solve<float>(p, st);
}
}  // namespace

extern "C" int gd_solve(gd_plan p, const double *const *f, double *const *x, const int32_t *pitch,
                        const double *scale, cudaStream_t st, gd_report *reports) {
  GD_REQUIRE(reports, GD_ERR_ARG, "gd_solve: bad arguments");
  const int rc = bind_solve(p, f, x, pitch, scale, st);
  if (rc != GD_OK) return rc;
  return collect_reports(p, reports);
}

extern "C" int gd_solve_async(gd_plan p, const double *const *f, double *const *x,
                              const int32_t *pitch, const double *scale, cudaStream_t st) {
  return bind_solve(p, f, x, pitch, scale, st);
}

extern "C" int gd_solve_finish(gd_plan p, gd_report *reports) {
  GD_REQUIRE(p && reports, GD_ERR_ARG, "gd_solve_finish: bad arguments");
  return collect_reports(p, reports);
}

namespace {
template <typename T>
int run_apply_vcycle(gd_plan p, int i, const double *r, double *z, int pitch, cudaStream_t st) {
  const InstInfo &I = p->inst[i];
  for (int k = 0; k < p->n; ++k) {
    std::memset(&p->h_st[k], 0, sizeof(InstState));
    p->h_st[k].status = (k == i) ? GD_ACTIVE : GD_CONVERGED;
    p->h_st[k].first = 1;
  }
  GD_CHECK_CUDA(cudaMemcpyAsync(p->ws + p->o_st, p->h_st, sizeof(InstState) * p->n,
                                cudaMemcpyHostToDevice, st));
  T *arena = reinterpret_cast<T *>(p->ws + p->o_arena);
  const int cells = I.ny * I.nx;
  k_load_r<T><<<ceil_div(cells, 256), 256, 0, st>>>(arena + I.r_off, I.pitch, r, pitch, I.ny,
                                                    I.nx);
  Runner<T>::dispatch_vcycle(p, Runner<T>::args(p), st);
  k_store_z<T><<<ceil_div(cells, 256), 256, 0, st>>>(z, pitch, arena + I.z_off, I.pitch, I.ny,
                                                     I.nx);
  GD_CHECK_LAUNCH();
  GD_CHECK_CUDA(cudaStreamSynchronize(st));
  return GD_OK;
}
}  // namespace

extern "C" int gd_plan_apply_vcycle(gd_plan p, int32_t i, const double *r, double *z,
                                    int32_t pitch, cudaStream_t st) {
  GD_REQUIRE(p && r && z && i >= 0 && i < p->n, GD_ERR_ARG, "gd_plan_apply_vcycle: bad arguments");
  GD_REQUIRE(p->ws && p->prepared, GD_ERR_STATE, "gd_plan_apply_vcycle: plan not prepared");
  GD_REQUIRE(pitch >= p->inst[i].nx, GD_ERR_ARG, "gd_plan_apply_vcycle: bad pitch");
  return p->fp64 ? run_apply_vcycle<double>(p, i, r, z, pitch, st)
                 : run_apply_vcycle<float>(p, i, r, z, pitch, st);
}

extern "C" int gd_plan_set_profiling(gd_plan p, int32_t enable) {
  GD_REQUIRE(p, GD_ERR_ARG, "gd_plan_set_profiling: null plan");
  p->profiling = enable != 0;
  for (int k = 0; k < GD_KERNEL_KINDS; ++k) {
    p->prof_ms[k] = 0.0;
    p->prof_cells[k] = 0.0;
    p->prof_launches[k] = 0;
  }
  for (gd_kernel_time &t : p->prof_level) t = gd_kernel_time{0, 0.0, 0.0};
  p->ev_used = 0;
  return GD_OK;
}

extern "C" int gd_plan_kernel_times(gd_plan p, gd_kernel_time *out, int32_t n) {
  GD_REQUIRE(p && out && n >= GD_KERNEL_KINDS, GD_ERR_ARG,
             "gd_plan_kernel_times: need room for %d entries", GD_KERNEL_KINDS);
  for (int k = 0; k < GD_KERNEL_KINDS; ++k) {
    out[k].launches = p->prof_launches[k];
    out[k].milliseconds = p->prof_ms[k];
    out[k].cells = p->prof_cells[k];
  }
  return GD_OK;
}

extern "C" int gd_plan_level_times(gd_plan p, gd_kernel_time *out, int32_t n) {
  GD_REQUIRE(p && out && n >= GD_KERNEL_KINDS * GD_PROFILE_LEVELS, GD_ERR_ARG,
             "gd_plan_level_times: need room for %d entries",
             GD_KERNEL_KINDS * GD_PROFILE_LEVELS);
  std::copy(p->prof_level, p->prof_level + GD_KERNEL_KINDS * GD_PROFILE_LEVELS, out);
  return GD_OK;
}

namespace {
// Self-test of the bounded waits of the bulk-copy rings: one warp arms an
// mbarrier for 16 bytes that no copy will deliver and waits for it with a limit
// of `tries` attempts.  The wait gives up, sets the error bit and returns;
// nothing is in flight when the block exits.
__global__ void k_wait_selftest(unsigned *err, int tries, int *completed) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) bulk::init(&bar, 1);
  bulk::init_fence();
  __syncwarp();
  if (threadIdx.x == 0) bulk::arrive_expect(&bar, 16);
  __syncwarp();
  const bool ok = bulk::wait(&bar, 0u, err, tries);
  if (threadIdx.x == 0) *completed = ok ? 1 : 0;
}
}  // namespace

extern "C" int gd_selftest_bounded_wait(int32_t tries, int32_t *err, int32_t *completed,
                                        cudaStream_t st) {
  GD_REQUIRE(err && completed && tries >= 1 && tries <= bulk::kWaitTries, GD_ERR_ARG,
             "gd_selftest_bounded_wait: bad arguments");
  k_wait_selftest<<<1, 32, 0, st>>>(reinterpret_cast<unsigned *>(err), tries, completed);
  GD_CHECK_LAUNCH();
  return GD_OK;
}
