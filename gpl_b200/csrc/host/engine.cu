// The device engine: HBM-resident Nesterov state, the trial's launches, the solves.
#include <algorithm>
#include <cstring>
#include <numeric>

#include "../kernels/b2b.h"
#include "../kernels/bicgstab.h"
#include "../kernels/common.cuh"
#include "../kernels/engine_kernels.h"
#include "engine.h"
#include "parallel.h"
#include "tune.h"

namespace gpl {
void progress(const char *fmt, ...) __attribute__((format(printf, 1, 2)));
}

namespace gpl {

struct Engine::Region {
  RegionArgs args{};
  int32_t *bx = nullptr, *by = nullptr;
  float *scaled = nullptr, *density = nullptr, *fx = nullptr, *fy = nullptr;
  float *np = nullptr, *npu = nullptr;
  int64_t *acc_inst = nullptr, *acc_fill = nullptr;
  float2 *slot[S_NUM] = {};
  int64_t cell_off = 0, n_cells = 0;
  PoissonPlan *plan = nullptr;
  double *part = nullptr;
  unsigned int *ticket = nullptr;  // arrivals of the finalize's and the gradients' blocks
  int nb_bins = 0, nb_cells = 0;
  __nv_bfloat16 *dens_split = nullptr;
  int split_ld = 0;
  std::vector<float> np_host, npu_host;  // staging of an update_bins copy
  unsigned int *spread = nullptr;  // the scatter's spread blocks (cleared by the finalize)
  int32_t *order = nullptr;        // each device cell's index at upload (since take_order)
  bool order_moved = false;
  double spread_base = 0;          // the spread blocks of the order as made
  bool need_base = true;           // the next scatter's count is that base
  int64_t reorder_trial = -1000;   // the trial of the last reorder
  // the scatter's form (shared tiles, straight to HBM, or straight to HBM pooled by bin: the
  // same int64 sums every way), timed in place; GPL_SCATTER=tiles|global|pooled fixes it
  std::unique_ptr<Tuner> scatter_tune = std::make_unique<Tuner>("scatter", std::vector<std::string>{"tiles", "global", "pooled"}, "GPL_SCATTER", 3, 64);
};

struct Engine::QueueEntry {
  int kind;
  int region;
  PackedRegion e;  // the phase's arguments as queued (the slots as they were then)
};

// Page-locked table slots between two trial reads (each packed launch's tables in a slot of
// their own, as the copies out of them may still be queued).
constexpr int kTableSlots = 8;

// A region's density solver: the split-BF16 tensor-core form takes grids of at least 512 bins
// a side; a smaller grid's GEMMs are a few tiles each, too few to fill the tensor cores, so it
// runs the FP32 form (which packed launches then solve with every other such region at once).
static int region_plan_mode(int mode, int nx, int ny) { return mode == 1 && (nx < 512 || ny < 512) ? 0 : mode; }

static int blocks_for(int64_t n, int per = kThreadsPerBlock) { return (int)std::max<int64_t>(1, (n + per - 1) / per); }

// Whether the scatter's shared tile can sum in 32 bits: a cell adds at most a bin's area to a
// bin (its overlap, times a scale of at most 1), once, so a block's sum for one bin stays below
// kThreadsPerBlock times the largest bin area.
bool narrow_tile(const std::vector<int32_t> &bx, const std::vector<int32_t> &by) {
  int64_t w = 0, h = 0;
  for (size_t k = 0; k + 1 < bx.size(); k++) w = std::max<int64_t>(w, (int64_t)bx[k + 1] - bx[k]);
  for (size_t k = 0; k + 1 < by.size(); k++) h = std::max<int64_t>(h, (int64_t)by[k + 1] - by[k]);
  return (double)w * (double)h * kThreadsPerBlock < 4294967295.0;
}

// The fixed areas as float (int64 -> float, round to nearest), as the bin density reads them.
static std::vector<float> as_float(const std::vector<int64_t> &v) {
  std::vector<float> out(v.size());
  for (size_t k = 0; k < v.size(); k++) out[k] = (float)v[k];
  return out;
}

void Engine::check(cudaError_t e, const char *where) {
  if (e != cudaSuccess && err_.code == cudaSuccess) {
    err_.code = e;
    err_.where = where;
  }
}

Engine::Engine(int device) : device_(device) {
  check(cudaSetDevice(device), "cudaSetDevice");
  // device buffers come from the device's pool, which keeps freed memory for the next run
  if (!failed()) keep_device_pool();
  // the trial's own stream at the highest priority and the WA's beside it at the lowest: when
  // both have blocks waiting, an SM that frees up takes the density solve's first
  int prio_lo = 0, prio_hi = 0;
  cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
  if (!failed()) check(cudaStreamCreateWithPriority(&stream_, cudaStreamNonBlocking, prio_hi), "cudaStreamCreate");
  if (!failed()) check(cudaStreamCreateWithPriority(&wa_stream_, cudaStreamNonBlocking, prio_lo), "cudaStreamCreate");
  if (!failed()) check(cudaStreamCreateWithPriority(&wa2_stream_, cudaStreamNonBlocking, prio_lo), "cudaStreamCreate");
  if (!failed()) check(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming), "cudaEventCreate");
  if (!failed()) check(cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming), "cudaEventCreate");
  if (!failed()) check(cudaEventCreateWithFlags(&ev_split_, cudaEventDisableTiming), "cudaEventCreate");
  if (!failed()) check(cudaEventCreateWithFlags(&ev_join2_, cudaEventDisableTiming), "cudaEventCreate");
  // the degree-2..4 nets' WA form, timed in place; GPL_WA_SMALL=lean|nets|pins fixes it
  if (!failed()) wa_tune_ = std::make_unique<Tuner>("small-net WA", std::vector<std::string>{"lean", "nets", "pins"}, "GPL_WA_SMALL", 3, 256);
  if (!failed()) pk_scatter_tune_ = std::make_unique<Tuner>("packed scatter", std::vector<std::string>{"tiles", "global", "pooled"}, "GPL_SCATTER", 3, 64);
  queue_ = new std::vector<QueueEntry>();
}

void Engine::join() {
  if (!wa_pending_) return;
  check(cudaStreamWaitEvent(stream_, ev_join_, 0), "join");
  check(cudaStreamWaitEvent(stream_, ev_join2_, 0), "join");
  wa_pending_ = false;
}

void Engine::prewarm(size_t bytes) {
  prewarm_join();
  const int dev = device_;
  prewarm_ = new std::thread([dev, bytes] {
    if (cudaSetDevice(dev) != cudaSuccess) return;
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return;
    keep_device_pool();
    void *p = nullptr;
    if (bytes && cudaMallocAsync(&p, bytes, s) == cudaSuccess) cudaFreeAsync(p, s);
    load_kernel_modules();
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    cudaGetLastError();  // nothing of it is an error of the command's
  });
}

void Engine::prewarm_join() {
  if (!prewarm_) return;
  prewarm_->join();
  delete prewarm_;
  prewarm_ = nullptr;
}

Engine::~Engine() {
  prewarm_join();
  release();
  delete queue_;
  if (pk_host_) cudaFreeHost(pk_host_);
  if (pk_dev_) cudaFree(pk_dev_);
  if (pinned_) cudaFreeHost(pinned_);
  if (wa_stream_) cudaStreamSynchronize(wa_stream_);
  if (wa2_stream_) cudaStreamSynchronize(wa2_stream_);
  if (stream_) cudaStreamDestroy(stream_);
  if (wa_stream_) cudaStreamDestroy(wa_stream_);
  if (wa2_stream_) cudaStreamDestroy(wa2_stream_);
  if (ev_split_) cudaEventDestroy(ev_split_);
  if (ev_join2_) cudaEventDestroy(ev_join2_);
  if (ev_fork_) cudaEventDestroy(ev_fork_);
  if (ev_join_) cudaEventDestroy(ev_join_);
}

template <class T>
static cudaError_t dmalloc(T **p, size_t n, cudaStream_t s) {
  *p = nullptr;
  if (n == 0) n = 1;
  return cudaMallocAsync((void **)p, n * sizeof(T), s);  // from the device's pool (kept)
}
static int64_t g_h2d = 0;  // bytes the uploads below copied (folded into the engine's counter)
template <class T, class A>
static cudaError_t upload_vec(T **p, const std::vector<T, A> &v, cudaStream_t s) {
  cudaError_t e = dmalloc(p, v.size(), s);
  if (e != cudaSuccess || v.empty()) return e;
  g_h2d += (int64_t)(v.size() * sizeof(T));
  return cudaMemcpyAsync(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

// ---------------------------------------------------------------- Nesterov state
void Engine::free_globals() {
  void *ptrs[] = {dc_, hx_, hy_, dscale_, area_, kind_, locked_, cell_pin_start_, net_start_, pin_cell_, pin_slot_, big_nets_, pin_base_, tiles_, net_weight_, pin_grad_, hpwl_acc_, dev_scal_};
  for (void *p : ptrs)
    if (p) cudaFreeAsync(p, stream_);
  dc_ = nullptr;
  hx_ = hy_ = nullptr;
  dscale_ = area_ = nullptr;
  kind_ = locked_ = nullptr;
  cell_pin_start_ = nullptr;
  net_start_ = nullptr;
  pin_cell_ = pin_slot_ = big_nets_ = nullptr;
  pin_base_ = nullptr;
  tiles_ = nullptr;
  n_tiles_ = n_big_ = 0;
  small_ = WaSmall{};
  net_weight_ = nullptr;
  pin_grad_ = nullptr;
  hpwl_acc_ = nullptr;
  dev_scal_ = nullptr;
}

void Engine::release() {
  flush();
  join();
  poisson_group_destroy(group_);
  group_ = nullptr;
  group_set_.clear();
  for (Region *r : regions_) {
    void *ptrs[] = {r->bx, r->by, r->scaled, r->density, r->fx, r->fy, r->np, r->npu, r->acc_inst, r->acc_fill, r->part, r->ticket, r->spread, r->order};
    for (void *p : ptrs)
      if (p) cudaFreeAsync(p, stream_);
    for (int k = 0; k < S_NUM; k++)
      if (r->slot[k]) cudaFreeAsync(r->slot[k], stream_);
    poisson_plan_destroy(r->plan);
    delete r;
  }
  if (!regions_.empty()) progress("  release: regions freed");
  regions_.clear();
  free_globals();
}

void Engine::upload(const EngineSetup &s) {
  prewarm_join();
  release();
  hpwl_ready_ = hpwl_fetched_ = false;  // the density centres move
  if (failed()) return;
  cudaStream_t st = stream_;
  n_cells_ = (int64_t)s.hx.size();
  n_pins_ = (int64_t)s.pin_cell.size();
  n_nets_ = (int32_t)(s.net_start.size() - 1);
  {
    std::vector<int2> dc(n_cells_);
    for (int64_t i = 0; i < n_cells_; i++) dc[i] = make_int2(s.dcx[i], s.dcy[i]);
    check(upload_vec(&dc_, dc, st), "upload cells");
  }
  check(upload_vec(&hx_, s.hx, st), "upload cells");
  check(upload_vec(&hy_, s.hy, st), "upload cells");
  check(upload_vec(&dscale_, s.dscale, st), "upload cells");
  check(upload_vec(&area_, s.area, st), "upload cells");
  check(upload_vec(&kind_, s.kind, st), "upload cells");
  any_locked_ = std::any_of(s.locked.begin(), s.locked.end(), [](uint8_t v) { return v != 0; });
  if (any_locked_) check(upload_vec(&locked_, s.locked, st), "upload cells");
  check(upload_vec(&cell_pin_start_, s.cell_pin_start, st), "upload cells");
  {
    // The nets in degree order, their pins following them: a WA tile then holds
    // nets of one degree, so its thread-per-net phases do not diverge. No result depends on
    // the order: each pin's force goes to its place in its cell's pin list (pin_slot), the
    // HPWL is an integer sum, a net's weight moves with it.
    // Within a degree, the nets in order of their lowest device cell (the cells are on a
    // Hilbert curve), so a warp's nets and their first pins' cells lie close together.
    std::vector<int64_t> by_deg;
    int64_t max_deg = 0;
    for (int32_t n = 0; n < n_nets_; n++) max_deg = std::max(max_deg, s.net_start[n + 1] - s.net_start[n]);
    std::vector<int32_t> low(n_nets_);
    parallel_for((size_t)n_nets_, [&](size_t a, size_t b) {
      for (size_t n = a; n < b; n++) {
        int32_t m = (int32_t)n_cells_;
        for (int64_t q = s.net_start[n]; q < s.net_start[n + 1]; q++)
          if (s.pin_cell[q] >= 0) m = std::min(m, s.pin_cell[q]);
        low[n] = m;
      }
    });
    std::vector<int32_t> by_cell(n_nets_);
    {
      std::vector<int64_t> cnt((size_t)n_cells_ + 2, 0);
      for (int32_t n = 0; n < n_nets_; n++) cnt[(size_t)low[n] + 1]++;
      for (size_t k = 1; k < cnt.size(); k++) cnt[k] += cnt[k - 1];
      for (int32_t n = 0; n < n_nets_; n++) by_cell[cnt[low[n]]++] = n;
    }
    net_order_.resize(n_nets_);
    if (max_deg <= (int64_t)1 << 20) {
      by_deg.assign(max_deg + 2, 0);
      for (int32_t n = 0; n < n_nets_; n++) by_deg[s.net_start[n + 1] - s.net_start[n] + 1]++;
      for (int64_t d = 0; d <= max_deg; d++) by_deg[d + 1] += by_deg[d];
      for (int32_t n : by_cell) net_order_[by_deg[s.net_start[n + 1] - s.net_start[n]]++] = n;
    } else {
      net_order_ = by_cell;
      std::stable_sort(net_order_.begin(), net_order_.end(), [&](int32_t a, int32_t b) { return s.net_start[a + 1] - s.net_start[a] < s.net_start[b + 1] - s.net_start[b]; });
    }
    // each pin's force goes to its place in its cell's pin list (cell_pins lists each pin once)
    std::vector<int32_t> slot;
    big_assign(slot, (size_t)n_pins_, -1);
    parallel_for(s.cell_pins.size(), [&](size_t a, size_t b) {
      for (size_t k = a; k < b; k++) slot[s.cell_pins[k]] = (int32_t)k;
    });
    std::vector<int64_t> ns(n_nets_ + 1, 0);
    parallel_for((size_t)n_nets_, [&](size_t a, size_t b) {
      for (size_t i = a; i < b; i++) ns[i + 1] = s.net_start[net_order_[i] + 1] - s.net_start[net_order_[i]];
    });
    for (int32_t i = 0; i < n_nets_; i++) ns[i + 1] += ns[i];
    std::vector<int32_t> pc, ps;
    std::vector<int2> pb;
    big_resize(pc, (size_t)n_pins_);
    big_resize(ps, (size_t)n_pins_);
    big_resize(pb, (size_t)n_pins_);
    std::vector<float> wt(n_nets_);
    parallel_for((size_t)n_nets_, [&](size_t a, size_t b) {
      for (size_t i = a; i < b; i++) {
        int32_t n = net_order_[i];
        int64_t at = ns[i];
        for (int64_t q = s.net_start[n]; q < s.net_start[n + 1]; q++, at++) {
          pc[at] = s.pin_cell[q];
          ps[at] = slot[q];
          pb[at] = make_int2(s.pin_base[2 * q], s.pin_base[2 * q + 1]);
        }
        wt[i] = s.net_weight[n];
      }
    });
    if (ns[n_nets_] >= ((int64_t)1 << 31)) check(cudaErrorInvalidValue, "upload nets: 2^31 pins or more");
    check(upload_vec(&net_start_, ns, st), "upload nets");
    // WA's tiles of consecutive nets, and the nets too large for a tile (already in degree
    // order, so a warp's threads walk nets of one length)
    // the degree-2..4 nets run a lane per pin (k_wa_pins); the tiles take the rest: the
    // nets below degree 2 and those above 4
    small_ = wa_small_ranges(ns.data(), n_nets_);
    const int32_t small_lo = small_.first[0], small_hi = small_.first[2] + small_.count[2];
    std::vector<int4> tiles;
    std::vector<int32_t> big;
    wa_tiles(ns.data(), 0, small_lo, tiles, big);
    wa_tiles(ns.data(), small_hi, n_nets_, tiles, big);
    n_tiles_ = (int32_t)tiles.size();
    n_big_ = (int32_t)big.size();
    check(upload_vec(&tiles_, tiles, st), "upload nets");
    check(upload_vec(&big_nets_, big, st), "upload nets");
    check(upload_vec(&pin_slot_, ps, st), "upload pins");
    check(upload_vec(&pin_cell_, pc, st), "upload pins");
    check(upload_vec(&pin_base_, pb, st), "upload pins");
    check(upload_vec(&net_weight_, wt, st), "upload nets");
    unit_weights_ = std::all_of(wt.begin(), wt.end(), [](float v) { return v == 1.0f; });
  }
  progress("  upload: cells, nets and pins");
  check(dmalloc(&pin_grad_, s.cell_pins.size(), st), "alloc pins");
  check(dmalloc(&hpwl_acc_, 1, st), "alloc");
  check(dmalloc(&dev_scal_, s.regions.size(), st), "alloc");
  host_scal_.assign(s.regions.size(), RegionScalars{});
  {
    size_t need = s.regions.size() * sizeof(RegionScalars) + sizeof(unsigned long long);
    if (need > pinned_bytes_) {
      if (pinned_) cudaFreeHost(pinned_);
      pinned_ = nullptr;
      pinned_bytes_ = 0;
      check(cudaHostAlloc((void **)&pinned_, need, cudaHostAllocDefault), "alloc pinned");
      if (pinned_) pinned_bytes_ = need;
    }
  }
  region_wx_.clear();
  region_wy_.clear();
  region_dims_.clear();
  for (const RegionSetup &rs : s.regions) {
    region_wx_.push_back(rs.wx);
    region_wy_.push_back(rs.wy);
    region_dims_.push_back({rs.nx, rs.ny});
    Region *r = new Region();
    regions_.push_back(r);
    int64_t nb = (int64_t)rs.nx * rs.ny;
    r->cell_off = rs.cell_off;
    r->n_cells = rs.n_cells;
    check(upload_vec(&r->bx, rs.bx, st), "upload bins");
    check(upload_vec(&r->by, rs.by, st), "upload bins");
    check(upload_vec(&r->scaled, rs.scaled, st), "upload bins");
    check(upload_vec(&r->np, as_float(rs.non_place), st), "upload bins");
    check(upload_vec(&r->npu, as_float(rs.non_place_u), st), "upload bins");
    check(dmalloc(&r->acc_inst, nb, st), "alloc bins");
    check(dmalloc(&r->acc_fill, nb, st), "alloc bins");
    check(dmalloc(&r->density, nb, st), "alloc bins");
    check(dmalloc(&r->fx, nb, st), "alloc bins");
    check(dmalloc(&r->fy, nb, st), "alloc bins");
    if (!failed()) {
      check(cudaMemsetAsync(r->acc_inst, 0, nb * sizeof(int64_t), st), "memset");
      check(cudaMemsetAsync(r->acc_fill, 0, nb * sizeof(int64_t), st), "memset");
    }
    for (int k = 0; k < S_NUM; k++) {
      check(dmalloc(&r->slot[k], rs.n_cells, st), "alloc slots");
      if (!failed()) check(cudaMemsetAsync(r->slot[k], 0, std::max<int64_t>(rs.n_cells, 1) * sizeof(float2), st), "memset");
    }
    r->nb_bins = rs.nx;  // the bin finalize runs one block per x row
    r->nb_cells = blocks_for(rs.n_cells);
    check(dmalloc(&r->part, (size_t)std::max(r->nb_bins * 2, r->nb_cells * 4), st), "alloc partials");
    check(dmalloc(&r->ticket, 1, st), "alloc partials");
    if (!failed()) check(cudaMemsetAsync(r->ticket, 0, sizeof(unsigned int), st), "memset");
    check(dmalloc(&r->spread, 1, st), "alloc partials");
    if (!failed()) check(cudaMemsetAsync(r->spread, 0, sizeof(unsigned int), st), "memset");
    check(dmalloc(&r->order, rs.n_cells, st), "alloc order");
    if (!failed() && rs.n_cells) k_iota<<<blocks_for(rs.n_cells), kThreadsPerBlock, 0, st>>>((int32_t)rs.n_cells, r->order);
    r->order_moved = false;
    if (!failed()) {
      cudaError_t pe = cudaSuccess;
      const int mode = region_plan_mode(poisson_mode_, rs.nx, rs.ny);
      r->plan = poisson_plan_create(rs.nx, rs.ny, rs.wx.data(), rs.wy.data(), mode, &pe);
      check(pe, mode == 0 ? "poisson plan (fp32)" : mode == 2 ? "poisson plan (fp64)" : "poisson plan (split-bf16 tcgen05)");
      if (r->plan) r->dens_split = poisson_split_input(r->plan, &r->split_ld);
      progress("  upload: region solver planned (%dx%d bins)", rs.nx, rs.ny);
    }
    RegionArgs &a = r->args;
    a.n_cells = (int32_t)rs.n_cells;
    a.nx = rs.nx;
    a.ny = rs.ny;
    a.lx = rs.lx;
    a.ly = rs.ly;
    a.ux = rs.ux;
    a.uy = rs.uy;
    a.size_x = rs.size_x;
    a.size_y = rs.size_y;
    a.inv_size_x = 1.0 / rs.size_x;
    a.inv_size_y = 1.0 / rs.size_y;
    a.narrow = narrow_tile(rs.bx, rs.by) ? 1 : 0;
    a.target_density = rs.target_density;
    a.bx = r->bx;
    a.by = r->by;
    a.scaled = r->scaled;
    a.non_place = r->np;
    a.non_place_u = r->npu;
    a.acc_inst = r->acc_inst;
    a.acc_fill = r->acc_fill;
    a.density = r->density;
    a.field_x = r->fx;
    a.field_y = r->fy;
    a.spread = r->spread;
  }
  check(cudaStreamSynchronize(st), "upload sync");
  h2d_bytes += g_h2d + n_pins_ * 8;
  g_h2d = 0;
}

void Engine::update_bins(int b, const RegionSetup &rs) {
  flush();
  join();
  Region *r = regions_[b];
  r->args.target_density = rs.target_density;
  size_t nb = rs.scaled.size();
  check(cudaMemcpyAsync(r->scaled, rs.scaled.data(), nb * sizeof(float), cudaMemcpyHostToDevice, stream_), "update bins");
  // staged in the region (the copy is asynchronous), converted as the density reads them
  r->np_host = as_float(rs.non_place);
  r->npu_host = as_float(rs.non_place_u);
  check(cudaMemcpyAsync(r->np, r->np_host.data(), nb * sizeof(float), cudaMemcpyHostToDevice, stream_), "update bins");
  check(cudaMemcpyAsync(r->npu, r->npu_host.data(), nb * sizeof(float), cudaMemcpyHostToDevice, stream_), "update bins");
  check(cudaStreamSynchronize(stream_), "update bins");
}

void Engine::rewrite_cells(const EngineSetup &s) {
  flush();
  join();
  // sizes and density sizes of every cell (routability's inflation and filler changes keep
  // the cell count of a region's block only when no filler moved; the caller re-uploads then)
  size_t n = s.hx.size();
  if ((int64_t)n != n_cells_) {
    check(cudaErrorInvalidValue, "rewrite_cells: cell count changed");
    return;
  }
  check(cudaMemcpyAsync(hx_, s.hx.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, stream_), "rewrite cells");
  check(cudaMemcpyAsync(hy_, s.hy.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, stream_), "rewrite cells");
  check(cudaMemcpyAsync(dscale_, s.dscale.data(), n * sizeof(float), cudaMemcpyHostToDevice, stream_), "rewrite cells");
  check(cudaMemcpyAsync(area_, s.area.data(), n * sizeof(float), cudaMemcpyHostToDevice, stream_), "rewrite cells");
}

static CellArgs cell_args(const int64_t off, int2 *dc, int32_t *hx, int32_t *hy, float *dscale, uint8_t *kind, uint8_t *locked, float *area, int64_t *ps, float2 *const *slot) {
  CellArgs c{};
  c.dc = dc + off;
  c.hx = hx + off;
  c.hy = hy + off;
  c.dscale = dscale + off;
  c.kind = kind + off;
  c.locked = locked ? locked + off : nullptr;
  c.area = area + off;
  c.pin_start = ps + off;
  c.cur_slp = slot[S_CUR_SLP];
  c.cur_slp_sum = slot[S_CUR_SLP_SUM];
  c.next_slp = slot[S_NEXT_SLP];
  c.next_slp_sum = slot[S_NEXT_SLP_SUM];
  c.prev_slp = slot[S_PREV_SLP];
  c.prev_slp_sum = slot[S_PREV_SLP_SUM];
  c.cur = slot[S_CUR];
  c.next = slot[S_NEXT];
  return c;
}

#define CELLS(r) cell_args((r)->cell_off, dc_, hx_, hy_, dscale_, kind_, locked_, area_, cell_pin_start_, (r)->slot)

void Engine::set_coords(int b, SlotId slot, const std::vector<float> &xy) {
  flush();
  join();
  Region *r = regions_[b];
  if (r->n_cells) check(cudaMemcpyAsync(r->slot[slot], xy.data(), r->n_cells * sizeof(float2), cudaMemcpyHostToDevice, stream_), "set_coords");
  h2d_bytes += r->n_cells * 8;
}

std::vector<float> Engine::get_coords(int b, SlotId slot) {
  flush();
  join();
  Region *r = regions_[b];
  std::vector<float> xy(2 * r->n_cells);
  if (r->n_cells) check(cudaMemcpyAsync(xy.data(), r->slot[slot], r->n_cells * sizeof(float2), cudaMemcpyDeviceToHost, stream_), "get_coords");
  d2h_bytes += r->n_cells * 8;
  check(cudaStreamSynchronize(stream_), "get_coords sync");
  return xy;
}

void Engine::fork_after_place() {
  if (!overlap_) return;
  check(cudaEventRecord(ev_fork_, stream_), "wa fork");
  fork_early_ = true;
}

void Engine::place_at(int b, SlotId slot) {
  flush();
  fork_early_ = false;
  join();
  if (failed()) return;
  hpwl_ready_ = hpwl_fetched_ = false;  // the density centres move
  Region *r = regions_[b];
  CellArgs c = CELLS(r);
  ph_begin(PH_PLACE);
  launches += (r->n_cells ? 1 : 0) + 1;
  RegionArgs a = r->args;
  a.scatter_form = r->scatter_tune->best();
  if (r->n_cells) k_place_cells<<<blocks_for(r->n_cells), kThreadsPerBlock, 0, stream_>>>(a, c, PLACE_AT, 0.0f, 0.0f, r->slot[slot]);
  ph_end(PH_PLACE);
  ph_begin(PH_FINALIZE);
  k_bins_finalize<<<r->nb_bins, kThreadsPerBlock, 0, stream_>>>(r->args, r->part, r->dens_split, r->split_ld, r->ticket, &dev_scal_[b].overflow);
  ph_end(PH_FINALIZE);
  check(cudaGetLastError(), "place_at");
}

void Engine::nesterov_step(int b, float step, float coeff) {
  join();
  if (failed()) return;
  {
    // the cells sorted again when the blocks that spread past the scatter's shared tile have
    // grown by 2 % of the blocks since the order was made (its own spread, in sparse patches,
    // is its base), at most once in 8 trials
    Region *rg = regions_[b];
    const double sp = host_scal_[b].spread_blocks;
    if (rg->need_base) {
      rg->spread_base = sp;
      rg->need_base = false;
    } else if (reorder_on_ && trials - rg->reorder_trial >= 8 && sp > rg->spread_base + 0.02 * rg->nb_cells) {
      reorder(b);
      rg->reorder_trial = trials;
      rg->need_base = true;
      if (failed()) return;
    }
  }
  hpwl_ready_ = hpwl_fetched_ = false;  // the density centres move
  Region *r = regions_[b];
  CellArgs c = CELLS(r);
  if (packed()) {
    QueueEntry q{};
    q.kind = Q_PLACE;
    q.region = b;
    q.e.r = r->args;
    q.e.c = c;
    q.e.step = step;
    q.e.coeff = coeff;
    q.e.partials = r->part;
    q.e.ticket = r->ticket;
    q.e.out = &dev_scal_[b].overflow;
    q.e.dens_split = r->dens_split;
    q.e.split_ld = r->split_ld;
    queue_->push_back(q);
    return;
  }
  ph_begin(PH_PLACE);
  launches += (r->n_cells ? 1 : 0) + 1;
  if (r->n_cells) {
    RegionArgs a = r->args;
    a.scatter_form = r->scatter_tune->start(stream_);
    k_place_cells<<<blocks_for(r->n_cells), kThreadsPerBlock, 0, stream_>>>(a, c, PLACE_NESTEROV, step, coeff, nullptr);
    fork_after_place();
    r->scatter_tune->stop(stream_);
  }
  ph_end(PH_PLACE);
  ph_begin(PH_FINALIZE);
  check(launch_chained(k_bins_finalize, dim3(r->nb_bins), dim3(kThreadsPerBlock), 0, stream_, r->args, r->part, r->dens_split, r->split_ld, r->ticket, &dev_scal_[b].overflow), "nesterov_step");
  ph_end(PH_FINALIZE);
  check(cudaGetLastError(), "nesterov_step");
}

void Engine::field(int b) {
  if (failed()) return;
  if (packed()) {
    QueueEntry q{};
    q.kind = Q_FIELD;
    q.region = b;
    queue_->push_back(q);
    return;
  }
  Region *r = regions_[b];
  ph_begin(PH_POISSON);
  check(poisson_solve(r->plan, r->density, r->fx, r->fy, stream_), "poisson");
  ph_end(PH_POISSON);
  launches += poisson_launches(r->plan);
}

WaArgs Engine::wa_args() const {
  WaArgs w{};
  w.n_nets = n_big_;
  w.net_start = net_start_;
  w.net_order = big_nets_;
  w.net_weight = unit_weights_ ? nullptr : net_weight_;  // x * 1.0f is x, bit for bit
  w.pin_cell = pin_cell_;
  w.pin_base = pin_base_;
  w.dc = dc_;
  w.pin_slot = pin_slot_;
  w.pin_grad = pin_grad_;
  w.n_tiles = n_tiles_;
  w.tiles = tiles_;
  w.small = small_;
  return w;
}

void Engine::wa(float cx, float cy) {
  flush();
  if (failed() || n_nets_ == 0) return;
  join();
  WaArgs w = wa_args();
  // forked after the work queued so far (the centres), joined by the forces' readers
  cudaStream_t st = overlap_ ? wa_stream_ : stream_;
  if (overlap_) {
    // the fork was recorded right after the last scatter (the new centres) when one ran since
    // the last WA: the WA then runs beside the bins' finalize too
    if (!fork_early_) check(cudaEventRecord(ev_fork_, stream_), "wa fork");
    check(cudaStreamWaitEvent(wa_stream_, ev_fork_, 0), "wa fork");
  }
  fork_early_ = false;
  // the kernels add the HPWL of these same positions: hpwl() reads it without a launch
  check(cudaMemsetAsync(hpwl_acc_, 0, sizeof(unsigned long long), st), "wa");
  w.hpwl_out = hpwl_acc_;
  hpwl_ready_ = true;
  hpwl_fetched_ = false;
  cudaStream_t st2 = st;
  if (overlap_) {
    check(cudaEventRecord(ev_split_, st), "wa split");
    check(cudaStreamWaitEvent(wa2_stream_, ev_split_, 0), "wa split");
    st2 = wa2_stream_;
  }
  ph_begin(PH_WA, st);
  if (wa_small_blocks(small_)) {
    launches += 1;
    const int form = wa_tune_->start(st2);
    launch_wa_small(w, cx, cy, 1, st2, form);
    wa_tune_->stop(st2);
  }
  if (n_tiles_) {
    launches += 1;
    launch_wa_tiles(w, cx, cy, st);
  }
  if (n_big_) {
    launches += 1;
    k_wa<<<blocks_for(n_big_), kThreadsPerBlock, 0, st>>>(w, cx, cy);
  }
  ph_end(PH_WA, st);
  check(cudaGetLastError(), "wa");
  if (overlap_) {
    check(cudaEventRecord(ev_join_, st), "wa join");
    check(cudaEventRecord(ev_join2_, st2), "wa join");
    wa_pending_ = true;
  }
}

void Engine::gradients(int b, SlotId out, float penalty, SlotId a1, SlotId b1, SlotId b2) {
  if (failed()) return;
  Region *r = regions_[b];
  CellArgs c = CELLS(r);
  const float2 *pa1 = a1 == S_NUM ? nullptr : r->slot[a1];
  const float2 *pb1 = b1 == S_NUM ? nullptr : r->slot[b1];
  const float2 *pb2 = b2 == S_NUM ? nullptr : r->slot[b2];
  if (packed()) {
    QueueEntry q{};
    q.kind = Q_GRAD;
    q.region = b;
    q.e.r = r->args;
    q.e.c = c;
    q.e.pin_grad = pin_grad_;
    q.e.penalty = penalty;
    q.e.out_sum = r->slot[out];
    q.e.a1 = pa1;
    q.e.b1 = pb1;
    q.e.b2 = pb2;
    q.e.partials = r->part;
    q.e.ticket = r->ticket;
    q.e.out = &dev_scal_[b].wl_sum;
    queue_->push_back(q);
    return;
  }
  join();
  if (r->n_cells) {
    ph_begin(PH_GRAD);
    launches += 1;
    check(launch_chained(k_gradients, dim3(r->nb_cells), dim3(kThreadsPerBlock), 0, stream_, r->args, c, pin_grad_, penalty, r->slot[out], pa1, pb1, pb2, r->part, r->ticket, &dev_scal_[b].wl_sum), "gradients");
    ph_end(PH_GRAD);
  } else {
    check(cudaMemsetAsync(&dev_scal_[b].wl_sum, 0, 4 * sizeof(double), stream_), "gradients");
  }
  check(cudaGetLastError(), "gradients");
}

void Engine::prev_slp(int b, float coef) {
  flush();
  join();
  if (failed()) return;
  Region *r = regions_[b];
  if (!r->n_cells) return;
  k_prev_slp<<<blocks_for(r->n_cells), kThreadsPerBlock, 0, stream_>>>(r->args, CELLS(r), coef);
  check(cudaGetLastError(), "prev_slp");
}

void Engine::hold_locked(int b) {
  flush();
  join();
  if (failed() || !any_locked_) return;
  Region *r = regions_[b];
  if (!r->n_cells) return;
  k_hold_locked<<<blocks_for(r->n_cells), kThreadsPerBlock, 0, stream_>>>(r->args, CELLS(r));
  check(cudaGetLastError(), "hold_locked");
}

void Engine::swap_slots(int b, SlotId a, SlotId c) { std::swap(regions_[b]->slot[a], regions_[b]->slot[c]); }

void Engine::copy_slot(int b, SlotId dst, SlotId src) {
  flush();
  join();
  Region *r = regions_[b];
  if (r->n_cells) check(cudaMemcpyAsync(r->slot[dst], r->slot[src], r->n_cells * sizeof(float2), cudaMemcpyDeviceToDevice, stream_), "copy_slot");
}

void Engine::fetch() {
  flush();
  join();
  if (failed() || host_scal_.empty()) return;
  const size_t bytes = host_scal_.size() * sizeof(RegionScalars);
  const bool with_hpwl = hpwl_ready_ && !hpwl_fetched_;
  check(cudaMemcpyAsync(pinned_, dev_scal_, bytes, cudaMemcpyDeviceToHost, stream_), "fetch");
  d2h_bytes += (int64_t)bytes;
  if (with_hpwl) {
    check(cudaMemcpyAsync(pinned_ + bytes, hpwl_acc_, sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream_), "fetch");
    d2h_bytes += (int64_t)sizeof(unsigned long long);
  }
  check(cudaStreamSynchronize(stream_), "fetch sync");
  if (failed()) return;
  std::memcpy(host_scal_.data(), pinned_, bytes);
  if (with_hpwl) {
    std::memcpy(&hpwl_host_, pinned_ + bytes, sizeof hpwl_host_);
    hpwl_fetched_ = true;
  }
  ph_flush();
  // the trial's timed launches have ended (the WA joined the stream before the copy)
  for (Region *r : regions_) r->scatter_tune->finish();
  wa_tune_->finish();
  pk_scatter_tune_->finish();
  pk_slot_ = 0;  // the stream has drained: every table slot is free
}

// ---- packed launches
bool Engine::stage_tables(size_t n) {
  const size_t need = (size_t)kTableSlots * n;
  if (need > pk_cap_) {
    check(cudaStreamSynchronize(stream_), "packed tables");
    if (pk_host_) cudaFreeHost(pk_host_);
    if (pk_dev_) cudaFree(pk_dev_);
    pk_host_ = nullptr;
    pk_dev_ = nullptr;
    pk_cap_ = 0;
    check(cudaMallocHost(&pk_host_, need * sizeof(PackedRegion)), "packed tables");
    check(cudaMalloc(&pk_dev_, need * sizeof(PackedRegion)), "packed tables");
    if (failed()) return false;
    pk_cap_ = need;
    pk_slot_ = 0;
  }
  if (pk_slot_ >= kTableSlots) {
    // every slot used since the last trial read: wait for the copies out of them
    check(cudaStreamSynchronize(stream_), "packed tables");
    pk_slot_ = 0;
  }
  return !failed();
}

void Engine::flush() {
  if (!queue_ || queue_->empty() || failed()) {
    if (queue_) queue_->clear();
    return;
  }
  std::vector<QueueEntry> q;
  q.swap(*queue_);
  size_t a = 0;
  while (a < q.size()) {
    // a run of one phase, each region at most once
    std::vector<char> seen(regions_.size(), 0);
    size_t b = a;
    while (b < q.size() && q[b].kind == q[a].kind && !seen[q[b].region]) seen[q[b].region] = 1, b++;
    if (q[a].kind == Q_PLACE)
      flush_place(q, a, b);
    else if (q[a].kind == Q_FIELD)
      flush_field(q, a, b);
    else
      flush_grad(q, a, b);
    a = b;
  }
}

// Table entries [first, first + n) of a slot copied to the device: the slot's device address.
static PackedRegion *copy_tables(Engine &eng, PackedRegion *host, PackedRegion *dev, size_t n, cudaStream_t s, int64_t &h2d) {
  eng.check(cudaMemcpyAsync(dev, host, n * sizeof(PackedRegion), cudaMemcpyHostToDevice, s), "packed tables");
  h2d += (int64_t)(n * sizeof(PackedRegion));
  return dev;
}

void Engine::flush_place(const std::vector<QueueEntry> &q, size_t a, size_t b) {
  join();  // the WA has read the centres this moves
  const size_t n = b - a;
  if (!stage_tables(2 * regions_.size())) return;
  PackedRegion *h = pk_host_ + (size_t)pk_slot_ * 2 * regions_.size(), *d = pk_dev_ + (size_t)pk_slot_ * 2 * regions_.size();
  pk_slot_++;
  // the scatter's table (regions with cells), then the finalize's (every region); the
  // scatter's form for every region (timed from the table's copy, the same for each form)
  bool any = false;
  for (size_t k = a; k < b; k++) any |= q[k].e.r.n_cells > 0;
  ph_begin(PH_PLACE);
  const int form = any ? pk_scatter_tune_->start(stream_) : 0;
  int ns = 0, blocks = 0;
  for (size_t k = a; k < b; k++) {
    const PackedRegion &e = q[k].e;
    if (e.r.n_cells <= 0) continue;
    h[ns] = e;
    h[ns].r.scatter_form = form;
    h[ns].first = blocks;
    h[ns].blocks = blocks_for(e.r.n_cells);
    blocks += h[ns].blocks;
    ns++;
  }
  int fb = 0;
  for (size_t k = a; k < b; k++) {
    PackedRegion &f = h[ns + (k - a)];
    f = q[k].e;
    f.first = fb;
    f.blocks = f.r.nx;  // one block per x row
    fb += f.blocks;
  }
  copy_tables(*this, h, d, ns + n, stream_, h2d_bytes);
  if (ns) {
    k_place_packed<<<blocks, kThreadsPerBlock, 0, stream_>>>(d, ns);
    fork_after_place();
    pk_scatter_tune_->stop(stream_);
    launches += 1;
  }
  ph_end(PH_PLACE);
  ph_begin(PH_FINALIZE);
  k_finalize_packed<<<fb, kThreadsPerBlock, 0, stream_>>>(d + ns, (int)n);
  launches += 1;
  ph_end(PH_FINALIZE);
  check(cudaGetLastError(), "packed place");
}

void Engine::flush_field(const std::vector<QueueEntry> &q, size_t a, size_t b) {
  // the FP32 solves as one group (made again when the set of regions changes), the others
  // one region a launch
  std::vector<char> set(regions_.size(), 0);
  std::vector<int> alone;
  for (size_t k = a; k < b; k++) {
    Region *r = regions_[q[k].region];
    if (r->plan && poisson_plan_mode(r->plan) == 0)
      set[q[k].region] = 1;
    else
      alone.push_back(q[k].region);
  }
  ph_begin(PH_POISSON);
  if (std::count(set.begin(), set.end(), 1)) {
    if (!group_ || set != group_set_) {
      check(cudaStreamSynchronize(stream_), "poisson group");
      poisson_group_destroy(group_);
      group_ = nullptr;
      std::vector<PoissonPlan *> plans;
      std::vector<const float *> dens;
      std::vector<float *> fx, fy;
      for (size_t k = 0; k < regions_.size(); k++)
        if (set[k]) {
          plans.push_back(regions_[k]->plan);
          dens.push_back(regions_[k]->density);
          fx.push_back(regions_[k]->fx);
          fy.push_back(regions_[k]->fy);
        }
      cudaError_t pe = cudaSuccess;
      group_ = poisson_group_create(plans.data(), dens.data(), fx.data(), fy.data(), (int)plans.size(), &pe);
      check(pe, "poisson group");
      group_set_ = set;
    }
    check(poisson_group_solve(group_, stream_), "poisson group");
    launches += poisson_group_launches(group_);
  }
  for (int k : alone) {
    Region *r = regions_[k];
    check(poisson_solve(r->plan, r->density, r->fx, r->fy, stream_), "poisson");
    launches += poisson_launches(r->plan);
  }
  ph_end(PH_POISSON);
}

void Engine::flush_grad(const std::vector<QueueEntry> &q, size_t a, size_t b) {
  join();  // the forces are the WA's
  if (!stage_tables(2 * regions_.size())) return;
  PackedRegion *h = pk_host_ + (size_t)pk_slot_ * 2 * regions_.size(), *d = pk_dev_ + (size_t)pk_slot_ * 2 * regions_.size();
  pk_slot_++;
  int n = 0, blocks = 0;
  for (size_t k = a; k < b; k++) {
    const PackedRegion &e = q[k].e;
    if (e.r.n_cells <= 0) {
      check(cudaMemsetAsync(e.out, 0, 4 * sizeof(double), stream_), "gradients");
      continue;
    }
    h[n] = e;
    h[n].first = blocks;
    h[n].blocks = blocks_for(e.r.n_cells);
    blocks += h[n].blocks;
    n++;
  }
  if (!n) return;
  copy_tables(*this, h, d, n, stream_, h2d_bytes);
  ph_begin(PH_GRAD);
  k_gradients_packed<<<blocks, kThreadsPerBlock, 0, stream_>>>(d, n);
  launches += 1;
  ph_end(PH_GRAD);
  check(cudaGetLastError(), "packed gradients");
}

void Engine::region_info(int b, int32_t out[4]) const {
  const Region *r = regions_[b];
  out[0] = region_dims_[b].first;
  out[1] = region_dims_[b].second;
  out[2] = (int32_t)r->n_cells;
  out[3] = r->plan ? poisson_plan_mode(r->plan) : -1;
}

std::string Engine::tuning() const {
  std::string s = wa_tune_ ? wa_tune_->report() : std::string();
  if (packed()) return s + "; " + pk_scatter_tune_->report();
  for (size_t b = 0; b < regions_.size(); b++)
    if (regions_[b]->n_cells) s += "; region " + std::to_string(b) + " " + regions_[b]->scatter_tune->report();
  return s;
}

int64_t Engine::hpwl() {
  flush();
  join();
  if (failed()) return 0;
  if (hpwl_ready_ && hpwl_fetched_) return (int64_t)hpwl_host_;  // read with the trial's scalars
  WaArgs w = wa_args();
  if (!hpwl_ready_) {
  check(cudaMemsetAsync(hpwl_acc_, 0, sizeof(unsigned long long), stream_), "hpwl");
  ph_begin(PH_HPWL);
  if (wa_small_blocks(small_)) {
    launches += 1;
    WaArgs wh = w;
    wh.hpwl_out = hpwl_acc_;
    launch_wa_small(wh, 0.0f, 0.0f, 0, stream_, wa_tune_->best());
  }
  if (n_tiles_) {
    launches += 1;
    k_hpwl_tiles<<<n_tiles_, kThreadsPerBlock, 0, stream_>>>(w, hpwl_acc_);
  }
  if (n_big_) {
    launches += 1;
    k_hpwl<<<blocks_for(n_big_), kThreadsPerBlock, 0, stream_>>>(w, hpwl_acc_);
  }
  ph_end(PH_HPWL);
  hpwl_ready_ = true;
  }
  unsigned long long h = 0;
  check(cudaMemcpyAsync(&h, hpwl_acc_, sizeof h, cudaMemcpyDeviceToHost, stream_), "hpwl");
  d2h_bytes += 8;
  check(cudaStreamSynchronize(stream_), "hpwl sync");
  ph_flush();
  if (!failed()) {
    hpwl_host_ = h;
    hpwl_fetched_ = true;
  }
  return (int64_t)h;
}

void Engine::centres(std::vector<int32_t> &dcx, std::vector<int32_t> &dcy) {
  flush();
  join();
  std::vector<int2> dc(n_cells_);
  if (n_cells_) {
    check(cudaMemcpyAsync(dc.data(), dc_, n_cells_ * sizeof(int2), cudaMemcpyDeviceToHost, stream_), "centres");
    d2h_bytes += n_cells_ * 8;
  }
  check(cudaStreamSynchronize(stream_), "centres sync");
  dcx.resize(n_cells_);
  dcy.resize(n_cells_);
  for (int64_t i = 0; i < n_cells_; i++) {
    dcx[i] = dc[i].x;
    dcy[i] = dc[i].y;
  }
}

void Engine::set_net_weights(const std::vector<float> &w) {
  flush();
  join();
  if (w.empty()) return;
  if (w.size() != net_order_.size()) {
    check(cudaErrorInvalidValue, "net weights");
    return;
  }
  // in the device's net order (a copy from pageable memory returns once the data is staged)
  std::vector<float> dw(w.size());
  for (size_t i = 0; i < w.size(); i++) dw[i] = w[net_order_[i]];
  unit_weights_ = std::all_of(dw.begin(), dw.end(), [](float v) { return v == 1.0f; });
  check(cudaMemcpyAsync(net_weight_, dw.data(), dw.size() * sizeof(float), cudaMemcpyHostToDevice, stream_), "net weights");
}

// The region's cells in a new device order (cell_order.cu): sorted by the Hilbert index of
// their density centres, stably; every per-cell array gathered through the permutation, the
// cell-major pin lists moved with their cells (each cell's pins keep their order), the pins'
// cell indices and slots remapped. Scratch from the device's pool, returned at the end.
void Engine::reorder(int b) {
  flush();
  join();
  Region *r = regions_[b];
  const int32_t n = (int32_t)r->n_cells;
  if (failed() || n < 2) return;
  cudaStream_t st = stream_;
  const int64_t off = r->cell_off;
  uint32_t *key0 = nullptr, *key1 = nullptr;
  int32_t *idx0 = nullptr, *idx1 = nullptr, *hist = nullptr, *inv = nullptr, *ord = nullptr, *hx = nullptr, *hy = nullptr;
  int2 *dc = nullptr;
  float *ds = nullptr, *ar = nullptr;
  uint8_t *kd = nullptr, *lk = nullptr;
  int64_t *cnt = nullptr, *tmp = nullptr;
  float2 *slot[S_NUM] = {};
  check(dmalloc(&key0, n, st), "reorder");
  check(dmalloc(&key1, n, st), "reorder");
  check(dmalloc(&idx0, n, st), "reorder");
  check(dmalloc(&idx1, n, st), "reorder");
  check(dmalloc(&hist, (size_t)64 * order_tiles(n), st), "reorder");
  check(dmalloc(&inv, n, st), "reorder");
  check(dmalloc(&ord, n, st), "reorder");
  check(dmalloc(&dc, n, st), "reorder");
  check(dmalloc(&hx, n, st), "reorder");
  check(dmalloc(&hy, n, st), "reorder");
  check(dmalloc(&ds, n, st), "reorder");
  check(dmalloc(&ar, n, st), "reorder");
  check(dmalloc(&kd, n, st), "reorder");
  if (locked_) check(dmalloc(&lk, n, st), "reorder");
  check(dmalloc(&cnt, (size_t)n + 1, st), "reorder");
  check(dmalloc(&tmp, scan_i64_tmp(n), st), "reorder");
  for (int k = 0; k < S_NUM; k++) check(dmalloc(&slot[k], n, st), "reorder");
  if (!failed()) {
    const RegionArgs &a = r->args;
    check(order_sort(n, dc_ + off, a.lx, a.ly, std::max(1.0, (double)(a.ux - a.lx) / 1024.0), std::max(1.0, (double)(a.uy - a.ly) / 1024.0), key0, idx0, key1, idx1, hist, st), "reorder sort");
    static_assert(S_NUM <= kMaxSlots, "the gather's slot table");
    CellGather g{};
    g.dc = dc_ + off;
    g.hx = hx_ + off;
    g.hy = hy_ + off;
    g.dscale = dscale_ + off;
    g.area = area_ + off;
    g.kind = kind_ + off;
    g.locked = locked_ ? locked_ + off : nullptr;
    g.pin_start = cell_pin_start_ + off;
    g.order = r->order;
    g.dc_out = dc;
    g.hx_out = hx;
    g.hy_out = hy;
    g.dscale_out = ds;
    g.area_out = ar;
    g.kind_out = kd;
    g.locked_out = lk;
    g.pins_out = cnt;
    g.inv = inv;
    g.order_out = ord;
    g.n_slots = S_NUM;
    for (int k = 0; k < S_NUM; k++) {
      g.slot[k] = r->slot[k];
      g.slot_out[k] = slot[k];
    }
    k_order_gather<<<blocks_for(n), kThreadsPerBlock, 0, st>>>(n, idx0, g);
    check(cudaGetLastError(), "reorder gather");
    // the new pin starts (relative to the region's first slot), then the pins remapped from
    // the old starts, then the old starts overwritten
    check(scan_i64(cnt, n, tmp, st), "reorder scan");
    if (n_pins_) k_order_pins<<<blocks_for(n_pins_), kThreadsPerBlock, 0, st>>>(n_pins_, (int32_t)off, n, inv, cell_pin_start_ + off, cnt, pin_cell_, pin_slot_);
    k_order_starts<<<blocks_for(n), kThreadsPerBlock, 0, st>>>(n, cnt, cell_pin_start_ + off);
    check(cudaGetLastError(), "reorder pins");
    auto back = [&](auto *dst, const auto *src, size_t elems) { check(cudaMemcpyAsync(dst, src, elems * sizeof(*src), cudaMemcpyDeviceToDevice, st), "reorder copy"); };
    back(dc_ + off, dc, n);
    back(hx_ + off, hx, n);
    back(hy_ + off, hy, n);
    back(dscale_ + off, ds, n);
    back(area_ + off, ar, n);
    back(kind_ + off, kd, n);
    if (locked_) back(locked_ + off, lk, n);
    std::swap(r->order, ord);
    for (int k = 0; k < S_NUM; k++) std::swap(r->slot[k], slot[k]);
    r->order_moved = true;
    reorders++;
    launches += 12;
  }
  void *bufs[] = {key0, key1, idx0, idx1, hist, inv, ord, dc, hx, hy, ds, ar, kd, lk, cnt, tmp};
  for (void *p : bufs)
    if (p) cudaFreeAsync(p, st);
  for (int k = 0; k < S_NUM; k++)
    if (slot[k]) cudaFreeAsync(slot[k], st);
}

bool Engine::take_order(int b, std::vector<int32_t> &order) {
  flush();
  join();
  Region *r = regions_[b];
  if (!r->order_moved || failed()) return false;
  order.resize((size_t)r->n_cells);
  if (r->n_cells) check(cudaMemcpyAsync(order.data(), r->order, r->n_cells * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_), "take_order");
  d2h_bytes += r->n_cells * 4;
  if (r->n_cells) k_iota<<<blocks_for(r->n_cells), kThreadsPerBlock, 0, stream_>>>((int32_t)r->n_cells, r->order);
  check(cudaStreamSynchronize(stream_), "take_order sync");
  r->order_moved = false;
  return !failed();
}

void Engine::rebuild_poisson(int mode) {
  flush();
  join();
  poisson_mode_ = mode;
  check(cudaStreamSynchronize(stream_), "rebuild sync");
  poisson_group_destroy(group_);
  group_ = nullptr;
  group_set_.clear();
  for (size_t b = 0; b < regions_.size(); b++) {
    Region *r = regions_[b];
    check(cudaStreamSynchronize(stream_), "rebuild sync");
    poisson_plan_destroy(r->plan);
    r->plan = nullptr;
    r->dens_split = nullptr;
    r->split_ld = 0;
    cudaError_t pe = cudaSuccess;
    const int rmode = region_plan_mode(mode, region_dims_[b].first, region_dims_[b].second);
    r->plan = poisson_plan_create(region_dims_[b].first, region_dims_[b].second, region_wx_[b].data(), region_wy_[b].data(), rmode, &pe);
    check(pe, rmode == 0 ? "poisson plan (fp32)" : rmode == 2 ? "poisson plan (fp64)" : "poisson plan (split-bf16 tcgen05)");
    if (r->plan) {
      r->dens_split = poisson_split_input(r->plan, &r->split_ld);
      // the current density into the new operand, the field recomputed
      if (r->dens_split) check(poisson_split_density(r->plan, r->density, stream_), "split density");
      check(poisson_solve(r->plan, r->density, r->fx, r->fy, stream_), "poisson");
    }
  }
  check(cudaStreamSynchronize(stream_), "rebuild sync");
}

void Engine::set_profile(bool on) {
  profile_ = on;
  for (int k = 0; k < PH_COUNT; k++) {
    ph_ms_[k] = 0;
    ph_n_[k] = 0;
  }
  ev_pending_.clear();
  ev_used_ = 0;
}

void Engine::ph_begin(int ph, cudaStream_t on) {
  if (!profile_) return;
  if (!on) on = stream_;
  if (ev_used_ + 2 > ev_.size()) {
    for (int k = 0; k < 64; k++) {
      cudaEvent_t e;
      check(cudaEventCreate(&e), "event");
      ev_.push_back(e);
    }
  }
  check(cudaEventRecord(ev_[ev_used_], on), "event record");
  ev_pending_.push_back({ph, ev_used_});
  ev_used_ += 2;
}

void Engine::ph_end(int ph, cudaStream_t on) {
  if (!profile_ || ev_pending_.empty()) return;
  check(cudaEventRecord(ev_[ev_pending_.back().second + 1], on ? on : stream_), "event record");
}

void Engine::ph_flush() {
  if (!profile_) return;
  for (auto &[ph, i] : ev_pending_) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, ev_[i], ev_[i + 1]) == cudaSuccess) {
      ph_ms_[ph] += ms;
      ph_n_[ph] += 1;
    }
  }
  ev_pending_.clear();
  ev_used_ = 0;
}

int Engine::profile_read(double *ms, int64_t *launches, int cap) {
  int n = std::min<int>(cap, PH_COUNT);
  for (int k = 0; k < n; k++) {
    ms[k] = ph_ms_[k];
    launches[k] = ph_n_[k];
  }
  return n;
}

}  // namespace gpl
