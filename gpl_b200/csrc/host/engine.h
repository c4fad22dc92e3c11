// The device half of the engine: the Nesterov state resident in HBM and the trial's kernels,
// and the initial placement's solve. The host control (nesterov.cpp) only sees scalars: the
// overflow and gradient sums, the step-length distances and the HPWL, read once per trial.
#pragma once
#include "pod_vector.h"
#include <cstdint>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "host.h"

namespace gpl {

struct PoissonPlan;
struct PoissonGroup;
struct WaArgs;
struct PackedRegion;
class Tuner;

// What the device needs of one region (a `NesterovBase`'s bin grid).
struct RegionSetup {
  int32_t lx = 0, ly = 0, ux = 0, uy = 0, nx = 0, ny = 0;
  double size_x = 0, size_y = 0;
  float target_density = 0;
  std::vector<int32_t> bx, by;                 // bin edges
  std::vector<float> scaled;                   // x-major: (float)area * target density
  std::vector<int64_t> non_place, non_place_u; // x-major
  std::vector<float> wx, wy;                   // wavenumbers
  int64_t cell_off = 0, n_cells = 0;           // the region's cells in the device order
};

// Every device cell (regions contiguous, in each region's cell order) and every pin.
struct EngineSetup {
  pod_vector<int32_t> hx, hy;     // half density size
  pod_vector<float> dscale, area; // density scale; (float)dx * (float)dy of the cell box
  pod_vector<uint8_t> kind;       // CELL_STD / CELL_MACRO / CELL_FILLER
  pod_vector<uint8_t> locked;
  pod_vector<int64_t> cell_pin_start;
  pod_vector<int32_t> cell_pins;
  pod_vector<int32_t> dcx, dcy;   // the density centres as set up
  pod_vector<int64_t> net_start;  // pins net-major
  pod_vector<int32_t> pin_cell;   // device cell, -1 for a pin with no moving cell
  pod_vector<int32_t> pin_base;   // 2 per pin: offset, or the fixed position
  pod_vector<float> net_weight;
  std::vector<RegionSetup> regions;
};

enum SlotId { S_CUR_SLP = 0, S_CUR_SLP_SUM, S_NEXT_SLP, S_NEXT_SLP_SUM, S_PREV_SLP, S_PREV_SLP_SUM, S_CUR, S_NEXT, S_SNAP_CUR, S_SNAP_SLP, S_SNAP_SLP_SUM, S_SNAP_PREV_SLP_SUM, S_NUM };

// Per-region scalars the trial reads back (doubles): the overflow sums of the last scatter,
// the two |gradient| sums and the two step-length distances of the last gradient update, and
// how many blocks of the last scatter found their cells spread past the shared tile.
struct RegionScalars {
  double overflow, overflow_u, wl_sum, den_sum, dist1, dist2, spread_blocks, pad1;
};

struct DeviceError {
  cudaError_t code;
  std::string where;
};

class Engine {
 public:
  explicit Engine(int device);
  ~Engine();
  int device() const { return device_; }
  cudaStream_t stream() const { return stream_; }
  void set_poisson_mode(int m) { poisson_mode_ = m; }
  int poisson_mode() const { return poisson_mode_; }


  // ---- Nesterov state
  void upload(const EngineSetup &s);
  void release();
  int regions() const { return (int)regions_.size(); }
  // While the host builds the placer: a thread that grows the device pool by `bytes` (kept
  // once freed, so the initial placement's and the regions' buffers come from it without
  // mapping new memory) and loads the kernels' modules (loaded at first use otherwise).
  // prewarm_join() waits for it; every device call of the command comes after that.
  void prewarm(size_t bytes);
  void prewarm_join();
  // Region b's bin grid, cells, and its density solver's form (0 FP32, 1 split-BF16, 2 FP64).
  void region_info(int b, int32_t out[4]) const;
  void set_coords(int b, SlotId slot, const std::vector<float> &xy);  // 2 floats per cell
  std::vector<float> get_coords(int b, SlotId slot);
  // The density centres at `slot` (PLACE_AT) and the bins; the overflow sums.
  void place_at(int b, SlotId slot);
  // nesterovUpdateCoordinates: next, next_slp from cur_slp, cur_slp_sum, cur; then the bins.
  void nesterov_step(int b, float step, float coeff);
  void field(int b);
  void wa(float coef_x, float coef_y);
  // updateGradients into `out` with the penalty; distances |a1 - b1| and |out - b2| (pass
  // S_NUM to skip one).
  void gradients(int b, SlotId out, float penalty, SlotId a1, SlotId b1, SlotId b2);
  void prev_slp(int b, float coef);
  void hold_locked(int b);
  void swap_slots(int b, SlotId a, SlotId c);
  void copy_slot(int b, SlotId dst, SlotId src);
  // Every region's scalars (one synchronisation).
  void fetch();
  const RegionScalars &scalars(int b) const { return host_scal_[b]; }
  int64_t hpwl();  // synchronises
  void centres(std::vector<int32_t> &dcx, std::vector<int32_t> &dcy);
  void set_net_weights(const std::vector<float> &w);
  // New bin targets and fixed areas (a target-density change), same grid.
  void update_bins(int b, const RegionSetup &r);
  // Cell data after a routability change: sizes, density sizes, scales, order (a region's
  // whole cell block is rewritten).
  void rewrite_cells(const EngineSetup &s);
  int64_t trials = 0;
  int64_t launches = 0, h2d_bytes = 0, d2h_bytes = 0;  // counters for the run's report
  // The density solvers rebuilt in another mode (0 FP32, 1 split-BF16 tensor cores).
  void rebuild_poisson(int mode);
  // The region's cells sorted again on the device by their current positions (a Hilbert
  // order), when the blocks the scatter finds spread past its shared tile have grown by 2 % of
  // the blocks since the order was made; on by default ("reorder" option). take_order() gives the upload-time index of each
  // device cell of the region since the last call (false: unchanged) and starts counting anew.
  void set_reorder(bool on) { reorder_on_ = on; }
  void reorder(int b);
  bool take_order(int b, std::vector<int32_t> &order);
  int64_t reorders = 0;
  // Per-phase device time (CUDA events on the engine's stream around each launch group).
  enum Phase { PH_PLACE = 0, PH_FINALIZE, PH_POISSON, PH_WA, PH_GRAD, PH_HPWL, PH_COUNT };
  void set_profile(bool on);
  void set_overlap(bool on) {
    join();
    overlap_ = on;
  }
  int profile_read(double *ms, int64_t *launches, int cap);
  // The tuners' choices and their candidates' median times: the small nets' WA form, each
  // region's scatter form.
  std::string tuning() const;
  // Packed launches (the default with more than one region): each region's scatter, bin
  // finalize, FP32 density solve and gradient update are queued and run as one launch per
  // phase over every region queued (the split-BF16 and FP64 solves stay one region a launch);
  // every result is the same as the region-by-region launches' bit for bit.
  void set_packed(int on) {
    flush();
    packed_opt_ = on;
  }
  bool packed() const { return packed_opt_ < 0 ? regions_.size() > 1 : packed_opt_ != 0; }
  bool failed() const { return err_.code != cudaSuccess; }
  const DeviceError &error() const { return err_; }
  void check(cudaError_t e, const char *where);

  // timing of the device phases (CUDA events on the engine's stream)
  float ms_poisson = 0;

 private:
  struct Region;
  int device_ = 0;
  int poisson_mode_ = 1;
  bool reorder_on_ = true;
  cudaStream_t stream_ = nullptr;
  DeviceError err_{cudaSuccess, ""};
  std::vector<Region *> regions_;
  std::vector<RegionScalars> host_scal_;
  RegionScalars *dev_scal_ = nullptr;
  // globals
  int64_t n_cells_ = 0, n_pins_ = 0;
  int32_t n_nets_ = 0;
  int2 *dc_ = nullptr;
  int32_t *hx_ = nullptr, *hy_ = nullptr;
  float *dscale_ = nullptr, *area_ = nullptr;
  uint8_t *kind_ = nullptr, *locked_ = nullptr;
  bool any_locked_ = false;
  int64_t *cell_pin_start_ = nullptr;
  // The device's nets (and their pins) in degree order, net_order_[i] being the i-th one's
  // index in the placer's order: WA tiles then hold nets of one degree.
  std::vector<int32_t> net_order_;
  int64_t *net_start_ = nullptr;
  int32_t *pin_cell_ = nullptr, *pin_slot_ = nullptr, *big_nets_ = nullptr;
  int2 *pin_base_ = nullptr;
  int4 *tiles_ = nullptr;
  int32_t n_tiles_ = 0, n_big_ = 0;
  WaSmall small_{};  // the degree-2..4 net ranges the thread-per-net WA takes
  float *net_weight_ = nullptr;
  bool unit_weights_ = true;  // every net weight is 1: the WA kernels skip the weight loads
  float2 *pin_grad_ = nullptr;  // the WA force of every pin of a cell, cell-major (cell_pins order)
  unsigned long long *hpwl_acc_ = nullptr;
  bool hpwl_ready_ = false;  // hpwl_acc_ holds the HPWL of the current centres (from the WA)
  // Page-locked read-back: the trial's region scalars and, beside them, the HPWL the WA
  // added up (hpwl_fetched_: that value is in hpwl_host_), so one copy and one wait serve
  // both each trial.
  uint8_t *pinned_ = nullptr;
  size_t pinned_bytes_ = 0;
  bool hpwl_fetched_ = false;
  unsigned long long hpwl_host_ = 0;
  // With overlap on (the default), the WA runs on its own stream beside the density solve
  // (it needs the centres, not the field) and everything that reads its forces or moves the
  // centres joins it first. Both kernels fill every SM, so the gain is small (a few percent
  // of a trial, measured); off runs them one after the other.
  cudaStream_t wa_stream_ = nullptr;
  // the small nets' WA beside the tiles' WA (disjoint pins; the HPWL adds are exact): a second
  // stream forked after the HPWL accumulator is cleared, joined with the first
  cudaStream_t wa2_stream_ = nullptr;
  cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr, ev_split_ = nullptr, ev_join2_ = nullptr;
  std::unique_ptr<Tuner> wa_tune_;
  std::thread *prewarm_ = nullptr;
  // packed launches: the queue of (phase, region) with each entry's arguments as queued, the
  // tables' page-locked staging and device copy, the grouped FP32 solves of the live set
  enum Queued { Q_PLACE = 0, Q_FIELD, Q_GRAD };
  struct QueueEntry;
  std::vector<QueueEntry> *queue_ = nullptr;
  int packed_opt_ = -1;  // -1: by the region count
  PackedRegion *pk_host_ = nullptr, *pk_dev_ = nullptr;
  size_t pk_cap_ = 0;
  int pk_slot_ = 0;
  PoissonGroup *group_ = nullptr;
  std::vector<char> group_set_;  // the regions group_ solves
  std::unique_ptr<Tuner> pk_scatter_tune_;
  void flush();
  void flush_place(const std::vector<QueueEntry> &q, size_t a, size_t b);
  void flush_field(const std::vector<QueueEntry> &q, size_t a, size_t b);
  void flush_grad(const std::vector<QueueEntry> &q, size_t a, size_t b);
  bool stage_tables(size_t n);
  bool wa_pending_ = false;
  bool fork_early_ = false;  // ev_fork_ holds the point right after the trial's last scatter
  void fork_after_place();
  bool overlap_ = true;
  void join();
  void free_globals();
  WaArgs wa_args() const;
  // profiling
  bool profile_ = false;
  std::vector<cudaEvent_t> ev_;
  size_t ev_used_ = 0;
  std::vector<std::pair<int, size_t>> ev_pending_;
  double ph_ms_[PH_COUNT] = {};
  int64_t ph_n_[PH_COUNT] = {};
  std::vector<std::vector<float>> region_wx_, region_wy_;
  std::vector<std::pair<int, int>> region_dims_;
  void ph_begin(int ph, cudaStream_t on = nullptr);
  void ph_end(int ph, cudaStream_t on = nullptr);
  void ph_flush();
};

}  // namespace gpl
