// The initial placement's device half: the bound-to-bound matrix of each axis assembled,
// collapsed into CSR and solved on the GPU, the coordinates updated there, and the report's
// HPWL over the instances' database boxes. The host loop (place.cpp) keeps the reference's
// control flow (`doBicgstabPlace`, src/initial_place.rs:420-446) and reads back scalars only.
#pragma once
#include "pod_vector.h"
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "bicgstab.h"
#include "tune.h"

namespace gpl {

// What the device needs, in the initial placement's own orders: instances in `Ip::place`
// order (e), pins net by net (`Ip::pins`).
struct IpSetup {
  // per placed instance e
  pod_vector<int4> box;       // lx, ly, ux, uy after the initial positions
  pod_vector<uint8_t> locked;
  pod_vector<int4> clamp;     // the group's region box, for grouped instances
  pod_vector<uint8_t> grouped;
  pod_vector<int4> db_box;    // the database box the report's HPWL reads (the design's at first)
  pod_vector<int2> db_size;   // the database box's width and height
  // per pin
  pod_vector<int32_t> pin_e;     // placed instance, -1 for none (port, fixed, outside the set)
  pod_vector<int32_t> pin_inst;  // placer instance (-1 for ports): the "same instance" test
  pod_vector<uint8_t> pin_mio;   // movable IO: left out of the matrix and the extremes
  pod_vector<int2> pin_off, pin_xy;
  pod_vector<uint8_t> pin_hp;    // report HPWL: 0 the instance's db box, 1 the static box, 2 none
  pod_vector<int4> pin_static;   // the static box (fixed instance, outside instance, port bbox)
  pod_vector<int64_t> net_start;
  int4 core{};                    // `updateCoordi` clamps to the core first
  int32_t max_fanout = 200, min_diff = 1500;
  float weight_scale = 800.0f;
};

// Exclusive scan of n int64 in place, data[n] receiving the total; tmp holds scan_i64_tmp(n)
// int64 (the block totals).
size_t scan_i64_tmp(int64_t n);
cudaError_t scan_i64(int64_t *data, int64_t n, int64_t *tmp, cudaStream_t s);

// Raises the current device's stream-ordered pool's release threshold (once per device), so
// memory freed with cudaFreeAsync stays in the pool for the next allocation instead of being
// unmapped.
void keep_device_pool();

struct IpAxisResult {
  int64_t triplets = 0;  // triplets assembled (the locked diagonal included)
  BicgResult solve{};
};

class IpDevice {
 public:
  explicit IpDevice(cudaStream_t s) : s_(s) {}
  ~IpDevice();
  cudaError_t upload(const IpSetup &s);
  // `updatePinInfo` then `createSparseMatrix` for both axes, each collapsed to CSR
  // (`Csr::from_triplets`), with its right-hand side and start vector.
  cudaError_t assemble(IpAxisResult out[2]);
  // Both axes' BiCGSTAB (src/bicgstab.rs:615-669), solved side by side.
  cudaError_t solve(int max_iters, IpAxisResult out[2]);
  // The report's HPWL over the database boxes (src/initial_place.rs:359-386).
  cudaError_t hpwl(int64_t *out);
  // `updateCoordi` (src/initial_place.rs:391-417) from both solutions.
  cudaError_t update();
  // The solution vector of an axis (for the trace's probe lines).
  cudaError_t solution(int axis, std::vector<float> &x);
  // The placed instances' boxes and database boxes.
  cudaError_t download(std::vector<int4> &box, std::vector<int4> &db_box);
  // `Csr::from_triplets` (src/bicgstab.rs:501-541) on its own, on device triplets: n rows,
  // nt triplets (row, col, val) in order; writes starts[n + 1] and the *nnz (host) entries of
  // cols and vals (device buffers of at least nt entries). For a device that holds no design.
  cudaError_t csr_from_triplets(int64_t n, int64_t nt, const int32_t *row, const int32_t *col, const float *val, int64_t *starts, int32_t *cols, float *vals, int64_t *nnz);
  int64_t launches = 0, h2d_bytes = 0, d2h_bytes = 0;
  // The SpMV tuner's choice and timings so far ("" before the first solve).
  std::string tuning() const { return spmv_fixed_ >= 0 ? "initial placement SpMV: form " + std::to_string(spmv_fixed_) + " (fixed)" : spmv_tune_ ? spmv_tune_->report() : std::string(); }

 private:
  cudaStream_t s_;
  // the solver's SpMV form, by the tuner (GPL_SPMV_FORM 0 rows, 1 tiled, 2 sliced fixes it)
  std::unique_ptr<Tuner> spmv_tune_;
  int spmv_fixed_ = -1;  // GPL_SPMV_FORM's form, or -1
  int64_t n_ = 0, n_pins_ = 0, n_locked_ = 0;
  int32_t n_nets_ = 0;
  IpSetup cfg_;
  // device state
  int4 *box_ = nullptr, *clamp_ = nullptr, *db_box_ = nullptr, *pin_static_ = nullptr;
  int2 *db_size_ = nullptr, *pin_off_ = nullptr, *pin_xy_ = nullptr;
  uint8_t *locked_ = nullptr, *grouped_ = nullptr, *pin_mio_ = nullptr, *pin_hp_ = nullptr, *pin_flag_ = nullptr;
  int32_t *pin_e_ = nullptr, *pin_inst_ = nullptr, *locked_rank_ = nullptr;
  int64_t *net_start_ = nullptr;
  // counts and offsets, triplets and right-hand-side terms of both axes, the collapse's work
  int64_t *cnt_ = nullptr;       // [4][n_nets + 1]: triplets x, triplets y, rhs x, rhs y
  int64_t *scan_tmp_ = nullptr;
  size_t scan_tmp_n_ = 0;
  int32_t *t_row_ = nullptr, *t_col_ = nullptr, *r_row_ = nullptr;
  float *t_val_ = nullptr, *r_val_ = nullptr;
  size_t t_cap_ = 0, r_cap_ = 0, w_cap_ = 0;
  unsigned long long *bucket_ = nullptr;  // (column << 32 | position) per triplet, by row
  unsigned long long *bucket2_ = nullptr; // the longest rows' merge scratch, as long
  int32_t *fill_ = nullptr;
  int64_t *row_off_ = nullptr, *ucount_ = nullptr;
  int32_t *tier_rows_ = nullptr;  // [3][n]: rows handed to the collapse's later tiers
  int *tier_n_ = nullptr;         // their counts
  int32_t *ucol_ = nullptr;
  float *uval_ = nullptr;
  struct Axis {
    int64_t *starts = nullptr;
    int32_t *cols = nullptr;
    float *vals = nullptr, *rhs = nullptr, *x = nullptr;
    size_t cap = 0;
    int64_t nnz = 0;
    // the sliced copy (bicgstab.h): row order and lengths, length counts, slice starts,
    // entries
    int64_t sl_long = 0;
    int32_t *sl_row = nullptr, *sl_len = nullptr, *sl_count = nullptr;
    int64_t *sl_start = nullptr;
    int2 *sl_ent = nullptr;
    size_t sl_cap = 0, sl_start_cap = 0, sl_row_cap = 0, sl_count_cap = 0;
    // the system in the solver's row order (see solve): rows, columns and vectors renumbered
    int64_t *p_starts = nullptr;
    int32_t *p_cols = nullptr;
    float *p_vals = nullptr, *p_rhs = nullptr, *p_x = nullptr;
    size_t p_cap = 0;
  } ax_[2];
  // The solver's row order (GPL_IP_ORDER=1; off by default): perm_[i'] = the row solved as
  // row i', inv_ its inverse; sorted again each round by the Hilbert index of the rows'
  // centres (the start point), so a warp's rows gather their x entries from a compact patch.
  int32_t *perm_ = nullptr, *inv_ = nullptr, *ord_idx_ = nullptr, *ord_hist_ = nullptr;
  uint32_t *ord_key0_ = nullptr, *ord_key1_ = nullptr;
  int64_t solves_ = 0;
  int ip_order_ = -1;
  cudaError_t solver_order();
  void *scratch_ = nullptr;
  size_t scratch_bytes_ = 0;
  int64_t *hpwl_acc_ = nullptr;
  void release();
  cudaError_t collapse(int64_t n_trip, const int32_t *row, const int32_t *col, const float *val, int64_t *starts_out, int32_t **cols, float **vals, size_t *cap, int64_t *nnz);
  cudaError_t scan(int64_t *data, int64_t n);
  cudaError_t slice(Axis &A, CsrDev m);  // the axis's sliced copy of m (its CSR, as solved)
};

}  // namespace gpl
