// Host side, part 2: the Nesterov placer's setup (src/nesterov.rs:787-2036: cells, pins, nets,
// fillers, the perturbation, the bin grid and its fixed area, density sizes) restated on the
// CPU, and the loop's control (src/nesterov.rs:2669-3168, 4440-4610) driving the device engine:
// every per-cell and per-bin vector lives in HBM; the host holds the loop's scalars and makes
// the reference's decisions (back-tracking, phi, divergence, snapshots, convergence) on them.
#include <algorithm>
#include <charconv>
#include <chrono>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <thread>

#include "../kernels/engine_kernels.h"
#include "engine.h"
#include "parallel.h"
#include "../kernels/b2b.h"
#include "../kernels/rudy.h"
#include "host.h"

namespace gpl {

struct FloatPoint {
  float x = 0, y = 0;
};


// `FFT::init`'s wavenumbers in x87 extended precision (src/nesterov.rs:351-361).
static const long double PI_L = 3.141592653589793238462643383279502884L;
static const long double SQRT2_L = 1.414213562373095048801L;
float wavenumber_x(int i, int nx) { return (float)((PI_L * (long double)(float)i) / (long double)(float)nx); }
float wavenumber_y(int i, int ny, float bin_x, float bin_y) {
  return (float)((((PI_L * (long double)(float)i) / (long double)(float)ny) * (long double)bin_y) / (long double)bin_x);
}


// ---------------------------------------------------------------- Nesterov records
// `GCell`, `GPin`, `GNet`, `Bin`, `BinGrid` (src/nesterov.rs:114-295).
struct GCell {
  int inst = -1;
  bool macro_ = false;
  int32_t lx = 0, ly = 0, ux = 0, uy = 0, dlx = 0, dly = 0, dux = 0, duy = 0;
  float density_scale = 0;
  bool locked = false;
  static GCell filler(int32_t cx, int32_t cy, int32_t dx, int32_t dy) {
    GCell g;
    g.lx = cx - dx / 2;
    g.ly = cy - dy / 2;
    g.ux = cx + dx / 2;
    g.uy = cy + dy / 2;
    g.dlx = g.lx;
    g.dly = g.ly;
    g.dux = g.ux;
    g.duy = g.uy;
    return g;
  }
  int32_t dx() const { return ux - lx; }
  int32_t dy() const { return uy - ly; }
  int32_t d_cx() const { return (dux + dlx) / 2; }
  int32_t d_cy() const { return (duy + dly) / 2; }
  int32_t d_dx() const { return dux - dlx; }
  int32_t d_dy() const { return duy - dly; }
  bool is_filler() const { return inst < 0; }
  bool is_instance() const { return inst >= 0; }
  bool is_macro() const { return inst >= 0 && macro_; }
  bool is_std() const { return inst >= 0 && !macro_; }
  void set_density_size(int32_t ddx, int32_t ddy) {
    int32_t cx = d_cx(), cy = d_cy();
    dlx = cx - ddx / 2;
    dly = cy - ddy / 2;
    dux = cx + ddx / 2;
    duy = cy + ddy / 2;
  }
};
struct GPin {
  int32_t cx = 0, cy = 0, off_x = 0, off_y = 0;
  int gcell = -1;
  bool has_min_x = false, has_max_x = false, has_min_y = false, has_max_y = false;
  float min_x = 0, max_x = 0, min_y = 0, max_y = 0;
};
struct GNet {
  std::vector<int> pins;
  int32_t lx = 0, ly = 0, ux = 0, uy = 0;
  float min_x = 0, x_min_x = 0, max_x = 0, x_max_x = 0, min_y = 0, y_min_y = 0, max_y = 0, y_max_y = 0;
  float custom_weight = 1, timing_weight = 1;
  float total_weight() const { return timing_weight * custom_weight; }
  int64_t hpwl() const {
    if (ux < lx) return 0;
    return ((int64_t)ux - (int64_t)lx) + ((int64_t)uy - (int64_t)ly);
  }
};
struct Bin {
  int32_t lx = 0, ly = 0, ux = 0, uy = 0;
  float target_density = 0, density = 0, field_x = 0, field_y = 0, phi = 0;
  int64_t non_place = 0, non_place_unscaled = 0, inst_placed = 0, inst_placed_unscaled = 0, filler = 0;
  int64_t area() const { return (int64_t)(ux - lx) * (int64_t)(uy - ly); }
};
struct BinGrid {
  int32_t lx = 0, ly = 0, ux = 0, uy = 0, cnt_x = 0, cnt_y = 0;
  double size_x = 0, size_y = 0;
  std::vector<Bin> bins;
  int64_t overflow = 0, overflow_unscaled = 0;
  std::pair<int32_t, int32_t> idx_x(int32_t a, int32_t b) const {
    int32_t lower = f2i((double)(a - lx) / size_x);
    int32_t upper = f2i(std::ceil((double)(b - lx) / size_x));
    return {std::max(lower, 0), std::min(upper, cnt_x)};
  }
  std::pair<int32_t, int32_t> idx_y(int32_t a, int32_t b) const {
    int32_t lower = f2i((double)(a - ly) / size_y);
    int32_t upper = f2i(std::ceil((double)(b - ly) / size_y));
    return {std::max(lower, 0), std::min(upper, cnt_y)};
  }
  std::pair<int32_t, int32_t> density_idx_x(const GCell &g) const { return idx_x(g.dlx, g.dux); }
  std::pair<int32_t, int32_t> density_idx_y(const GCell &g) const { return idx_y(g.dly, g.duy); }
};

// `getOverlapDensityArea` (src/nesterov.rs:298-305).
static float overlap_density_area(const Bin &b, const GCell &c) {
  int32_t lx = std::max(b.lx, c.dlx), ly = std::max(b.ly, c.dly);
  int32_t ux = std::min(b.ux, c.dux), uy = std::min(b.uy, c.duy);
  if (lx >= ux || ly >= uy) return 0.0f;
  return (float)(ux - lx) * (float)(uy - ly);
}

// `fastExp` (src/nesterov.rs:308-314).
float fast_exp(float x) {
  float e = 1.0f + x / 1024.0f;
  for (int i = 0; i < 10; i++) e *= e;
  return e;
}

// `getDistance` (src/nesterov.rs:319-330).
static float distance(const std::vector<FloatPoint> &a, const std::vector<FloatPoint> &b) {
  float sum = 0.0f;
  for (size_t i = 0; i < a.size(); i++) {
    sum += (a[i].x - b[i].x) * (a[i].x - b[i].x);
    sum += (a[i].y - b[i].y) * (a[i].y - b[i].y);
  }
  size_t n = a.size();
  if (n == 0) return 0.0f;
  return (float)std::sqrt((double)sum / (2.0 * (double)n));
}

// `calculateBiVariateNormalCDF` (src/nesterov.rs:338-348).
static float bivariate_normal_cdf(float mean_x, float mean_y, float sigma_x, float sigma_y, float lx, float ly, float ux, float uy) {
  double s2 = std::sqrt(2.0);
  float x1 = (float)((double)(mean_x - lx) / (s2 * (double)sigma_x));
  float x2 = (float)((double)(mean_x - ux) / (s2 * (double)sigma_x));
  float y1 = (float)((double)(mean_y - ly) / (s2 * (double)sigma_y));
  float y2 = (float)((double)(mean_y - uy) / (s2 * (double)sigma_y));
  float s = erff(x1) * erff(y1) + erff(x2) * erff(y2) - erff(x1) * erff(y2) - erff(x2) * erff(y1);
  return (float)(0.25 * (double)s);
}

static uint32_t round_down_to_power_of_two(uint32_t x) {
  x |= x >> 1;
  x |= x >> 2;
  x |= x >> 4;
  x |= x >> 8;
  x |= x >> 16;
  return x ^ (x >> 1);
}
static double dbu_area(const Design &d, double a) { return a / ((double)d.dbu * (double)d.dbu); }

// ---------------------------------------------------------------- routability records
struct RouteVars {  // `RouteBaseVars` (src/route_base.rs:13-45)
  bool use_rudy = true;
  float target_rc = 1.01f, inflation_ratio_coef = 2.0f, max_inflation_ratio = 3.0f, max_density = 0.99f, ignore_edge_ratio = 0.8f, min_congestion_for_inflation = 0.95f, max_inflation_total = 0.30f, net_weight_max = 1.0f, congested_nets_percentage = 1.0f;
  float rc_k[4] = {1.0f, 1.0f, 0.0f, 0.0f};
};

struct Opts {  // `Opts` (src/nesterov.rs:35-82)
  float density = 0.7f;
  bool uniform_density = false;
  int bin_cnt = -1;
  float init_density_penalty = 0.00008f, init_wirelength_coef = 0.25f, min_phi_coef = 0.95f, max_phi_coef = 1.05f, overflow = 0.1f, reference_hpwl = 0.0f;
  int max_iter = 5000, seed = 1;
  float perturb_dist = -1.0f;
  bool disable_revert_if_diverge = false;
  int32_t pad_left = 0;
  bool routability = false;
  RouteVars rv;
  float routability_end_overflow = 0.3f, routability_snapshot_overflow = 0.6f;
};

struct RemovedFiller {
  int cell;
  FloatPoint vals[14];
  bool has_snapshot;
  FloatPoint snap[4];
};

// One region's `NesterovBase` (src/nesterov.rs:451-523).
struct Nb {
  std::vector<int> cells;
  int group = -1;
  std::string group_name;
  BinGrid bg;
  std::vector<float> wx, wy;  // the solver's wavenumbers
  int64_t cell_off = 0;         // the region's first device cell
  int32_t filler_dx = 0, filler_dy = 0;
  int64_t fillers = 0;
  float target_density = 0, uniform_target_density = 0;
  int64_t white_space_area = 0, movable_area = 0, total_filler_area = 0, std_insts_area = 0, macro_insts_area = 0, non_place_insts_area = 0;
  std::vector<Instance> fixed;
  int32_t dbu = 0;
  std::vector<RemovedFiller> removed_fillers;
  float max_phi_coef = 0;
  bool max_phi_coef_changed = false;
  std::vector<FloatPoint> cur_slp, cur_slp_wl, cur_slp_den, cur_slp_sum, next_slp, next_slp_wl, next_slp_den, next_slp_sum, prev_slp, prev_slp_wl, prev_slp_den, prev_slp_sum, cur, next;
  std::vector<FloatPoint> snapshot, snapshot_slp, snapshot_slp_sum, snapshot_prev_slp_sum;
  float snapshot_density_penalty = 0, snapshot_step_length = 0;
  float step_length = 0, density_penalty = 0, wl_grad_sum = 0, density_grad_sum = 0, sum_overflow = 0, sum_overflow_unscaled = 0, base_wl_coef_nb = 0;
  int64_t prev_hpwl = 0, prev_reported_hpwl = 0;
  float prev_reported_overflow_unscaled = 0, min_sum_overflow = 1e30f, hpwl_with_min_sum_overflow = 1e30f, coordi_distance = 0, peak_coordi_distance = 0;
  bool reprint_header = false, is_converged = false, is_diverged = false;
  Mt19937 generator{1};
  std::vector<FloatPoint> *per_cell(int k) {
    std::vector<FloatPoint> *v[14] = {&cur_slp, &cur_slp_wl, &cur_slp_den, &cur_slp_sum, &next_slp, &next_slp_wl, &next_slp_den, &next_slp_sum, &prev_slp, &prev_slp_wl, &prev_slp_den, &prev_slp_sum, &cur, &next};
    return v[k];
  }
  std::vector<FloatPoint> *snaps(int k) {
    std::vector<FloatPoint> *v[4] = {&snapshot, &snapshot_slp, &snapshot_slp_sum, &snapshot_prev_slp_sum};
    return v[k];
  }
  template <class T>
  static T swap_remove(std::vector<T> &v, size_t i) {
    T x = v[i];
    v[i] = v.back();
    v.pop_back();
    return x;
  }
  // `destroyFillerGCell` (src/nesterov.rs:552-568).
  RemovedFiller swap_pop(size_t i) {
    RemovedFiller f;
    f.cell = swap_remove(cells, i);
    for (int k = 0; k < 14; k++) f.vals[k] = swap_remove(*per_cell(k), i);
    f.has_snapshot = snapshot.size() > i;
    if (f.has_snapshot)
      for (int k = 0; k < 4; k++) f.snap[k] = swap_remove(*snaps(k), i);
    return f;
  }
  // `restoreRemovedFillers`' per filler (src/nesterov.rs:602-614).
  void push_back(const RemovedFiller &f) {
    bool grow = snapshot.size() == cur_slp.size();
    cells.push_back(f.cell);
    for (int k = 0; k < 14; k++) per_cell(k)->push_back(f.vals[k]);
    if (grow)
      for (int k = 0; k < 4; k++) snaps(k)->push_back(f.has_snapshot ? f.snap[k] : FloatPoint{});
  }
};

// `NesterovBase::getNesterovInstsArea` (src/nesterov.rs:1683-1685).
static int64_t nesterov_insts_area(const Nb &nb) { return nb.std_insts_area + (int64_t)std::round((float)nb.macro_insts_area * nb.target_density); }

// `Rudy` (src/route_base.rs:130-265).
struct Rudy {
  int32_t die[4] = {0, 0, 0, 0};
  int32_t cnt_x = 0, cnt_y = 0, tile_size = 0, wire_width = 0;
  std::vector<std::array<int32_t, 4>> rects;
  std::vector<float> demand, blockage;
  void init(const int32_t d4[4], int32_t xg, int32_t yg, int32_t ts, const std::vector<int32_t> &pitches) {
    double pitch_terms = 0.0;
    for (int32_t p : pitches) pitch_terms += 1.0 / (double)p;
    wire_width = pitch_terms != 0.0 ? f2i((1.0 / pitch_terms) * 1.25) : 100;
    std::memcpy(die, d4, sizeof die);
    cnt_x = xg;
    cnt_y = yg;
    tile_size = ts;
    make_grid();
  }
  void make_grid() {  // `makeGrid` (src/route_base.rs:157-176)
    int32_t x_extra = die[2] - cnt_x * tile_size, y_extra = die[3] - cnt_y * tile_size;
    rects.clear();
    int32_t cur_x = die[0];
    for (int32_t x = 0; x < cnt_x; x++) {
      int32_t cur_y = die[1];
      for (int32_t y = 0; y < cnt_y; y++) {
        int32_t xe = x == cnt_x - 1 ? x_extra : 0, ye = y == cnt_y - 1 ? y_extra : 0;
        rects.push_back({cur_x, cur_y, cur_x + tile_size + xe, cur_y + tile_size + ye});
        cur_y += tile_size;
      }
      cur_x += tile_size;
    }
    demand.assign((size_t)cnt_x * cnt_y, 0.0f);
    blockage.assign((size_t)cnt_x * cnt_y, 0.0f);
  }
  size_t at(int32_t x, int32_t y) const { return (size_t)(x * cnt_y + y); }
  // The demand map on the device (kernels/rudy.cu: the same deposits, added atomically), the
  // blockage on the host from the router's (capacity, reduction) bytes.
  cudaStream_t stream = nullptr;
  int4 *d_boxes = nullptr;
  float *d_demand = nullptr;
  size_t box_cap = 0;
  Rudy() = default;
  Rudy(const Rudy &) = delete;
  Rudy &operator=(const Rudy &) = delete;
  ~Rudy() {
    if (d_boxes) cudaFree(d_boxes);
    if (d_demand) cudaFree(d_demand);
  }
  // `resource_reductions` (src/route_base.rs:184-188): min(reduction / capacity, 1), 1 where the
  // capacity is 0.
  void set_blockage(const std::vector<uint8_t> &cap_red) {
    std::fill(blockage.begin(), blockage.end(), 0.0f);
    for (size_t i = 0; i < blockage.size() && 2 * i + 1 < cap_red.size(); i++) {
      uint8_t cap = cap_red[2 * i], red = cap_red[2 * i + 1];
      blockage[i] = cap == 0 ? 1.0f : fminr((float)red / (float)cap, 1.0f);
    }
  }
  void calculate(const std::vector<uint8_t> &cap_red, const std::vector<std::array<int32_t, 4>> &nets) {
    std::fill(demand.begin(), demand.end(), 0.0f);
    set_blockage(cap_red);
    auto ok = [](cudaError_t e, const char *where) {
      if (e != cudaSuccess) throw std::runtime_error(std::string("device: ") + cudaGetErrorString(e) + " in " + where);
    };
    if (!d_demand) ok(cudaMalloc((void **)&d_demand, std::max<size_t>(demand.size(), 1) * sizeof(float)), "rudy alloc");
    if (nets.size() > box_cap) {
      if (d_boxes) cudaFree(d_boxes);
      d_boxes = nullptr;
      box_cap = nets.size();
      ok(cudaMalloc((void **)&d_boxes, std::max<size_t>(box_cap, 1) * sizeof(int4)), "rudy alloc");
    }
    if (!nets.empty()) ok(cudaMemcpyAsync(d_boxes, nets.data(), nets.size() * sizeof(int4), cudaMemcpyHostToDevice, stream), "rudy boxes");
    RudyGrid g{die[0], die[1], die[2], die[3], cnt_x, cnt_y, tile_size, wire_width};
    ok(rudy_demand(g, (int64_t)nets.size(), d_boxes, d_demand, stream), "rudy");
    ok(cudaMemcpyAsync(demand.data(), d_demand, demand.size() * sizeof(float), cudaMemcpyDeviceToHost, stream), "rudy demand");
    ok(cudaStreamSynchronize(stream), "rudy sync");
  }
  float congestion(int32_t x, int32_t y) const {
    size_t i = at(x, y);
    float available = 1.0f - blockage[i];
    if (available <= 0.0f) return INFINITY;
    return (demand[i] / 100.0f) / available;
  }
};

// `top_averages` (src/route_base.rs:686-699).
std::array<double, 4> top_averages(const std::vector<double> &desc) {
  double n = (double)desc.size();
  const double shares[4] = {0.005, 0.01, 0.02, 0.05};
  double sums[4] = {0, 0, 0, 0};
  for (size_t i = 0; i < desc.size(); i++)
    for (int s = 0; s < 4; s++)
      if ((double)i < shares[s] * n) sums[s] += desc[i];
  return {sums[0] / std::ceil(0.005 * n), sums[1] / std::ceil(0.010 * n), sums[2] / std::ceil(0.020 * n), sums[3] / std::ceil(0.050 * n)};
}

struct Tile {
  int32_t x, y;
  float inflation_ratio = 1.0f, inflated_ratio = 0.0f;
  bool actionable = true;
};

static void router_check(int rc, const char *what) {
  if (rc != 0) refuse(std::string("the router failed: ") + what);
}

// `RouteBase` (src/route_base.rs:280-558), the RUDY path.
struct RouteBase {
  RouteVars vars;
  bool have_rudy = false;
  Rudy rudy;
  std::vector<Tile> tiles;
  int32_t cnt_x = 0, cnt_y = 0, size = 0, size_y = 0;
  int32_t revert_count = 0;
  float final_average_rc = 0, min_rc = 1e30f;
  int32_t min_rc_violated = 0;
  std::vector<float> min_rc_target_density;
  std::vector<int64_t> inflated_delta, accumulated, min_rc_inflated;
  int64_t original_movable_area = 0;
  size_t overflowed_tiles_count = 0, actionable_tiles_count = 0;
  double total_route_overflow = 0;
  void init(size_t regions, int64_t area) {
    min_rc_target_density.assign(regions, 0.0f);
    inflated_delta.assign(regions, 0);
    accumulated.assign(regions, 0);
    min_rc_inflated.assign(regions, 0);
    original_movable_area = area;
  }
  int64_t total_inflation() const {
    int64_t s = 0;
    for (auto a : accumulated) s += a;
    return s;
  }
  void reset_resources() { std::fill(inflated_delta.begin(), inflated_delta.end(), 0); }
  int tile_at(int32_t x, int32_t y) const {
    int32_t ix = std::min(x / size, cnt_x - 1), iy = std::min(y / size_y, cnt_y - 1);
    if (ix < 0 || iy < 0) return -1;
    size_t i = (size_t)iy * cnt_x + ix;
    return i < tiles.size() ? (int)i : -1;
  }
  bool inflated_ratio_at(int32_t x, int32_t y, float &r) const {
    int i = tile_at(x, y);
    if (i < 0) return false;
    r = tiles[i].inflated_ratio;
    return true;
  }
  void set_inflated_ratios() {
    for (auto &t : tiles) t.inflated_ratio = t.inflation_ratio > 1.0f ? t.inflation_ratio : 1.0f;
  }
  void scale_inflated(double scale) {
    for (auto &t : tiles)
      if (t.inflated_ratio > 1.0f) t.inflated_ratio = (float)(1.0 + scale * ((double)t.inflated_ratio - 1.0));
  }
  // `calculateRudyTiles` (src/route_base.rs:443-488).
  void calculate_rudy_tiles(const gpl_router_t *router, const std::vector<std::array<int32_t, 3>> &locs, const std::vector<std::pair<int32_t, int32_t>> &centres) {
    router_check(router->write_locations(router->user, (int64_t)locs.size(), locs.empty() ? nullptr : &locs[0][0]), "write_locations");
    if (!have_rudy) {
      int32_t d4[4], xg, yg, ts, np;
      int32_t p[32];
      router_check(router->rudy_inputs(router->user, d4, &xg, &yg, &ts, &np, p), "rudy_inputs");
      rudy.init(d4, xg, yg, ts, std::vector<int32_t>(p, p + np));
      have_rudy = true;
    }
    std::vector<uint8_t> cap_red((size_t)rudy.cnt_x * rudy.cnt_y * 2);
    router_check(router->capacity_reduction(router->user, cap_red.data(), (int64_t)rudy.cnt_x * rudy.cnt_y), "capacity_reduction");
    int64_t nn = router->net_term_boxes(router->user, nullptr, nullptr, 0);
    std::vector<int32_t> idx(nn), boxes(4 * nn);
    if (nn > 0) router->net_term_boxes(router->user, idx.data(), boxes.data(), nn);
    std::vector<std::array<int32_t, 4>> nets(nn);
    for (int64_t k = 0; k < nn; k++) nets[k] = {boxes[4 * k], boxes[4 * k + 1], boxes[4 * k + 2], boxes[4 * k + 3]};
    rudy.calculate(cap_red, nets);
    cnt_x = rudy.cnt_x;
    cnt_y = rudy.cnt_y;
    size = rudy.tile_size;
    size_y = rudy.tile_size;
    tiles.clear();
    for (int32_t y = 0; y < cnt_y; y++)
      for (int32_t x = 0; x < cnt_x; x++) tiles.push_back(Tile{x, y, 1.0f, 0.0f, false});
    for (auto &[cx, cy] : centres) {
      int i = tile_at(cx, cy);
      if (i >= 0) tiles[i].actionable = true;
    }
    // each tile's own flags and ratio: the tiles in parallel
    parallel_for(tiles.size(), [&](size_t a, size_t b) {
      for (size_t k = a; k < b; k++) {
        Tile &t = tiles[k];
        if (rudy.blockage[rudy.at(t.x, t.y)] >= vars.ignore_edge_ratio) t.actionable = false;
        if (!t.actionable) continue;
        float ratio = rudy.congestion(t.x, t.y);
        if (vars.min_congestion_for_inflation > 0.0f && ratio >= vars.min_congestion_for_inflation) {
          float r = std::pow(ratio / vars.min_congestion_for_inflation, vars.inflation_ratio_coef);
          t.inflation_ratio = fminr(r, vars.max_inflation_ratio);
        }
      }
    });
  }
  // `updateRudyAverage` (src/route_base.rs:493-536).
  void update_rudy_average() {
    double total_overflow = 0.0;
    size_t overflowed = 0;
    std::vector<double> cong;
    for (auto &t : tiles) {
      if (!t.actionable) continue;
      float ratio = rudy.congestion(t.x, t.y);
      if (std::isfinite(ratio) && ratio >= 0.0f) {
        total_overflow += std::fmax(0.0, -1.0 + (double)ratio);
        cong.push_back((double)ratio);
        if (ratio > 1.0f) overflowed++;
      }
    }
    total_route_overflow = total_overflow;
    overflowed_tiles_count = overflowed;
    actionable_tiles_count = cong.size();
    if (cong.empty()) {
      final_average_rc = 0.0f;
      return;
    }
    // only the top 5 % are summed (in descending order): sort those alone
    const size_t top = std::min(cong.size(), (size_t)std::ceil(0.05 * (double)cong.size()) + 1);
    std::partial_sort(cong.begin(), cong.begin() + top, cong.end(), [](double a, double b) { return a > b; });
    auto a = top_averages(cong);
    const float *k = vars.rc_k;
    double weighted = ((double)k[0] * a[0] + (double)k[1] * a[1] + (double)k[2] * a[2] + (double)k[3] * a[3]) / (double)(k[0] + k[1] + k[2] + k[3]);
    final_average_rc = (float)weighted;
  }
  // `RouteBase::measure` (src/route_base.rs:542-557).
  float measure(Log &log, const gpl_router_t *router, const std::vector<std::array<int32_t, 3>> &locs, const std::vector<std::pair<int32_t, int32_t>> &centres) {
    revert_count++;
    calculate_rudy_tiles(router, locs, centres);
    update_rudy_average();
    float cur_rc = final_average_rc;
    size_t over = overflowed_tiles_count, act = actionable_tiles_count;
    double pct = act > 0 ? (double)over / (double)act * 100.0 : 0.0;
    log.info("GPL", 40, sfmt("Routability pass %d: weighted congestion %.4f (target %.4f), %zu of %zu actionable tiles overflowed (%.1f%%).", revert_count, (double)cur_rc, (double)vars.target_rc, over, act, pct));
    return cur_rc;
  }
};

struct LoopSnapshots {  // src/nesterov.rs:4428-4437
  bool route_saved = false;
  float route_coef[2] = {0, 0};
  float route_a = 0;
  int route_attempts = 0;
  bool diverge_saved = false;
  float diverge_coef[2] = {0, 0};
  int64_t diverge_hpwl = 0;
  int diverge_reverts = 0;
};
enum class DivergeAction { None, Resume, Stop };
enum class DivergeFallback { RevertAndResume, RevertAndStop, Error };
static const int MAX_DIVERGE_REVERTS = 3, MAX_ROUTABILITY_DIVERGE_ATTEMPTS = 2;
static const float SETTLE_FRACTION = 0.6f;

// `diverge_fallback` (src/nesterov.rs:4406-4414).
DivergeFallback diverge_fallback(const LoopSnapshots &s, bool disable_revert) {
  if (!disable_revert && s.diverge_saved && s.diverge_reverts < MAX_DIVERGE_REVERTS) return DivergeFallback::RevertAndResume;
  if (!disable_revert && s.diverge_reverts > 0) return DivergeFallback::RevertAndStop;
  return DivergeFallback::Error;
}
// `routability_recovery_attempt` (src/nesterov.rs:4382-4390): 0 for none.
int routability_recovery_attempt(const LoopSnapshots &s, bool need) {
  if (!s.route_saved || s.route_attempts >= MAX_ROUTABILITY_DIVERGE_ATTEMPTS) return 0;
  if (!need && (s.diverge_saved || s.diverge_reverts > 0)) return 0;
  return need ? s.route_attempts + 1 : MAX_ROUTABILITY_DIVERGE_ATTEMPTS;
}
// `max_iter_takes_min_hpwl_snapshot` (src/nesterov.rs:4420-4422).
bool max_iter_takes_min_hpwl_snapshot(int iter, int max_iter, bool disable_revert, const LoopSnapshots &s, float snapshot_overflow, float overflow, int64_t hpwl) {
  return iter >= max_iter && !disable_revert && (s.diverge_saved || s.diverge_reverts > 0) && snapshot_overflow <= overflow && s.diverge_hpwl < hpwl;
}
// `settle_wait_step` (src/nesterov.rs:4364-4372): event 0 nothing, 1 started, 2 finished.
std::pair<int, int> settle_wait_step(int start, int iter, bool active, bool settled, int &extra) {
  if (active && !settled && start == -1) return {iter, 1};
  if (settled && start != -1) {
    extra = iter - start;
    return {-1, 2};
  }
  return {start, 0};
}
// `derived_reference_hpwl` (src/nesterov.rs:96-98).
float derived_reference_hpwl(float user, int64_t design_hpwl) { return user > 0.0f ? user : fmaxr(446000000.0f, 0.01f * (float)design_hpwl); }

static void set_size(GCell &g, int32_t dx, int32_t dy) {  // src/nesterov.rs:3754-3760
  int32_t cx = (g.lx + g.ux) / 2, cy = (g.ly + g.uy) / 2;
  g.lx = cx - dx / 2;
  g.ly = cy - dy / 2;
  g.ux = cx + dx / 2;
  g.uy = cy + dy / 2;
}

// `NesterovBase::updateDensitySize` (src/nesterov.rs:2022-2036) for one cell.
static void update_density_size_one(GCell &g, const Nb &nb) {
  double bsx = nb.bg.size_x, bsy = nb.bg.size_y;
  long double thr_x = SQRT2_L * (long double)bsx, thr_y = SQRT2_L * (long double)bsy;
  float size_x = (float)(SQRT2_L * (long double)(float)bsx), size_y = (float)(SQRT2_L * (long double)(float)bsy);
  int32_t dx = g.dx(), dy = g.dy();
  float scale_x, dsx, scale_y, dsy;
  if ((long double)(uint64_t)(int64_t)dx < thr_x) {
    scale_x = (float)dx / (float)thr_x;
    dsx = size_x;
  } else {
    scale_x = 1.0f;
    dsx = (float)dx;
  }
  if ((long double)(uint64_t)(int64_t)dy < thr_y) {
    scale_y = (float)dy / (float)thr_y;
    dsy = size_y;
  } else {
    scale_y = 1.0f;
    dsy = (float)dy;
  }
  g.set_density_size(f2i(dsx), f2i(dsy));
  g.density_scale = scale_x * scale_y;
}

// `union_area` (src/nesterov.rs:1901-1928).
int64_t union_area(const std::vector<std::array<int32_t, 4>> &rects) {
  std::vector<int32_t> xs;
  for (auto &r : rects) {
    xs.push_back(r[0]);
    xs.push_back(r[2]);
  }
  std::sort(xs.begin(), xs.end());
  xs.erase(std::unique(xs.begin(), xs.end()), xs.end());
  int64_t area = 0;
  for (size_t w = 0; w + 1 < xs.size(); w++) {
    int32_t x0 = xs[w], x1 = xs[w + 1];
    std::vector<std::pair<int32_t, int32_t>> spans;
    for (auto &r : rects)
      if (r[0] <= x0 && r[2] >= x1) spans.push_back({r[1], r[3]});
    std::sort(spans.begin(), spans.end());
    int64_t covered = 0;
    bool have = false;
    int32_t ca = 0, cb = 0;
    for (auto &[a, b] : spans) {
      if (have && a <= cb)
        cb = std::max(cb, b);
      else {
        if (have) covered += (int64_t)(cb - ca);
        ca = a;
        cb = b;
        have = true;
      }
    }
    if (have) covered += (int64_t)(cb - ca);
    area += covered * (int64_t)(x1 - x0);
  }
  return area;
}

// `getOverlapArea` (src/nesterov.rs:1933-1951).
static int64_t overlap_area(const Bin &b, const Instance &i, int32_t dbu) {
  int32_t lx = std::max(b.lx, i.lx), ly = std::max(b.ly, i.ly), ux = std::min(b.ux, i.ux), uy = std::min(b.uy, i.uy);
  if (lx >= ux || ly >= uy) return 0;
  if (i.macro_) {
    float f = (float)dbu;
    float mean_x = (float)(i.cx() - i.lx) / f, mean_y = (float)(i.cy() - i.ly) / f;
    float cdf = bivariate_normal_cdf(mean_x, mean_y, mean_x / 6.0f, mean_y / 6.0f, (float)(lx - i.lx) / f, (float)(ly - i.ly) / f, (float)(ux - i.lx) / f, (float)(uy - i.ly) / f);
    float original = (float)(ux - lx) * (float)(uy - ly);
    float scaled = cdf * (float)(i.ux - i.lx) * (float)(i.uy - i.ly);
    if (scaled >= original) return f2l(fminr(scaled, (float)((double)original * 1.10)));
    return f2l(original);
  }
  return (int64_t)(ux - lx) * (int64_t)(uy - ly);
}

// `BinGrid::updateBinsNonPlaceArea` (src/nesterov.rs:1956-2018).
static void update_bins_non_place_area(Nb &nb) {
  auto &bg = nb.bg;
  const auto &fixed = nb.fixed;
  const size_t n = bg.bins.size();
  // each bin's touching fixed instances in instance order (counts, their scan, a fill)
  std::vector<int64_t> start(n + 1, 0);
  auto each_bin = [&](const Instance &i, auto &&f) {
    auto [x0, x1] = bg.idx_x(i.lx, i.ux);
    auto [y0, y1] = bg.idx_y(i.ly, i.uy);
    for (int32_t y = y0; y < y1; y++)
      for (int32_t x = x0; x < x1; x++) f((size_t)(y * bg.cnt_x + x));
  };
  for (const Instance &i : fixed)
    if (i.lx < i.ux && i.ly < i.uy) each_bin(i, [&](size_t b) { start[b + 1]++; });
  for (size_t b = 0; b < n; b++) start[b + 1] += start[b];
  std::vector<int32_t> touching((size_t)start[n]);
  {
    std::vector<int64_t> at(start.begin(), start.end() - 1);
    for (size_t k = 0; k < fixed.size(); k++)
      if (fixed[k].lx < fixed[k].ux && fixed[k].ly < fixed[k].uy) each_bin(fixed[k], [&](size_t b) { touching[(size_t)at[b]++] = (int32_t)k; });
  }
  // per bin: the union of the touching boxes (the cap), and the sum of their overlaps (a
  // degenerate instance overlaps nothing, so the touching ones give the whole sum)
  parallel_for(n, [&](size_t b0, size_t b1) {
    std::vector<std::array<int32_t, 4>> rects;
    for (size_t b = b0; b < b1; b++) {
      Bin &bin = bg.bins[b];
      bin.non_place = 0;
      bin.non_place_unscaled = 0;
      if (start[b] == start[b + 1]) continue;
      rects.clear();
      int64_t raw = 0;
      for (int64_t t = start[b]; t < start[b + 1]; t++) {
        const Instance &i = fixed[(size_t)touching[(size_t)t]];
        std::array<int32_t, 4> r = {std::max(i.lx, bin.lx), std::max(i.ly, bin.ly), std::min(i.ux, bin.ux), std::min(i.uy, bin.uy)};
        if (r[0] < r[2] && r[1] < r[3]) rects.push_back(r);
        raw += overlap_area(bin, i, nb.dbu);
      }
      const int64_t uni = union_area(rects);
      bin.non_place_unscaled = f2l((float)uni * bin.target_density);
      if (raw != 0) bin.non_place += f2l((float)raw * bin.target_density);
      const int64_t cap = f2l((float)uni * bin.target_density * 1.10f);
      if (bin.non_place > cap) bin.non_place = cap;
    }
  }, 1024);
}

enum Slot { SLOT_PREV, SLOT_CUR, SLOT_NEXT };


// `initFillerGCells` (src/nesterov.rs:1690-1753).
static std::vector<GCell> init_filler_gcells(Log &log, const Design &d, const Common &c, const Base &base, Nb &nb, const Opts &o) {
  std::vector<int32_t> dxs, dys;
  dxs.reserve(base.place_insts.size());
  dys.reserve(base.place_insts.size());
  for (int k : base.place_insts) {
    dxs.push_back(c.insts[k].dx());
    dys.push_back(c.insts[k].dy());
  }
  size_t n = dxs.size();
  int32_t lo = f2i((double)n * 0.05), hi = f2i((double)n * 0.95);
  if (lo == hi) {
    lo = 0;
    hi = (int32_t)n;
  }
  if (lo == hi) refuse("a region with no placeable instance (no filler size) is not modelled");
  // the sorted sizes' ranks [lo, hi): two partitions put exactly those values there (their
  // integer sum needs no further order)
  for (auto *v : {&dxs, &dys}) {
    if (lo > 0) std::nth_element(v->begin(), v->begin() + lo, v->end());
    if ((size_t)hi < n) std::nth_element(v->begin() + lo, v->begin() + hi, v->end());
  }
  int64_t sx = 0, sy = 0;
  for (int32_t i = lo; i < hi; i++) {
    sx += dxs[i];
    sy += dys[i];
  }
  nb.filler_dx = (int32_t)(sx / (int64_t)(hi - lo));
  nb.filler_dy = (int32_t)(sy / (int64_t)(hi - lo));
  nb.white_space_area = base.region_area - base.non_place_insts_area;
  float tmp_target = (float)((double)((float)nb.std_insts_area / (float)(nb.white_space_area - nb.macro_insts_area)) + 0.01);
  nb.target_density = o.uniform_density ? tmp_target : o.density;
  int64_t nia = nesterov_insts_area(nb);
  int64_t movable = f2l((float)nb.white_space_area * nb.target_density);
  int64_t total_filler = movable - nia;
  nb.uniform_target_density = (float)nia / (float)nb.white_space_area;
  nb.uniform_target_density = std::ceil(nb.uniform_target_density * 100.0f) / 100.0f;
  if (total_filler < 0) {
    log.warn("GPL", 302, sfmt("Target density %.4f is too low for the available free area.\nAutomatically adjusting to uniform density %.4f.", (double)nb.target_density, (double)nb.uniform_target_density));
    nb.target_density = nb.uniform_target_density;
    movable = f2l((float)nb.white_space_area * nb.target_density);
    total_filler = movable - nia;
  }
  double scale = std::sqrt((double)total_filler / (10.0 * (double)nia));
  if (scale > 1.0) {
    int32_t max_x = std::max(f2i((double)d.core.dx() / 1024.0), nb.filler_dx);
    int32_t max_y = std::max(f2i((double)d.core.dy() / 1024.0), nb.filler_dy);
    nb.filler_dx = f2i((double)nb.filler_dx * scale);
    nb.filler_dy = f2i((double)nb.filler_dy * scale);
    nb.filler_dx = std::min(nb.filler_dx, max_x);
    nb.filler_dy = std::min(nb.filler_dy, max_y);
  }
  nb.movable_area = movable;
  nb.total_filler_area = total_filler;
  int32_t count = (int32_t)(total_filler / (int64_t)(int32_t)((uint32_t)nb.filler_dx * (uint32_t)nb.filler_dy));
  Mt19937 rng(0);
  Rect r = base.region_bbox;
  std::vector<GCell> fillers;
  for (int32_t k = 0; k < count; k++) {
    uint32_t rx = rng.next_u32(), ry = rng.next_u32();
    int32_t cx = (int32_t)((rx % (uint32_t)r.dx()) + (uint32_t)r.lx);
    int32_t cy = (int32_t)((ry % (uint32_t)r.dy()) + (uint32_t)r.ly);
    fillers.push_back(GCell::filler(cx, cy, nb.filler_dx, nb.filler_dy));
  }
  return fillers;
}

// The constructor's perturbation (src/nesterov.rs:1761-1826), no clusters.
static void perturb_place_insts(const Design &d, Common &c, Ip &ip, const Base &base, const std::vector<int> &inst_cell, std::vector<GCell> &gcells, const Opts &o, Mt19937 &rng) {
  float dist = o.perturb_dist;
  bool draws = c.site_y > 0 && dist != 0.0f;
  double r = dist > 0.0f ? (double)dist * ((double)d.dbu / 1000.0) : std::min(0.5 * (double)d.dbu, (double)c.site_y);
  double sigma = r * 0.3071963263271184;
  // the draws in the reference's order, then each instance moved (its own instance, pins and
  // cell: the instances are independent)
  const size_t m = base.place_insts.size();
  std::vector<int2> off(m, int2{0, 0});
  if (draws)
    for (size_t j = 0; j < m; j++) {
      double ddx = normal(rng, 0.0, sigma);
      double ddy = normal(rng, 0.0, sigma);
      off[j] = int2{f2i(std::round(ddx)), f2i(std::round(ddy))};
    }
  parallel_for(m, [&](size_t j0, size_t j1) {
    for (size_t j = j0; j < j1; j++) {
      const int k = base.place_insts[j];
      const int32_t xo = off[j].x, yo = off[j].y;
      int gi = inst_cell[k];
      if (!c.insts[k].locked) {
        int32_t nx = c.insts[k].lx + xo, ny = c.insts[k].ly + yo;
        Instance &i = c.insts[k];
        int32_t w = i.dx(), h = i.dy();
        i.lx = nx;
        i.ly = ny;
        i.ux = i.lx + w;
        i.uy = i.ly + h;
        int32_t icx = i.cx(), icy = i.cy();
        for (int p : ip.inst_pins[k]) {
          ip.pins[p].cx = icx + ip.pins[p].off_x;
          ip.pins[p].cy = icy + ip.pins[p].off_y;
        }
      }
      const Instance &i = c.insts[k];
      GCell &cell = gcells[gi];
      cell.lx = i.lx;
      cell.ly = i.ly;
      cell.ux = i.ux;
      cell.uy = i.uy;
      cell.dlx = i.lx;
      cell.dly = i.ly;
      cell.dux = i.ux;
      cell.duy = i.uy;
    }
  }, 4096);
}

// `BinGrid::initBins` (src/nesterov.rs:1830-1898).
static void init_bins(Log &log, const Design &d, const Common &c, const Base &base, Nb &nb, const Opts &o) {
  Rect r = base.region_bbox;
  BinGrid bg;
  bg.lx = r.lx;
  bg.ly = r.ly;
  bg.ux = r.ux;
  bg.uy = r.uy;
  int64_t total_bin_area = (int64_t)(r.ux - r.lx) * (int64_t)(r.uy - r.ly);
  int64_t avg = 0;
  if (base.place_insts.empty())
    log.warn("GPL", 306, "GPL component has no placed instances.");
  else
    avg = base.place_insts_area / (int64_t)base.place_insts.size();
  int64_t ideal_bin_area = nb.target_density != 0.0f ? f2l(std::round((float)avg / nb.target_density)) : 0;
  int32_t ideal_cnt = std::max(ideal_bin_area != 0 ? (int32_t)(total_bin_area / ideal_bin_area) : 0, 4);
  log.info("GPL", 23, sfmt("Placement target density:   %10.4f", (double)nb.target_density));
  log.info("GPL", 24, sfmt("Movable insts average area: %10.3f um^2", dbu_area(d, (double)avg)));
  log.info("GPL", 25, sfmt("Ideal bin area:             %10.3f um^2", dbu_area(d, (double)ideal_bin_area)));
  log.info("GPL", 26, sfmt("Ideal bin count:            %10d", ideal_cnt));
  log.info("GPL", 27, sfmt("Total bin area:             %10.3f um^2", dbu_area(d, (double)total_bin_area)));
  if (o.bin_cnt >= 0) {
    bg.cnt_x = o.bin_cnt;
    bg.cnt_y = o.bin_cnt;
  } else {
    int32_t w = r.ux - r.lx, h = r.uy - r.ly;
    int32_t ratio = (int32_t)round_down_to_power_of_two((uint32_t)(std::max(w, h) / std::min(w, h)));
    int32_t found = 2;
    while (found <= 1024) {
      if ((found == 2 || found * (found * ratio) <= ideal_cnt) && 4 * found * (found * ratio) > ideal_cnt) break;
      found *= 2;
    }
    if (w > h) {
      bg.cnt_x = found * ratio;
      bg.cnt_y = found;
    } else {
      bg.cnt_x = found;
      bg.cnt_y = found * ratio;
    }
  }
  log.info("GPL", 28, sfmt("%-21s %7d , %6d", "Bin count (X, Y):", bg.cnt_x, bg.cnt_y));
  bg.size_x = (double)(r.ux - r.lx) / (double)bg.cnt_x;
  bg.size_y = (double)(r.uy - r.ly) / (double)bg.cnt_y;
  log.info("GPL", 29, sfmt("%-21s %7.3f * %6.3f um", "Bin size (W * H):", bg.size_x / (double)d.dbu, bg.size_y / (double)d.dbu));
  big_resize(bg.bins, (size_t)bg.cnt_x * bg.cnt_y);
  parallel_for((size_t)bg.cnt_y, [&](size_t y0, size_t y1) {
    for (int32_t y = (int32_t)y0; y < (int32_t)y1; y++)
      for (int32_t x = 0; x < bg.cnt_x; x++) {
        Bin &b = bg.bins[(size_t)y * bg.cnt_x + x];
        b.lx = r.lx + f2i(std::round((double)x * bg.size_x));
        b.ly = r.ly + f2i(std::round((double)y * bg.size_y));
        b.ux = r.lx + f2i(std::round((double)(x + 1) * bg.size_x));
        b.uy = r.ly + f2i(std::round((double)(y + 1) * bg.size_y));
        b.target_density = nb.target_density;
      }
  }, 16);
  for (size_t k = 0; k < bg.bins.size(); k++) {
    const Bin &b = bg.bins[k];
    if (b.ux - b.lx < 0 || b.uy - b.ly < 0) log.warn("GPL", 34, sfmt("Bin (center: %d,%d, index: %zu) has negative size: %d, %d", (b.lx + b.ux) / 2, (b.ly + b.uy) / 2, k, b.ux - b.lx, b.uy - b.ly));
  }
  log.info("GPL", 30, sfmt("Number of bins:             %10zu", bg.bins.size()));
  progress("    bins: grid");
  nb.bg = std::move(bg);
  nb.fixed.clear();
  for (int k : base.fixed_insts) nb.fixed.push_back(c.insts[k]);
  for (auto &dm : base.dummies) nb.fixed.push_back(dm);
  nb.dbu = d.dbu;
  update_bins_non_place_area(nb);
}


// ---------------------------------------------------------------- run.rs
static const char *KEYS[] = {"-bin_grid_count", "-density", "-init_density_penalty", "-init_wirelength_coef", "-min_phi_coef", "-max_phi_coef", "-overflow", "-reference_hpwl", "-initial_place_max_iter", "-initial_place_max_fanout", "-routability_check_overflow", "-routability_snapshot_overflow", "-routability_max_density", "-routability_target_rc_metric", "-routability_inflation_ratio_coef", "-routability_max_inflation_ratio", "-routability_min_congestion_for_inflation", "-routability_max_inflation_total", "-routability_net_weight_max", "-routability_congested_nets_percentage", "-routability_rc_coefficients", "-timing_driven_net_reweight_overflow", "-timing_driven_net_weight_max", "-timing_driven_nets_percentage", "-timing_driven_repair_tns_end_percent", "-keep_resize_below_overflow", "-virtual_cts_max_skew_fraction", "-random_seed", "-perturb_dist", "-pad_left", "-pad_right", nullptr};
static const char *FLAGS[] = {"-skip_initial_place", "-force_center_initial_place", "-skip_nesterov_place", "-timing_driven", "-timing_driven_repair_timing", "-routability_driven", "-virtual_cts", "-routability_use_grt", "-skip_io", "-place_ios", "-incremental", "-disable_revert_if_diverge", "-disable_pin_density_adjust", "-enable_routing_congestion", nullptr};

// `parse_key_args` (src/run.rs:53-88).
static void parse_key_args(Log &log, const std::vector<std::string> &args, std::map<std::string, std::string> &keys, std::vector<std::string> &flags) {
  bool positional = false;
  auto keyword = [](const std::string &a) { return a.size() >= 2 && a[0] == '-' && std::isalpha((unsigned char)a[1]); };
  auto in = [](const char **list, const std::string &a) {
    for (int i = 0; list[i]; i++)
      if (a == list[i]) return true;
    return false;
  };
  auto first_prefix = [](const char **list, const std::string &a) -> const char * {
    for (int i = 0; list[i]; i++)
      if (std::string(list[i]).rfind(a, 0) == 0) return list[i];
    return nullptr;
  };
  size_t i = 0;
  while (i < args.size()) {
    const std::string &a = args[i];
    if (!keyword(a)) {
      positional = true;
      i++;
      continue;
    }
    const char *key = in(KEYS, a) ? a.c_str() : (in(FLAGS, a) ? nullptr : first_prefix(KEYS, a));
    const char *flag = nullptr;
    if (!key) flag = in(FLAGS, a) ? a.c_str() : first_prefix(FLAGS, a);
    if (key) {
      std::string ks = key;
      if (i + 1 >= args.size()) log.error("STA", in(KEYS, a) ? 560 : 561, "global_placement " + ks + " missing value.");
      keys[ks] = args[i + 1];
      i += 2;
    } else if (flag) {
      flags.push_back(flag);
      i++;
    } else {
      log.error("STA", 562, "global_placement " + a + " is not a known keyword or flag.");
    }
  }
  if (positional) log.error("STA", 564, "global_placement positional arguments not supported.");
}

static std::string trim(const std::string &s) {
  size_t a = s.find_first_not_of(" \t\n\r"), b = s.find_last_not_of(" \t\n\r");
  return a == std::string::npos ? "" : s.substr(a, b - a + 1);
}
// Rust's `str::parse::<f32>` / `parse::<i32>` on trimmed text.
static bool parse_f32(const std::string &s, float &out) {
  std::string t = trim(s);
  if (t.empty()) return false;
  auto r = std::from_chars(t.data(), t.data() + t.size(), out);
  return r.ec == std::errc() && r.ptr == t.data() + t.size();
}
static bool parse_i32(const std::string &s, int32_t &out) {
  std::string t = trim(s);
  if (!t.empty() && t[0] == '+') t = t.substr(1);
  if (t.empty()) return false;
  auto r = std::from_chars(t.data(), t.data() + t.size(), out);
  return r.ec == std::errc() && r.ptr == t.data() + t.size();
}

// `nesterov_opts` (src/run.rs:225-272).
static Opts nesterov_opts(const std::map<std::string, std::string> &keys, const std::vector<std::string> &flags, const Vars &v) {
  auto flag = [&](const char *f) { return std::find(flags.begin(), flags.end(), f) != flags.end(); };
  if (flag("-enable_routing_congestion")) refuse("global_placement -enable_routing_congestion is not modelled");
  auto fl = [&](const char *k, float dflt) {
    auto it = keys.find(k);
    if (it == keys.end()) return dflt;
    float x;
    if (!parse_f32(it->second, x)) refuse(std::string(k) + " " + it->second + ": not a number");
    return x;
  };
  auto in = [&](const char *k, int32_t dflt) {
    auto it = keys.find(k);
    if (it == keys.end()) return dflt;
    int32_t x;
    if (!parse_i32(it->second, x)) refuse(std::string(k) + " " + it->second + ": not an integer");
    return x;
  };
  Opts o;
  auto dens = keys.find("-density");
  if (dens != keys.end()) {
    if (dens->second == "uniform")
      o.uniform_density = true;
    else
      o.density = fl("-density", 0.7f);
  }
  if (keys.count("-bin_grid_count")) o.bin_cnt = in("-bin_grid_count", 0);
  o.init_density_penalty = fl("-init_density_penalty", o.init_density_penalty);
  o.init_wirelength_coef = fl("-init_wirelength_coef", o.init_wirelength_coef);
  o.min_phi_coef = fl("-min_phi_coef", o.min_phi_coef);
  o.max_phi_coef = fl("-max_phi_coef", o.max_phi_coef);
  o.overflow = fl("-overflow", o.overflow);
  o.reference_hpwl = fl("-reference_hpwl", o.reference_hpwl);
  o.seed = in("-random_seed", o.seed);
  o.perturb_dist = fl("-perturb_dist", o.perturb_dist);
  o.disable_revert_if_diverge = flag("-disable_revert_if_diverge");
  o.pad_left = v.pad_left;
  o.routability_end_overflow = fl("-routability_check_overflow", o.routability_end_overflow);
  o.routability_snapshot_overflow = fl("-routability_snapshot_overflow", o.routability_snapshot_overflow);
  if (flag("-routability_driven") && !v.skip_io) {
    RouteVars r;
    r.use_rudy = !flag("-routability_use_grt");
    r.target_rc = fl("-routability_target_rc_metric", r.target_rc);
    r.max_density = fl("-routability_max_density", r.max_density);
    r.inflation_ratio_coef = fl("-routability_inflation_ratio_coef", r.inflation_ratio_coef);
    r.max_inflation_ratio = fl("-routability_max_inflation_ratio", r.max_inflation_ratio);
    r.min_congestion_for_inflation = fl("-routability_min_congestion_for_inflation", r.min_congestion_for_inflation);
    r.max_inflation_total = fl("-routability_max_inflation_total", r.max_inflation_total);
    r.net_weight_max = fl("-routability_net_weight_max", r.net_weight_max);
    r.congested_nets_percentage = fl("-routability_congested_nets_percentage", r.congested_nets_percentage);
    auto it = keys.find("-routability_rc_coefficients");
    if (it != keys.end()) {
      std::vector<float> k;
      size_t p = 0;
      std::string s = it->second;
      while (p < s.size()) {
        size_t q = s.find_first_not_of(" \t\n", p);
        if (q == std::string::npos) break;
        size_t e = s.find_first_of(" \t\n", q);
        float x;
        if (!parse_f32(s.substr(q, e == std::string::npos ? std::string::npos : e - q), x)) refuse("-routability_rc_coefficients " + s + ": not four numbers");
        k.push_back(x);
        p = e == std::string::npos ? s.size() : e;
      }
      if (k.size() != 4) refuse("-routability_rc_coefficients " + s + ": not four numbers");
      for (int q = 0; q < 4; q++) r.rc_k[q] = k[q];
    }
    if (!r.use_rudy) refuse("-routability_use_grt needs the global router, which is not modelled");
    o.routability = true;
    o.rv = r;
  }
  return o;
}


// ---------------------------------------------------------------- the placer on the device
// `NesterovPlace` with every per-cell vector on the device (Engine): the same decisions as
// src/nesterov.rs, taken on the scalars the trial reads back.
// The routability pass's state and services (the reference's RouteBase with its router).
struct Routability {
  RouteBase rb;
  const gpl_router_t *router = nullptr;
  const Common *common = nullptr;
};

struct Placer {
  Opts o;
  Engine &eng;
  std::vector<GCell> gcells;  // host copy: sizes and, after the loop, the placed centres
  std::vector<GPin> gpins;
  PinLists net_pins;
  PinLists inst_pins;  // each instance's pins (a cell's are those of its instance)
  std::vector<int> pin_net;
  std::vector<Nb> nbs;
  std::vector<int64_t> dev_of_gcell;  // gcell -> device cell (-1: in no region)
  std::vector<int> gcell_of_dev;
  float wl_coef_x = 0, wl_coef_y = 0, base_wl_coef = 0;
  int recursion_wl = 0, recursion_init_slp = 0;
  float initial_prev_coordi_update_coef = 100.0f, reference_hpwl = 0;
  int max_iter = 0;
  float average_overflow = 0, average_overflow_unscaled = 0;
  int64_t min_hpwl = INT64_MAX;
  bool is_min_hpwl = false;
  int diverge_snapshot_iter = 0;
  float diverge_snapshot_overflow = 0;
  int num_region_diverged = 0;
  int diverge_code = 0;
  std::string diverge_msg;
  int64_t trials = 0;
  int64_t hpwl_cache = 0;
  bool hpwl_dirty = true;

  explicit Placer(Engine &e) : eng(e) {}

  void device_check() {
    if (eng.failed()) throw std::runtime_error("device: " + std::string(cudaGetErrorString(eng.error().code)) + " in " + eng.error().where);
  }
  int64_t hpwl() {
    if (hpwl_dirty) {
      hpwl_cache = eng.hpwl();
      device_check();
      hpwl_dirty = false;
    }
    return hpwl_cache;
  }
  void place_at(int b, SlotId s) {
    eng.place_at(b, s);
    hpwl_dirty = true;
  }
  // `updateWireLengthCoef` (src/nesterov.rs:2532-2542).
  void update_wirelength_coef(float overflow) {
    float c;
    if (overflow > 1.0f)
      c = (float)0.1;
    else if ((double)overflow < 0.1)
      c = 10.0f;
    else
      c = (float)(1.0 / std::pow(10.0, ((double)overflow - 0.1) * 20.0 / 9.0 - 1.0));
    wl_coef_x = c * base_wl_coef;
    wl_coef_y = c * base_wl_coef;
  }
  void wa() { eng.wa(wl_coef_x, wl_coef_y); }
  float dist(double sum, int b) const {  // getDistance's sqrt(sum / 2n), as float
    int64_t n = (int64_t)nbs[b].cells.size();
    if (n == 0) return 0.0f;
    return (float)std::sqrt(sum / (2.0 * (double)n));
  }
  // updateGradients (src/nesterov.rs:2455-2507) into `out`, and its sums read back.
  void update_gradients(int b, SlotId out, SlotId a1, SlotId b1, SlotId b2) {
    if (nbs[b].is_converged) return;
    eng.gradients(b, out, nbs[b].density_penalty, a1, b1, b2);
    eng.fetch();
    device_check();
    read_grad_sums(b);
  }
  void read_grad_sums(int b) {
    const RegionScalars &s = eng.scalars(b);
    nbs[b].wl_grad_sum = (float)s.wl_sum;
    nbs[b].density_grad_sum = (float)s.den_sum;
  }
  // npUpdate*Gradient (src/nesterov.rs:2512-2528): a zero WA sum halves the coefficients.
  // `batched`: the region's gradient was computed with the others and already read back.
  void np_update_gradient(int b, SlotId out, SlotId a1, SlotId b1, SlotId b2, bool batched) {
    if (!batched) update_gradients(b, out, a1, b1, b2);
    while (nbs[b].wl_grad_sum == 0.0f && recursion_wl < 10) {
      wl_coef_x = (float)((double)wl_coef_x * 0.5);
      wl_coef_y = (float)((double)wl_coef_y * 0.5);
      base_wl_coef = (float)((double)base_wl_coef * 0.5);
      wa();
      recursion_wl++;
      update_gradients(b, out, a1, b1, b2);
      wa_changed = true;
    }
    auto bad = [](float v) { return std::isnan(v) || std::isinf(v); };
    if (bad(nbs[b].wl_grad_sum) || bad(nbs[b].density_grad_sum)) {
      diverge_code = 306;
      diverge_msg = "RePlAce diverged at wire/density gradient Sum. An internal value is NaN or Inf.";
      num_region_diverged = 1;
    }
  }
  bool wa_changed = false;

  // initDensity1 (src/nesterov.rs:2546-2580).
  void init_density1(int b) {
    Nb &nb = nbs[b];
    size_t n = nb.cells.size();
    std::vector<float> xy(2 * n);
    // each of the region's device cells moves its own host cell (gcell_of_dev is a permutation)
    parallel_for(n, [&](size_t a, size_t e) {
      for (size_t i = a; i < e; i++) {
        GCell &g = gcells[gcell_of_dev[nb.cell_off + i]];  // the device's order of the region's cells
        // updateDensityCoordiLayoutInside (:2173-2185) on the host copy of the density box
        float tlx = fmaxr((float)g.dlx, (float)nb.bg.lx), tly = fmaxr((float)g.dly, (float)nb.bg.ly);
        if (tlx + (float)g.d_dx() > (float)nb.bg.ux) tlx = (float)(nb.bg.ux - g.d_dx());
        if (tly + (float)g.d_dy() > (float)nb.bg.uy) tly = (float)(nb.bg.uy - g.d_dy());
        int32_t lx = f2i(tlx), ly = f2i(tly);
        g.dux = lx + (g.dux - g.dlx);
        g.duy = ly + (g.duy - g.dly);
        g.dlx = lx;
        g.dly = ly;
        xy[2 * i] = (float)g.d_cx();
        xy[2 * i + 1] = (float)g.d_cy();
      }
    });
    eng.set_coords(b, S_CUR_SLP, xy);
    eng.copy_slot(b, S_PREV_SLP, S_CUR_SLP);
    eng.copy_slot(b, S_CUR, S_CUR_SLP);
    place_at(b, S_CUR_SLP);
    nbs[b].prev_hpwl = hpwl();
    eng.field(b);
    eng.fetch();
    device_check();
    Nb &q = nbs[b];
    q.base_wl_coef_nb = (float)((double)o.init_wirelength_coef / ((double)(float)(q.bg.size_x + q.bg.size_y) * 0.5));
    float nia = (float)nesterov_insts_area(q);
    q.sum_overflow = (float)eng.scalars(b).overflow / nia;
    q.sum_overflow_unscaled = (float)eng.scalars(b).overflow_u / nia;
  }
  // NesterovPlace::init (src/nesterov.rs:2674-2714).
  void np_init(Log &log) {
    float total_sum_overflow = 0.0f, total_base_wl_coef = 0.0f;
    for (size_t b = 0; b < nbs.size(); b++) {
      init_density1((int)b);
      total_sum_overflow += nbs[b].sum_overflow;
      total_base_wl_coef += nbs[b].base_wl_coef_nb;
    }
    float n = (float)nbs.size();
    average_overflow = total_sum_overflow / n;
    base_wl_coef = total_base_wl_coef / n;
    progress("    init: density");
    update_wirelength_coef(average_overflow);
    wa();
    progress("    init: wirelength");
    for (size_t b = 0; b < nbs.size(); b++) {
      np_update_gradient((int)b, S_CUR_SLP_SUM, S_NUM, S_NUM, S_NUM, false);
      eng.prev_slp((int)b, initial_prev_coordi_update_coef);
      place_at((int)b, S_PREV_SLP);
      eng.field((int)b);
    }
    progress("    init: first gradients");
    wa();
    for (size_t b = 0; b < nbs.size(); b++) np_update_gradient((int)b, S_PREV_SLP_SUM, S_PREV_SLP, S_CUR_SLP, S_CUR_SLP_SUM, false);
    progress("    init: second gradients");
    for (size_t b = 0; b < nbs.size(); b++) {
      float step = init_density2((int)b);
      bool bad = std::isnan(step) || std::isinf(step);
      if (bad && recursion_init_slp < 10) {
        initial_prev_coordi_update_coef *= 10.0f;
        recursion_init_slp++;
        sync_host_centres();
        np_init(log);
        break;
      }
      if (bad) log.error("GPL", 304, "RePlAce diverged at initial iteration with steplength being " + rust_f32(step) + ". Re-run with a smaller init_density_penalty value.");
    }
  }
  // initDensity2 (src/nesterov.rs:2600-2617).
  float init_density2(int b) {
    if (nbs[b].wl_grad_sum == 0.0f) {
      nbs[b].density_penalty = o.init_density_penalty;
      update_gradients(b, S_PREV_SLP_SUM, S_PREV_SLP, S_CUR_SLP, S_CUR_SLP_SUM);
    }
    Nb &nb = nbs[b];
    if (nb.wl_grad_sum != 0.0f) nb.density_penalty = (nb.wl_grad_sum / nb.density_grad_sum) * o.init_density_penalty;
    float nia = (float)nesterov_insts_area(nb);
    nb.sum_overflow = (float)eng.scalars(b).overflow / nia;
    nb.sum_overflow_unscaled = (float)eng.scalars(b).overflow_u / nia;
    nb.coordi_distance = dist(eng.scalars(b).dist1, b);
    float grad = dist(eng.scalars(b).dist2, b);
    nb.step_length = nb.coordi_distance / grad;
    return nb.step_length;
  }
  // The host's map of the device's cell order, after the engine sorted cells again.
  void apply_device_order() {
    std::vector<int32_t> ord;
    for (size_t b = 0; b < nbs.size(); b++) {
      if (!eng.take_order((int)b, ord)) continue;
      const int64_t off = nbs[b].cell_off;
      std::vector<int> was(gcell_of_dev.begin() + off, gcell_of_dev.begin() + off + (int64_t)ord.size());
      for (size_t i = 0; i < ord.size(); i++) {
        const int g = was[ord[i]];
        gcell_of_dev[off + i] = g;
        dev_of_gcell[g] = off + (int64_t)i;
      }
    }
    device_check();
  }
  // The device's density centres into the host's density boxes.
  void sync_host_centres() {
    apply_device_order();
    std::vector<int32_t> cx, cy;
    eng.centres(cx, cy);
    device_check();
    // gcell_of_dev is a permutation: each device cell writes its own host cell
    parallel_for(gcell_of_dev.size(), [&](size_t a, size_t b) {
      for (size_t d = a; d < b; d++) {
        GCell &g = gcells[gcell_of_dev[d]];
        int32_t hx = g.d_dx() / 2, hy = g.d_dy() / 2;
        g.dlx = cx[d] - hx;
        g.dux = cx[d] + hx;
        g.dly = cy[d] - hy;
        g.duy = cy[d] + hy;
      }
    });
  }
  // nesterovUpdateStepLength (src/nesterov.rs:2750-2772).
  bool nesterov_update_step_length(int b) {
    Nb &nb = nbs[b];
    if (nb.is_converged) return true;
    nb.coordi_distance = dist(eng.scalars(b).dist1, b);
    float grad = dist(eng.scalars(b).dist2, b);
    float nw = nb.coordi_distance / grad;
    if (std::isnan(nw) || std::isinf(nw)) {
      nb.is_diverged = true;
      return false;
    }
    if ((double)nw > (double)nb.step_length * 0.95) {
      nb.step_length = nw;
      return false;
    }
    if ((double)nw < 0.01) {
      nb.step_length = (float)0.01;
      return false;
    }
    nb.step_length = nw;
    return true;
  }
  // doBackTracking (src/nesterov.rs:2776-2808): every region's trial launched, one read-back.
  void do_back_tracking(float coeff) {
    for (int nbt = 0; nbt < 10; nbt++) {
      trials++;
      eng.trials++;
      for (size_t b = 0; b < nbs.size(); b++)
        if (!nbs[b].is_converged) eng.nesterov_step((int)b, nbs[b].step_length, coeff);
      hpwl_dirty = true;
      wa();  // beside the density solves: it needs the new centres, not the field
      for (size_t b = 0; b < nbs.size(); b++)
        if (!nbs[b].is_converged) eng.field((int)b);
      for (size_t b = 0; b < nbs.size(); b++)
        if (!nbs[b].is_converged) eng.gradients((int)b, S_NEXT_SLP_SUM, nbs[b].density_penalty, S_CUR_SLP, S_NEXT_SLP, S_CUR_SLP_SUM);
      eng.fetch();
      device_check();
      num_region_diverged = 0;
      wa_changed = false;
      for (size_t b = 0; b < nbs.size(); b++) {
        bool batched = !wa_changed;
        if (batched && !nbs[b].is_converged) read_grad_sums((int)b);
        np_update_gradient((int)b, S_NEXT_SLP_SUM, S_CUR_SLP, S_NEXT_SLP, S_CUR_SLP_SUM, batched);
        num_region_diverged += nbs[b].is_diverged ? 1 : 0;
      }
      if (num_region_diverged > 0) {
        diverge_code = 306;
        diverge_msg = "RePlAce diverged at wire/density gradient Sum.";
        break;
      }
      size_t ok = 0;
      num_region_diverged = 0;
      for (size_t b = 0; b < nbs.size(); b++) {
        ok += nesterov_update_step_length((int)b) ? 1 : 0;
        num_region_diverged += nbs[b].is_diverged ? 1 : 0;
      }
      if (num_region_diverged > 0) {
        diverge_code = 305;
        diverge_msg = "RePlAce diverged during gradient descent calculation, resulting in an invalid step length (Inf or NaN). This is often caused by numerical instability or high placement density. Consider reducing placement density to potentially resolve the issue.";
        break;
      }
      if (ok != nbs.size()) break;
    }
  }
  void nesterov_adjust_phi(int b) {  // src/nesterov.rs:2812-2824
    Nb &nb = nbs[b];
    if (nb.is_converged) return;
    if (!nb.max_phi_coef_changed && nb.sum_overflow_unscaled < 0.35f) {
      nb.max_phi_coef_changed = true;
      nb.max_phi_coef = (float)((double)nb.max_phi_coef * 0.99);
    }
    if (nb.max_phi_coef <= 1.0f) nb.max_phi_coef = 1.01f;
  }
  float phi_coef(int b, float scaled_diff_hpwl) const {  // src/nesterov.rs:2827-2831
    float m = nbs[b].max_phi_coef;
    float r = scaled_diff_hpwl < 0.0f ? (float)(double)m : (float)((double)m * std::pow((double)m, -(double)scaled_diff_hpwl));
    return fmaxr(o.min_phi_coef, r);
  }
  // NesterovBase::updateNextIter (src/nesterov.rs:2837-2903).
  void nb_update_next_iter(Log &log, const Design &d, int b, int iter) {
    if (nbs[b].is_converged) return;
    {
      Nb &nb = nbs[b];
      eng.swap_slots(b, S_PREV_SLP, S_CUR_SLP);
      eng.swap_slots(b, S_PREV_SLP_SUM, S_CUR_SLP_SUM);
      eng.hold_locked(b);
      eng.swap_slots(b, S_CUR_SLP, S_NEXT_SLP);
      eng.swap_slots(b, S_CUR_SLP_SUM, S_NEXT_SLP_SUM);
      eng.swap_slots(b, S_CUR, S_NEXT);
      float fraction = (float)iter / (float)max_iter;
      float denom = fmaxr((float)nesterov_insts_area(nb), fraction * (float)nb.non_place_insts_area * 0.05f);
      nb.sum_overflow = (float)eng.scalars(b).overflow / denom;
      nb.sum_overflow_unscaled = (float)eng.scalars(b).overflow_u / denom;
    }
    int64_t h = hpwl();
    Nb &nb = nbs[b];
    if (iter == 0 || iter % 10 == 0) {
      float pct = 0.0f;
      if (nb.prev_reported_hpwl != 0) pct = (float)((double)(h - nb.prev_reported_hpwl) / (double)nb.prev_reported_hpwl * 100.0);
      nb.prev_reported_hpwl = h;
      nb.prev_reported_overflow_unscaled = nb.sum_overflow_unscaled;
      std::string group = nb.group >= 0 ? " (" + nb.group_name + ")" : "";
      if ((iter == 0 || nb.reprint_header) && nb.group < 0) {
        if (iter == 0) log.info("GPL", 31, "HPWL: Half-Perimeter Wirelength");
        log.report(sfmt("%9s | %8s | %13s | %8s | %9s | %5s", "Iteration", "Overflow", "HPWL (um)", "HPWL(%)", "Penalty", "Group"));
        log.report("---------------------------------------------------------------");
        nb.reprint_header = false;
      }
      log.report(sfmt("%9d | %8.4f | %s | %+7.2f%% | %s | %5s", iter, (double)nb.sum_overflow_unscaled, fmt_e((double)h / (double)d.dbu, 6, 13).c_str(), (double)pct, fmt_e((double)nb.density_penalty, 2, 9).c_str(), group.c_str()));
    }
    float scaled = (float)(h - nb.prev_hpwl) / reference_hpwl;
    float phi = phi_coef(b, scaled);
    nb.density_penalty *= phi;
    nb.prev_hpwl = h;
    nb.peak_coordi_distance = fmaxr(nb.peak_coordi_distance, nb.coordi_distance);
    if (iter > 50 && nb.min_sum_overflow > nb.sum_overflow_unscaled) {
      nb.min_sum_overflow = nb.sum_overflow_unscaled;
      nb.hpwl_with_min_sum_overflow = (float)nb.prev_hpwl;
    }
  }
  // NesterovPlace::updateNextIter (src/nesterov.rs:2907-2930).
  void np_update_next_iter(Log &log, const Design &d, int iter) {
    float total = 0.0f, total_unscaled = 0.0f;
    for (size_t b = 0; b < nbs.size(); b++) {
      nb_update_next_iter(log, d, (int)b, iter);
      total += nbs[b].sum_overflow;
      total_unscaled += nbs[b].sum_overflow_unscaled;
    }
    float n = (float)nbs.size();
    average_overflow = total / n;
    average_overflow_unscaled = total_unscaled / n;
    update_wirelength_coef(average_overflow);
    if (!o.disable_revert_if_diverge) {
      int64_t h = hpwl();
      if (h < min_hpwl && (double)average_overflow_unscaled <= 0.25) {
        min_hpwl = h;
        diverge_snapshot_overflow = average_overflow_unscaled;
        diverge_snapshot_iter = iter + 1;
        is_min_hpwl = true;
      } else {
        is_min_hpwl = false;
      }
    }
  }
  void save_snapshot(int b) {  // src/nesterov.rs:2933-2947
    Nb &nb = nbs[b];
    if (nb.is_converged) return;
    eng.copy_slot(b, S_SNAP_CUR, S_CUR);
    eng.copy_slot(b, S_SNAP_SLP, S_CUR_SLP);
    eng.copy_slot(b, S_SNAP_SLP_SUM, S_CUR_SLP_SUM);
    eng.copy_slot(b, S_SNAP_PREV_SLP_SUM, S_PREV_SLP_SUM);
    has_snapshot.resize(nbs.size(), 0);
    has_snapshot[b] = 1;
    nb.snapshot_density_penalty = nb.density_penalty;
    nb.snapshot_step_length = nb.step_length;
  }
  void revert_to_snapshot(int b) {  // src/nesterov.rs:2950-2973
    if (nbs[b].is_converged) return;
    Nb &nb = nbs[b];
    eng.copy_slot(b, S_CUR, S_SNAP_CUR);
    eng.copy_slot(b, S_CUR_SLP, S_SNAP_SLP);
    eng.copy_slot(b, S_CUR_SLP_SUM, S_SNAP_SLP_SUM);
    eng.copy_slot(b, S_PREV_SLP_SUM, S_SNAP_PREV_SLP_SUM);
    nb.density_penalty = nb.snapshot_density_penalty;
    nb.step_length = nb.snapshot_step_length;
    place_at(b, S_CUR);
    eng.field(b);
    nb.is_diverged = false;
    nb.prev_reported_hpwl = 0;
    nb.prev_reported_overflow_unscaled = 0.0f;
  }
  bool check_divergence(Log &log, int b) {  // src/nesterov.rs:2976-2991
    Nb &nb = nbs[b];
    if (nb.sum_overflow_unscaled < 0.2f && nb.sum_overflow_unscaled - nb.min_sum_overflow >= 0.02f && nb.hpwl_with_min_sum_overflow * 1.2f < (float)nb.prev_hpwl) {
      nb.is_diverged = true;
      log.warn("GPL", 323, "Divergence detected between consecutive iterations");
    }
    if (nb.prev_reported_overflow_unscaled > 0.0f && nb.prev_reported_hpwl > 0) {
      float change = nb.sum_overflow_unscaled - nb.prev_reported_overflow_unscaled;
      float increase = (float)(nb.prev_hpwl - nb.prev_reported_hpwl) / (float)nb.prev_reported_hpwl;
      if (change >= 0.05f && increase >= 0.25f) {
        nb.is_diverged = true;
        log.warn("GPL", 324, "Divergence detected between reported values. Overflow change: " + fmt_g((double)change) + ", HPWL increase: " + fmt_g((double)(increase * 100.0f)) + "%.");
      }
    }
    return nb.is_diverged;
  }
  void reset_min_sum_overflow(int b) {
    nbs[b].min_sum_overflow = 1e30f;
    nbs[b].hpwl_with_min_sum_overflow = 1e30f;
  }
  void revert_to_diverge_snapshot(Log &log, const LoopSnapshots &s) {  // src/nesterov.rs:3093-3102
    log.warn("GPL", 999, sfmt("Revert to iter: %4d overflow: %.3f HPWL: %ld", diverge_snapshot_iter, (double)diverge_snapshot_overflow, (long)s.diverge_hpwl));
    wl_coef_x = s.diverge_coef[0];
    wl_coef_y = s.diverge_coef[1];
    wa();
    for (size_t b = 0; b < nbs.size(); b++) {
      revert_to_snapshot((int)b);
      reset_min_sum_overflow((int)b);
    }
  }
  // isDiverged (src/nesterov.rs:3009-3052).
  DivergeAction np_is_diverged(Log &log, LoopSnapshots &s, float &cur_a, Routability *route) {
    num_region_diverged = 0;
    for (size_t b = 0; b < nbs.size(); b++) num_region_diverged += check_divergence(log, (int)b) ? 1 : 0;
    bool routability_off = !o.routability || !routability_need;
    if (num_region_diverged == 0 && is_min_hpwl && !o.disable_revert_if_diverge && routability_off) {
      s.diverge_coef[0] = wl_coef_x;
      s.diverge_coef[1] = wl_coef_y;
      s.diverge_hpwl = min_hpwl;
      for (size_t b = 0; b < nbs.size(); b++) save_snapshot((int)b);
      s.diverge_saved = true;
    }
    if (num_region_diverged == 0) return DivergeAction::None;
    log.report(sfmt("Divergence occured in %d regions.", num_region_diverged));
    if (!o.disable_revert_if_diverge && try_routability_diverge_recovery(log, s, cur_a, route)) {
      num_region_diverged = 0;
      return DivergeAction::Resume;
    }
    switch (diverge_fallback(s, o.disable_revert_if_diverge)) {
      case DivergeFallback::RevertAndResume:
        s.diverge_reverts++;
        log.warn("GPL", 998, sfmt("Divergence detected, reverting to snapshot with min hpwl and resuming (%d of %d reverts allowed).", s.diverge_reverts, MAX_DIVERGE_REVERTS));
        revert_to_diverge_snapshot(log, s);
        cur_a = 1.0f;
        s.diverge_saved = false;
        num_region_diverged = 0;
        return DivergeAction::Resume;
      case DivergeFallback::RevertAndStop:
        log.warn("GPL", 997, "Divergence detected again, reverting to snapshot with min hpwl and stopping.");
        revert_to_diverge_snapshot(log, s);
        num_region_diverged = 0;
        return DivergeAction::Stop;
      default:
        diverge_code = 307;
        diverge_msg = "RePlAce divergence detected: Current overflow is low and increasing relative to minimum,and the HPWL has significantly worsened. Consider re-running with a smaller max_phi_cof value.";
        return DivergeAction::Stop;
    }
  }
  // ---- routability (src/nesterov.rs:3771-4093). It runs between device iterations on the
  // host's copy of the state: pull_state() brings the device's coordinate slots and density
  // centres into the regions' per-cell vectors (in each region's own cell order), the
  // reference's host logic resizes cells, removes or restores fillers and moves target
  // densities, and push_state() rebuilds the device from the result.
  bool routability_need = true;
  int routability_settle_wait_start_iter = -1;
  std::vector<std::pair<int32_t, int32_t>> min_rc_cell_size;
  std::vector<uint8_t> has_snapshot;  // per region: the snapshot slots hold a saved snapshot
  std::vector<FloatPoint> *slot_vec(Nb &nb, int k) {
    std::vector<FloatPoint> *v[12] = {&nb.cur_slp, &nb.cur_slp_sum, &nb.next_slp, &nb.next_slp_sum, &nb.prev_slp, &nb.prev_slp_sum, &nb.cur, &nb.next, &nb.snapshot, &nb.snapshot_slp, &nb.snapshot_slp_sum, &nb.snapshot_prev_slp_sum};
    return v[k];
  }
  static SlotId slot_id(int k) {
    static const SlotId ids[12] = {S_CUR_SLP, S_CUR_SLP_SUM, S_NEXT_SLP, S_NEXT_SLP_SUM, S_PREV_SLP, S_PREV_SLP_SUM, S_CUR, S_NEXT, S_SNAP_CUR, S_SNAP_SLP, S_SNAP_SLP_SUM, S_SNAP_PREV_SLP_SUM};
    return ids[k];
  }
  void pull_state() {
    sync_host_centres();
    has_snapshot.resize(nbs.size(), 0);
    for (size_t b = 0; b < nbs.size(); b++) {
      Nb &nb = nbs[b];
      size_t n = nb.cells.size();
      for (int k = 0; k < 12; k++) {
        std::vector<FloatPoint> *v = slot_vec(nb, k);
        if (k >= 8 && !has_snapshot[b]) {
          v->clear();
          continue;
        }
        std::vector<float> xy = eng.get_coords((int)b, slot_id(k));
        device_check();
        v->assign(n, FloatPoint{});
        for (size_t i = 0; i < n; i++) {
          int64_t dv = dev_of_gcell[nb.cells[i]] - nb.cell_off;
          (*v)[i] = FloatPoint{xy[2 * dv], xy[2 * dv + 1]};
        }
      }
      // the gradient's two parts are not kept on the device; sized for the filler moves
      for (auto *v : {&nb.cur_slp_wl, &nb.cur_slp_den, &nb.next_slp_wl, &nb.next_slp_den, &nb.prev_slp_wl, &nb.prev_slp_den}) v->resize(n);
    }
  }
  void push_state();  // after engine_setup (below)
  bool is_std_instance(int gi) const { return gcells[gi].is_instance() && !gcells[gi].macro_; }
  void set_target_density(int b, float density) {  // src/nesterov.rs:3795-3802
    nbs[b].target_density = density;
    for (auto &bin : nbs[b].bg.bins) bin.target_density = density;
    update_bins_non_place_area(nbs[b]);
  }
  void update_areas(int b) {  // src/nesterov.rs:3805-3821
    int64_t st = 0, mac = 0;
    for (int gi : nbs[b].cells) {
      const GCell &g = gcells[gi];
      if (!g.is_instance()) continue;
      int64_t a = (int64_t)g.dx() * (int64_t)g.dy();
      if (g.macro_)
        mac += a;
      else
        st += a;
    }
    nbs[b].std_insts_area = st;
    nbs[b].macro_insts_area = mac;
  }
  void update_density_size_nb(int b) {
    for (int gi : nbs[b].cells) update_density_size_one(gcells[gi], nbs[b]);
  }
  // `cutFillerCells` (src/nesterov.rs:3826-3869).
  void cut_filler_cells(Log &log, const Design &d, int b, int64_t inflation_area) {
    if (inflation_area < 0) {
      log.warn("GPL", 313, "Negative area provided to remove fillers: " + rust_f64(dbu_area(d, (double)inflation_area)) + ". Expected positive value, ignoring.");
      return;
    }
    int64_t single = (int64_t)nbs[b].filler_dx * (int64_t)nbs[b].filler_dy;
    int64_t max_remove = std::min(inflation_area / single, nbs[b].fillers);
    int64_t available = single * nbs[b].fillers;
    int64_t removed = 0;
    int64_t i = (int64_t)nbs[b].cells.size() - 1;
    while (i >= 0 && removed < max_remove) {
      int gi = nbs[b].cells[i];
      if (gcells[gi].is_filler()) {
        RemovedFiller f = nbs[b].swap_pop((size_t)i);
        nbs[b].removed_fillers.push_back(f);
        nbs[b].fillers--;
        available -= single;
        removed++;
      }
      i--;
    }
    nbs[b].total_filler_area = available;
    Nb &nb = nbs[b];
    if (single * nb.fillers != nb.total_filler_area) log.warn("GPL", 312, "Unexpected filler area! The value " + rust_f64(dbu_area(d, (double)(single * nb.fillers))) + ", should be equal to totalFillerArea_ " + rust_f64(dbu_area(d, (double)nb.total_filler_area)) + ".");
    int64_t removed_area = single * removed;
    int64_t remaining = inflation_area - removed_area;
    if (remaining > single) {
      int64_t total = nesterov_insts_area(nb) + removed_area + nb.total_filler_area + remaining;
      float density = (float)total / (float)nb.white_space_area;
      set_target_density(b, density);
      nbs[b].movable_area = f2l((float)nbs[b].white_space_area * nbs[b].target_density);
    }
  }
  // `restoreRemovedFillers` (src/nesterov.rs:3873-3892).
  void restore_removed_fillers(int b) {
    Nb &nb = nbs[b];
    if (nb.removed_fillers.empty()) return;
    int64_t single = (int64_t)nb.filler_dx * (int64_t)nb.filler_dy;
    std::vector<RemovedFiller> removed;
    std::swap(removed, nb.removed_fillers);
    for (auto &f : removed) {
      nb.push_back(f);
      nb.fillers++;
      nb.total_filler_area += single;
    }
  }
  // `applyNetWeights` (src/nesterov.rs:3926-3939): no net is reweighted (weights of 1), which
  // the device's net weights already hold after a rebuild.
  void apply_net_weights(const RouteBase &) {}
  // `revertToMinCongestion` (src/nesterov.rs:3897-3922).
  void revert_to_min_congestion(Log &log, RouteBase &rb) {
    if (rb.revert_count < 1) return;
    float first = rb.min_rc_target_density.empty() ? 0.0f : rb.min_rc_target_density[0];
    log.info("GPL", 55, sfmt("Reverting inflation and target density to the pass with the minimum observed routing congestion (%.4f), target density %.4f.", (double)rb.min_rc, (double)first));
    for (size_t gi = 0; gi < gcells.size(); gi++)
      if (is_std_instance((int)gi)) set_size(gcells[gi], min_rc_cell_size[gi].first, min_rc_cell_size[gi].second);
    for (size_t b = 0; b < nbs.size(); b++) {
      set_target_density((int)b, rb.min_rc_target_density[b]);
      restore_removed_fillers((int)b);
      update_density_size_nb((int)b);
      rb.accumulated[b] = rb.min_rc_inflated[b];
    }
    apply_net_weights(rb);
    rb.reset_resources();
  }
  // `scaleInflationToBudget` (src/nesterov.rs:3945-3975).
  bool scale_inflation_to_budget(RouteBase &rb) {
    if (rb.original_movable_area <= 0) return false;
    double budget = (double)rb.original_movable_area * (double)rb.vars.max_inflation_total;
    double spent = (double)rb.total_inflation();
    double allowed = std::min(budget / 6.0, budget - spent);
    double wanted = 0.0;
    for (auto &nb : nbs)
      for (int gi : nb.cells) {
        if (!is_std_instance(gi)) continue;
        const GCell &g = gcells[gi];
        float ratio;
        if (!rb.inflated_ratio_at(g.d_cx(), g.d_cy(), ratio)) continue;
        if ((double)ratio <= 1.0) continue;
        wanted += (double)g.dx() * (double)g.dy() * ((double)ratio - 1.0);
      }
    if (wanted <= 0.0 || wanted <= allowed) return spent + wanted >= budget;
    double scale = std::fmax(0.0, allowed / wanted);
    rb.scale_inflated(scale);
    return spent + allowed >= budget;
  }
  std::vector<std::pair<int32_t, int32_t>> std_centres() const {
    std::vector<std::pair<int32_t, int32_t>> out;
    for (auto &nb : nbs)
      for (int gi : nb.cells) {
        const GCell &g = gcells[gi];
        if (g.is_instance() && !g.macro_) out.push_back({g.d_cx(), g.d_cy()});
      }
    return out;
  }
  // `placed_locations` (src/nesterov.rs:4099-4110) from the host's density centres.
  std::vector<std::array<int32_t, 3>> host_locations(const Common &c) const {
    std::vector<std::array<int32_t, 3>> out;
    for (auto &g : gcells) {
      if (g.inst < 0) continue;
      const Instance &i = c.insts[g.inst];
      out.push_back({i.db, g.d_cx() - i.dx() / 2 + c.site_x * o.pad_left, g.d_cy() - i.dy() / 2});
    }
    return out;
  }
  // `RouteBase::routability` (src/nesterov.rs:3985-4093) on the pulled state.
  std::pair<bool, bool> routability(Log &log, const Design &d, Routability &r, int revert_count) {
    float cur_rc = r.rb.measure(log, r.router, host_locations(*r.common), std_centres());
    RouteVars v = r.rb.vars;
    if (cur_rc < v.target_rc) {
      log.info("GPL", 50, sfmt("Weighted routing congestion is lower than target routing congestion(%.4f), end routability optimization.", (double)v.target_rc));
      r.rb.reset_resources();
      return {false, false};
    }
    if ((r.rb.min_rc - cur_rc) > r.rb.min_rc * 0.005f) {
      log.info("GPL", 48, "Congestion improved on previous minimum (" + fmt_g_prec((double)r.rb.min_rc, 4) + "); updating minimum.");
      r.rb.min_rc = cur_rc;
      r.rb.min_rc_violated = 0;
      for (size_t b = 0; b < nbs.size(); b++) {
        r.rb.min_rc_target_density[b] = nbs[b].target_density;
        nbs[b].removed_fillers.clear();
      }
      for (size_t gi = 0; gi < gcells.size(); gi++)
        if (is_std_instance((int)gi)) min_rc_cell_size[gi] = {gcells[gi].dx(), gcells[gi].dy()};
      r.rb.min_rc_inflated = r.rb.accumulated;
    } else {
      r.rb.min_rc_violated++;
      log.info("GPL", 49, sfmt("No improvement on minimum (%.4f); consecutive non-improvement count: %d.", (double)r.rb.min_rc, r.rb.min_rc_violated));
    }
    r.rb.set_inflated_ratios();
    bool budget_spent = scale_inflation_to_budget(r.rb);
    size_t n = nbs.size();
    for (size_t b = 0; b < n; b++) {
      r.rb.inflated_delta[b] = 0;
      for (size_t k = 0; k < nbs[b].cells.size(); k++) {
        int gi = nbs[b].cells[k];
        if (!is_std_instance(gi)) continue;
        const GCell &g = gcells[gi];
        float ratio;
        if (!r.rb.inflated_ratio_at(g.d_cx(), g.d_cy(), ratio)) continue;
        if ((double)ratio <= 1.0) continue;
        int64_t prev = (int64_t)g.dx() * (int64_t)g.dy();
        float root = std::sqrt(ratio);
        int32_t nx = f2i(std::round((float)g.dx() * root)), ny = f2i(std::round((float)g.dy() * root));
        set_size(gcells[gi], nx, ny);
        r.rb.inflated_delta[b] += (int64_t)gcells[gi].dx() * (int64_t)gcells[gi].dy() - prev;
      }
      r.rb.accumulated[b] += r.rb.inflated_delta[b];
      int64_t delta = r.rb.inflated_delta[b];
      float pct = ((float)delta / (float)nesterov_insts_area(nbs[b])) * 100.0f;
      float delta_um2 = (float)dbu_area(d, (double)delta);
      cut_filler_cells(log, d, (int)b, delta);
      {
        const Nb &nb = nbs[b];
        double spent = r.rb.original_movable_area > 0 ? 100.0 * (double)r.rb.total_inflation() / (double)r.rb.original_movable_area : 0.0;
        std::string group = nb.group >= 0 ? " in group " + nb.group_name : "";
        log.info("GPL", 86, sfmt("Inflation %+.3f um^2 (%+.2f%% of movable), %.2f%% of the %.2f%% budget spent; target density %.4f%s.", (double)delta_um2, (double)pct, spent, 100.0 * (double)v.max_inflation_total, (double)nb.target_density, group.c_str()));
      }
      if (nbs[b].target_density > v.max_density) {
        const Nb &nb = nbs[b];
        std::string group = nb.group >= 0 ? " in group " + nb.group_name : "";
        log.info("GPL", 53, sfmt("Target density %.4f exceeds the maximum allowed %.4f%s.", (double)nb.target_density, (double)v.max_density, group.c_str()));
        revert_to_min_congestion(log, r.rb);
        return {false, true};
      }
    }
    if (revert_count >= 50) {
      log.info("GPL", 91, sfmt("Routability mode reached the maximum allowed reverts %d", revert_count));
      revert_to_min_congestion(log, r.rb);
      return {false, true};
    }
    if (r.rb.min_rc_violated >= 3) {
      log.info("GPL", 54, sfmt("No improvement in routing congestion for %d consecutive iterations (limit is %d).", r.rb.min_rc_violated, 3));
      revert_to_min_congestion(log, r.rb);
      return {false, true};
    }
    for (size_t b = 0; b < n; b++) {
      update_areas((int)b);
      update_density_size_nb((int)b);
    }
    if (v.net_weight_max > 1.0f && v.congested_nets_percentage > 0.0f) refuse("routability net reweighting (-routability_net_weight_max above 1) is not modelled");
    apply_net_weights(r.rb);
    r.rb.reset_resources();
    if (budget_spent) {
      log.info("GPL", 97, sfmt("Total routability inflation %.2f%% of the movable area spent the %.2f%% budget, ending routability.", 100.0 * (double)r.rb.total_inflation() / (double)r.rb.original_movable_area, 100.0 * (double)r.rb.vars.max_inflation_total));
      revert_to_min_congestion(log, r.rb);
    }
    return {!budget_spent, true};
  }
  // `tryRoutabilityDivergeRecovery` (src/nesterov.rs:3061-3088).
  bool try_routability_diverge_recovery(Log &log, LoopSnapshots &s, float &cur_a, Routability *route) {
    int attempt = routability_recovery_attempt(s, routability_need);
    if (attempt == 0) return false;
    s.route_attempts = attempt;
    bool last = s.route_attempts == MAX_ROUTABILITY_DIVERGE_ATTEMPTS;
    if (routability_need && route) {
      pull_state();
      revert_to_min_congestion(log, route->rb);
      push_state();
    }
    if (last) routability_need = false;
    log.warn("GPL", 112, sfmt("Divergence detected, reverting to the routability snapshot (attempt %d of %d), further inflation %s.", s.route_attempts, MAX_ROUTABILITY_DIVERGE_ATTEMPTS, last ? "disabled" : "still allowed"));
    wl_coef_x = s.route_coef[0];
    wl_coef_y = s.route_coef[1];
    wa();
    for (size_t b = 0; b < nbs.size(); b++) {
      revert_to_snapshot((int)b);
      reset_min_sum_overflow((int)b);
    }
    cur_a = 1.0f;
    routability_settle_wait_start_iter = -1;
    min_hpwl = INT64_MAX;
    is_min_hpwl = false;
    return true;
  }
  bool is_placement_settled() const {
    for (auto &nb : nbs)
      if (!(nb.peak_coordi_distance > 0.0f && nb.coordi_distance <= SETTLE_FRACTION * nb.peak_coordi_distance)) return false;
    return true;
  }
  float worst_settle_ratio() const {
    float w = 0.0f;
    for (auto &nb : nbs) w = fmaxr(w, nb.peak_coordi_distance <= 0.0f ? 1.0f : nb.coordi_distance / nb.peak_coordi_distance);
    return w;
  }
  bool check_convergence(Log &log, const Design &d, int b, int iter, Routability *route, int route_iters) {  // src/nesterov.rs:3107-3159
    if (nbs[b].is_converged) return true;
    if (nbs[b].sum_overflow_unscaled > o.overflow) return false;
    int64_t h = hpwl();
    const Nb &nb = nbs[b];
    log.report(sfmt("%9d | %8.4f | %s | %8s | %s | %5s", iter, (double)nb.sum_overflow_unscaled, fmt_e((double)h / (double)d.dbu, 6, 13).c_str(), "", fmt_e((double)nb.density_penalty, 2, 9).c_str(), nb.group >= 0 ? nb.group_name.c_str() : ""));
    log.report("---------------------------------------------------------------");
    if (nb.group >= 0)
      log.info("GPL", 1016, sfmt("Region '%s' placement finished at iteration %d", nb.group_name.c_str(), iter));
    else {
      log.info("GPL", 1001, sfmt("Global placement finished at iteration %d", iter));
      if (o.routability) log.info("GPL", 1017, sfmt("Routability mode iteration count: %d", route_iters));
    }
    if (route) {
      sync_host_centres();
      route->rb.calculate_rudy_tiles(route->router, host_locations(*route->common), std_centres());
      route->rb.update_rudy_average();
      log.info("GPL", 1005, sfmt("Routability final weighted congestion: %.4f", (double)route->rb.final_average_rc));
    }
    int64_t nia = nesterov_insts_area(nb);
    log.info("GPL", 1002, sfmt("Placed Cell Area            %10.4f", dbu_area(d, (double)nia)));
    log.info("GPL", 1003, sfmt("Available Free Area         %10.4f", dbu_area(d, (double)nb.white_space_area)));
    log.info("GPL", 1004, sfmt("Minimum Feasible Density        %.4f (cell_area / free_area)", (double)nb.uniform_target_density));
    log.info("GPL", 1006, "  Suggested Target Densities:");
    double w = (double)nb.white_space_area;
    log.info("GPL", 1007, sfmt("    - For 90%% usage of free space: %.4f", (double)nia / (w * 0.90)));
    log.info("GPL", 1008, sfmt("    - For 80%% usage of free space: %.4f", (double)nia / (w * 0.80)));
    if ((double)nia / (w * 0.50) <= 1.0) log.info("GPL", 1009, sfmt("    - For 50%% usage of free space: %.4f", (double)nia / (w * 0.50)));
    if (nb.uniform_target_density > 0.95f) log.warn("GPL", 1015, sfmt("High uniform density (>%.2f) may cause congestion or legalization issues.", (double)nb.uniform_target_density));
    for (int gi : nbs[b].cells)
      if (gcells[gi].is_instance()) gcells[gi].locked = true;
    nbs[b].is_converged = true;
    return true;
  }
};

// Builds the placer (init_nesterov_place + nesterov_base, src/nesterov.rs:787-933) on the
// host and uploads it.
static void init_nesterov_place(Log &log, const Design &d, Common &c, Ip &ip, const std::vector<Base> &bases, Placer &P) {
  const Opts &o = P.o;
  std::vector<int> inst_cell(c.insts.size(), -1);
  for (size_t q = 0; q < ip.place.size(); q++) inst_cell[ip.place[q]] = (int)q;
  reserve_huge(P.gcells, ip.place.size() + ip.place.size() / 4);
  P.gcells.resize(ip.place.size());
  parallel_for(ip.place.size(), [&](size_t a, size_t b) {
    for (size_t q = a; q < b; q++) {
      int k = ip.place[q];
      const Instance &i = c.insts[k];
      GCell &g = P.gcells[q];
      g.inst = k;
      g.macro_ = i.macro_;
      g.lx = g.dlx = i.lx;
      g.ly = g.dly = i.ly;
      g.ux = g.dux = i.ux;
      g.uy = g.duy = i.uy;
      g.locked = i.locked;
    }
  });
  big_resize(P.gpins, ip.pins.size());
  parallel_for(ip.pins.size(), [&](size_t a, size_t b) {
    for (size_t q = a; q < b; q++) {
      const Pin &p = ip.pins[q];
      GPin &g = P.gpins[q];
      g.cx = p.cx;
      g.cy = p.cy;
      g.off_x = p.off_x;
      g.off_y = p.off_y;
      g.gcell = p.inst >= 0 ? inst_cell[p.inst] : -1;
    }
  });
  P.net_pins = std::move(ip.net_pins);  // the initial placement is done with them
  for (auto &b : bases)
    for (int k : b.place_insts)
      if (inst_cell[k] < 0) refuse("a placer region holding an instance outside the common placed set is not modelled");
  P.max_iter = o.max_iter;
  for (auto &base : bases) {
    std::string gname = base.group >= 0 ? d.groups[base.group].name : "";
    log.info("GPL", 33, "---- Initialize Nesterov Region: " + (base.group >= 0 ? gname : std::string("Top-level")));
    Nb nb;
    nb.group = base.group;
    nb.group_name = gname;
    nb.std_insts_area = base.std_insts_area;
    nb.macro_insts_area = base.macro_insts_area;
    nb.non_place_insts_area = base.non_place_insts_area;
    nb.max_phi_coef = o.max_phi_coef;
    nb.generator = Mt19937((uint32_t)o.seed);
    progress("  region set-up: cells and pins copied");
    std::vector<GCell> fillers = init_filler_gcells(log, d, c, base, nb, o);
    progress("  region set-up: %zu fillers", fillers.size());
    perturb_place_insts(d, c, ip, base, inst_cell, P.gcells, o, nb.generator);
    progress("  region set-up: instances perturbed");
    nb.fillers = (int64_t)fillers.size();
    for (int k : base.place_insts) nb.cells.push_back(inst_cell[k]);
    for (auto &f : fillers) {
      nb.cells.push_back((int)P.gcells.size());
      P.gcells.push_back(f);
    }
    init_bins(log, d, c, base, nb, o);
    progress("  region set-up: bins");
    nb.wx.resize(nb.bg.cnt_x);
    nb.wy.resize(nb.bg.cnt_y);
    for (int i = 0; i < nb.bg.cnt_x; i++) nb.wx[i] = wavenumber_x(i, nb.bg.cnt_x);
    for (int i = 0; i < nb.bg.cnt_y; i++) nb.wy[i] = wavenumber_y(i, nb.bg.cnt_y, (float)nb.bg.size_x, (float)nb.bg.size_y);
    for (int gi : nb.cells) update_density_size_one(P.gcells[gi], nb);
    P.nbs.push_back(std::move(nb));
  }
  P.inst_pins = std::move(ip.inst_pins);  // the perturbation above moves pins through them
}

static RegionSetup region_setup(const Nb &nb) {
  RegionSetup r;
  const BinGrid &bg = nb.bg;
  r.lx = bg.lx;
  r.ly = bg.ly;
  r.ux = bg.ux;
  r.uy = bg.uy;
  r.nx = bg.cnt_x;
  r.ny = bg.cnt_y;
  r.size_x = bg.size_x;
  r.size_y = bg.size_y;
  r.target_density = nb.target_density;
  r.bx.resize(bg.cnt_x + 1);
  r.by.resize(bg.cnt_y + 1);
  for (int32_t x = 0; x < bg.cnt_x; x++) r.bx[x] = bg.bins[x].lx;
  r.bx[bg.cnt_x] = bg.cnt_x ? bg.bins[bg.cnt_x - 1].ux : bg.lx;
  for (int32_t y = 0; y < bg.cnt_y; y++) r.by[y] = bg.bins[(size_t)y * bg.cnt_x].ly;
  r.by[bg.cnt_y] = bg.cnt_y ? bg.bins[(size_t)(bg.cnt_y - 1) * bg.cnt_x].uy : bg.ly;
  size_t n = (size_t)bg.cnt_x * bg.cnt_y;
  r.scaled.resize(n);
  r.non_place.resize(n);
  r.non_place_u.resize(n);
  for (int32_t y = 0; y < bg.cnt_y; y++)
    for (int32_t x = 0; x < bg.cnt_x; x++) {
      const Bin &b = bg.bins[(size_t)y * bg.cnt_x + x];
      size_t k = (size_t)x * bg.cnt_y + y;  // x-major on the device
      r.scaled[k] = (float)b.area() * b.target_density;
      r.non_place[k] = b.non_place;
      r.non_place_u[k] = b.non_place_unscaled;
    }
  r.wx = nb.wx;
  r.wy = nb.wy;
  r.cell_off = nb.cell_off;
  r.n_cells = (int64_t)nb.cells.size();
  return r;
}

// The device's view of the placer: cells in region order, pins net-major.
static EngineSetup engine_setup(Placer &P, bool rebuild = false) {
  EngineSetup s;
  P.dev_of_gcell.assign(P.gcells.size(), -1);
  P.gcell_of_dev.clear();
  // Device order: each region's cells along a Hilbert curve of their density centres over
  // its bin grid (1/16 bin steps), so a warp's and a block's cells lie close together (their
  // bins and their pins' cells share cache lines and shared-memory tiles); a Hilbert curve's
  // runs stay compact where a Z curve's jump across quadrant seams. The order is the
  // device's only: the region's own cell order (nb.cells) is kept for everything the
  // reference orders by. The engine sorts the cells again as they move (Engine::reorder).
  auto hilbert = [](uint32_t x, uint32_t y) {
    const uint32_t n = 1u << 16;
    uint64_t d = 0;
    for (uint32_t q = n >> 1; q > 0; q >>= 1) {
      const uint32_t rx = (x & q) ? 1u : 0u, ry = (y & q) ? 1u : 0u;
      d += (uint64_t)q * q * ((3u * rx) ^ ry);
      if (ry == 0) {
        if (rx == 1) {
          x = n - 1 - x;
          y = n - 1 - y;
        }
        std::swap(x, y);
      }
    }
    return d;
  };
  for (auto &nb : P.nbs) {
    nb.cell_off = (int64_t)P.gcell_of_dev.size();
    const size_t m = nb.cells.size();
    std::vector<uint32_t> key(m), key2(m);
    std::vector<int> idx(m), idx2(m);
    parallel_for(m, [&](size_t a, size_t b) {
      for (size_t k = a; k < b; k++) {
        const GCell &g = P.gcells[nb.cells[k]];
        double fx = 16.0 * ((double)g.d_cx() - nb.bg.lx) / std::max(nb.bg.size_x, 1.0);
        double fy = 16.0 * ((double)g.d_cy() - nb.bg.ly) / std::max(nb.bg.size_y, 1.0);
        uint32_t qx = (uint32_t)std::min(std::max(fx, 0.0), 65535.0), qy = (uint32_t)std::min(std::max(fy, 0.0), 65535.0);
        key[k] = (uint32_t)hilbert(qx, qy);  // below 2^32 on a 2^16 square
        idx[k] = nb.cells[k];
      }
    });
    // stable: four LSD passes of 8-bit digits (the order of a stable sort by key), each pass
    // over fixed chunks in parallel: the chunks' digit counts, their offsets digit by digit in
    // chunk order, then each chunk scattering its keys in order
    const size_t T = std::max<size_t>(1, std::min<size_t>(host_threads(), m / 16384));
    const size_t chunk = (m + T - 1) / T;
    std::vector<size_t> hist(T * 256);
    for (int shift = 0; shift < 32; shift += 8) {
      std::fill(hist.begin(), hist.end(), 0);
      parallel_for(T, [&](size_t t0, size_t t1) {
        for (size_t t = t0; t < t1; t++)
          for (size_t k = t * chunk; k < std::min(m, (t + 1) * chunk); k++) hist[t * 256 + ((key[k] >> shift) & 0xffu)]++;
      }, 1);
      size_t run = 0;
      for (size_t dgt = 0; dgt < 256; dgt++)
        for (size_t t = 0; t < T; t++) {
          const size_t c = hist[t * 256 + dgt];
          hist[t * 256 + dgt] = run;
          run += c;
        }
      parallel_for(T, [&](size_t t0, size_t t1) {
        for (size_t t = t0; t < t1; t++)
          for (size_t k = t * chunk; k < std::min(m, (t + 1) * chunk); k++) {
            const size_t at = hist[t * 256 + ((key[k] >> shift) & 0xffu)]++;
            key2[at] = key[k];
            idx2[at] = idx[k];
          }
      }, 1);
      key.swap(key2);
      idx.swap(idx2);
    }
    for (int gi : idx) {
      P.dev_of_gcell[gi] = (int64_t)P.gcell_of_dev.size();
      P.gcell_of_dev.push_back(gi);
    }
  }
  progress("  device set-up: cells in Hilbert order");
  size_t n = P.gcell_of_dev.size();
  big_resize(s.hx, n);
  big_resize(s.hy, n);
  big_resize(s.dscale, n);
  big_resize(s.area, n);
  big_resize(s.kind, n);
  big_resize(s.locked, n);
  big_resize(s.dcx, n);
  big_resize(s.dcy, n);
  big_assign(s.cell_pin_start, n + 1, (int64_t)0);
  auto cell_pins = [&](const GCell &g) { return g.is_filler() ? PinLists::Span{} : P.inst_pins[g.inst]; };
  parallel_for(n, [&](size_t a, size_t b) {
    for (size_t dv = a; dv < b; dv++) s.cell_pin_start[dv + 1] = (int64_t)cell_pins(P.gcells[P.gcell_of_dev[dv]]).size();
  });
  for (size_t dv = 0; dv < n; dv++) s.cell_pin_start[dv + 1] += s.cell_pin_start[dv];
  big_resize(s.cell_pins, (size_t)s.cell_pin_start[n]);
  parallel_for(n, [&](size_t a, size_t b) {
    for (size_t dv = a; dv < b; dv++) {
      const GCell &g = P.gcells[P.gcell_of_dev[dv]];
      s.hx[dv] = g.d_dx() / 2;
      s.hy[dv] = g.d_dy() / 2;
      s.dscale[dv] = g.density_scale;
      s.area[dv] = (float)g.dx() * (float)g.dy();
      s.kind[dv] = g.is_filler() ? CELL_FILLER : (g.macro_ ? CELL_MACRO : CELL_STD);
      s.locked[dv] = g.locked ? 1 : 0;
      s.dcx[dv] = g.d_cx();
      s.dcy[dv] = g.d_cy();
      // a cell's pins sit where the placer copied them (before the perturbation); a rebuild
      // keeps the current centres
      PinLists::Span pins = cell_pins(g);
      if (!rebuild && !pins.empty()) {
        const GPin &q = P.gpins[pins[0]];
        s.dcx[dv] = q.cx - q.off_x;
        s.dcy[dv] = q.cy - q.off_y;
      }
      std::copy(pins.begin(), pins.end(), s.cell_pins.begin() + s.cell_pin_start[dv]);
    }
  });
  s.net_start.assign(P.net_pins.start.begin(), P.net_pins.start.end());
  size_t np = P.gpins.size();
  big_assign(s.pin_cell, np, -1);
  big_assign(s.pin_base, 2 * np, 0);
  // pins are numbered net-major already (the placer's pins are made net by net)
  {
    bool net_major = true;
    parallel_for(P.net_pins.items.size(), [&](size_t a, size_t b) {
      bool ok = true;
      for (size_t q = a; q < b; q++) ok &= P.net_pins.items[q] == (int)q;
      if (!ok) __atomic_store_n(&net_major, false, __ATOMIC_RELAXED);
    });
    if (!net_major) refuse("pins not numbered net by net");
  }
  parallel_for(np, [&](size_t a, size_t b) {
    for (size_t p = a; p < b; p++) {
      const GPin &q = P.gpins[p];
      int64_t dv = q.gcell >= 0 ? P.dev_of_gcell[q.gcell] : -1;
      if (dv >= 0) {
        s.pin_cell[p] = (int32_t)dv;
        s.pin_base[2 * p] = q.off_x;
        s.pin_base[2 * p + 1] = q.off_y;
      } else {
        s.pin_base[2 * p] = q.cx;
        s.pin_base[2 * p + 1] = q.cy;
      }
    }
  });
  s.net_weight.assign(P.net_pins.size(), 1.0f);
  progress("  device set-up: cells and pins");
  for (auto &nb : P.nbs) s.regions.push_back(region_setup(nb));
  progress("  device set-up: regions");
  return s;
}

// The device rebuilt from the host's state (after a routability change): cells, pins and bins
// uploaded again, the coordinate slots written back in the new device order.
void Placer::push_state() {
  eng.upload(engine_setup(*this, true));
  device_check();
  for (size_t b = 0; b < nbs.size(); b++) {
    Nb &nb = nbs[b];
    size_t n = nb.cells.size();
    for (int k = 0; k < 12; k++) {
      std::vector<FloatPoint> *v = slot_vec(nb, k);
      if (v->size() != n) continue;  // a snapshot never saved stays zero
      std::vector<float> xy(2 * n);
      for (size_t i = 0; i < n; i++) {
        int64_t dv = dev_of_gcell[nb.cells[i]] - nb.cell_off;
        xy[2 * dv] = (*v)[i].x;
        xy[2 * dv + 1] = (*v)[i].y;
      }
      eng.set_coords((int)b, slot_id(k), xy);
    }
  }
  device_check();
  hpwl_dirty = true;
}

// `resume_nesterov_place` (src/nesterov.rs:4440-4610) from iteration 0, cut into its
// prologue, one loop iteration at a time, and its epilogue (so a caller can step it).
struct NesterovLoop {
  LoopSnapshots snaps;
  float cur_a = 1.0f;
  int iter = 0;
  int route_iters = 0, route_reverts = 0;
  int64_t original_area = 0;
  bool done = false;

  void begin(Log &log, Placer &P) {
    log.info("GPL", 84, "---- Execute Nesterov Global Placement.");
    if (P.num_region_diverged > 0) log.error("GPL", P.diverge_code, P.diverge_msg);
    for (auto &nb : P.nbs) {
      nb.max_phi_coef_changed = false;
      nb.min_sum_overflow = 1e30f;
      nb.hpwl_with_min_sum_overflow = 1e30f;
      nb.is_converged = false;
      original_area += nesterov_insts_area(nb);
    }
  }
  // One pass of the loop's body; false once the loop has ended.
  bool step(Log &log, const Design &d, Placer &P, Routability *route) {
    if (done || iter >= P.max_iter) return !(done = true);
    if (iter % 50 == 0) progress("iteration %d: overflow %.4f, %ld trials, %ld cell reorders", iter, (double)P.average_overflow_unscaled, (long)P.trials, (long)P.eng.reorders);
    float prev_a = cur_a;
    cur_a = (float)((1.0 + std::sqrt(4.0 * (double)prev_a * (double)prev_a + 1.0)) * 0.5);
    float coeff = (float)(((double)prev_a - 1.0) / (double)cur_a);
    P.do_back_tracking(coeff);
    for (size_t b = 0; b < P.nbs.size(); b++) P.nesterov_adjust_phi((int)b);
    if (P.num_region_diverged > 0) return !(done = true);
    P.np_update_next_iter(log, d, iter);
    bool routability = P.o.routability;
    bool routability_gpl_iter = snaps.route_saved && P.average_overflow_unscaled > P.o.routability_end_overflow;
    if (routability_gpl_iter) {
      route_iters++;
      P.max_iter++;
    }
    DivergeAction act = P.np_is_diverged(log, snaps, cur_a, route);
    if (act == DivergeAction::Stop) return !(done = true);
    if (act == DivergeAction::Resume) {
      iter++;
      return true;
    }
    if (routability && !snaps.route_saved && P.o.routability_snapshot_overflow >= P.average_overflow_unscaled) {
      snaps.route_coef[0] = P.wl_coef_x;
      snaps.route_coef[1] = P.wl_coef_y;
      snaps.route_a = cur_a;
      snaps.route_saved = true;
      for (size_t b = 0; b < P.nbs.size(); b++) P.save_snapshot((int)b);
      log.info("GPL", 38, sfmt("Routability snapshot saved at iter = %d", iter + 1));
      int64_t h = P.hpwl();
      log.report(sfmt("%9d | %8.4f | %s | %-8s | %-9s | %5s", iter, (double)P.average_overflow_unscaled, fmt_e((double)h / (double)d.dbu, 6, 13).c_str(), " ", " ", " "));
    }
    if (route) {
      bool active = P.routability_need && P.average_overflow_unscaled <= P.o.routability_end_overflow;
      bool settled = active && P.is_placement_settled();
      int extra = 0;
      auto [start, event] = settle_wait_step(P.routability_settle_wait_start_iter, iter, active, settled, extra);
      P.routability_settle_wait_start_iter = start;
      if (event == 1)
        log.info("GPL", 99, sfmt("Routability end extended at iter = %d: overflow %.4f reached %.4f, but cells are still moving at %.0f%% of peak displacement (waiting for %.0f%%).", iter + 1, (double)P.average_overflow_unscaled, (double)P.o.routability_end_overflow, (double)(P.worst_settle_ratio() * 100.0f), (double)(SETTLE_FRACTION * 100.0f)));
      else if (event == 2)
        log.info("GPL", 103, sfmt("Routability end extension finished at iter = %d after %d extra iterations: overflow %.4f, cells moving at %.0f%% of peak displacement.", iter + 1, extra, (double)P.average_overflow_unscaled, (double)(P.worst_settle_ratio() * 100.0f)));
      if (settled) {
        P.nbs[0].reprint_header = true;
        route_reverts++;
        progress("routability pass %d at iteration %d", route_reverts, iter);
        P.pull_state();
        auto [need, revert_init] = P.routability(log, d, *route, route_reverts);
        P.routability_need = need;
        P.min_hpwl = INT64_MAX;
        P.is_min_hpwl = false;
        if (need || revert_init) {
          P.push_state();
          cur_a = snaps.route_a;
          P.wl_coef_x = snaps.route_coef[0];
          P.wl_coef_y = snaps.route_coef[1];
          P.wa();
          for (size_t b = 0; b < P.nbs.size(); b++) {
            P.revert_to_snapshot((int)b);
            P.reset_min_sum_overflow((int)b);
          }
        }
        if (need && revert_init) log.info("GPL", 87, "Routability end iteration: increase inflation and revert back to snapshot.");
        if (!need && revert_init) log.info("GPL", 89, "Routability finished. Reverting to minimal observed routing congestion, could not reach target.");
        if (!need && !revert_init) log.info("GPL", 90, "Routability finished. Target routing congestion achieved succesfully.");
      }
    }
    int converged = 0;
    for (size_t b = 0; b < P.nbs.size(); b++) converged += P.check_convergence(log, d, (int)b, iter, route, route_iters) ? 1 : 0;
    if (converged == (int)P.nbs.size()) return !(done = true);
    iter++;
    return true;
  }
  int end(Log &log, const Design &d, Placer &P, Routability *route) {
    if (max_iter_takes_min_hpwl_snapshot(iter, P.max_iter, P.o.disable_revert_if_diverge, snaps, P.diverge_snapshot_overflow, P.average_overflow_unscaled, P.hpwl())) {
      log.warn("GPL", 121, "Reached the maximum number of iterations, reverting to snapshot with min hpwl.");
      P.revert_to_diverge_snapshot(log, snaps);
    }
    if (iter >= P.max_iter) log.warn("GPL", 1010, sfmt("GPL reached the maximum number of iterations for nesterov %d. Placement may have failed to converge.", P.max_iter));
    if (route) log.info("GPL", 1011, sfmt("Original area (um^2): %.2f", dbu_area(d, (double)original_area)));
    if (route) {
      int64_t inflation = route->rb.total_inflation();
      float pct = (float)(100.0 * (double)inflation / (double)original_area);
      log.info("GPL", 1012, sfmt("Total routability artificial inflation: %.2f (%+.2f%%)", dbu_area(d, (double)inflation), (double)pct));
    }
    int64_t new_area = 0;
    for (auto &nb : P.nbs) new_area += nesterov_insts_area(nb);
    float diff = (float)(100.0 * (double)(new_area - original_area) / (double)original_area);
    log.info("GPL", 1014, sfmt("Final placement area: %.2f (%+.2f%%)", dbu_area(d, (double)new_area), (double)diff));
    if (P.num_region_diverged > 0) log.error("GPL", P.diverge_code, P.diverge_msg);
    return iter;
  }
};

// `placed_locations` (src/nesterov.rs:4099-4110) from the device's density centres.
static std::vector<std::array<int32_t, 3>> placed_locations(const Common &c, Placer &P) {
  P.sync_host_centres();
  // the instances' cells in cell order: their ranks by a scan, then the rows in parallel
  const size_t n = P.gcells.size();
  std::vector<int64_t> at(n + 1, 0);
  for (size_t q = 0; q < n; q++) at[q + 1] = at[q] + (P.gcells[q].inst >= 0 ? 1 : 0);
  std::vector<std::array<int32_t, 3>> out((size_t)at[n]);
  parallel_for(n, [&](size_t a, size_t b) {
    for (size_t q = a; q < b; q++) {
      const GCell &g = P.gcells[q];
      if (g.inst < 0) continue;
      const Instance &i = c.insts[g.inst];
      out[(size_t)at[q]] = {i.db, g.d_cx() - i.dx() / 2 + c.site_x * P.o.pad_left, g.d_cy() - i.dy() / 2};
    }
  });
  return out;
}

struct RunResult {
  int status = GPL_PLACED;
  int outcome = GPL_OUTCOME_PLACED;
  std::string code, reason;
  Log log;
  int64_t insts = 0, nets = 0, pins = 0;
  int iterations = -1;
  std::vector<std::array<int32_t, 4>> bases;
  std::vector<std::array<int32_t, 3>> locations;
  int64_t final_hpwl = 0;
  float final_overflow = 0;
  int64_t trials = 0;
  double t_ip = 0, t_np = 0;
  int64_t h2d = 0, d2h = 0, launches = 0;
};

// One run of the command: `global_placement` (src/run.rs:115-201) with `do_initial_place`
// (:292-308) in `open`, the Nesterov loop stepped by `step`, and the report in `close`.
struct Run {
  RunResult res;
  Engine &eng;
  Design d;
  Common c;
  std::vector<Base> bases;
  Ip ip;
  std::unique_ptr<Placer> P;
  std::unique_ptr<Routability> route;
  NesterovLoop loop;
  bool nesterov = false;
  bool ended = false;
  std::chrono::steady_clock::time_point t2;
  explicit Run(Engine &e) : eng(e) {}

  void open(const std::vector<std::string> &args, const gpl_router_t *router) {
    Log &log = res.log;
    std::map<std::string, std::string> keys;
    std::vector<std::string> flags;
    parse_key_args(log, args, keys, flags);
    auto flag = [&](const char *f) { return std::find(flags.begin(), flags.end(), f) != flags.end(); };
    if (flag("-place_ios")) {
      if (flag("-skip_io")) log.error("GPL", 169, "-place_ios cannot be used with -skip_io placement.");
      if (flag("-incremental")) log.error("GPL", 170, "-place_ios cannot be used with -incremental placement.");
      if (flag("-skip_nesterov_place")) log.error("GPL", 182, "-place_ios cannot be used with -skip_nesterov_place placement.");
    }
    auto in = [&](const char *k) -> int32_t {
      auto it = keys.find(k);
      if (it == keys.end()) return 0;
      int32_t x;
      if (!parse_i32(it->second, x)) refuse(std::string(k) + " " + it->second + ": not an integer");
      return x;
    };
    Vars vars;
    vars.pad_left = in("-pad_left");
    vars.pad_right = in("-pad_right");
    vars.skip_io = flag("-skip_io");
    vars.place_ios = flag("-place_ios");
    vars.disable_pin_density_adjust = flag("-disable_pin_density_adjust");
    IpVars ipv;
    ipv.force_center = flag("-force_center_initial_place");
    if (flag("-skip_initial_place")) ipv.max_iter = 0;
    if (keys.count("-initial_place_max_iter")) ipv.max_iter = std::max(in("-initial_place_max_iter"), 0);
    if (keys.count("-initial_place_max_fanout")) ipv.max_fanout = std::max(in("-initial_place_max_fanout"), 0);
    if (flag("-skip_io")) ipv.max_iter = 0;
    if (flag("-incremental")) refuse("-incremental placement is outside this engine's path");
    if (flag("-place_ios")) refuse("-place_ios (concurrent IO placement) is outside this engine's path");
    if (flag("-timing_driven")) refuse("-timing_driven needs the design database's resizer");
    bool skip_nesterov = flag("-skip_nesterov_place");
    Opts o;
    if (!skip_nesterov) o = nesterov_opts(keys, flags, vars);
    if (o.routability && !router) refuse("-routability_driven / -timing_driven need the design database");
    bool has_core_row = false;
    for (auto &r : d.rows)
      if (!r.pad) has_core_row = true;
    if (!has_core_row) log.error("GPL", 130, "No rows defined in design. Use initialize_floorplan to add rows.");
    c = placer_base_common(log, d, vars);
    progress("placer common built");
    bases.push_back(placer_base(log, d, c, -1, true));
    for (auto &reg : d.regions)
      for (int g : reg.groups) bases.push_back(placer_base(log, d, c, g, true));
    if (bases[0].place_insts.empty()) {
      log.warn("GPL", 123, "No placeable instances in the top-level region. Removing it.");
      bases.erase(bases.begin());
    }
    progress("placer built: %zu instances, %zu nets, %zu bases", c.insts.size(), c.nets.size(), bases.size());
    auto t0 = std::chrono::steady_clock::now();
    {
      eng.prewarm_join();
      IpDevice dev(eng.stream());
      ip = do_bicgstab_place_device(log, d, c, vars, ipv, dev);
      eng.launches += dev.launches;
      eng.h2d_bytes += dev.h2d_bytes;
      eng.d2h_bytes += dev.d2h_bytes;
      progress("initial placement applied on the host");
    }
    progress("initial placement device memory released");
    auto t1 = std::chrono::steady_clock::now();
    res.t_ip = std::chrono::duration<double>(t1 - t0).count();
    res.insts = (int64_t)c.insts.size();
    res.nets = (int64_t)c.nets.size();
    res.pins = c.pins;
    for (auto &b : bases) res.bases.push_back({b.group, (int32_t)b.place_insts.size(), (int32_t)b.fixed_insts.size(), (int32_t)b.dummies.size()});
    if (skip_nesterov) {
      res.outcome = GPL_OUTCOME_INITIALLY_PLACED;
      for (int k : ip.place) {
        int di = c.insts[k].db;
        res.locations.push_back({di, ip.db_bbox[di].lx, ip.db_bbox[di].ly});
      }
      return;
    }
    P = std::make_unique<Placer>(eng);
    P->o = o;
    progress("initial placement done");
    init_nesterov_place(log, d, c, ip, bases, *P);
    progress("placer regions built");
    if (o.routability) {
      route = std::make_unique<Routability>();
      route->rb.vars = o.rv;
      route->router = router;
      route->common = &c;
      int64_t area = 0;
      for (auto &nb : P->nbs) area += nesterov_insts_area(nb);
      route->rb.init(P->nbs.size(), area);
      P->min_rc_cell_size.assign(P->gcells.size(), {0, 0});
    }
    // the first HPWL (the reference HPWL's base) over the pins as the placer copied them
    int64_t design_hpwl = 0;
    for (size_t nn = 0; nn < P->net_pins.size(); nn++) {
      int32_t lx = INT32_MAX, ly = INT32_MAX, ux = INT32_MIN, uy = INT32_MIN;
      for (int p : P->net_pins[nn]) {
        lx = std::min(lx, P->gpins[p].cx);
        ly = std::min(ly, P->gpins[p].cy);
        ux = std::max(ux, P->gpins[p].cx);
        uy = std::max(uy, P->gpins[p].cy);
      }
      if (ux >= lx) design_hpwl += ((int64_t)ux - lx) + ((int64_t)uy - ly);
    }
    t2 = std::chrono::steady_clock::now();
    progress("nesterov set up: %zu cells, %zu regions", P->gcells.size(), P->nbs.size());
    eng.upload(engine_setup(*P));
    P->device_check();
    progress("uploaded");
    P->reference_hpwl = derived_reference_hpwl(o.reference_hpwl, design_hpwl);
    P->np_init(log);
    progress("nesterov init done");
    loop.begin(log, *P);
    nesterov = true;
  }
  bool step() {
    if (!nesterov || ended) return false;
    bool more = loop.step(res.log, d, *P, route.get());
    if (!more) ended = true;
    return more;
  }
  void close() {
    if (!nesterov) return;
    while (step()) {
    }
    progress("loop done");
    int iter = loop.end(res.log, d, *P, route.get());
    progress("loop ended");
    res.locations = placed_locations(c, *P);
    progress("placement written");
    auto t3 = std::chrono::steady_clock::now();
    res.t_np = std::chrono::duration<double>(t3 - t2).count();
    res.iterations = iter;
    res.final_hpwl = P->hpwl();
    res.final_overflow = P->average_overflow_unscaled;
    res.trials = P->trials;
  }
};

}  // namespace gpl

// ---------------------------------------------------------------- the C ABI
using namespace gpl;

struct gpl_ctx {
  std::unique_ptr<Engine> eng;
  int poisson_mode = 1;
  bool trace = false;
  // A finished command's host state (the design copy and the placer's arrays, about 1 GB in
  // some millions of blocks at 1M cells) is freed on a thread of its own once the result is
  // written; nothing of it touches the engine or the device (the routability state, which
  // holds device buffers, is freed on the caller's thread first). One at a time; the context's
  // end waits for it.
  std::thread reaper;
  void reap(std::unique_ptr<Run> run) {
    if (run) run->route.reset();
    settle();
    reaper = std::thread([r = std::move(run)]() mutable { r.reset(); });
  }
  void settle() {
    if (reaper.joinable()) reaper.join();
  }
  ~gpl_ctx() { settle(); }
};

static char *dupstr(const std::string &s) {
  char *p = (char *)malloc(s.size() + 1);
  std::memcpy(p, s.c_str(), s.size() + 1);
  return p;
}

static void fill_result(RunResult &r, gpl_result_t *out) {
  std::memset(out, 0, sizeof *out);
  out->status = r.status;
  out->outcome = r.outcome;
  std::snprintf(out->code, sizeof out->code, "%s", r.code.c_str());
  out->reason = dupstr(r.reason);
  std::string lines, trace;
  for (auto &l : r.log.lines) lines += l + "\n";
  for (auto &l : r.log.trace) trace += l + "\n";
  out->lines = dupstr(lines);
  out->trace = dupstr(trace);
  out->insts = r.insts;
  out->nets = r.nets;
  out->pins = r.pins;
  out->iterations = r.iterations;
  out->n_bases = (int32_t)r.bases.size();
  out->bases = (int32_t *)malloc(sizeof(int32_t) * 4 * (r.bases.size() + 1));
  for (size_t b = 0; b < r.bases.size(); b++)
    for (int q = 0; q < 4; q++) out->bases[4 * b + q] = r.bases[b][q];
  out->n_locations = (int64_t)r.locations.size();
  out->locations = (int32_t *)malloc(sizeof(int32_t) * 3 * (r.locations.size() + 1));
  for (size_t k = 0; k < r.locations.size(); k++)
    for (int q = 0; q < 3; q++) out->locations[3 * k + q] = r.locations[k][q];
  out->final_hpwl = r.final_hpwl;
  out->final_overflow = r.final_overflow;
  out->trials = r.trials;
  out->seconds_initial_place = r.t_ip;
  out->seconds_nesterov = r.t_np;
  out->h2d_bytes = r.h2d;
  out->d2h_bytes = r.d2h;
  out->launches = r.launches;
}

// Runs `f` and turns a stop into the result's status: the reference's error, a refusal, or a
// device fault.
template <class F>
static void guarded(RunResult &r, F f) {
  try {
    f();
  } catch (const StopEx &s) {
    if (s.error) {
      r.status = GPL_ERROR;
      r.code = sfmt("%s-%04d", s.tool.c_str(), s.id);
    } else {
      r.status = GPL_REFUSED;
      r.reason = s.why;
    }
  } catch (const std::exception &e) {
    r.status = GPL_DEVICE_FAULT;
    r.reason = e.what();
  }
}

struct gpl_session {
  gpl_ctx *ctx;
  std::unique_ptr<Run> run;
};

extern "C" {

gpl_ctx *gpl_create(int device) {
  auto *c = new gpl_ctx();
  c->eng = std::make_unique<Engine>(device);
  if (c->eng->failed()) {
    delete c;
    return nullptr;
  }
  return c;
}

void gpl_destroy(gpl_ctx *c) { delete c; }

int gpl_set_option(gpl_ctx *c, const char *name, const char *value) {
  std::string n = name, v = value;
  if (n == "poisson") {
    if (v == "mixed")
      c->poisson_mode = 1;
    else if (v == "fp32")
      c->poisson_mode = 0;
    else if (v == "fp64")
      c->poisson_mode = 2;
    else
      return -1;
    return 0;
  }
  if (n == "trace") {
    c->trace = v == "1";
    return 0;
  }
  if (n == "reorder") {
    if (v != "0" && v != "1") return -1;
    c->eng->set_reorder(v == "1");
    return 0;
  }
  if (n == "packed") {
    if (v != "0" && v != "1" && v != "auto") return -1;
    c->eng->set_packed(v == "auto" ? -1 : v == "1" ? 1 : 0);
    return 0;
  }
  return -1;
}

// The device memory a command on this design takes at most, about: the initial placement's
// triplets, collapse and solver copies (some 400 bytes a pin), which the Nesterov state then
// reuses from the pool.
static size_t prewarm_bytes(const gpl_design_t *cd) {
  const int64_t pins = cd->n_nets > 0 && cd->net_iterm_start ? cd->net_iterm_start[cd->n_nets] : 0;
  return (size_t)std::max<int64_t>(pins, 0) * 400 + ((size_t)64 << 20);
}

static void reset_counters(Engine &e) {
  e.launches = 0;
  e.h2d_bytes = 0;
  e.d2h_bytes = 0;
  e.trials = 0;
}

int gpl_global_placement(gpl_ctx *ctx, const gpl_design_t *cd, int argc, const char *const *argv, const gpl_router_t *router, gpl_result_t *out) {
  ctx->eng->set_poisson_mode(ctx->poisson_mode);
  reset_counters(*ctx->eng);
  auto run = std::make_unique<Run>(*ctx->eng);
  run->res.log.trace_on = ctx->trace;
  guarded(run->res, [&] {
    progress("command start");
    ctx->eng->prewarm(prewarm_bytes(cd));
    run->d = design_from_c(cd);
    progress("design read: %zu instances, %zu nets", run->d.insts.size(), run->d.nets.size());
    run->open(std::vector<std::string>(argv, argv + argc), router);
    run->close();
    progress("command done (%s)", ctx->eng->tuning().substr(0, 400).c_str());
  });
  run->res.h2d = ctx->eng->h2d_bytes;
  run->res.d2h = ctx->eng->d2h_bytes;
  run->res.launches = ctx->eng->launches;
  progress("  release: start");
  ctx->eng->release();
  progress("device memory released");
  fill_result(run->res, out);
  progress("result written");
  ctx->reap(std::move(run));
  progress("host state handed off");
  return out->status;
}

gpl_session *gpl_session_open(gpl_ctx *ctx, const gpl_design_t *cd, int argc, const char *const *argv, const gpl_router_t *router) {
  ctx->eng->set_poisson_mode(ctx->poisson_mode);
  reset_counters(*ctx->eng);
  auto *s = new gpl_session{ctx, std::make_unique<Run>(*ctx->eng)};
  s->run->res.log.trace_on = ctx->trace;
  guarded(s->run->res, [&] {
    ctx->eng->prewarm(prewarm_bytes(cd));
    s->run->d = design_from_c(cd);
    s->run->open(std::vector<std::string>(argv, argv + argc), router);
  });
  return s;
}

int gpl_session_iterate(gpl_session *s, int n, int *done) {
  int k = 0;
  if (s->run->res.status != GPL_PLACED) {
    *done = 1;
    return 0;
  }
  guarded(s->run->res, [&] {
    while (k < n && s->run->step()) k++;
  });
  *done = (s->run->ended || !s->run->nesterov || s->run->res.status != GPL_PLACED) ? 1 : 0;
  return k;
}

int gpl_session_set_option(gpl_session *s, const char *name, const char *value) {
  std::string n = name, v = value;
  if (n == "poisson") {
    int mode = v == "fp32" ? 0 : v == "mixed" ? 1 : v == "fp64" ? 2 : -1;
    if (mode < 0) return -1;
    if (!s->run->nesterov) return -1;
    s->ctx->eng->rebuild_poisson(mode);
    return s->ctx->eng->failed() ? -1 : 0;
  }
  if (n == "profile") {
    s->ctx->eng->set_profile(v == "1");
    return 0;
  }
  if (n == "overlap") {  // the WA beside the density solve (1, the default) or after it (0)
    s->ctx->eng->set_overlap(v != "0");
    return 0;
  }
  if (n == "reorder") {  // the device cell order kept coherent (1, the default) or fixed (0)
    s->ctx->eng->set_reorder(v != "0");
    return 0;
  }
  if (n == "packed") {  // every region's phase in one launch ("auto", the default: with regions)
    if (v != "0" && v != "1" && v != "auto") return -1;
    s->ctx->eng->set_packed(v == "auto" ? -1 : v == "1" ? 1 : 0);
    return 0;
  }
  return -1;
}

int gpl_session_profile(gpl_session *s, double *ms, int64_t *launches, int cap) {
  return s->ctx->eng->profile_read(ms, launches, cap);
}

void *gpl_session_stream(gpl_session *s) { return (void *)s->ctx->eng->stream(); }

void gpl_session_counters(gpl_session *s, int64_t out[6]) {
  out[0] = s->ctx->eng->launches;
  out[1] = s->ctx->eng->h2d_bytes;
  out[2] = s->ctx->eng->d2h_bytes;
  out[3] = s->run->P ? (int64_t)s->run->P->gcell_of_dev.size() : 0;
  out[4] = s->ctx->eng->trials;
  out[5] = s->ctx->eng->reorders;
}

int gpl_session_regions(gpl_session *s, int32_t *out, int cap) {
  Engine &e = *s->ctx->eng;
  for (int b = 0; b < e.regions() && b < cap; b++) e.region_info(b, out + 4 * b);
  return e.regions();
}

int gpl_session_tuning(gpl_session *s, char *buf, int cap) {
  const std::string t = s->ctx->eng->tuning();
  if (buf && cap > 0) std::snprintf(buf, (size_t)cap, "%s", t.c_str());
  return (int)t.size();
}

void gpl_session_discard(gpl_session *s) {
  s->ctx->eng->release();
  delete s;
}

int gpl_session_close(gpl_session *s, gpl_result_t *out) {
  if (s->run->res.status == GPL_PLACED) guarded(s->run->res, [&] { s->run->close(); });
  s->run->res.h2d = s->ctx->eng->h2d_bytes;
  s->run->res.d2h = s->ctx->eng->d2h_bytes;
  s->run->res.launches = s->ctx->eng->launches;
  s->ctx->eng->release();
  fill_result(s->run->res, out);
  s->ctx->reap(std::move(s->run));
  delete s;
  return out->status;
}

void gpl_result_free(gpl_result_t *out) {
  free(out->reason);
  free(out->lines);
  free(out->trace);
  free(out->bases);
  free(out->locations);
  std::memset(out, 0, sizeof *out);
}

}  // extern "C"

// ---- test-only exports (not in include/gpl.h): the engine's own host rules, so the tests can
// check them against the reference's unit-test vectors directly, not only through the oracle's
// restatement. Each takes the same arguments as the oracle's function of the same suffix.
extern "C" {
using namespace gpl;
uint32_t gpl_rules_mt19937_nth(uint32_t seed, int64_t n) {
  Mt19937 e(seed);
  uint32_t last = 0;
  for (int64_t i = 0; i < n; i++) last = e.next_u32();
  return last;
}
uint32_t gpl_rules_normal_draws(uint32_t seed, double sigma, int k, double *out) {
  Mt19937 e(seed);
  for (int i = 0; i < k; i++) {
    double v = normal(e, 0.0, sigma);
    if (out) out[i] = v;
  }
  return e.next_u32();
}
void gpl_rules_uniform_int_draws(uint32_t seed, int nr, const int32_t *ranges, int per, int32_t *out) {
  Mt19937 e(seed);
  for (int r = 0; r < nr; r++)
    for (int i = 0; i < per; i++) out[r * per + i] = uniform_int(e, -ranges[r], ranges[r]);
}
void gpl_rules_min_max_idx(int32_t ll, int32_t uu, int32_t core_ll, int32_t site, int32_t mn, int32_t mx, int32_t *out2) {
  auto [a, b] = min_max_idx(ll, uu, core_ll, site, mn, mx);
  out2[0] = a;
  out2[1] = b;
}
static Instance instance_of(const int32_t *box4) {
  Instance i;
  i.db = 0;
  i.lx = box4[0];
  i.ly = box4[1];
  i.ux = box4[2];
  i.uy = box4[3];
  return i;
}
static void box_of(const Instance &i, int32_t *box4) {
  box4[0] = i.lx;
  box4[1] = i.ly;
  box4[2] = i.ux;
  box4[3] = i.uy;
}
void gpl_rules_snap_outward(int32_t *box4, int32_t ox, int32_t oy, int32_t sx, int32_t sy) {
  Instance i = instance_of(box4);
  i.snap_outward(ox, oy, sx, sy);
  box_of(i, box4);
}
int64_t gpl_rules_extend_size_by_scale(int32_t *box4, double scale) {
  Instance i = instance_of(box4);
  int64_t d = i.extend_size_by_scale(scale);
  box_of(i, box4);
  return d;
}
void gpl_rules_orient_point(int orient, int32_t x, int32_t y, int32_t *out2) {
  auto [a, b] = orient_point(orient, x, y);
  out2[0] = a;
  out2[1] = b;
}
int gpl_rules_fmt(const char *which, double v, int a, int b, char *buf, int cap) {
  std::string s, w = which;
  if (w == "fmt_e")
    s = fmt_e(v, a, b);
  else if (w == "fmt_g")
    s = fmt_g(v);
  else if (w == "fmt_g_prec")
    s = fmt_g_prec(v, a);
  else if (w == "log_f32")
    s = log_fmt_f32((float)v);
  else if (w == "log_f64")
    s = log_fmt_f64(v);
  else if (w == "log_e")
    s = log_fmt_e(v, a);
  else if (w == "rust_f32")
    s = rust_f32((float)v);
  else
    return -1;
  std::snprintf(buf, cap, "%s", s.c_str());
  return (int)s.size();
}
int gpl_rules_diverge_fallback(int saved, int reverts, int disable) {
  LoopSnapshots s;
  s.diverge_saved = saved;
  s.diverge_reverts = reverts;
  return (int)diverge_fallback(s, disable);
}
int gpl_rules_routability_recovery_attempt(int route_saved, int attempts, int saved, int reverts, int need) {
  LoopSnapshots s;
  s.route_saved = route_saved;
  s.route_attempts = attempts;
  s.diverge_saved = saved;
  s.diverge_reverts = reverts;
  return routability_recovery_attempt(s, need);
}
int gpl_rules_max_iter_takes_snapshot(int iter, int max_iter, int disable, int saved, int reverts, int64_t snap_hpwl, float snap_ov, float ov, int64_t hpwl) {
  LoopSnapshots s;
  s.diverge_saved = saved;
  s.diverge_reverts = reverts;
  s.diverge_hpwl = snap_hpwl;
  return max_iter_takes_min_hpwl_snapshot(iter, max_iter, disable, s, snap_ov, ov, hpwl);
}
void gpl_rules_settle_wait_step(int start, int iter, int active, int settled, int *out3) {
  int extra = 0;
  auto [s, e] = settle_wait_step(start, iter, active, settled, extra);
  out3[0] = s;
  out3[1] = e;
  out3[2] = extra;
}
float gpl_rules_fast_exp(float x) { return fast_exp(x); }
float gpl_rules_wavenumber_x(int i, int nx) { return wavenumber_x(i, nx); }
float gpl_rules_wavenumber_y(int i, int ny, float bx, float by) { return wavenumber_y(i, ny, bx, by); }
uint32_t gpl_rules_round_down_pow2(uint32_t x) { return round_down_to_power_of_two(x); }
int64_t gpl_rules_union_area(int n, const int32_t *rects) {
  std::vector<std::array<int32_t, 4>> r(n);
  for (int i = 0; i < n; i++) r[i] = {rects[4 * i], rects[4 * i + 1], rects[4 * i + 2], rects[4 * i + 3]};
  return union_area(r);
}
float gpl_rules_distance(int n, const float *a, const float *b) {
  std::vector<FloatPoint> x(n), y(n);
  for (int i = 0; i < n; i++) {
    x[i] = {a[2 * i], a[2 * i + 1]};
    y[i] = {b[2 * i], b[2 * i + 1]};
  }
  return distance(x, y);
}
float gpl_rules_derived_reference_hpwl(float user, int64_t h) { return derived_reference_hpwl(user, h); }
void gpl_rules_set_size(int32_t *box4, int32_t dx, int32_t dy) {
  GCell g;
  g.lx = box4[0];
  g.ly = box4[1];
  g.ux = box4[2];
  g.uy = box4[3];
  set_size(g, dx, dy);
  box4[0] = g.lx;
  box4[1] = g.ly;
  box4[2] = g.ux;
  box4[3] = g.uy;
}
void gpl_rules_top_averages(int n, const double *desc, double *out4) {
  auto a = top_averages(std::vector<double>(desc, desc + n));
  for (int k = 0; k < 4; k++) out4[k] = a[k];
}
// RUDY's host half (src/route_base.rs:144-188, :257-264): wire width, tile rects (x-major),
// blockage and congestion for the given demand.
void gpl_rules_rudy_grid(const int32_t die4[4], int32_t xg, int32_t yg, int32_t ts, int np, const int32_t *pitches, const uint8_t *cap_red, const float *demand, int32_t *wire_width, int32_t *rects, float *blockage, float *congestion) {
  Rudy r;
  r.init(die4, xg, yg, ts, std::vector<int32_t>(pitches, pitches + np));
  *wire_width = r.wire_width;
  for (size_t k = 0; k < r.rects.size(); k++)
    for (int q = 0; q < 4; q++) rects[4 * k + q] = r.rects[k][q];
  r.set_blockage(std::vector<uint8_t>(cap_red, cap_red + 2 * r.blockage.size()));
  std::copy(demand, demand + r.demand.size(), r.demand.begin());
  for (int32_t x = 0; x < xg; x++)
    for (int32_t y = 0; y < yg; y++) {
      blockage[r.at(x, y)] = r.blockage[r.at(x, y)];
      congestion[r.at(x, y)] = r.congestion(x, y);
    }
}
}  // extern "C"
