// The per-kernel C entry points (include/gpl.h) and the synthetic router.
#include <algorithm>
#include <climits>
#include <cstring>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../../include/gpl.h"
#include "../kernels/b2b.h"
#include "../kernels/bicgstab.h"
#include "../kernels/engine_kernels.h"
#include "../kernels/rudy.h"
#include "parallel.h"

using namespace gpl;

extern "C" {

int gpl_kernel_density_scatter(int64_t n_cells, const int32_t *cx, const int32_t *cy, const int32_t *hx, const int32_t *hy, const float *scale, const uint8_t *kind, int32_t nx, int32_t ny, int32_t grid_lx, int32_t grid_ly, const int32_t *bx, const int32_t *by, double size_x, double size_y, float target_density, int64_t *inst, int64_t *filler, void *stream) {
  cudaStream_t s = (cudaStream_t)stream;
  size_t nb = (size_t)nx * ny;
  cudaError_t e = cudaMemsetAsync(inst, 0, nb * sizeof(int64_t), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(filler, 0, nb * sizeof(int64_t), s);
  if (e != cudaSuccess) return (int)e;
  if (n_cells <= 0) return 0;
  RegionArgs r{};
  r.n_cells = (int32_t)n_cells;
  r.nx = nx;
  r.ny = ny;
  r.lx = grid_lx;
  r.ly = grid_ly;
  r.size_x = size_x;
  r.size_y = size_y;
  r.inv_size_x = 1.0 / size_x;
  r.inv_size_y = 1.0 / size_y;
  {
    std::vector<int32_t> hbx(nx + 1), hby(ny + 1);
    e = cudaMemcpyAsync(hbx.data(), bx, hbx.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hby.data(), by, hby.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return (int)e;
    r.narrow = narrow_tile(hbx, hby) ? 1 : 0;
  }
  r.target_density = target_density;
  // GPL_SCATTER=global|pooled: the scatter's other forms (the engine's tuner picks per region)
  if (const char *f = std::getenv("GPL_SCATTER")) r.scatter_form = std::string(f) == "global" ? 1 : std::string(f) == "pooled" ? 2 : 0;
  r.bx = bx;
  r.by = by;
  r.acc_inst = inst;
  r.acc_fill = filler;
  // the engine keeps a cell's centre as one int2: pack the caller's two arrays
  int2 *dc = nullptr;
  e = cudaMallocAsync((void **)&dc, (size_t)n_cells * sizeof(int2), s);
  if (e != cudaSuccess) return (int)e;
  unsigned blocks = (unsigned)((n_cells + kThreadsPerBlock - 1) / kThreadsPerBlock);
  k_pack_centres<<<blocks, kThreadsPerBlock, 0, s>>>(n_cells, cx, cy, dc);
  CellArgs c{};
  c.dc = dc;
  c.hx = hx;
  c.hy = hy;
  c.dscale = scale;
  c.kind = kind;
  k_place_cells<<<blocks, kThreadsPerBlock, 0, s>>>(r, c, PLACE_GIVEN, 0.0f, 0.0f, nullptr);
  e = cudaGetLastError();
  cudaError_t e2 = cudaFreeAsync(dc, s);
  return (int)(e != cudaSuccess ? e : e2);
}

// A grid of the caller's bins as the trial kernels read it; its edges are read back here (the
// scatter's 32-bit tile test and the grid's upper corner).
static cudaError_t region_args(RegionArgs &r, int64_t n_cells, int32_t nx, int32_t ny, int32_t grid_lx, int32_t grid_ly, const int32_t *bx, const int32_t *by, double size_x, double size_y, float target_density, cudaStream_t s) {
  if (n_cells < 0 || n_cells >= ((int64_t)1 << 31) || nx <= 0 || ny <= 0) return cudaErrorInvalidValue;
  r = RegionArgs{};
  r.n_cells = (int32_t)n_cells;
  r.nx = nx;
  r.ny = ny;
  r.lx = grid_lx;
  r.ly = grid_ly;
  r.size_x = size_x;
  r.size_y = size_y;
  r.inv_size_x = 1.0 / size_x;
  r.inv_size_y = 1.0 / size_y;
  std::vector<int32_t> hbx(nx + 1), hby(ny + 1);
  cudaError_t e = cudaMemcpyAsync(hbx.data(), bx, hbx.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hby.data(), by, hby.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  r.ux = hbx[nx];
  r.uy = hby[ny];
  r.narrow = narrow_tile(hbx, hby) ? 1 : 0;
  r.target_density = target_density;
  // GPL_SCATTER=global|pooled: the scatter's other forms (the engine's tuner picks per region)
  if (const char *f = std::getenv("GPL_SCATTER")) r.scatter_form = std::string(f) == "global" ? 1 : std::string(f) == "pooled" ? 2 : 0;
  r.bx = bx;
  r.by = by;
  return cudaSuccess;
}

static bool aligned8(const void *p) { return ((uintptr_t)p & 7u) == 0; }

int gpl_kernel_nesterov_step(int64_t n_cells, const float *cur_slp, const float *cur_slp_sum, const float *cur, const int32_t *hx, const int32_t *hy, const float *scale, const uint8_t *kind, const uint8_t *locked, int32_t nx, int32_t ny, int32_t grid_lx, int32_t grid_ly, const int32_t *bx, const int32_t *by, double size_x, double size_y, float target_density, float step, float coeff, float *next, float *next_slp, int32_t *centre, int64_t *inst, int64_t *filler, void *stream) {
  cudaStream_t s = (cudaStream_t)stream;
  RegionArgs r;
  cudaError_t e = region_args(r, n_cells, nx, ny, grid_lx, grid_ly, bx, by, size_x, size_y, target_density, s);
  if (e != cudaSuccess) return (int)e;
  for (const void *p : {(const void *)cur_slp, (const void *)cur_slp_sum, (const void *)cur, (const void *)next, (const void *)next_slp, (const void *)centre})
    if (!aligned8(p)) return (int)cudaErrorMisalignedAddress;  // read and written as pairs
  size_t nb = (size_t)nx * ny;
  e = cudaMemsetAsync(inst, 0, nb * sizeof(int64_t), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(filler, 0, nb * sizeof(int64_t), s);
  if (e != cudaSuccess || n_cells == 0) return (int)e;
  r.acc_inst = inst;
  r.acc_fill = filler;
  CellArgs c{};
  c.dc = reinterpret_cast<int2 *>(centre);
  c.hx = hx;
  c.hy = hy;
  c.dscale = scale;
  c.kind = kind;
  c.locked = locked;
  // the kernel reads cur_slp, cur_slp_sum and cur and writes next and next_slp only
  c.cur_slp = reinterpret_cast<float2 *>(const_cast<float *>(cur_slp));
  c.cur_slp_sum = reinterpret_cast<float2 *>(const_cast<float *>(cur_slp_sum));
  c.cur = reinterpret_cast<float2 *>(const_cast<float *>(cur));
  c.next = reinterpret_cast<float2 *>(next);
  c.next_slp = reinterpret_cast<float2 *>(next_slp);
  unsigned blocks = (unsigned)((n_cells + kThreadsPerBlock - 1) / kThreadsPerBlock);
  k_place_cells<<<blocks, kThreadsPerBlock, 0, s>>>(r, c, PLACE_NESTEROV, step, coeff, nullptr);
  return (int)cudaGetLastError();
}

int gpl_kernel_gradients(int64_t n_cells, const int32_t *centre, const int32_t *hx, const int32_t *hy, const float *scale, const float *area, const int64_t *cell_pin_start, const float *pin_force, int32_t nx, int32_t ny, int32_t grid_lx, int32_t grid_ly, const int32_t *bx, const int32_t *by, double size_x, double size_y, const float *field_x, const float *field_y, float penalty, float *sum, const float *a1, const float *b1, const float *b2, double *sums, void *stream) {
  cudaStream_t s = (cudaStream_t)stream;
  for (int k = 0; k < 4; k++) sums[k] = 0.0;
  RegionArgs r;
  cudaError_t e = region_args(r, n_cells, nx, ny, grid_lx, grid_ly, bx, by, size_x, size_y, 1.0f, s);
  if (e != cudaSuccess) return (int)e;
  for (const void *p : {(const void *)centre, (const void *)pin_force, (const void *)sum, (const void *)a1, (const void *)b1, (const void *)b2})
    if (!aligned8(p)) return (int)cudaErrorMisalignedAddress;
  if ((a1 == nullptr) != (b1 == nullptr)) return (int)cudaErrorInvalidValue;
  if (n_cells == 0) return 0;
  r.field_x = const_cast<float *>(field_x);
  r.field_y = const_cast<float *>(field_y);
  CellArgs c{};
  c.dc = reinterpret_cast<int2 *>(const_cast<int32_t *>(centre));
  c.hx = hx;
  c.hy = hy;
  c.dscale = scale;
  c.area = area;
  c.pin_start = cell_pin_start;
  const int blocks = (int)((n_cells + kThreadsPerBlock - 1) / kThreadsPerBlock);
  // the block partials, the arrival ticket and the four sums, in one scratch block
  const size_t bytes = (size_t)(4 * blocks + 4) * sizeof(double) + 256;
  uint8_t *scratch = nullptr;
  e = cudaMallocAsync((void **)&scratch, bytes, s);
  if (e != cudaSuccess) return (int)e;
  double *partials = reinterpret_cast<double *>(scratch), *out = partials + 4 * blocks;
  unsigned int *ticket = reinterpret_cast<unsigned int *>(out + 4);
  e = cudaMemsetAsync(ticket, 0, sizeof(unsigned int), s);
  if (e == cudaSuccess) {
    k_gradients<<<blocks, kThreadsPerBlock, 0, s>>>(r, c, reinterpret_cast<const float2 *>(pin_force), penalty, reinterpret_cast<float2 *>(sum), reinterpret_cast<const float2 *>(a1),
                                                    reinterpret_cast<const float2 *>(b1), reinterpret_cast<const float2 *>(b2), partials, ticket, out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(sums, out, 4 * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaError_t e2 = cudaFreeAsync(scratch, s);
  return (int)(e != cudaSuccess ? e : e2);
}

int gpl_kernel_poisson(int32_t nx, int32_t ny, const float *wx, const float *wy, const float *density, float *field_x, float *field_y, int mode, void *stream) {
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaSuccess;
  PoissonPlan *p = poisson_plan_create(nx, ny, wx, wy, mode, &e);
  if (!p) return (int)e;
  int ld = 0;
  __nv_bfloat16 *split = poisson_split_input(p, &ld);
  if (split) {
    // the tensor-core path reads the density as split bf16: convert it
    e = poisson_split_density(p, density, s);
  }
  if (e == cudaSuccess) e = poisson_solve(p, density, field_x, field_y, s);
  cudaError_t e2 = cudaStreamSynchronize(s);
  poisson_plan_destroy(p);
  return (int)(e != cudaSuccess ? e : e2);
}

// The caller's nets on the device as the engine holds them: in degree order (stable), their
// pins following them, each pin's slot its index in the caller's order (so a force goes back to
// its own place); the degree-2..4 ranges, the tiles and the nets too large for a tile.
struct DeviceNets {
  cudaStream_t s;
  cudaError_t e = cudaSuccess;
  int64_t *d_ns = nullptr;
  int32_t *d_xy = nullptr, *d_slot = nullptr, *d_big = nullptr;
  int4 *d_tiles = nullptr;
  float *d_wt = nullptr;
  WaSmall small{};
  size_t n_tiles = 0, n_big = 0;
  int64_t n_pins = 0;
  explicit DeviceNets(cudaStream_t st) : s(st) {}
  ~DeviceNets() {
    void *bufs[] = {d_ns, d_xy, d_slot, d_tiles, d_big, d_wt};
    for (void *p : bufs)
      if (p) cudaFreeAsync(p, s);
  }
  cudaError_t build(int64_t n_nets, const int64_t *net_start, const int32_t *pin_xy, const float *net_weight) {
    std::vector<int64_t> starts((size_t)n_nets + 1);
    e = cudaMemcpyAsync(starts.data(), net_start, starts.size() * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
    const int64_t np = starts[n_nets];
    n_pins = np;
    if (np >= ((int64_t)1 << 31)) return e = cudaErrorInvalidValue;  // pin numbers are 32-bit
    std::vector<int32_t> order((size_t)n_nets);
    for (int64_t n = 0; n < n_nets; n++) order[n] = (int32_t)n;
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return starts[x + 1] - starts[x] < starts[y + 1] - starts[y]; });
    std::vector<int32_t> xy((size_t)np * 2), xy2((size_t)np * 2), slot((size_t)np);
    std::vector<float> wt, wt2;
    if (np) e = cudaMemcpyAsync(xy.data(), pin_xy, xy.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && net_weight) {
      wt.resize((size_t)n_nets);
      wt2.resize((size_t)n_nets);
      e = cudaMemcpyAsync(wt.data(), net_weight, wt.size() * sizeof(float), cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
    std::vector<int64_t> ns((size_t)n_nets + 1, 0);
    int64_t at = 0;
    for (int64_t i = 0; i < n_nets; i++) {
      const int32_t n = order[i];
      for (int64_t q = starts[n]; q < starts[n + 1]; q++, at++) {
        xy2[2 * at] = xy[2 * q];
        xy2[2 * at + 1] = xy[2 * q + 1];
        slot[at] = (int32_t)q;
      }
      ns[i + 1] = at;
      if (net_weight) wt2[i] = wt[n];
    }
    std::vector<int4> tiles;
    std::vector<int32_t> big;
    small = wa_small_ranges(ns.data(), (int32_t)n_nets);
    wa_tiles(ns.data(), 0, small.first[0], tiles, big);
    wa_tiles(ns.data(), small.first[2] + small.count[2], (int32_t)n_nets, tiles, big);
    n_tiles = tiles.size();
    n_big = big.size();
    auto put = [&](auto **d, const auto &v) {
      if (e != cudaSuccess) return;
      e = cudaMallocAsync((void **)d, std::max<size_t>(v.size(), 1) * sizeof(v[0]), s);
      if (e == cudaSuccess && !v.empty()) e = cudaMemcpyAsync(*d, v.data(), v.size() * sizeof(v[0]), cudaMemcpyHostToDevice, s);
    };
    put(&d_ns, ns);
    put(&d_xy, xy2);
    put(&d_slot, slot);
    put(&d_tiles, tiles);
    put(&d_big, big);
    if (net_weight) put(&d_wt, wt2);
    // the host vectors above are freed on return: the copies must have read them
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e;
  }
  WaArgs args(float *grad) const {
    WaArgs w{};
    w.n_nets = (int32_t)n_big;
    w.net_start = d_ns;
    w.net_order = d_big;
    w.net_weight = d_wt;
    w.pin_base = reinterpret_cast<const int2 *>(d_xy);
    w.pin_slot = d_slot;
    w.pin_grad = reinterpret_cast<float2 *>(grad);
    w.n_tiles = (int32_t)n_tiles;
    w.tiles = d_tiles;
    w.small = small;
    return w;
  }
};

int gpl_kernel_wa(int64_t n_nets, const int64_t *net_start, const int32_t *pin_xy, const float *net_weight, float coef_x, float coef_y, float *grad, void *stream) {
  if (n_nets <= 0) return 0;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e;
  {
    DeviceNets d(s);
    e = d.build(n_nets, net_start, pin_xy, net_weight);
    if (e == cudaSuccess) {
      WaArgs w = d.args(grad);
      launch_wa_small(w, coef_x, coef_y, 1, s);
      if (w.n_tiles) launch_wa_tiles(w, coef_x, coef_y, s);
      if (w.n_nets) k_wa<<<(unsigned)((w.n_nets + kThreadsPerBlock - 1) / kThreadsPerBlock), kThreadsPerBlock, 0, s>>>(w, coef_x, coef_y);
      e = cudaGetLastError();
    }
  }
  cudaError_t e2 = cudaStreamSynchronize(s);
  return (int)(e != cudaSuccess ? e : e2);
}

int gpl_kernel_hpwl(int64_t n_nets, const int64_t *net_start, const int32_t *pin_xy, int32_t fused, int64_t *hpwl, void *stream) {
  *hpwl = 0;
  if (n_nets <= 0) return 0;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e;
  unsigned long long h = 0;
  {
    DeviceNets d(s);
    unsigned long long *acc = nullptr;
    float *grad = nullptr;
    e = d.build(n_nets, net_start, pin_xy, nullptr);
    if (e == cudaSuccess) e = cudaMallocAsync((void **)&acc, sizeof(unsigned long long), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(acc, 0, sizeof(unsigned long long), s);
    if (e == cudaSuccess && fused) e = cudaMallocAsync((void **)&grad, (size_t)std::max<int64_t>(d.n_pins, 1) * 2 * sizeof(float), s);
    if (e == cudaSuccess) {
      WaArgs w = d.args(grad);
      w.hpwl_out = acc;
      const unsigned nbig = (unsigned)((w.n_nets + kThreadsPerBlock - 1) / kThreadsPerBlock);
      const float c = 1e-4f;  // any coefficient: the HPWL is the pins' boxes
      if (fused) {
        // the HPWL the WA kernels add up beside the forces (the trial's read-back)
        launch_wa_small(w, c, c, 1, s);
        if (w.n_tiles) launch_wa_tiles(w, c, c, s);
        if (w.n_nets) k_wa<<<nbig, kThreadsPerBlock, 0, s>>>(w, c, c);
      } else {
        // the HPWL kernels of an iteration without a WA pass
        launch_wa_small(w, 0.0f, 0.0f, 0, s);
        if (w.n_tiles) k_hpwl_tiles<<<(unsigned)w.n_tiles, kThreadsPerBlock, 0, s>>>(w, acc);
        if (w.n_nets) k_hpwl<<<nbig, kThreadsPerBlock, 0, s>>>(w, acc);
      }
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaMemcpyAsync(&h, acc, sizeof h, cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (acc) cudaFreeAsync(acc, s);
    if (grad) cudaFreeAsync(grad, s);
  }
  cudaError_t e2 = cudaStreamSynchronize(s);
  if (e == cudaSuccess && e2 == cudaSuccess) *hpwl = (int64_t)h;
  return (int)(e != cudaSuccess ? e : e2);
}

int gpl_kernel_csr_from_triplets(int64_t n, int64_t nt, const int32_t *rows, const int32_t *cols, const float *vals, int64_t *row_start, int32_t *out_cols, float *out_vals, int64_t *nnz, void *stream) {
  if (n < 0 || nt < 0 || nt >= ((int64_t)1 << 32)) return (int)cudaErrorInvalidValue;  // positions are 32-bit
  IpDevice dev((cudaStream_t)stream);
  return (int)dev.csr_from_triplets(n, nt, rows, cols, vals, row_start, out_cols, out_vals, nnz);
}

static_assert(GPL_SPMV_ROWS == kSpmvRows && GPL_SPMV_TILED == kSpmvTiled, "the C ABI's SpMV forms");

int gpl_kernel_spmv(int64_t n, const int64_t *row_start, const int32_t *cols, const float *vals, const float *x, float *y, int32_t form, void *stream) {
  CsrDev A{n, row_start, cols, vals};
  cudaStream_t s = (cudaStream_t)stream;
  if (form != kSpmvSliced || n <= 0) return (int)spmv(A, x, y, form, s);
  // the sliced copy: the order by length and the slice widths on the device, their
  // exclusive scan here, the entries
  int64_t *starts = nullptr;
  int32_t *row = nullptr, *len = nullptr, *count = nullptr;
  int2 *ent = nullptr;
  int32_t n_long = 0;
  cudaError_t e = cudaMalloc(&row, (size_t)n * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMalloc(&len, (size_t)n * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMalloc(&count, (size_t)(kSliceLenCap + 1) * sizeof(int32_t));
  if (e == cudaSuccess) e = csr_slice_order(A, row, len, count, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&n_long, count + kSliceLongRow + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  const int64_t ns = (n - n_long + kSliceRows - 1) / kSliceRows;
  std::vector<int64_t> h((size_t)ns + 1, 0);
  if (e == cudaSuccess) e = cudaMalloc(&starts, (size_t)(ns + 1) * sizeof(int64_t));
  if (e == cudaSuccess) e = csr_slice_widths(n, n_long, len, starts, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), starts, (size_t)ns * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) {
    int64_t run = 0;
    for (int64_t k = 0; k < ns; k++) {
      const int64_t w = h[(size_t)k];
      h[(size_t)k] = run;
      run += w;
    }
    h[(size_t)ns] = run;
    e = cudaMemcpyAsync(starts, h.data(), (size_t)(ns + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s);
  }
  const size_t total = (size_t)std::max<int64_t>(h[(size_t)ns], 1);
  if (e == cudaSuccess) e = cudaMalloc(&ent, total * sizeof(int2));
  if (e == cudaSuccess) {
    A.sl_long = n_long;
    A.sl_row = row;
    A.sl_len = len;
    A.sl_start = starts;
    e = csr_slice_fill(A, ent, s);
  }
  if (e == cudaSuccess) {
    A.sl_ent = ent;
    e = spmv(A, x, y, form, s);
  }
  cudaError_t e2 = cudaStreamSynchronize(s);
  for (void *p : {(void *)starts, (void *)row, (void *)len, (void *)count, (void *)ent}) cudaFree(p);
  return (int)(e != cudaSuccess ? e : e2);
}

int gpl_kernel_bicgstab(int64_t n, const int64_t *row_start, const int32_t *cols, const float *vals, const float *rhs, float *x, int32_t max_iters, int32_t *iterations, float *error, void *stream) {
  cudaStream_t s = (cudaStream_t)stream;
  void *scratch = nullptr;
  cudaError_t e = cudaMalloc(&scratch, bicgstab_scratch_bytes(n));
  if (e != cudaSuccess) return (int)e;
  CsrDev A{n, row_start, cols, vals};
  BicgResult r{};
  e = bicgstab_solve(A, rhs, x, max_iters, scratch, s, &r);
  cudaError_t e2 = cudaStreamSynchronize(s);
  cudaFree(scratch);
  *iterations = r.iterations;
  *error = r.error;
  return (int)(e != cudaSuccess ? e : e2);
}

int gpl_kernel_rudy(int64_t n_nets, const int32_t *boxes, int32_t die_lx, int32_t die_ly, int32_t die_ux, int32_t die_uy, int32_t cnt_x, int32_t cnt_y, int32_t tile_size, int32_t wire_width, float *demand, void *stream) {
  RudyGrid g{die_lx, die_ly, die_ux, die_uy, cnt_x, cnt_y, tile_size, wire_width};
  return (int)rudy_demand(g, n_nets, reinterpret_cast<const int4 *>(boxes), demand, (cudaStream_t)stream);
}

// ---------------------------------------------------------------- the synthetic router
struct SynthRouter {
  gpl_router_t r;
  int32_t die[4];
  int32_t tile;
  std::vector<int32_t> pitches;
  uint8_t capacity;
  std::vector<int32_t> inst_xy;   // lower-left per design instance
  std::vector<int64_t> net_iterm_start, net_bterm_start;
  std::vector<int32_t> iterm_inst, iterm_shape, bterm_box;
  std::vector<uint8_t> bterm_placed;
};

static int sr_write(void *u, int64_t n, const int32_t *loc) {
  SynthRouter *s = (SynthRouter *)u;
  for (int64_t k = 0; k < n; k++) {
    int32_t di = loc[3 * k];
    if (di < 0 || (size_t)di * 2 + 1 >= s->inst_xy.size()) return 1;
    s->inst_xy[2 * di] = loc[3 * k + 1];
    s->inst_xy[2 * di + 1] = loc[3 * k + 2];
  }
  return 0;
}
static int sr_inputs(void *u, int32_t die[4], int32_t *xg, int32_t *yg, int32_t *ts, int32_t *np, int32_t p[32]) {
  SynthRouter *s = (SynthRouter *)u;
  std::memcpy(die, s->die, sizeof s->die);
  *xg = std::max(1, (s->die[2] - s->die[0]) / s->tile);
  *yg = std::max(1, (s->die[3] - s->die[1]) / s->tile);
  *ts = s->tile;
  *np = (int32_t)std::min<size_t>(32, s->pitches.size());
  for (int i = 0; i < *np; i++) p[i] = s->pitches[i];
  return 0;
}
static int sr_cap(void *u, uint8_t *cr, int64_t n) {
  SynthRouter *s = (SynthRouter *)u;
  for (int64_t i = 0; i < n; i++) {
    cr[2 * i] = s->capacity;
    cr[2 * i + 1] = 0;
  }
  return 0;
}
static int64_t sr_boxes(void *u, int32_t *idx, int32_t *boxes, int64_t cap) {
  SynthRouter *s = (SynthRouter *)u;
  int64_t nn = (int64_t)s->net_iterm_start.size() - 1;
  if (!boxes) return nn;
  // each net's box from its own terminals: the nets in parallel
  parallel_for((size_t)std::min(nn, cap), [&](size_t n0, size_t n1) {
  for (int64_t n = (int64_t)n0; n < (int64_t)n1; n++) {
    int32_t lx = INT32_MAX, ly = INT32_MAX, ux = INT32_MIN, uy = INT32_MIN;
    for (int64_t t = s->net_iterm_start[n]; t < s->net_iterm_start[n + 1]; t++) {
      int32_t i = s->iterm_inst[t];
      const int32_t *sh = &s->iterm_shape[4 * t];
      int32_t x = s->inst_xy[2 * i], y = s->inst_xy[2 * i + 1];
      lx = std::min(lx, x + sh[0]);
      ly = std::min(ly, y + sh[1]);
      ux = std::max(ux, x + sh[2]);
      uy = std::max(uy, y + sh[3]);
    }
    for (int64_t t = s->net_bterm_start[n]; t < s->net_bterm_start[n + 1]; t++) {
      if (!s->bterm_placed[t]) continue;
      const int32_t *b = &s->bterm_box[4 * t];
      lx = std::min(lx, b[0]);
      ly = std::min(ly, b[1]);
      ux = std::max(ux, b[2]);
      uy = std::max(uy, b[3]);
    }
    idx[n] = (int32_t)n;
    boxes[4 * n] = lx;
    boxes[4 * n + 1] = ly;
    boxes[4 * n + 2] = ux;
    boxes[4 * n + 3] = uy;
  }
  });
  return std::min(nn, cap);
}

gpl_router_t *gpl_synthetic_router_create(const gpl_design_t *d, int32_t tile_size, int32_t n_pitches, const int32_t *pitches, uint8_t capacity) {
  if (tile_size <= 0) return nullptr;
  SynthRouter *s = new SynthRouter();
  std::memcpy(s->die, d->die, sizeof s->die);
  s->tile = tile_size;
  s->pitches.assign(pitches, pitches + std::max(0, n_pitches));
  s->capacity = capacity;
  s->inst_xy.resize(2 * (size_t)d->n_insts);
  for (int32_t i = 0; i < d->n_insts; i++) {
    s->inst_xy[2 * i] = d->inst_box[4 * i];
    s->inst_xy[2 * i + 1] = d->inst_box[4 * i + 1];
  }
  s->net_iterm_start.assign(d->net_iterm_start, d->net_iterm_start + d->n_nets + 1);
  s->net_bterm_start.assign(d->net_bterm_start, d->net_bterm_start + d->n_nets + 1);
  int64_t nt = s->net_iterm_start.back(), nb = s->net_bterm_start.back();
  s->iterm_inst.assign(d->iterm_inst, d->iterm_inst + nt);
  s->iterm_shape.assign(d->iterm_shape, d->iterm_shape + 4 * nt);
  s->bterm_box.assign(d->bterm_box, d->bterm_box + 4 * nb);
  s->bterm_placed.resize(nb);
  for (int64_t t = 0; t < nb; t++) s->bterm_placed[t] = d->bterm_flags[t] & GPL_BTERM_PLACED;
  s->r.user = s;
  s->r.write_locations = sr_write;
  s->r.rudy_inputs = sr_inputs;
  s->r.capacity_reduction = sr_cap;
  s->r.net_term_boxes = sr_boxes;
  return &s->r;
}

void gpl_synthetic_router_destroy(gpl_router_t *r) {
  if (r) delete (SynthRouter *)r->user;
}

}  // extern "C"
