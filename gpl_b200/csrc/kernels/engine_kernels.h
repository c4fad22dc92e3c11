// Kernel argument blocks and launchers shared by the engine's host code and its kernels.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <vector>

namespace gpl {

constexpr int kThreadsPerBlock = 256;  // the block size every launch uses

enum CellKind : uint8_t { CELL_STD = 0, CELL_MACRO = 1, CELL_FILLER = 2 };
enum PlaceMode { PLACE_AT = 0, PLACE_NESTEROV = 1, PLACE_GIVEN = 2 };  // GIVEN: the centres in dc

// WA and HPWL run over tiles of consecutive nets (pins are net-major, so a tile's pins are
// contiguous): at most kWaTilePins pins and kWaTileNets nets per tile, one block per tile.
// A net with more pins than a tile holds runs in the thread-per-net kernels instead.
constexpr int kWaTilePins = 512;
constexpr int kWaTileNets = 256;

// One region's bin grid (`BinGrid`, src/nesterov.rs:260-295) and its cell count.
struct RegionArgs {
  int32_t n_cells;
  int32_t nx, ny;
  int32_t lx, ly, ux, uy;        // the grid's box
  double size_x, size_y;
  double inv_size_x, inv_size_y; // 1 / size, rounded (the bin span's fast path)
  int32_t narrow;                // a block's sum into one bin fits 32 bits (the scatter's tile)
  float target_density;
  // the scatter's form: 0 shared tiles (a block's or a warp's, else straight to HBM); 1 every
  // addend straight to HBM; 2 straight to HBM, a warp's lanes that hit one bin pooled first
  int32_t scatter_form;
  const int32_t *bx, *by;        // bin edges, nx+1 and ny+1
  const float *scaled;           // bin area * target density (float)
  const float *non_place, *non_place_u;  // the fixed areas (int64) as float, as the density reads them
  int64_t *acc_inst, *acc_fill;  // scatter accumulators (cleared by the finalize)
  float *density, *field_x, *field_y;
  // blocks of the last scatter whose cells spread past the shared tile (NULL: not counted);
  // the finalize reports the count (out[6]) and clears it
  unsigned int *spread;
};

// One region's cells, SoA, region-local index.
struct CellArgs {
  int2 *dc;                      // density centre (the integer box centre)
  const int32_t *hx, *hy;        // half density size
  const float *dscale;           // density scale
  const uint8_t *kind;           // CellKind
  const uint8_t *locked;         // may be NULL
  const float *area;             // (float)dx * (float)dy of the cell box, for the preconditioner
  const int64_t *pin_start;      // the cell's pins (CSR, the cell's own order): its WA forces
  float2 *cur_slp, *cur_slp_sum, *next_slp, *next_slp_sum, *prev_slp, *prev_slp_sum, *cur, *next;
};

// The nets and pins (all regions): pins net-major.
// Nets of degree 2, 3 and 4 (most of a netlist) run a thread per net with their pins in
// registers (k_wa_small, no shared memory and no barriers): one range of consecutive device
// nets per degree (the device orders its nets by degree).
struct WaSmall {
  int32_t first[3], count[3];  // degree 2 + k: nets [first[k], first[k] + count[k])
  int64_t pin0[3];             // and their pins from pin0[k], 2 + k a net in net order
};

struct WaArgs {
  int32_t n_nets;                // nets the thread-per-net kernels walk (net_order, or 0..n)
  const int64_t *net_start;
  const int32_t *net_order;      // NULL: natural order
  const float *net_weight;       // NULL: 1
  const int32_t *pin_cell;       // global device cell index, -1 for a pin with no cell (NULL: none)
  const int2 *pin_base;          // offset from the cell's centre, or the fixed position
  const int2 *dc;                // global device cell centres
  const int32_t *pin_slot;       // where a pin's force goes (-1: nowhere); NULL: at the pin
  float2 *pin_grad;
  int32_t n_tiles;               // tiles of consecutive nets: first net, end net, first pin, pins
  const int4 *tiles;
  unsigned long long *hpwl_out;  // WA adds the HPWL of the same pin positions here (NULL: not)
  WaSmall small;                 // the degree-2..4 ranges (zero counts: none)
};

// One region's entry in a packed launch (a phase of every live region in one launch): its
// arguments, and its first block and block count in the launch's grid.
struct PackedRegion {
  RegionArgs r;
  CellArgs c;
  int32_t first, blocks;
  float step, coeff;                 // the scatter (PLACE_NESTEROV)
  double *partials, *out;            // the finalize's or the gradients' partials and sums
  unsigned int *ticket;
  __nv_bfloat16 *dens_split;         // the finalize
  int32_t split_ld;
  float penalty;                     // the gradients
  const float2 *pin_grad;
  float2 *out_sum;
  const float2 *a1, *b1, *b2;
};
// The packed phases: k_place_cells (PLACE_NESTEROV), k_bins_finalize and k_gradients of n
// regions, each region's blocks doing exactly what its own launch's would.
__global__ void k_place_packed(const PackedRegion *t, int n);
__global__ void k_finalize_packed(const PackedRegion *t, int n);
__global__ void k_gradients_packed(const PackedRegion *t, int n);
__global__ void k_place_cells(RegionArgs r, CellArgs c, int mode, float step, float coeff, const float2 *coords);
__global__ void k_bins_finalize(RegionArgs r, double *partials, __nv_bfloat16 *dens_split, int split_ld, unsigned int *ticket, double *out);
__global__ void k_wa(WaArgs w, float cx, float cy);
__global__ void k_wa_tiles(WaArgs w, float cx, float cy);
// The nets of w.small, a thread per net: their forces (forces != 0) and their HPWL into
// w.hpwl_out. Launch with wa_small_blocks(w.small) blocks.
__global__ void k_wa_small(WaArgs w, float cx, float cy, int forces);
int wa_small_blocks(const WaSmall &s);
// The same nets, a lane per pin (32 / D nets per warp): forces and HPWL bit for bit as
// k_wa_small's. Launch with wa_pins_blocks(w.small) blocks.
__global__ void k_wa_pins(WaArgs w, float cx, float cy, int forces);
int wa_pins_blocks(const WaSmall &s);
// The degree-2..4 nets' WA (forces != 0) or HPWL alone: k_wa_lean, or k_wa_small / k_wa_pins
// when the environment sets GPL_WA_SMALL=nets / pins (the same results; a timing comparison).
__global__ void k_wa_lean(WaArgs w, float cx, float cy, int forces);
// The degree-2..4 nets' WA in one of its three forms (0 k_wa_lean, 1 k_wa_small, 2 k_wa_pins;
// -1: GPL_WA_SMALL's "nets" / "pins", else the first), which give the same forces and HPWL.
void launch_wa_small(const WaArgs &w, float cx, float cy, int forces, cudaStream_t s, int form = -1);
// The degree-2..4 ranges of nets already in degree order.
WaSmall wa_small_ranges(const int64_t *net_start, int32_t n_nets);
// k_wa_tiles over every tile: a persistent grid of the blocks the device holds at once.
void launch_wa_tiles(const WaArgs &w, float cx, float cy, cudaStream_t s);
__global__ void k_gradients(RegionArgs r, CellArgs c, const float2 *pin_grad, float penalty, float2 *out_sum,
                            const float2 *a1, const float2 *b1, const float2 *b2, double *partials, unsigned int *ticket, double *out);
__global__ void k_prev_slp(RegionArgs r, CellArgs c, float coef);
__global__ void k_hpwl(WaArgs w, unsigned long long *out);
__global__ void k_hpwl_tiles(WaArgs w, unsigned long long *out);
__global__ void k_pack_centres(int64_t n, const int32_t *x, const int32_t *y, int2 *out);

// ---- the device cell order (cell_order.cu): a region's cells sorted again by a coarse Z key
// of their density centres, stably; the per-cell arrays gathered through the permutation.
constexpr int kMaxSlots = 12;
struct CellGather {
  const int2 *dc;
  const int32_t *hx, *hy;
  const float *dscale, *area;
  const uint8_t *kind, *locked;
  const int64_t *pin_start;  // n + 1
  const int32_t *order;
  int2 *dc_out;
  int32_t *hx_out, *hy_out;
  float *dscale_out, *area_out;
  uint8_t *kind_out, *locked_out;
  int64_t *pins_out;          // each cell's pin count (n, scanned afterwards)
  int32_t *inv, *order_out;   // old -> new; the upload-time index of each new cell
  int n_slots;
  const float2 *slot[kMaxSlots];
  float2 *slot_out[kMaxSlots];
};
int order_tiles(int32_t n);
// Sorts the cells [0, n) by the Hilbert index of their density centres on a 1024 x 1024 grid
// of tile_w x tile_h cells from (lx, ly); the old indices in new order end in idx0
// (key0/key1/idx1: n each; hist: 64 * order_tiles(n)).
cudaError_t order_sort(int32_t n, const int2 *dc, int32_t lx, int32_t ly, double tile_w, double tile_h, uint32_t *key0, int32_t *idx0, uint32_t *key1, int32_t *idx1, int32_t *hist, cudaStream_t s);
// The same sort of n float centres (x[i], y[i]) over the box from (lx, ly), tile_w x tile_h a
// grid step.
cudaError_t order_sort_xy(int32_t n, const float *x, const float *y, double lx, double ly, double tile_w, double tile_h, uint32_t *key0, int32_t *idx0, uint32_t *key1, int32_t *idx1, int32_t *hist, cudaStream_t s);
__global__ void k_order_gather(int32_t n, const int32_t *perm, CellGather g);
__global__ void k_order_pins(int64_t n_pins, int32_t off, int32_t n, const int32_t *inv, const int64_t *old_start, const int64_t *new_start, int32_t *pin_cell, int32_t *pin_slot);
__global__ void k_order_starts(int32_t n, const int64_t *rel, int64_t *start);
__global__ void k_iota(int32_t n, int32_t *a);

// Whether a grid's bins are small enough for the scatter's 32-bit shared tile.
bool narrow_tile(const std::vector<int32_t> &bx, const std::vector<int32_t> &by);

// Tiles of the consecutive nets [first, last) (at most kWaTilePins pins and kWaTileNets nets
// each) and the nets too large for a tile, from the nets' pin starts; appended to both lists.
void wa_tiles(const int64_t *net_start, int32_t first, int32_t last, std::vector<int4> &tiles, std::vector<int32_t> &big);
__global__ void k_hold_locked(RegionArgs r, CellArgs c);

// The density solver (Fft::solve without the potential): FP32 SIMT GEMMs or split-BF16
// tcgen05 GEMMs. Workspace layout and basis matrices are the solver's own.
struct PoissonPlan;
PoissonPlan *poisson_plan_create(int nx, int ny, const float *wx_host, const float *wy_host, int mode, cudaError_t *err);
void poisson_plan_destroy(PoissonPlan *p);
cudaError_t poisson_solve(PoissonPlan *p, const float *density, float *field_x, float *field_y, cudaStream_t s);
// The split-BF16 density operand the bin finalize can write directly (NULL in FP32 mode).
__nv_bfloat16 *poisson_split_input(PoissonPlan *p, int *ld);
// Fill the split-BF16 operand from a float density (when no bin finalize wrote it).
cudaError_t poisson_split_density(PoissonPlan *p, const float *density, cudaStream_t s);
size_t poisson_workspace_bytes(int nx, int ny);
// Loads the modules of the engine's kernels (each translation unit's), which the driver
// otherwise loads at their first launch.
void load_kernel_modules();
void load_module_b2b();
void load_module_bicgstab();
void load_module_poisson();
void load_module_poisson_tc();
void load_module_cell_order();
// Kernel launches one poisson_solve makes.
int poisson_launches(const PoissonPlan *p);
// The FP32 solves of n plans (mode 0) with their densities and fields fixed, as five
// launches in all: each GEMM stage over every plan's problems, the spectral step over every
// plan's spectrum (the fields equal poisson_solve's bit for bit).
struct PoissonGroup;
PoissonGroup *poisson_group_create(PoissonPlan *const *plans, const float *const *density, float *const *field_x, float *const *field_y, int n, cudaError_t *err);
void poisson_group_destroy(PoissonGroup *g);
cudaError_t poisson_group_solve(const PoissonGroup *g, cudaStream_t s);
int poisson_group_launches(const PoissonGroup *g);
int poisson_plan_mode(const PoissonPlan *p);

}  // namespace gpl
