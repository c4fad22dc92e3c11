// The device order of a region's cells, kept spatially coherent as the cells move.
//
// The trial kernels rely on a block's 256 consecutive cells lying close together: the
// scatter sums them in a shared-memory tile of the bins they cover, and the gradient kernel
// reads the same bins' fields. The order is a Z curve over the cells' positions when the
// design is uploaded; as the loop moves cells (most of all from a spread start, where the
// wirelength forces pull every cell toward its nets) a block's cells drift apart and the
// scatter falls back to smaller tiles and global atomics. When the scatter reports that, the
// engine sorts the region's cells again by the Hilbert index of their current density centres
// on a 1024 x 1024 grid over the region, stably, so the sort is deterministic: four LSD passes
// of 6-bit digits, each a per-tile digit histogram, one exclusive scan, and a stable scatter
// that ranks a tile's
// elements in input order (a warp's items round by round, lanes with the same digit ranked by
// a warp match). Then every per-cell array is gathered through the permutation and the pins'
// cell indices and cell-major slots are remapped. Nothing computed per cell depends on the
// order; only the cross-cell double sums see their terms in another order.
#include "common.cuh"
#include "engine_kernels.h"

namespace gpl {

namespace {

constexpr int kItems = 8;                       // elements per thread in a sort tile
constexpr int kTile = kThreads * kItems;        // 2048
constexpr int kDigits = 64;                     // 6-bit digits
constexpr int kWarps = kThreads / 32;

constexpr int kOrderBits = 10;                  // the Hilbert grid: 1024 x 1024 cells of the region
constexpr int kPasses = (2 * kOrderBits + 5) / 6;  // 6-bit digits of the 20-bit key (even: 4)
static_assert(kPasses % 2 == 0, "the sorted pairs end where they started");

// The distance of (x, y) along the Hilbert curve over a 2^kOrderBits square: any run of it
// lies in a compact patch, unlike a Z curve, whose runs jump across quadrant seams.
__device__ __forceinline__ uint32_t hilbert(uint32_t x, uint32_t y) {
  constexpr uint32_t n = 1u << kOrderBits;
  uint32_t d = 0;
  for (uint32_t s = n >> 1; s > 0; s >>= 1) {
    const uint32_t rx = (x & s) ? 1u : 0u, ry = (y & s) ? 1u : 0u;
    d += s * s * ((3u * rx) ^ ry);
    if (ry == 0) {
      if (rx == 1) {
        x = n - 1 - x;
        y = n - 1 - y;
      }
      const uint32_t t = x;
      x = y;
      y = t;
    }
  }
  return d;
}

}  // namespace

__global__ void k_order_keys(int32_t n, const int2 *__restrict__ dc, int32_t lx, int32_t ly, double tile_w, double tile_h, uint32_t *__restrict__ key, int32_t *__restrict__ idx) {
  const int32_t i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= n) return;
  const int2 c = dc[i];
  const double hi = (double)((1 << kOrderBits) - 1);
  const double fx = ((double)c.x - (double)lx) / tile_w, fy = ((double)c.y - (double)ly) / tile_h;
  key[i] = hilbert((uint32_t)fmin(fmax(fx, 0.0), hi), (uint32_t)fmin(fmax(fy, 0.0), hi));
  idx[i] = i;
}

// Per tile of kTile elements: how many hold each digit, at hist[digit * tiles + tile].
__global__ void __launch_bounds__(kThreads) k_order_hist(int32_t n, const uint32_t *__restrict__ key, int shift, int32_t tiles, int32_t *__restrict__ hist) {
  __shared__ int32_t h[kDigits];
  if (threadIdx.x < kDigits) h[threadIdx.x] = 0;
  __syncthreads();
  const int32_t base = blockIdx.x * kTile;
  for (int k = 0; k < kItems; k++) {
    const int32_t e = base + k * kThreads + threadIdx.x;
    if (e < n) atomicAdd(&h[(key[e] >> shift) & (kDigits - 1)], 1);
  }
  __syncthreads();
  if (threadIdx.x < kDigits) hist[threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of hist[0 .. m) in place (one block; each thread a contiguous run).
__global__ void __launch_bounds__(1024) k_order_scan(int32_t m, int32_t *__restrict__ hist) {
  __shared__ int32_t part[1024];
  const int32_t per = (m + 1023) / 1024;
  const int32_t b = threadIdx.x * per, e = min(m, b + per);
  int32_t s = 0;
  for (int32_t k = b; k < e; k++) s += hist[k];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const int32_t v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int32_t run = part[threadIdx.x] - s;
  for (int32_t k = b; k < e; k++) {
    const int32_t v = hist[k];
    hist[k] = run;
    run += v;
  }
}

// The stable scatter of one digit pass: a tile's elements keep their input order within a
// digit. Warp w ranks items [w * 256, w * 256 + 256) of the tile, 32 at a time in order.
__global__ void __launch_bounds__(kThreads) k_order_scatter(int32_t n, const uint32_t *__restrict__ key, const int32_t *__restrict__ idx, int shift, int32_t tiles, const int32_t *__restrict__ off,
                                                            uint32_t *__restrict__ key_out, int32_t *__restrict__ idx_out) {
  __shared__ int32_t wcount[kWarps][kDigits];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = threadIdx.x; k < kWarps * kDigits; k += kThreads) (&wcount[0][0])[k] = 0;
  __syncthreads();
  const int32_t base = blockIdx.x * kTile + warp * (32 * kItems);
  int32_t rank[kItems];
  uint32_t dig[kItems];
#pragma unroll
  for (int r = 0; r < kItems; r++) {
    const int32_t e = base + r * 32 + lane;
    const bool live = e < n;
    const uint32_t d = live ? (key[e] >> shift) & (kDigits - 1) : kDigits;  // kDigits: none
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int below = __popc(peers & ((1u << lane) - 1u));
    const int leader = __ffs(peers) - 1;
    int32_t start = 0;
    if (live && lane == leader) start = wcount[warp][d];
    start = __shfl_sync(0xffffffffu, start, leader);
    rank[r] = start + below;
    dig[r] = d;
    __syncwarp();
    if (live && lane == leader) wcount[warp][d] = start + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // each digit's warps in order: the warps before this one, per digit
  if (threadIdx.x < kDigits) {
    int32_t run = 0;
    for (int w = 0; w < kWarps; w++) {
      const int32_t c = wcount[w][threadIdx.x];
      wcount[w][threadIdx.x] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kItems; r++) {
    const int32_t e = base + r * 32 + lane;
    if (e >= n) continue;
    const uint32_t d = dig[r];
    const int32_t at = off[d * tiles + blockIdx.x] + wcount[warp][d] + rank[r];
    key_out[at] = key[e];
    idx_out[at] = idx[e];
  }
}

// The region's per-cell arrays through the permutation perm (new local index -> old): into
// the temporaries, and each cell's pin count.
__global__ void k_order_gather(int32_t n, const int32_t *__restrict__ perm, CellGather g) {
  const int32_t i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= n) return;
  const int32_t s = perm[i];
  g.dc_out[i] = g.dc[s];
  g.hx_out[i] = g.hx[s];
  g.hy_out[i] = g.hy[s];
  g.dscale_out[i] = g.dscale[s];
  g.area_out[i] = g.area[s];
  g.kind_out[i] = g.kind[s];
  if (g.locked) g.locked_out[i] = g.locked[s];
  g.pins_out[i] = g.pin_start[s + 1] - g.pin_start[s];
  g.inv[s] = i;
  g.order_out[i] = g.order[s];
#pragma unroll 1
  for (int k = 0; k < g.n_slots; k++) g.slot_out[k][i] = g.slot[k][s];
}

// The pins of the region's cells: new cell index and new cell-major slot.
__global__ void k_order_pins(int64_t n_pins, int32_t off, int32_t n, const int32_t *__restrict__ inv, const int64_t *__restrict__ old_start, const int64_t *__restrict__ new_start, int32_t *__restrict__ pin_cell,
                             int32_t *__restrict__ pin_slot) {
  const int64_t p = blockIdx.x * (int64_t)kThreads + threadIdx.x;
  if (p >= n_pins) return;
  const int32_t c = pin_cell[p] - off;
  if (c < 0 || c >= n) return;
  const int32_t i = inv[c];
  pin_cell[p] = off + i;
  if (pin_slot[p] >= 0) pin_slot[p] = (int32_t)(old_start[0] + new_start[i] + (pin_slot[p] - old_start[c]));
}

// The region's new pin starts: the old first slot plus the scanned counts (the start after the
// region's last cell is unchanged).
__global__ void k_order_starts(int32_t n, const int64_t *__restrict__ rel, int64_t *__restrict__ start) {
  const int32_t i = blockIdx.x * kThreads + threadIdx.x;
  if (i == 0 || i >= n) return;
  start[i] = start[0] + rel[i];
}

__global__ void k_iota(int32_t n, int32_t *__restrict__ a) {
  const int32_t i = blockIdx.x * kThreads + threadIdx.x;
  if (i < n) a[i] = i;
}

// The same key from float centres (the initial placement's solution vectors).
__global__ void k_order_keys_xy(int32_t n, const float *__restrict__ x, const float *__restrict__ y, double lx, double ly, double tile_w, double tile_h, uint32_t *__restrict__ key, int32_t *__restrict__ idx) {
  const int32_t i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= n) return;
  const double hi = (double)((1 << kOrderBits) - 1);
  const double fx = ((double)x[i] - lx) / tile_w, fy = ((double)y[i] - ly) / tile_h;
  // a NaN centre takes key 0 (fmax and fmin return the number)
  key[i] = hilbert((uint32_t)fmin(fmax(fx, 0.0), hi), (uint32_t)fmin(fmax(fy, 0.0), hi));
  idx[i] = i;
}

int order_tiles(int32_t n) { return (n + kTile - 1) / kTile; }

static cudaError_t order_passes(int32_t n, uint32_t *key0, int32_t *idx0, uint32_t *key1, int32_t *idx1, int32_t *hist, cudaStream_t s);

cudaError_t order_sort(int32_t n, const int2 *dc, int32_t lx, int32_t ly, double tile_w, double tile_h, uint32_t *key0, int32_t *idx0, uint32_t *key1, int32_t *idx1, int32_t *hist, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const unsigned eb = (unsigned)((n + kThreads - 1) / kThreads);
  k_order_keys<<<eb, kThreads, 0, s>>>(n, dc, lx, ly, tile_w, tile_h, key0, idx0);
  return order_passes(n, key0, idx0, key1, idx1, hist, s);
}

cudaError_t order_sort_xy(int32_t n, const float *x, const float *y, double lx, double ly, double tile_w, double tile_h, uint32_t *key0, int32_t *idx0, uint32_t *key1, int32_t *idx1, int32_t *hist, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const unsigned eb = (unsigned)((n + kThreads - 1) / kThreads);
  k_order_keys_xy<<<eb, kThreads, 0, s>>>(n, x, y, lx, ly, tile_w, tile_h, key0, idx0);
  return order_passes(n, key0, idx0, key1, idx1, hist, s);
}

static cudaError_t order_passes(int32_t n, uint32_t *key0, int32_t *idx0, uint32_t *key1, int32_t *idx1, int32_t *hist, cudaStream_t s) {
  const int32_t tiles = order_tiles(n);
  for (int pass = 0; pass < kPasses; pass++) {
    const int shift = 6 * pass;
    const bool odd = pass & 1;
    const uint32_t *ki = odd ? key1 : key0;
    const int32_t *ii = odd ? idx1 : idx0;
    uint32_t *ko = odd ? key0 : key1;
    int32_t *io = odd ? idx0 : idx1;
    k_order_hist<<<tiles, kThreads, 0, s>>>(n, ki, shift, tiles, hist);
    k_order_scan<<<1, 1024, 0, s>>>(kDigits * tiles, hist);
    k_order_scatter<<<tiles, kThreads, 0, s>>>(n, ki, ii, shift, tiles, hist, ko, io);
  }
  return cudaGetLastError();  // the sorted (key, old index) pairs are back in key0, idx0
}


// Loads this file's module (the driver loads a module at its first launch otherwise).
void load_module_cell_order() {
  cudaFuncAttributes a;
  cudaFuncGetAttributes(&a, k_order_scatter);
}

}  // namespace gpl
