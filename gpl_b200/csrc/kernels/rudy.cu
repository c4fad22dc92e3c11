// RUDY (`Rudy::calculate` / `visitNetTiles`, src/route_base.rs:191-253): each net's terminal
// box spreads hpwl * wire_width / area over the tiles it strictly overlaps, scaled by the share
// of each tile it covers, times 100; tiles x-major (x * cnt_y + y) from the die's lower-left,
// the last column and row stretched to the die's upper-right.
//
// The share is separable: the box covers ox(x) of column x's width and oy(y) of row y's
// height, so a net adds c fx(x) fy(y), c = 100 hpwl wire_width / area, fx = ox / width,
// fy = oy / height; fx is 1 on the columns strictly inside the box and partial only on its two
// edge columns, fy likewise. So a net's deposit is at most 3 x 3 rectangles of tiles with one
// value each (edge column or interior, by edge row or interior), added to a 2D difference array
// at the corners they share, and one inclusive 2D prefix sum gives every tile's demand: work in
// nets plus tiles instead of in the boxes' tile counts (a net spanning a fifth of a 1024 x 1024
// grid covers some 40,000 tiles). The differences and the sums are in double, so a tile's
// demand is the reference's float sum to within its own rounding.
#include "common.cuh"
#include "rudy.h"

namespace gpl {

__device__ __forceinline__ void tile_rect(const RudyGrid &g, int32_t x, int32_t y, int32_t &l, int32_t &b, int32_t &r, int32_t &t) {
  l = g.lx + x * g.tile;
  b = g.ly + y * g.tile;
  r = l + g.tile + (x == g.cnt_x - 1 ? g.ux - g.cnt_x * g.tile : 0);
  t = b + g.tile + (y == g.cnt_y - 1 ? g.uy - g.cnt_y * g.tile : 0);
}

// A net's columns (or rows) as up to three runs of one share each: the first, the interior
// (share 1), the last; n the count. share(i) of tile i is its overlap over its width.
struct Runs {
  int32_t a[3], b[3];
  double f[3];
  int n;
};
__device__ __forceinline__ void runs_of(int32_t lo, int32_t hi, int32_t g0, int32_t tile, int32_t cnt, int32_t gend, int32_t i0, int32_t i1, Runs &r) {
  r.n = 0;
  auto share = [&](int32_t i) {
    const int32_t t0 = g0 + i * tile, t1 = t0 + tile + (i == cnt - 1 ? gend - cnt * tile : 0);
    const int32_t o = min(hi, t1) - max(lo, t0);
    return o > 0 ? (double)o / (double)(t1 - t0) : 0.0;
  };
  if (i0 > i1) return;
  const double f0 = share(i0);
  if (f0 > 0.0) r.a[r.n] = r.b[r.n] = i0, r.f[r.n++] = f0;
  if (i1 - i0 >= 2) r.a[r.n] = i0 + 1, r.b[r.n] = i1 - 1, r.f[r.n++] = 1.0;
  if (i1 > i0) {
    const double f1 = share(i1);
    if (f1 > 0.0) r.a[r.n] = r.b[r.n] = i1, r.f[r.n++] = f1;
  }
}

// Each net's rectangles into the difference array diff[(cnt_x + 1) x (cnt_y + 1)].
__global__ void k_rudy_rects(RudyGrid g, int64_t n_nets, const int4 *__restrict__ boxes, double *__restrict__ diff) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n_nets) return;
  const int4 bx = boxes[k];
  const int32_t xl = bx.x, yl = bx.y, xh = bx.z, yh = bx.w;
  if (xl > xh || yl > yh) return;
  const int64_t area = (int64_t)(xh - xl) * (int64_t)(yh - yl);
  if (area == 0) return;
  const double c = 100.0 * (double)((xh - xl) + (yh - yl)) * (double)g.wire_width / (double)area;
  const int32_t min_x = max(0, (xl - g.lx) / g.tile), max_x = min(g.cnt_x - 1, (xh - g.lx) / g.tile);
  const int32_t min_y = max(0, (yl - g.ly) / g.tile), max_y = min(g.cnt_y - 1, (yh - g.ly) / g.tile);
  Runs rx, ry;
  runs_of(xl, xh, g.lx, g.tile, g.cnt_x, g.ux - g.lx, min_x, max_x, rx);
  runs_of(yl, yh, g.ly, g.tile, g.cnt_y, g.uy - g.ly, min_y, max_y, ry);
  // The runs are contiguous (run k spans [B_k, B_{k+1})), so the rectangles' corners fall on
  // the (n + 1) x (m + 1) breakpoints, where the difference of the piecewise-constant deposit is
  // c (f_i - f_{i-1}) (g_j - g_{j-1}) (f and g zero outside the runs): at most 16 adds a net
  // instead of four for each of up to nine rectangles.
  if (rx.n == 0 || ry.n == 0) return;
  const int64_t w = g.cnt_y + 1;
  int32_t px[4], py[4];
  double dfx[4], dfy[4];
  for (int i = 0; i <= rx.n; i++) {
    px[i] = i < rx.n ? rx.a[i] : rx.b[rx.n - 1] + 1;
    dfx[i] = (i < rx.n ? rx.f[i] : 0.0) - (i > 0 ? rx.f[i - 1] : 0.0);
  }
  for (int j = 0; j <= ry.n; j++) {
    py[j] = j < ry.n ? ry.a[j] : ry.b[ry.n - 1] + 1;
    dfy[j] = (j < ry.n ? ry.f[j] : 0.0) - (j > 0 ? ry.f[j - 1] : 0.0);
  }
  for (int i = 0; i <= rx.n; i++) {
    if (dfx[i] == 0.0) continue;
    for (int j = 0; j <= ry.n; j++)
      if (dfy[j] != 0.0) atomicAdd(&diff[(int64_t)px[i] * w + py[j]], c * dfx[i] * dfy[j]);
  }
}

// The prefix sum along y of every x row (a block per row, its threads over chunks of y).
__global__ void __launch_bounds__(256) k_prefix_y(int32_t rows, int32_t len, double *__restrict__ a) {
  __shared__ double part[256];
  double *row = a + (int64_t)blockIdx.x * len;
  const int per = (len + 255) / 256, b = threadIdx.x * per, e = min(len, b + per);
  double s = 0.0;
  for (int i = b; i < e; i++) s += row[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < 256; o <<= 1) {
    const double v = threadIdx.x >= o ? part[threadIdx.x - o] : 0.0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  double run = part[threadIdx.x] - s;
  for (int i = b; i < e; i++) {
    run += row[i];
    row[i] = run;
  }
}

// The prefix sum along x of every y column in kChunks chunks of rows: each thread (a column)
// sums its chunk, then adds the chunks before it and writes the running sums, as floats, into
// the demand (tiles x < cnt_x, y < cnt_y).
constexpr int kChunks = 32;
__global__ void k_prefix_x_chunks(int32_t rows, int32_t len, const double *__restrict__ a, double *__restrict__ chunk) {
  const int32_t y = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (y >= len) return;
  const int32_t per = (rows + kChunks - 1) / kChunks, x0 = c * per, x1 = min(rows, x0 + per);
  double s = 0.0;
  for (int32_t x = x0; x < x1; x++) s += a[(int64_t)x * len + y];
  chunk[(int64_t)c * len + y] = s;
}
__global__ void k_prefix_x_out(int32_t rows, int32_t len, int32_t cnt_x, int32_t cnt_y, const double *__restrict__ a, const double *__restrict__ chunk, float *__restrict__ demand) {
  const int32_t y = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (y >= len) return;
  double run = 0.0;
  for (int q = 0; q < c; q++) run += chunk[(int64_t)q * len + y];
  const int32_t per = (rows + kChunks - 1) / kChunks, x0 = c * per, x1 = min(rows, x0 + per);
  for (int32_t x = x0; x < x1; x++) {
    run += a[(int64_t)x * len + y];
    if (x < cnt_x && y < cnt_y) demand[(int64_t)x * cnt_y + y] = (float)run;
  }
}

// The reference's visit, one thread per net straight into the float demand (the form the
// difference array replaces; kept for the per-net visits' tests).
__global__ void k_rudy(RudyGrid g, int64_t n_nets, const int4 *__restrict__ boxes, float *__restrict__ demand) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n_nets) return;
  int4 bx = boxes[k];
  int32_t xl = bx.x, yl = bx.y, xh = bx.z, yh = bx.w;
  if (xl > xh || yl > yh) return;
  int64_t area = (int64_t)(xh - xl) * (int64_t)(yh - yl);
  if (area == 0) return;
  float hpwl = (float)((xh - xl) + (yh - yl));
  float nc = __fdiv_rn(__fmul_rn(hpwl, (float)g.wire_width), (float)area);
  int32_t min_x = max(0, (xl - g.lx) / g.tile), max_x = min(g.cnt_x - 1, (xh - g.lx) / g.tile);
  int32_t min_y = max(0, (yl - g.ly) / g.tile), max_y = min(g.cnt_y - 1, (yh - g.ly) / g.tile);
  for (int32_t x = min_x; x <= max_x; x++)
    for (int32_t y = min_y; y <= max_y; y++) {
      int32_t tl, tb, tr, tt;
      tile_rect(g, x, y, tl, tb, tr, tt);
      if (!(tr > xl && tl < xh && tt > yl && tb < yh)) continue;
      int64_t inter = (int64_t)(min(xh, tr) - max(xl, tl)) * (int64_t)(min(yh, tt) - max(yl, tb));
      int64_t tarea = (int64_t)(tr - tl) * (int64_t)(tt - tb);
      float ratio = __fdiv_rn((float)inter, (float)tarea);
      atomicAdd(&demand[(size_t)x * g.cnt_y + y], __fmul_rn(__fmul_rn(nc, ratio), 100.0f));
    }
}

// Congestion per tile (`getTileCongestion`, :257-264): demand / 100 / (1 - blockage).
__global__ void k_rudy_congestion(RudyGrid g, const float *__restrict__ demand, const float *__restrict__ blockage, float *__restrict__ cong) {
  int64_t n = (int64_t)g.cnt_x * g.cnt_y;
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float avail = __fsub_rn(1.0f, blockage[i]);
  cong[i] = avail <= 0.0f ? __int_as_float(0x7f800000) : __fdiv_rn(__fdiv_rn(demand[i], 100.0f), avail);
}

cudaError_t rudy_demand(const RudyGrid &g, int64_t n_nets, const int4 *boxes, float *demand, cudaStream_t s) {
  const int32_t rows = g.cnt_x + 1, len = g.cnt_y + 1;
  if (g.cnt_x <= 0 || g.cnt_y <= 0) return cudaSuccess;
  double *diff = nullptr, *chunk = nullptr;
  cudaError_t e = cudaMallocAsync((void **)&diff, (size_t)rows * len * sizeof(double), s);
  if (e == cudaSuccess) e = cudaMallocAsync((void **)&chunk, (size_t)kChunks * len * sizeof(double), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(diff, 0, (size_t)rows * len * sizeof(double), s);
  if (e == cudaSuccess) {
    if (n_nets > 0) k_rudy_rects<<<(unsigned)((n_nets + 255) / 256), 256, 0, s>>>(g, n_nets, boxes, diff);
    k_prefix_y<<<rows, 256, 0, s>>>(rows, len, diff);
    const dim3 grid((unsigned)((len + 255) / 256), kChunks);
    k_prefix_x_chunks<<<grid, 256, 0, s>>>(rows, len, diff, chunk);
    k_prefix_x_out<<<grid, 256, 0, s>>>(rows, len, g.cnt_x, g.cnt_y, diff, chunk, demand);
    e = cudaGetLastError();
  }
  if (diff) cudaFreeAsync(diff, s);
  if (chunk) cudaFreeAsync(chunk, s);
  return e;
}

cudaError_t rudy_demand_direct(const RudyGrid &g, int64_t n_nets, const int4 *boxes, float *demand, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(demand, 0, (size_t)g.cnt_x * g.cnt_y * sizeof(float), s);
  if (e != cudaSuccess) return e;
  if (n_nets > 0) k_rudy<<<(unsigned)((n_nets + 255) / 256), 256, 0, s>>>(g, n_nets, boxes, demand);
  return cudaGetLastError();
}

cudaError_t rudy_congestion(const RudyGrid &g, const float *demand, const float *blockage, float *cong, cudaStream_t s) {
  int64_t n = (int64_t)g.cnt_x * g.cnt_y;
  if (n > 0) k_rudy_congestion<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(g, demand, blockage, cong);
  return cudaGetLastError();
}

}  // namespace gpl
