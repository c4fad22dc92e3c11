// RUDY (`Rudy::calculate` / `visitNetTiles`, src/route_base.rs:191-253): each net's terminal
// box spreads hpwl * wire_width / area over the tiles it strictly overlaps, scaled by the share
// of each tile it covers, times 100; tiles x-major (x * cnt_y + y) from the die's lower-left,
// the last column and row stretched to the die's upper-right. One thread per net; the float
// deposits are atomic adds, so a tile's sum is the reference's up to the order of addition.
#include "common.cuh"
#include "rudy.h"

namespace gpl {

__device__ __forceinline__ void tile_rect(const RudyGrid &g, int32_t x, int32_t y, int32_t &l, int32_t &b, int32_t &r, int32_t &t) {
  l = g.lx + x * g.tile;
  b = g.ly + y * g.tile;
  r = l + g.tile + (x == g.cnt_x - 1 ? g.ux - g.cnt_x * g.tile : 0);
  t = b + g.tile + (y == g.cnt_y - 1 ? g.uy - g.cnt_y * g.tile : 0);
}

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
