// RUDY's tile grid and kernels (src/route_base.rs:130-265).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gpl {

struct RudyGrid {
  int32_t lx, ly, ux, uy;  // the die
  int32_t cnt_x, cnt_y, tile, wire_width;
};
// Every tile's demand (float, x-major) from the nets' boxes: the rectangles' difference array
// and its prefix sums, in double.
cudaError_t rudy_demand(const RudyGrid &g, int64_t n_nets, const int4 *boxes, float *demand, cudaStream_t s);
// The same by the reference's visit of each box's tiles, float atomics.
cudaError_t rudy_demand_direct(const RudyGrid &g, int64_t n_nets, const int4 *boxes, float *demand, cudaStream_t s);
cudaError_t rudy_congestion(const RudyGrid &g, const float *demand, const float *blockage, float *cong, cudaStream_t s);

}  // namespace gpl
