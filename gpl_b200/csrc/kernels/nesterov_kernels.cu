// The Nesterov trial's data-parallel stages (src/nesterov.rs:2139-2507, 2718-2772), one
// region's cells per launch. Cells are SoA in region-contiguous order; bins are x-major
// (index x*ny + y, the solver's layout, src/nesterov.rs:2283-2293).
//
// Compiled with --fmad=false: every float expression below is the reference's, in its order,
// and the per-cell results (coordinates, density boxes, the int64 bin addends, the density
// and WA gradients) are bit-identical to the reference's for identical inputs. Only the
// cross-cell sums (overflow, |gradient| sums, step-length distances) are taken in double and
// in a different order.
#include <cstdlib>
#include <string>

#include "common.cuh"
#include "engine_kernels.h"

namespace gpl {

// ---- cells: Nesterov step (nesterovUpdateCoordinates, :2718-2746) or a given point, then the
// density centre (setDensityCenterLocation, :2139-2153, truncated) and the bin scatter
// (updateBinsGCellDensityArea, :2218-2250): each (cell, bin) overlap times the density scale
// (times the bin's target density for a macro), truncated to int64 and added atomically —
// integer adds, so the accumulators equal the reference's in any order.
__device__ __forceinline__ float inside_axis(float c, float half, float lo, float hi) {
  float adj = c;
  if (__fsub_rn(c, half) < lo) adj = __fadd_rn(lo, half);
  if (__fadd_rn(c, half) > hi) adj = __fsub_rn(hi, half);
  return adj;
}

// The block's cells lie close together (the device orders each region's cells along a Z
// curve): the block first sums its addends in a shared-memory tile of the bins its cells
// cover, then adds each touched bin to HBM once. A block whose cells spread over more than
// kTileBins bins adds straight to HBM. Into the tile, a warp's lanes walk their cells' bins
// in step, and lanes that hit the same bin in a step pool their addends first (one shared
// atomic per distinct bin): after the initial placement many cells share a bin. The tile
// holds 32-bit sums when a block's sum for one bin cannot reach 2^32 (RegionArgs::narrow).
// Integer adds throughout: the same accumulators in any order.
constexpr int kTileBins = 2048;

// Exact conversions on the FMA and integer pipes for the small values the addends take (the
// conversion pipe is the scatter's busiest): an int in [0, 2^23) to float through the
// 2^23 exponent pattern; a float in [0, 2^23) truncated through a round-down add of 2^23
// (every float in [2^23, 2^24) is an integer). Larger values take the conversion pipe.
__device__ __forceinline__ float small_i2f(int32_t v) {
  return v < (1 << 23) ? __fsub_rn(__int_as_float(0x4B000000 | v), 8388608.0f) : (float)v;
}
__device__ __forceinline__ int64_t small_f2l_rz(float a) {
  return a < 8388608.0f ? (int64_t)(__float_as_int(__fadd_rd(a, 8388608.0f)) - 0x4B000000) : f2l_rz(a);
}

// One cell's addend to one bin (N4): the overlap area in float (the widths converted, then
// multiplied), times the cell's density scale (and the bin's target density for a macro),
// truncated to int64. Areas and widths are non-negative.
__device__ __forceinline__ int64_t cell_bin_addend(const RegionArgs &r, int32_t dlx, int32_t dux, int32_t dly, int32_t duy, int32_t x, int32_t y, float scale, uint8_t kind) {
  int32_t blx = r.bx[x], bux = r.bx[x + 1], bly = r.by[y], buy = r.by[y + 1];
  int32_t olx = dlx > blx ? dlx : blx, oux = dux < bux ? dux : bux;
  int32_t oly = dly > bly ? dly : bly, ouy = duy < buy ? duy : buy;
  float a = 0.0f;
  if (olx < oux && oly < ouy) a = __fmul_rn(small_i2f(oux - olx), small_i2f(ouy - oly));
  a = __fmul_rn(a, scale);
  if (kind == CELL_MACRO) a = __fmul_rn(a, r.target_density);
  return small_f2l_rz(a);
}

// The lanes' addends summed in a shared tile of th x tw bins (y fastest) from bin (tx0, ty0):
// slots [0, cap) for cells, [cap, 2 cap) for fillers, 32-bit when narrow; then every nonzero
// slot added to the HBM accumulators once. BLOCK: the block's threads share the tile; else
// the warp's lanes alone (their own slice of the block's tile). The warp's lanes walk their
// cells' bins in step (x outer, y inner), and lanes that hit the same bin in a step pool
// their addends first (one shared atomic per distinct bin). Integer adds throughout.
template <bool BLOCK>
__device__ __forceinline__ void tile_scatter(const RegionArgs &r, bool narrow, unsigned long long *s64, unsigned int *s32, unsigned long long *s_red, int cap, int32_t tx0, int32_t ty0, int32_t th,
                                             int32_t tw, bool any, int32_t x0, int32_t x1, int32_t y0, int32_t y1, int32_t dlx, int32_t dux, int32_t dly, int32_t duy, float scale, uint8_t kind) {
  const int lane = threadIdx.x & 31;
  const int start = BLOCK ? (int)threadIdx.x : lane, stride = BLOCK ? (int)blockDim.x : 32;
  const int nt = tw * th;
  {
    // zeroed 16 bytes a store (the slots this tile uses, rounded up to a multiple of 16 bytes)
    uint4 *c4 = reinterpret_cast<uint4 *>(narrow ? (void *)s32 : (void *)s64);
    uint4 *f4 = reinterpret_cast<uint4 *>(narrow ? (void *)(s32 + cap) : (void *)(s64 + cap));
    const int n4 = narrow ? (nt + 3) / 4 : (nt + 1) / 2;
    for (int k = start; k < n4; k += stride) c4[k] = f4[k] = make_uint4(0u, 0u, 0u, 0u);
  }
  if (BLOCK)
    __syncthreads();
  else
    __syncwarp();
  const int nb = any ? (x1 - x0) * (y1 - y0) : 0;
  const int rounds = __reduce_max_sync(0xffffffffu, nb);
  int32_t x = x0, y = y0;
  for (int q = 0; q < rounds; q++) {
    int key = -1;
    unsigned long long v = 0;
    if (q < nb) {
      int64_t a = cell_bin_addend(r, dlx, dux, dly, duy, x, y, scale, kind);
      if (a) {
        v = (unsigned long long)a;
        key = (((x - tx0) * th + (y - ty0)) << 1) | (kind == CELL_FILLER ? 1 : 0);
      }
      if (++y == y1) {
        y = y0;
        x++;
      }
    }
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    if (narrow) {
      // a block's sum for one bin stays below 2^32: each group of same-bin lanes adds its
      // addends with one warp reduction, its first lane one shared atomic
      const unsigned sum = __reduce_add_sync(peers, (unsigned)v);
      if (key >= 0 && lane == __ffs(peers) - 1) atomicAdd(&s32[(key & 1) * cap + (key >> 1)], sum);
    } else {
      s_red[threadIdx.x] = v;
      __syncwarp();
      if (key >= 0 && lane == __ffs(peers) - 1) {
        unsigned long long sum = 0;
        for (unsigned m = peers; m; m &= m - 1) sum += s_red[(threadIdx.x & ~31) + __ffs(m) - 1];
        atomicAdd(&s64[(key & 1) * cap + (key >> 1)], sum);
      }
      __syncwarp();
    }
  }
  if (BLOCK)
    __syncthreads();
  else
    __syncwarp();
  // the slot's bin (x, y) followed step by step (one division per thread, not per slot)
  const int dxs = stride / th, dys = stride - dxs * th;
  int xk = start / th, yk = start - xk * th;
  for (int k = start; k < nt; k += stride) {
    unsigned long long vi = narrow ? s32[k] : s64[k];
    unsigned long long vf = narrow ? s32[cap + k] : s64[cap + k];
    if (vi | vf) {
      const size_t g = (size_t)(tx0 + xk) * r.ny + (ty0 + yk);
      if (vi) atomicAdd((unsigned long long *)&r.acc_inst[g], vi);
      if (vf) atomicAdd((unsigned long long *)&r.acc_fill[g], vf);
    }
    xk += dxs;
    yk += dys;
    if (yk >= th) {
      yk -= th;
      xk++;
    }
  }
}

// Every addend straight to the HBM accumulators, the warp's lanes walking their cells' bins in
// step (x outer, y inner) and lanes that hit the same bin in a step pooling their addends first
// (one global atomic per distinct bin and step): the form for cells piled on few bins, where
// the atomics on one address would queue. Integer adds throughout.
__device__ __forceinline__ void pooled_scatter(const RegionArgs &r, bool narrow, unsigned long long *s_red, bool any, int32_t x0, int32_t x1, int32_t y0, int32_t y1, int32_t dlx, int32_t dux,
                                               int32_t dly, int32_t duy, float scale, uint8_t kind) {
  const int lane = threadIdx.x & 31;
  const int nb = any ? (x1 - x0) * (y1 - y0) : 0;
  const int rounds = __reduce_max_sync(0xffffffffu, nb);
  unsigned long long *acc = (unsigned long long *)(kind == CELL_FILLER ? r.acc_fill : r.acc_inst);
  int32_t x = x0, y = y0;
  for (int q = 0; q < rounds; q++) {
    long long key = -1;  // the accumulator slot, fillers' apart
    unsigned long long v = 0;
    size_t at = 0;
    if (q < nb) {
      const int64_t a = cell_bin_addend(r, dlx, dux, dly, duy, x, y, scale, kind);
      if (a) {
        v = (unsigned long long)a;
        at = (size_t)x * r.ny + y;
        key = ((long long)at << 1) | (kind == CELL_FILLER ? 1 : 0);
      }
      if (++y == y1) {
        y = y0;
        x++;
      }
    }
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const bool lead = key >= 0 && lane == __ffs(peers) - 1;
    if (narrow) {
      // a block's sum for one bin stays below 2^32, so a warp's does
      const unsigned sum = __reduce_add_sync(peers, (unsigned)v);
      if (lead) atomicAdd(&acc[at], (unsigned long long)sum);
    } else {
      s_red[threadIdx.x] = v;
      __syncwarp();
      if (lead) {
        unsigned long long sum = 0;
        for (unsigned m = peers; m; m &= m - 1) sum += s_red[(threadIdx.x & ~31) + __ffs(m) - 1];
        atomicAdd(&acc[at], sum);
      }
      __syncwarp();
    }
  }
}

// One block of a region's scatter: block `blk` of the region's cells.
__device__ __forceinline__ void place_cells_block(const RegionArgs &r, const CellArgs &c, int mode, float step, float coeff, const float2 *__restrict__ coords, int blk) {
  __shared__ __align__(16) unsigned long long s_tile[2 * kTileBins];  // cells then fillers; 32-bit when narrow
  __shared__ unsigned long long s_red[kThreads];
  __shared__ int s_box[5];  // the block's bin box, and its cells' (cell, bin) addends
  int i = blk * blockDim.x + threadIdx.x;
  const bool valid = i < r.n_cells;
  int32_t x0 = INT32_MAX, x1 = INT32_MIN, y0 = INT32_MAX, y1 = INT32_MIN;
  int32_t dlx = 0, dux = 0, dly = 0, duy = 0;
  float scale = 0.0f;
  uint8_t kind = 0;
  if (valid) {
    // the cell's constants first: after the stores below the compiler could not move these
    // loads ahead of them (the cell arrays are not marked restrict), each would be a round trip
    // of its own
    const int32_t hx = c.hx[i], hy = c.hy[i];
    scale = c.dscale[i];
    kind = c.kind[i];
    float2 p = make_float2(0.0f, 0.0f);
    if (mode == PLACE_AT) {
      p = coords[i];
    } else if (mode == PLACE_GIVEN) {
    } else {
      float2 cs = c.cur_slp[i];
      if (c.locked && c.locked[i]) {
        c.next[i] = c.cur[i];
        c.next_slp[i] = cs;
        p = cs;
      } else {
        float2 g = c.cur_slp_sum[i], cu = c.cur[i];
        float nx = __fadd_rn(cs.x, __fmul_rn(step, g.x));
        float ny = __fadd_rn(cs.y, __fmul_rn(step, g.y));
        float sx = __fadd_rn(nx, __fmul_rn(coeff, __fsub_rn(nx, cu.x)));
        float sy = __fadd_rn(ny, __fmul_rn(coeff, __fsub_rn(ny, cu.y)));
        const float fhx = (float)hx, fhy = (float)hy;
        float glx = (float)r.lx, gly = (float)r.ly, gux = (float)r.ux, guy = (float)r.uy;
        c.next[i] = make_float2(inside_axis(nx, fhx, glx, gux), inside_axis(ny, fhy, gly, guy));
        p = make_float2(inside_axis(sx, fhx, glx, gux), inside_axis(sy, fhy, gly, guy));
        c.next_slp[i] = p;
      }
    }
    int32_t cx, cy;
    if (mode == PLACE_GIVEN) {
      int2 d = c.dc[i];
      cx = d.x;
      cy = d.y;
    } else {
      cx = f2i_rz(p.x);
      cy = f2i_rz(p.y);
      c.dc[i] = make_int2(cx, cy);
    }
    dlx = cx - hx;
    dux = cx + hx;
    dly = cy - hy;
    duy = cy + hy;
    bin_span(dlx, dux, r.lx, r.size_x, r.inv_size_x, r.nx, x0, x1);
    bin_span(dly, duy, r.ly, r.size_y, r.inv_size_y, r.ny, y0, y1);
  }
  // the block's bin box
  if (threadIdx.x == 0) {
    s_box[0] = INT32_MAX;
    s_box[1] = INT32_MIN;
    s_box[2] = INT32_MAX;
    s_box[3] = INT32_MIN;
    s_box[4] = 0;
  }
  __syncthreads();
  const bool any = valid && x0 < x1 && y0 < y1;
  const int nb_cell = any ? (x1 - x0) * (y1 - y0) : 0;
  const int w_addends = __reduce_add_sync(0xffffffffu, nb_cell);
  int32_t wx0 = __reduce_min_sync(0xffffffffu, any ? x0 : INT32_MAX), wx1 = __reduce_max_sync(0xffffffffu, any ? x1 : INT32_MIN);
  int32_t wy0 = __reduce_min_sync(0xffffffffu, any ? y0 : INT32_MAX), wy1 = __reduce_max_sync(0xffffffffu, any ? y1 : INT32_MIN);
  const int lane = threadIdx.x & 31;
  if (lane == 0) {
    atomicMin(&s_box[0], wx0);
    atomicMax(&s_box[1], wx1);
    atomicMin(&s_box[2], wy0);
    atomicMax(&s_box[3], wy1);
    atomicAdd(&s_box[4], w_addends);
  }
  __syncthreads();
  // The block's cells share one tile when their bins fit it (32-bit slots hold twice as many
  // bins) and the tile is not mostly empty (at most twice as many slots as addends: a sparse
  // block's slots would cost more to clear and flush than its addends); else each warp takes a
  // slice of the tile for its own cells on the same terms, and a warp whose cells spread
  // wider adds straight to HBM.
  const bool narrow = r.narrow != 0;
  const int bcap = narrow ? 2 * kTileBins : kTileBins;
  const int64_t b_nt = (int64_t)(s_box[1] - s_box[0]) * (s_box[3] - s_box[2]);
  // (the other forms add straight to HBM; the spread count is the same in every form)
  const bool tile = s_box[1] > s_box[0] && s_box[3] > s_box[2] && b_nt <= bcap && b_nt <= 2 * (int64_t)s_box[4];
  unsigned int *t32 = reinterpret_cast<unsigned int *>(s_tile);
  const bool tiles = r.scatter_form == 0;
  if (tile && tiles) {
    tile_scatter<true>(r, narrow, s_tile, t32, s_red, bcap, s_box[0], s_box[2], s_box[3] - s_box[2], s_box[1] - s_box[0], any, x0, x1, y0, y1, dlx, dux, dly, duy, scale, kind);
    return;
  }
  if (!tile && threadIdx.x == 0 && r.spread) atomicAdd(r.spread, 1u);
  const int wcap = bcap / (kThreads / 32);
  const int64_t w_nt = (int64_t)(wx1 - wx0) * (wy1 - wy0);
  const bool wtile = wx1 > wx0 && wy1 > wy0 && w_nt <= wcap && w_nt <= 2 * (int64_t)w_addends;  // warp-uniform
  if (wtile && tiles) {
    const int w = threadIdx.x >> 5;
    tile_scatter<false>(r, narrow, s_tile + (size_t)w * 2 * wcap, t32 + (size_t)w * 2 * wcap, s_red, wcap, wx0, wy0, wy1 - wy0, wx1 - wx0, any, x0, x1, y0, y1, dlx, dux, dly, duy, scale, kind);
    return;
  }
  if (r.scatter_form == 2) {
    pooled_scatter(r, narrow, s_red, any, x0, x1, y0, y1, dlx, dux, dly, duy, scale, kind);
    return;
  }
  if (any) {
    unsigned long long *acc = (unsigned long long *)(kind == CELL_FILLER ? r.acc_fill : r.acc_inst);
    for (int32_t y = y0; y < y1; y++)
      for (int32_t x = x0; x < x1; x++) {
        int64_t v = cell_bin_addend(r, dlx, dux, dly, duy, x, y, scale, kind);
        if (v) atomicAdd(&acc[(size_t)x * r.ny + y], (unsigned long long)v);
      }
  }
}

__global__ void __launch_bounds__(kThreads) k_place_cells(RegionArgs r, CellArgs c, int mode, float step, float coeff, const float2 *__restrict__ coords) {
  place_cells_block(r, c, mode, step, coeff, coords, blockIdx.x);
}

// A packed launch's block: its region's entry (the last whose first block is at most this
// block) copied into shared memory.
__device__ __forceinline__ void packed_entry(const PackedRegion *__restrict__ t, int n, PackedRegion &e) {
  __shared__ int s_k;
  if (threadIdx.x == 0) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (t[mid].first <= (int)blockIdx.x) lo = mid; else hi = mid - 1;
    }
    s_k = lo;
  }
  __syncthreads();
  static_assert(sizeof(PackedRegion) % 8 == 0, "copied as 8-byte words");
  const unsigned long long *src = reinterpret_cast<const unsigned long long *>(t + s_k);
  unsigned long long *dst = reinterpret_cast<unsigned long long *>(&e);
  for (int k = threadIdx.x; k < (int)(sizeof(PackedRegion) / 8); k += blockDim.x) dst[k] = src[k];
  __syncthreads();
}

__global__ void __launch_bounds__(kThreads) k_place_packed(const PackedRegion *__restrict__ t, int n) {
  __shared__ PackedRegion e;
  packed_entry(t, n, e);
  place_cells_block(e.r, e.c, PLACE_NESTEROV, e.step, e.coeff, nullptr, (int)blockIdx.x - e.first);
}

// ---- bins: density and overflow (:2252-2262), accumulators cleared for the next scatter.
// Optionally the density split into bf16 hi/lo for the tensor-core solver. One block per x
// row (threads along y, kBinsPerThread bins each with their loads issued together), so no
// index is divided; block partials of the two overflow sums.
constexpr int kBinsPerThread = 4;

// One block (bin row x = blk) of a region's finalize over nblk rows.
__device__ __forceinline__ void bins_finalize_block(const RegionArgs &r, double *__restrict__ partials, __nv_bfloat16 *__restrict__ dens_split, int split_ld, unsigned int *ticket, double *out, int blk, int nblk) {
  __shared__ double sh[kThreads / 32];
  double o_sum = 0.0, ou_sum = 0.0;
  const int32_t x = blk;
  const size_t row = (size_t)x * r.ny;
  for (int32_t y0 = threadIdx.x; y0 < r.ny; y0 += blockDim.x * kBinsPerThread) {
    int64_t inst[kBinsPerThread], fill[kBinsPerThread];
    float fn[kBinsPerThread], fnu[kBinsPerThread], sc[kBinsPerThread];
#pragma unroll
    for (int q = 0; q < kBinsPerThread; q++) {
      int32_t y = y0 + q * blockDim.x;
      if (y < r.ny) {
        size_t k = row + y;
        inst[q] = r.acc_inst[k];
        fill[q] = r.acc_fill[k];
        fn[q] = r.non_place[k];
        fnu[q] = r.non_place_u[k];
        sc[q] = r.scaled[k];
      }
    }
#pragma unroll
    for (int q = 0; q < kBinsPerThread; q++) {
      int32_t y = y0 + q * blockDim.x;
      if (y >= r.ny) continue;
      size_t k = row + y;
      r.acc_inst[k] = 0;
      r.acc_fill[k] = 0;
      float fi = __ll2float_rn(inst[q]);
      float d = __fdiv_rn(__fadd_rn(__fadd_rn(fi, __ll2float_rn(fill[q])), fn[q]), sc[q]);
      r.density[k] = d;
      if (dens_split) {
        __nv_bfloat16 hi = __float2bfloat16_rn(d);
        __nv_bfloat16 lo = __float2bfloat16_rn(d - __bfloat162float(hi));
        dens_split[(size_t)x * split_ld + y] = hi;
        dens_split[(size_t)x * split_ld + r.ny + y] = lo;
      }
      float o = fmaxf(0.0f, __fsub_rn(__fadd_rn(fi, fn[q]), sc[q]));
      float ou = fmaxf(0.0f, __fsub_rn(__fadd_rn(fi, fnu[q]), sc[q]));
      o_sum += (double)o;
      ou_sum += (double)ou;
    }
  }
  double a = block_sum<kThreads>(o_sum, sh);
  double b = block_sum<kThreads>(ou_sum, sh);
  if (threadIdx.x == 0) {
    partials[2 * blk] = a;
    partials[2 * blk + 1] = b;
  }
  // the last block to finish sums the blocks' partials (the overflow sums) and reports the
  // scatter's spread blocks
  if (last_block_done(ticket, nblk)) {
    reduce_rows<kThreads>(partials, nblk, 2, out, sh);
    if (threadIdx.x == 0 && r.spread) {
      out[6] = (double)*r.spread;
      *r.spread = 0u;
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_bins_finalize(RegionArgs r, double *__restrict__ partials, __nv_bfloat16 *__restrict__ dens_split, int split_ld, unsigned int *ticket, double *out) {
  chain_enter();
  bins_finalize_block(r, partials, dens_split, split_ld, ticket, out, blockIdx.x, gridDim.x);
}

__global__ void __launch_bounds__(kThreads) k_finalize_packed(const PackedRegion *__restrict__ t, int n) {
  __shared__ PackedRegion e;
  packed_entry(t, n, e);
  bins_finalize_block(e.r, e.partials, e.dens_split, e.split_ld, e.ticket, e.out, (int)blockIdx.x - e.first, e.blocks);
}

// ---- WA wirelength (updateWireLengthForceWA :2325-2388 + getWireLengthGradientPinWA
// :2392-2414): one thread per net, nets in degree order so a warp's nets are alike; each
// net's sums over its pins in the net's order (the reference's float order), then each pin's
// force in double, times the net's weight. Pin position: its cell's density centre plus the
// pin's offset, or a fixed point for a pin with no cell.
__device__ __forceinline__ int2 pin_pos(const WaArgs &w, int64_t p) {
  int32_t cell = w.pin_cell ? w.pin_cell[p] : -1;
  int2 b = w.pin_base[p];
  if (cell >= 0) {
    int2 d = w.dc[cell];
    b.x += d.x;
    b.y += d.y;
  }
  return b;
}

__device__ __forceinline__ void wa_store(const WaArgs &w, int64_t p, float2 g) {
  int64_t at = w.pin_slot ? (int64_t)w.pin_slot[p] : p;
  if (at >= 0) w.pin_grad[at] = g;
}

// One pin's force from its net's sums (getWireLengthGradientPinWA :2392-2414): each quotient
// in double, rounded to float; gmin - gmax per axis, times the net weight.
__device__ __forceinline__ float wa_term_min(float s, float sx, float v, float c, float q) {
  double num = __dadd_rn(__dmul_rn((double)s, __dmul_rn((double)v, __dsub_rn(1.0, (double)__fmul_rn(c, q)))), (double)__fmul_rn(__fmul_rn(c, v), sx));
  return __double2float_rn(__ddiv_rn(num, (double)__fmul_rn(s, s)));
}
__device__ __forceinline__ float wa_term_max(float s, float sx, float v, float c, float q) {
  double num = __dsub_rn(__dmul_rn((double)s, __dmul_rn((double)v, __dadd_rn(1.0, (double)__fmul_rn(c, q)))), (double)__fmul_rn(__fmul_rn(c, v), sx));
  return __double2float_rn(__ddiv_rn(num, (double)__fmul_rn(s, s)));
}

__global__ void k_wa(WaArgs w, float cx, float cy) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= w.n_nets) return;
  int32_t n = w.net_order ? w.net_order[t] : t;
  int64_t b = w.net_start[n], e = w.net_start[n + 1];
  int32_t lx = INT32_MAX, ly = INT32_MAX, ux = INT32_MIN, uy = INT32_MIN;
  for (int64_t p = b; p < e; p++) {
    int2 q = pin_pos(w, p);
    lx = min(lx, q.x);
    ly = min(ly, q.y);
    ux = max(ux, q.x);
    uy = max(uy, q.y);
  }
  if (w.hpwl_out && ux >= lx) atomicAdd(w.hpwl_out, (unsigned long long)(((long long)ux - lx) + ((long long)uy - ly)));
  const float BAR = -300.0f;
  float s_minx = 0, s_xminx = 0, s_maxx = 0, s_xmaxx = 0, s_miny = 0, s_yminy = 0, s_maxy = 0, s_ymaxy = 0;
  for (int64_t p = b; p < e; p++) {
    int2 q = pin_pos(w, p);
    float emin_x = __fmul_rn((float)(lx - q.x), cx), emax_x = __fmul_rn((float)(q.x - ux), cx);
    float emin_y = __fmul_rn((float)(ly - q.y), cy), emax_y = __fmul_rn((float)(q.y - uy), cy);
    if (emin_x > BAR) {
      float v = fast_exp(emin_x);
      s_minx = __fadd_rn(s_minx, v);
      s_xminx = __fadd_rn(s_xminx, __fmul_rn((float)q.x, v));
    }
    if (emax_x > BAR) {
      float v = fast_exp(emax_x);
      s_maxx = __fadd_rn(s_maxx, v);
      s_xmaxx = __fadd_rn(s_xmaxx, __fmul_rn((float)q.x, v));
    }
    if (emin_y > BAR) {
      float v = fast_exp(emin_y);
      s_miny = __fadd_rn(s_miny, v);
      s_yminy = __fadd_rn(s_yminy, __fmul_rn((float)q.y, v));
    }
    if (emax_y > BAR) {
      float v = fast_exp(emax_y);
      s_maxy = __fadd_rn(s_maxy, v);
      s_ymaxy = __fadd_rn(s_ymaxy, __fmul_rn((float)q.y, v));
    }
  }
  float wt = w.net_weight ? w.net_weight[n] : 1.0f;
  for (int64_t p = b; p < e; p++) {
    int2 q = pin_pos(w, p);
    float qx = (float)q.x, qy = (float)q.y;
    float emin_x = __fmul_rn((float)(lx - q.x), cx), emax_x = __fmul_rn((float)(q.x - ux), cx);
    float emin_y = __fmul_rn((float)(ly - q.y), cy), emax_y = __fmul_rn((float)(q.y - uy), cy);
    float gmin_x = 0, gmax_x = 0, gmin_y = 0, gmax_y = 0;
    if (emin_x > BAR) {
      float v = fast_exp(emin_x);
      double num = __dadd_rn(__dmul_rn((double)s_minx, __dmul_rn((double)v, __dsub_rn(1.0, (double)__fmul_rn(cx, qx)))), (double)__fmul_rn(__fmul_rn(cx, v), s_xminx));
      gmin_x = __double2float_rn(__ddiv_rn(num, (double)__fmul_rn(s_minx, s_minx)));
    }
    if (emax_x > BAR) {
      float v = fast_exp(emax_x);
      double num = __dsub_rn(__dmul_rn((double)s_maxx, __dmul_rn((double)v, __dadd_rn(1.0, (double)__fmul_rn(cx, qx)))), (double)__fmul_rn(__fmul_rn(cx, v), s_xmaxx));
      gmax_x = __double2float_rn(__ddiv_rn(num, (double)__fmul_rn(s_maxx, s_maxx)));
    }
    if (emin_y > BAR) {
      float v = fast_exp(emin_y);
      double num = __dadd_rn(__dmul_rn((double)s_miny, __dmul_rn((double)v, __dsub_rn(1.0, (double)__fmul_rn(cy, qy)))), (double)__fmul_rn(__fmul_rn(cy, v), s_yminy));
      gmin_y = __double2float_rn(__ddiv_rn(num, (double)__fmul_rn(s_miny, s_miny)));
    }
    if (emax_y > BAR) {
      float v = fast_exp(emax_y);
      double num = __dsub_rn(__dmul_rn((double)s_maxy, __dmul_rn((double)v, __dadd_rn(1.0, (double)__fmul_rn(cy, qy)))), (double)__fmul_rn(__fmul_rn(cy, v), s_ymaxy));
      gmax_y = __double2float_rn(__ddiv_rn(num, (double)__fmul_rn(s_maxy, s_maxy)));
    }
    wa_store(w, p, make_float2(__fmul_rn(__fsub_rn(gmin_x, gmax_x), wt), __fmul_rn(__fsub_rn(gmin_y, gmax_y), wt)));
  }
}

// The same WA over a tile of consecutive nets, one block per tile, the pin work spread over
// the block's threads and each net's sums still taken by one thread in pin order:
//   1. pins' positions into shared memory (coalesced; one gather of the cell centre each);
//   2. a thread per net: the net's box, and each pin's net;
//   3. a thread per pin: the four exp terms (zero where the exponent is at or below -300,
//      which leaves a sum unchanged: the reference skips those terms), which of them the
//      reference takes (a mask beside the pin's net), and the position as floats;
//   4. a thread per net: the eight sums in pin order (the reference's float order);
//   5. a thread per pin: its force.
// The engine orders its nets by degree, so a tile's nets are alike and the thread-per-net
// phases run without divergence. The results are the thread-per-net kernel's bit for bit.
static_assert(kWaTileNets <= 256, "a pin's net index in the tile is kept in 8 bits");
static_assert(kWaTilePins <= 2 * kThreads, "a thread holds at most two of a tile's pins");

__global__ void __launch_bounds__(kThreads) k_wa_tiles(WaArgs w, float cx, float cy) {
  __shared__ int2 s_pos[kWaTilePins];        // phases 1-3: the position; 3-5: its floats' bits
  __shared__ float4 s_v[kWaTilePins];
  __shared__ uint16_t s_pnet[kWaTilePins];   // the pin's net in the tile | taken-terms mask << 8
  __shared__ int32_t s_nstart[kWaTileNets + 1];
  __shared__ int4 s_box[kWaTileNets];
  __shared__ float s_sum[8][kWaTileNets];
  // Persistent: the block walks tiles blockIdx.x, + gridDim.x, ...; the next tile's record and
  // its pins' cells load while this tile computes, so a tile starts with one round trip (the
  // cell centres) instead of three.
  const int ja = threadIdx.x, jb = threadIdx.x + kThreads;
  int tile = blockIdx.x;
  if (tile >= w.n_tiles) return;
  int4 t = w.tiles[tile];
  int32_t ca = -1, cb = -1;  // this tile's pins' cells
  if (w.pin_cell) {
    if (ja < t.w) ca = w.pin_cell[t.z + ja];
    if (jb < t.w) cb = w.pin_cell[t.z + jb];
  }
  for (;;) {
    const int32_t nn = t.y - t.x, np = t.w;
    const int64_t p0 = t.z;
    // the nets' starts and the pins' positions load together, and each pin's place in its
    // cell's list for the end
    for (int j = threadIdx.x; j <= nn; j += blockDim.x) s_nstart[j] = (int32_t)(w.net_start[t.x + j] - p0);
    int32_t slot_a = -1, slot_b = -1;
    if (ja < np) {
      const bool two = jb < np;
      slot_a = w.pin_slot ? w.pin_slot[p0 + ja] : (int32_t)(p0 + ja);
      if (two) slot_b = w.pin_slot ? w.pin_slot[p0 + jb] : (int32_t)(p0 + jb);
      int2 ba = w.pin_base[p0 + ja];
      int2 bb = two ? w.pin_base[p0 + jb] : make_int2(0, 0);
      const int2 da = ca >= 0 ? w.dc[ca] : make_int2(0, 0);
      const int2 db = cb >= 0 ? w.dc[cb] : make_int2(0, 0);
      s_pos[ja] = make_int2(ba.x + da.x, ba.y + da.y);
      if (two) s_pos[jb] = make_int2(bb.x + db.x, bb.y + db.y);
    }
    __syncthreads();
    const int next = tile + gridDim.x;
    const int4 tn = next < w.n_tiles ? w.tiles[next] : make_int4(0, 0, 0, 0);
    long long h = 0;  // the same pins' HPWL, for the iteration's report
    for (int j = threadIdx.x; j < nn; j += blockDim.x) {
      int32_t lx = INT32_MAX, ly = INT32_MAX, ux = INT32_MIN, uy = INT32_MIN;
      for (int32_t k = s_nstart[j]; k < s_nstart[j + 1]; k++) {
        int2 q = s_pos[k];
        lx = min(lx, q.x);
        ly = min(ly, q.y);
        ux = max(ux, q.x);
        uy = max(uy, q.y);
        s_pnet[k] = (uint16_t)j;
      }
      s_box[j] = make_int4(lx, ly, ux, uy);
      if (ux >= lx) h += ((long long)ux - lx) + ((long long)uy - ly);
    }
    if (w.hpwl_out) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) h += __shfl_down_sync(0xffffffffu, h, o);
      if ((threadIdx.x & 31) == 0 && h) atomicAdd(w.hpwl_out, (unsigned long long)h);
    }
    __syncthreads();
    const float BAR = -300.0f;
    for (int j = threadIdx.x; j < np; j += blockDim.x) {
      int2 q = s_pos[j];
      uint32_t n = s_pnet[j];
      int4 b = s_box[n];
      float emin_x = __fmul_rn((float)(b.x - q.x), cx), emax_x = __fmul_rn((float)(q.x - b.z), cx);
      float emin_y = __fmul_rn((float)(b.y - q.y), cy), emax_y = __fmul_rn((float)(q.y - b.w), cy);
      uint32_t m = (emin_x > BAR ? 1u : 0u) | (emax_x > BAR ? 2u : 0u) | (emin_y > BAR ? 4u : 0u) | (emax_y > BAR ? 8u : 0u);
      float4 v;
      v.x = (m & 1u) ? fast_exp(emin_x) : 0.0f;
      v.y = (m & 2u) ? fast_exp(emax_x) : 0.0f;
      v.z = (m & 4u) ? fast_exp(emin_y) : 0.0f;
      v.w = (m & 8u) ? fast_exp(emax_y) : 0.0f;
      s_v[j] = v;
      s_pnet[j] = (uint16_t)(n | (m << 8));
      s_pos[j] = make_int2(__float_as_int((float)q.x), __float_as_int((float)q.y));
    }
    __syncthreads();
    // the next tile's pins' cells (its record has arrived)
    int32_t can = -1, cbn = -1;
    if (w.pin_cell) {
      if (ja < tn.w) can = w.pin_cell[tn.z + ja];
      if (jb < tn.w) cbn = w.pin_cell[tn.z + jb];
    }
    for (int j = threadIdx.x; j < nn; j += blockDim.x) {
      float s_minx = 0, s_xminx = 0, s_maxx = 0, s_xmaxx = 0, s_miny = 0, s_yminy = 0, s_maxy = 0, s_ymaxy = 0;
      for (int32_t k = s_nstart[j]; k < s_nstart[j + 1]; k++) {
        int2 q = s_pos[k];
        float4 v = s_v[k];
        float qx = __int_as_float(q.x), qy = __int_as_float(q.y);
        s_minx = __fadd_rn(s_minx, v.x);
        s_xminx = __fadd_rn(s_xminx, __fmul_rn(qx, v.x));
        s_maxx = __fadd_rn(s_maxx, v.y);
        s_xmaxx = __fadd_rn(s_xmaxx, __fmul_rn(qx, v.y));
        s_miny = __fadd_rn(s_miny, v.z);
        s_yminy = __fadd_rn(s_yminy, __fmul_rn(qy, v.z));
        s_maxy = __fadd_rn(s_maxy, v.w);
        s_ymaxy = __fadd_rn(s_ymaxy, __fmul_rn(qy, v.w));
      }
      s_sum[0][j] = s_minx;
      s_sum[1][j] = s_xminx;
      s_sum[2][j] = s_maxx;
      s_sum[3][j] = s_xmaxx;
      s_sum[4][j] = s_miny;
      s_sum[5][j] = s_yminy;
      s_sum[6][j] = s_maxy;
      s_sum[7][j] = s_ymaxy;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < np; j += blockDim.x) {
      int2 q = s_pos[j];
      float4 v = s_v[j];
      uint32_t pn = s_pnet[j];
      uint32_t n = pn & 0xffu, m = pn >> 8;
      float qx = __int_as_float(q.x), qy = __int_as_float(q.y);
      float gmin_x = (m & 1u) ? wa_term_min(s_sum[0][n], s_sum[1][n], v.x, cx, qx) : 0.0f;
      float gmax_x = (m & 2u) ? wa_term_max(s_sum[2][n], s_sum[3][n], v.y, cx, qx) : 0.0f;
      float gmin_y = (m & 4u) ? wa_term_min(s_sum[4][n], s_sum[5][n], v.z, cy, qy) : 0.0f;
      float gmax_y = (m & 8u) ? wa_term_max(s_sum[6][n], s_sum[7][n], v.w, cy, qy) : 0.0f;
      float wt = w.net_weight ? w.net_weight[t.x + n] : 1.0f;
      const int32_t at = j == ja ? slot_a : slot_b;
      if (at >= 0) w.pin_grad[at] = make_float2(__fmul_rn(__fsub_rn(gmin_x, gmax_x), wt), __fmul_rn(__fsub_rn(gmin_y, gmax_y), wt));
    }
    if (next >= w.n_tiles) break;
    __syncthreads();  // every read of this tile's shared arrays ends before the next tile's writes
    tile = next;
    t = tn;
    ca = can;
    cb = cbn;
  }
}

// One net of degree D, a thread's own (the nets of the small ranges): its positions in
// registers, the box and the HPWL, the exp terms, the sums in pin order and each pin's force,
// the same operations in the same order as the tiles' phases.
template <int D>
__device__ __forceinline__ long long wa_net(const WaArgs &w, int32_t n, int64_t p0, float cx, float cy, bool forces) {
  int2 q[D];
#pragma unroll
  for (int k = 0; k < D; k++) q[k] = pin_pos(w, p0 + k);
  int32_t lx = INT32_MAX, ly = INT32_MAX, ux = INT32_MIN, uy = INT32_MIN;
#pragma unroll
  for (int k = 0; k < D; k++) {
    lx = min(lx, q[k].x);
    ly = min(ly, q[k].y);
    ux = max(ux, q[k].x);
    uy = max(uy, q[k].y);
  }
  const long long h = ((long long)ux - lx) + ((long long)uy - ly);  // ux >= lx: D >= 1 pins
  if (!forces) return h;
  const float BAR = -300.0f;
  float4 v[D];
  uint32_t m[D];
#pragma unroll
  for (int k = 0; k < D; k++) {
    float emin_x = __fmul_rn((float)(lx - q[k].x), cx), emax_x = __fmul_rn((float)(q[k].x - ux), cx);
    float emin_y = __fmul_rn((float)(ly - q[k].y), cy), emax_y = __fmul_rn((float)(q[k].y - uy), cy);
    m[k] = (emin_x > BAR ? 1u : 0u) | (emax_x > BAR ? 2u : 0u) | (emin_y > BAR ? 4u : 0u) | (emax_y > BAR ? 8u : 0u);
    v[k].x = (m[k] & 1u) ? fast_exp(emin_x) : 0.0f;
    v[k].y = (m[k] & 2u) ? fast_exp(emax_x) : 0.0f;
    v[k].z = (m[k] & 4u) ? fast_exp(emin_y) : 0.0f;
    v[k].w = (m[k] & 8u) ? fast_exp(emax_y) : 0.0f;
  }
  float s_minx = 0, s_xminx = 0, s_maxx = 0, s_xmaxx = 0, s_miny = 0, s_yminy = 0, s_maxy = 0, s_ymaxy = 0;
#pragma unroll
  for (int k = 0; k < D; k++) {
    float qx = (float)q[k].x, qy = (float)q[k].y;
    s_minx = __fadd_rn(s_minx, v[k].x);
    s_xminx = __fadd_rn(s_xminx, __fmul_rn(qx, v[k].x));
    s_maxx = __fadd_rn(s_maxx, v[k].y);
    s_xmaxx = __fadd_rn(s_xmaxx, __fmul_rn(qx, v[k].y));
    s_miny = __fadd_rn(s_miny, v[k].z);
    s_yminy = __fadd_rn(s_yminy, __fmul_rn(qy, v[k].z));
    s_maxy = __fadd_rn(s_maxy, v[k].w);
    s_ymaxy = __fadd_rn(s_ymaxy, __fmul_rn(qy, v[k].w));
  }
  const float wt = w.net_weight ? w.net_weight[n] : 1.0f;
#pragma unroll
  for (int k = 0; k < D; k++) {
    float qx = (float)q[k].x, qy = (float)q[k].y;
    float gmin_x = (m[k] & 1u) ? wa_term_min(s_minx, s_xminx, v[k].x, cx, qx) : 0.0f;
    float gmax_x = (m[k] & 2u) ? wa_term_max(s_maxx, s_xmaxx, v[k].y, cx, qx) : 0.0f;
    float gmin_y = (m[k] & 4u) ? wa_term_min(s_miny, s_yminy, v[k].z, cy, qy) : 0.0f;
    float gmax_y = (m[k] & 8u) ? wa_term_max(s_maxy, s_ymaxy, v[k].w, cy, qy) : 0.0f;
    wa_store(w, p0 + k, make_float2(__fmul_rn(__fsub_rn(gmin_x, gmax_x), wt), __fmul_rn(__fsub_rn(gmin_y, gmax_y), wt)));
  }
  return h;
}

__global__ void __launch_bounds__(kThreads) k_wa_small(WaArgs w, float cx, float cy, int forces) {
  // blocks of degree-2 nets, then degree 3, then degree 4 (the ranges read with constant
  // indices: the kernel's parameters stay out of local memory)
  const int nb0 = (w.small.count[0] + kThreads - 1) / kThreads, nb1 = (w.small.count[1] + kThreads - 1) / kThreads;
  const int b = blockIdx.x;
  const int k = b < nb0 ? 0 : b < nb0 + nb1 ? 1 : 2;
  const int t = (b - (k == 0 ? 0 : k == 1 ? nb0 : nb0 + nb1)) * kThreads + threadIdx.x;
  const int32_t count = k == 0 ? w.small.count[0] : k == 1 ? w.small.count[1] : w.small.count[2];
  const int32_t first = k == 0 ? w.small.first[0] : k == 1 ? w.small.first[1] : w.small.first[2];
  const int64_t pin0 = k == 0 ? w.small.pin0[0] : k == 1 ? w.small.pin0[1] : w.small.pin0[2];
  long long h = 0;
  if (t < count) {
    // a range's nets all have 2 + k pins, in net order: the net's first pin without a load
    const int32_t n = first + t;
    const int64_t p0 = pin0 + (int64_t)t * (2 + k);
    if (k == 0)
      h = wa_net<2>(w, n, p0, cx, cy, forces != 0);
    else if (k == 1)
      h = wa_net<3>(w, n, p0, cx, cy, forces != 0);
    else
      h = wa_net<4>(w, n, p0, cx, cy, forces != 0);
  }
  // the block's HPWL: warp sums, then one atomic per block (integer: any order)
  __shared__ long long s_h[kThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) h += __shfl_down_sync(0xffffffffu, h, o);
  if ((threadIdx.x & 31) == 0) s_h[threadIdx.x >> 5] = h;
  __syncthreads();
  if (threadIdx.x == 0 && w.hpwl_out) {
    long long sum = 0;
#pragma unroll
    for (int j = 0; j < kThreads / 32; j++) sum += s_h[j];
    if (sum) atomicAdd(w.hpwl_out, (unsigned long long)sum);
  }
}

// The same nets, a thread per net as wa_net, but with the pins' positions in shared memory and
// only the net's box and sums in registers across its passes: each pin's exp terms are formed
// again for its force instead of kept, for fewer registers (4 blocks per SM instead of 3) at a fifth more
// arithmetic. The same operations on the same values: wa_net's results bit for bit.
template <int D>
__device__ __forceinline__ long long wa_net_lean(const WaArgs &w, int32_t n, int64_t p0, float cx, float cy, bool forces, int2 *s_q) {
  // s_q: this thread's D positions, k-th at s_q[k * kThreads] (a warp's k-th positions in one
  // run of shared memory)
  int32_t lx = INT32_MAX, ly = INT32_MAX, ux = INT32_MIN, uy = INT32_MIN;
#pragma unroll
  for (int k = 0; k < D; k++) {
    const int2 q = pin_pos(w, p0 + k);
    s_q[k * kThreads] = q;
    lx = min(lx, q.x);
    ly = min(ly, q.y);
    ux = max(ux, q.x);
    uy = max(uy, q.y);
  }
  const long long h = ((long long)ux - lx) + ((long long)uy - ly);
  if (!forces) return h;
  const float BAR = -300.0f;
  float s_minx = 0, s_xminx = 0, s_maxx = 0, s_xmaxx = 0, s_miny = 0, s_yminy = 0, s_maxy = 0, s_ymaxy = 0;
#pragma unroll 1
  for (int k = 0; k < D; k++) {
    const int2 q = s_q[k * kThreads];
    const float qx = (float)q.x, qy = (float)q.y;
    const float emin_x = __fmul_rn((float)(lx - q.x), cx), emax_x = __fmul_rn((float)(q.x - ux), cx);
    const float emin_y = __fmul_rn((float)(ly - q.y), cy), emax_y = __fmul_rn((float)(q.y - uy), cy);
    const float vx = emin_x > BAR ? fast_exp(emin_x) : 0.0f, vy = emax_x > BAR ? fast_exp(emax_x) : 0.0f;
    const float vz = emin_y > BAR ? fast_exp(emin_y) : 0.0f, vw = emax_y > BAR ? fast_exp(emax_y) : 0.0f;
    s_minx = __fadd_rn(s_minx, vx);
    s_xminx = __fadd_rn(s_xminx, __fmul_rn(qx, vx));
    s_maxx = __fadd_rn(s_maxx, vy);
    s_xmaxx = __fadd_rn(s_xmaxx, __fmul_rn(qx, vy));
    s_miny = __fadd_rn(s_miny, vz);
    s_yminy = __fadd_rn(s_yminy, __fmul_rn(qy, vz));
    s_maxy = __fadd_rn(s_maxy, vw);
    s_ymaxy = __fadd_rn(s_ymaxy, __fmul_rn(qy, vw));
  }
  const float wt = w.net_weight ? w.net_weight[n] : 1.0f;
#pragma unroll 1
  for (int k = 0; k < D; k++) {
    const int2 q = s_q[k * kThreads];
    const float qx = (float)q.x, qy = (float)q.y;
    const float emin_x = __fmul_rn((float)(lx - q.x), cx), emax_x = __fmul_rn((float)(q.x - ux), cx);
    const float emin_y = __fmul_rn((float)(ly - q.y), cy), emax_y = __fmul_rn((float)(q.y - uy), cy);
    float gmin_x = 0.0f, gmax_x = 0.0f, gmin_y = 0.0f, gmax_y = 0.0f;
    if (emin_x > BAR) gmin_x = wa_term_min(s_minx, s_xminx, fast_exp(emin_x), cx, qx);
    if (emax_x > BAR) gmax_x = wa_term_max(s_maxx, s_xmaxx, fast_exp(emax_x), cx, qx);
    if (emin_y > BAR) gmin_y = wa_term_min(s_miny, s_yminy, fast_exp(emin_y), cy, qy);
    if (emax_y > BAR) gmax_y = wa_term_max(s_maxy, s_ymaxy, fast_exp(emax_y), cy, qy);
    wa_store(w, p0 + k, make_float2(__fmul_rn(__fsub_rn(gmin_x, gmax_x), wt), __fmul_rn(__fsub_rn(gmin_y, gmax_y), wt)));
  }
  return h;
}

__global__ void __launch_bounds__(kThreads, 4) k_wa_lean(WaArgs w, float cx, float cy, int forces) {
  const int nb0 = (w.small.count[0] + kThreads - 1) / kThreads, nb1 = (w.small.count[1] + kThreads - 1) / kThreads;
  const int b = blockIdx.x;
  const int k = b < nb0 ? 0 : b < nb0 + nb1 ? 1 : 2;
  const int t = (b - (k == 0 ? 0 : k == 1 ? nb0 : nb0 + nb1)) * kThreads + threadIdx.x;
  const int32_t count = k == 0 ? w.small.count[0] : k == 1 ? w.small.count[1] : w.small.count[2];
  const int32_t first = k == 0 ? w.small.first[0] : k == 1 ? w.small.first[1] : w.small.first[2];
  const int64_t pin0 = k == 0 ? w.small.pin0[0] : k == 1 ? w.small.pin0[1] : w.small.pin0[2];
  __shared__ int2 s_q[4 * kThreads];
  long long h = 0;
  if (t < count) {
    const int32_t n = first + t;
    const int64_t p0 = pin0 + (int64_t)t * (2 + k);
    if (k == 0)
      h = wa_net_lean<2>(w, n, p0, cx, cy, forces != 0, s_q + threadIdx.x);
    else if (k == 1)
      h = wa_net_lean<3>(w, n, p0, cx, cy, forces != 0, s_q + threadIdx.x);
    else
      h = wa_net_lean<4>(w, n, p0, cx, cy, forces != 0, s_q + threadIdx.x);
  }
  __shared__ long long s_h[kThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) h += __shfl_down_sync(0xffffffffu, h, o);
  if ((threadIdx.x & 31) == 0) s_h[threadIdx.x >> 5] = h;
  __syncthreads();
  if (threadIdx.x == 0 && w.hpwl_out) {
    long long sum = 0;
#pragma unroll
    for (int j = 0; j < kThreads / 32; j++) sum += s_h[j];
    if (sum) atomicAdd(w.hpwl_out, (unsigned long long)sum);
  }
}

// The same nets of degree D = 2, 3, 4, a lane per pin: a warp holds 32 / D nets, each net's D
// lanes consecutive, so the pins' loads are coalesced and every lane waits on one chain (its
// pin's cell, then that cell's centre) instead of D. The net's positions and exp terms reach
// its lanes by shuffles; every lane of a net forms the net's box and its eight sums in pin
// order itself (the reference's float order), then its own pin's force. Registers stay low
// enough for 6 blocks per SM. Results are k_wa_small's bit for bit.
template <int D>
__device__ __forceinline__ long long wa_lane(const WaArgs &w, int32_t first, int32_t count, int64_t pin0, int blk, float cx, float cy, bool forces) {
  constexpr int G = 32 / D;  // nets per warp
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane / D, j = lane - g * D;
  const int32_t t = (blk * (kThreads / 32) + warp) * G + g;  // the net's index in its range
  const bool active = g < G && t < count;
  const int64_t p = pin0 + (int64_t)t * D + j;
  int2 q = make_int2(0, 0);
  int32_t at = -1;
  if (active) {
    q = pin_pos(w, p);
    at = w.pin_slot ? w.pin_slot[p] : (int32_t)p;
  }
  const int base = g * D;  // the net's first lane (lanes past the last group read lane 0..: unused)
  int32_t X[D], Y[D];
#pragma unroll
  for (int i = 0; i < D; i++) {
    X[i] = __shfl_sync(0xffffffffu, q.x, (base + i) & 31);
    Y[i] = __shfl_sync(0xffffffffu, q.y, (base + i) & 31);
  }
  int32_t lx = X[0], ly = Y[0], ux = X[0], uy = Y[0];
#pragma unroll
  for (int i = 1; i < D; i++) {
    lx = min(lx, X[i]);
    ly = min(ly, Y[i]);
    ux = max(ux, X[i]);
    uy = max(uy, Y[i]);
  }
  const long long h = active && j == 0 ? ((long long)ux - lx) + ((long long)uy - ly) : 0;
  if (!forces) return h;
  const float BAR = -300.0f;
  float emin_x = __fmul_rn((float)(lx - q.x), cx), emax_x = __fmul_rn((float)(q.x - ux), cx);
  float emin_y = __fmul_rn((float)(ly - q.y), cy), emax_y = __fmul_rn((float)(q.y - uy), cy);
  const uint32_t m = (emin_x > BAR ? 1u : 0u) | (emax_x > BAR ? 2u : 0u) | (emin_y > BAR ? 4u : 0u) | (emax_y > BAR ? 8u : 0u);
  float4 v;
  v.x = (m & 1u) ? fast_exp(emin_x) : 0.0f;
  v.y = (m & 2u) ? fast_exp(emax_x) : 0.0f;
  v.z = (m & 4u) ? fast_exp(emin_y) : 0.0f;
  v.w = (m & 8u) ? fast_exp(emax_y) : 0.0f;
  float s_minx = 0, s_xminx = 0, s_maxx = 0, s_xmaxx = 0, s_miny = 0, s_yminy = 0, s_maxy = 0, s_ymaxy = 0;
#pragma unroll
  for (int i = 0; i < D; i++) {
    const int src = (base + i) & 31;
    const float vx = __shfl_sync(0xffffffffu, v.x, src), vy = __shfl_sync(0xffffffffu, v.y, src);
    const float vz = __shfl_sync(0xffffffffu, v.z, src), vw = __shfl_sync(0xffffffffu, v.w, src);
    const float qx = (float)X[i], qy = (float)Y[i];
    s_minx = __fadd_rn(s_minx, vx);
    s_xminx = __fadd_rn(s_xminx, __fmul_rn(qx, vx));
    s_maxx = __fadd_rn(s_maxx, vy);
    s_xmaxx = __fadd_rn(s_xmaxx, __fmul_rn(qx, vy));
    s_miny = __fadd_rn(s_miny, vz);
    s_yminy = __fadd_rn(s_yminy, __fmul_rn(qy, vz));
    s_maxy = __fadd_rn(s_maxy, vw);
    s_ymaxy = __fadd_rn(s_ymaxy, __fmul_rn(qy, vw));
  }
  if (active) {
    const float qx = (float)q.x, qy = (float)q.y;
    const float wt = w.net_weight ? w.net_weight[first + t] : 1.0f;
    float gmin_x = (m & 1u) ? wa_term_min(s_minx, s_xminx, v.x, cx, qx) : 0.0f;
    float gmax_x = (m & 2u) ? wa_term_max(s_maxx, s_xmaxx, v.y, cx, qx) : 0.0f;
    float gmin_y = (m & 4u) ? wa_term_min(s_miny, s_yminy, v.z, cy, qy) : 0.0f;
    float gmax_y = (m & 8u) ? wa_term_max(s_maxy, s_ymaxy, v.w, cy, qy) : 0.0f;
    if (at >= 0) w.pin_grad[at] = make_float2(__fmul_rn(__fsub_rn(gmin_x, gmax_x), wt), __fmul_rn(__fsub_rn(gmin_y, gmax_y), wt));
  }
  return h;
}

// Blocks per degree range of k_wa_pins: a block holds kThreads / 32 warps of 32 / D nets.
__host__ __device__ __forceinline__ int wa_pins_range_blocks(int32_t count, int d) { return (int)((count + (kThreads / 32) * (32 / d) - 1) / ((kThreads / 32) * (32 / d))); }

__global__ void __launch_bounds__(kThreads, 6) k_wa_pins(WaArgs w, float cx, float cy, int forces) {
  const int nb0 = wa_pins_range_blocks(w.small.count[0], 2), nb1 = wa_pins_range_blocks(w.small.count[1], 3);
  const int b = blockIdx.x;
  long long h;
  if (b < nb0)
    h = wa_lane<2>(w, w.small.first[0], w.small.count[0], w.small.pin0[0], b, cx, cy, forces != 0);
  else if (b < nb0 + nb1)
    h = wa_lane<3>(w, w.small.first[1], w.small.count[1], w.small.pin0[1], b - nb0, cx, cy, forces != 0);
  else
    h = wa_lane<4>(w, w.small.first[2], w.small.count[2], w.small.pin0[2], b - nb0 - nb1, cx, cy, forces != 0);
  __shared__ long long s_h[kThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) h += __shfl_down_sync(0xffffffffu, h, o);
  if ((threadIdx.x & 31) == 0) s_h[threadIdx.x >> 5] = h;
  __syncthreads();
  if (threadIdx.x == 0 && w.hpwl_out) {
    long long sum = 0;
#pragma unroll
    for (int j = 0; j < kThreads / 32; j++) sum += s_h[j];
    if (sum) atomicAdd(w.hpwl_out, (unsigned long long)sum);
  }
}

int wa_pins_blocks(const WaSmall &s) { return wa_pins_range_blocks(s.count[0], 2) + wa_pins_range_blocks(s.count[1], 3) + wa_pins_range_blocks(s.count[2], 4); }

// GPL_WA_SMALL picks the degree-2..4 nets' kernel: "nets" k_wa_small, "pins" k_wa_pins, else
// (the default) k_wa_lean; all three give the same forces and HPWL.
static int wa_small_form() {
  const char *f = std::getenv("GPL_WA_SMALL");
  if (f && std::string(f) == "nets") return 1;
  if (f && std::string(f) == "pins") return 2;
  return 0;
}

void launch_wa_small(const WaArgs &w, float cx, float cy, int forces, cudaStream_t s, int form) {
  if (form < 0) form = wa_small_form();
  if (form == 2) {
    if (const int nb = wa_pins_blocks(w.small)) k_wa_pins<<<nb, kThreads, 0, s>>>(w, cx, cy, forces);
  } else if (const int nb = wa_small_blocks(w.small)) {
    if (form == 1)
      k_wa_small<<<nb, kThreads, 0, s>>>(w, cx, cy, forces);
    else
      k_wa_lean<<<nb, kThreads, 0, s>>>(w, cx, cy, forces);
  }
}

// The WA tiles' launch: a persistent grid of as many blocks as fit on the device at once.
void launch_wa_tiles(const WaArgs &w, float cx, float cy, cudaStream_t s) {
  if (w.n_tiles <= 0) return;
  static int resident = 0;  // blocks per device at once (the devices of a run are alike)
  if (!resident) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_wa_tiles, kThreads, 0);
    resident = std::max(1, sms * std::max(per, 1));
  }
  k_wa_tiles<<<std::min(w.n_tiles, resident), kThreads, 0, s>>>(w, cx, cy);
}

// ---- cells: updateGradients (:2455-2507): the WA force over the cell's pins in its order,
// the density force over its bins (x outer, y inner), the preconditioned sum; block partials
// of |wl|, |density| and the two step-length distances (getDistance :319-330):
// |a1 - b1|^2 and |out - b2|^2.
// A block's cells are consecutive, so their pins' forces (cell-major) are one run: staged in
// shared memory with coalesced loads when the run fits kGradPinTile, then each cell sums its
// own in order. A cell over at most 2 x 2 bins loads its bins' boundaries and fields before
// the ordered sums; larger cells walk their bins.
constexpr int kGradPinTile = 2048;

// One block (cells blk * 256 ..) of a region's gradient update over nblk blocks.
__device__ __forceinline__ void gradients_block(const RegionArgs &r, const CellArgs &c, const float2 *__restrict__ pin_grad, float penalty, float2 *__restrict__ out_sum, const float2 *__restrict__ a1, const float2 *__restrict__ b1,
                                                const float2 *__restrict__ b2, double *__restrict__ partials, unsigned int *ticket, double *out, int blk, int nblk) {
  __shared__ double4 sh[kThreads / 32];
  __shared__ float2 s_pg[kGradPinTile];
  const int i0 = blk * blockDim.x;
  const int i = i0 + threadIdx.x;
  const int i1 = min(r.n_cells, i0 + (int)blockDim.x);
  const int64_t p0 = c.pin_start[i0], p1 = c.pin_start[i1];
  const bool staged = p1 - p0 <= kGradPinTile;
  if (staged)
    for (int k = threadIdx.x; k < (int)(p1 - p0); k += blockDim.x) s_pg[k] = pin_grad[p0 + k];
  __syncthreads();
  double s_wl = 0, s_den = 0, s_d1 = 0, s_d2 = 0;
  if (i < r.n_cells) {
    const int64_t pb = c.pin_start[i], pe = c.pin_start[i + 1];
    float wlx = 0.0f, wly = 0.0f;
    if (staged) {
      for (int k = (int)(pb - p0); k < (int)(pe - p0); k++) {
        float2 t = s_pg[k];
        wlx = __fadd_rn(wlx, t.x);
        wly = __fadd_rn(wly, t.y);
      }
    } else {
      for (int64_t k = pb; k < pe; k++) {
        float2 t = pin_grad[k];
        wlx = __fadd_rn(wlx, t.x);
        wly = __fadd_rn(wly, t.y);
      }
    }
    int2 d = c.dc[i];
    int32_t cx = d.x, cy = d.y, hx = c.hx[i], hy = c.hy[i];
    int32_t dlx = cx - hx, dux = cx + hx, dly = cy - hy, duy = cy + hy;
    int32_t x0, x1, y0, y1;
    bin_span(dlx, dux, r.lx, r.size_x, r.inv_size_x, r.nx, x0, x1);
    bin_span(dly, duy, r.ly, r.size_y, r.inv_size_y, r.ny, y0, y1);
    float scale = c.dscale[i];
    float fx = 0.0f, fy = 0.0f;
    // one bin's term in the reference's order: overlap area (float), times the scale, times
    // the field, added to the running sums
    auto term = [&](int32_t blx, int32_t bux, int32_t bly, int32_t buy, float ex, float ey) {
      int32_t olx = dlx > blx ? dlx : blx, oux = dux < bux ? dux : bux;
      int32_t oly = dly > bly ? dly : bly, ouy = duy < buy ? duy : buy;
      float a = 0.0f;
      if (olx < oux && oly < ouy) a = __fmul_rn((float)(oux - olx), (float)(ouy - oly));
      a = __fmul_rn(a, scale);
      fx = __fadd_rn(fx, __fmul_rn(a, ex));
      fy = __fadd_rn(fy, __fmul_rn(a, ey));
    };
    if (x1 - x0 <= 2 && y1 - y0 <= 2 && x1 > x0 && y1 > y0) {
      // every load first (the boundaries and up to four bins' fields), then the sums in order
      const int xb = min(x0 + 1, x1 - 1), yb = min(y0 + 1, y1 - 1);
      const int32_t bx0 = r.bx[x0], bx1 = r.bx[x0 + 1], bx2 = r.bx[xb + 1];
      const int32_t by0 = r.by[y0], by1 = r.by[y0 + 1], by2 = r.by[yb + 1];
      const size_t k00 = (size_t)x0 * r.ny + y0, k01 = (size_t)x0 * r.ny + yb, k10 = (size_t)xb * r.ny + y0, k11 = (size_t)xb * r.ny + yb;
      const float e00x = r.field_x[k00], e00y = r.field_y[k00], e01x = r.field_x[k01], e01y = r.field_y[k01];
      const float e10x = r.field_x[k10], e10y = r.field_y[k10], e11x = r.field_x[k11], e11y = r.field_y[k11];
      term(bx0, bx1, by0, by1, e00x, e00y);
      if (y1 - y0 == 2) term(bx0, bx1, by1, by2, e01x, e01y);
      if (x1 - x0 == 2) {
        term(bx1, bx2, by0, by1, e10x, e10y);
        if (y1 - y0 == 2) term(bx1, bx2, by1, by2, e11x, e11y);
      }
    } else {
      for (int32_t x = x0; x < x1; x++) {
        int32_t blx = r.bx[x], bux = r.bx[x + 1];
        for (int32_t y = y0; y < y1; y++) {
          size_t k = (size_t)x * r.ny + y;
          term(blx, bux, r.by[y], r.by[y + 1], r.field_x[k], r.field_y[k]);
        }
      }
    }
    float sx = __fadd_rn(wlx, __fmul_rn(penalty, fx));
    float sy = __fadd_rn(wly, __fmul_rn(penalty, fy));
    float wl_pre = (float)(pe - pb);
    float pre = fmaxf(__fadd_rn(wl_pre, __fmul_rn(penalty, c.area[i])), 1.0f);
    sx = __fdiv_rn(sx, pre);
    sy = __fdiv_rn(sy, pre);
    out_sum[i] = make_float2(sx, sy);
    s_wl = (double)fabsf(wlx) + (double)fabsf(wly);
    s_den = (double)fabsf(fx) + (double)fabsf(fy);
    if (a1) {
      float2 p = a1[i], q = b1[i];
      float dx = __fsub_rn(p.x, q.x), dy = __fsub_rn(p.y, q.y);
      s_d1 = (double)__fmul_rn(dx, dx) + (double)__fmul_rn(dy, dy);
    }
    if (b2) {
      float2 q = b2[i];
      float dx = __fsub_rn(sx, q.x), dy = __fsub_rn(sy, q.y);
      s_d2 = (double)__fmul_rn(dx, dx) + (double)__fmul_rn(dy, dy);
    }
  }
  double4 v = block_sum4<kThreads>(make_double4(s_wl, s_den, s_d1, s_d2), sh);
  if (threadIdx.x == 0) {
    partials[4 * blk + 0] = v.x;
    partials[4 * blk + 1] = v.y;
    partials[4 * blk + 2] = v.z;
    partials[4 * blk + 3] = v.w;
  }
  // the last block to finish sums the blocks' partials (|wl|, |density|, the two distances)
  __shared__ double shr[kThreads / 32];
  if (last_block_done(ticket, nblk)) reduce_rows<kThreads>(partials, nblk, 4, out, shr);
}

__global__ void __launch_bounds__(kThreads, 6) k_gradients(RegionArgs r, CellArgs c, const float2 *__restrict__ pin_grad, float penalty, float2 *__restrict__ out_sum, const float2 *__restrict__ a1, const float2 *__restrict__ b1, const float2 *__restrict__ b2, double *__restrict__ partials, unsigned int *ticket, double *out) {
  chain_enter();
  gradients_block(r, c, pin_grad, penalty, out_sum, a1, b1, b2, partials, ticket, out, blockIdx.x, gridDim.x);
}

__global__ void __launch_bounds__(kThreads, 6) k_gradients_packed(const PackedRegion *__restrict__ t, int n) {
  __shared__ PackedRegion e;
  packed_entry(t, n, e);
  gradients_block(e.r, e.c, e.pin_grad, e.penalty, e.out_sum, e.a1, e.b1, e.b2, e.partials, e.ticket, e.out, (int)blockIdx.x - e.first, e.blocks);
}

// ---- updateInitialPrevSLPCoordi (:2583-2595): a back-step along the current gradient.
__global__ void k_prev_slp(RegionArgs r, CellArgs c, float coef) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r.n_cells) return;
  float2 cs = c.cur_slp[i];
  if (c.locked && c.locked[i]) {
    c.prev_slp[i] = cs;
    return;
  }
  float2 g = c.cur_slp_sum[i];
  float px = __fsub_rn(cs.x, __fmul_rn(coef, g.x));
  float py = __fsub_rn(cs.y, __fmul_rn(coef, g.y));
  c.prev_slp[i] = make_float2(inside_axis(px, (float)c.hx[i], (float)r.lx, (float)r.ux), inside_axis(py, (float)c.hy[i], (float)r.ly, (float)r.uy));
}

// ---- getHpwl (:2297-2304): every net's pin box, summed (int64, exact).
__global__ void k_hpwl(WaArgs w, unsigned long long *__restrict__ out) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  long long h = 0;
  if (t < w.n_nets) {
    int32_t n = w.net_order ? w.net_order[t] : t;
    int64_t b = w.net_start[n], e = w.net_start[n + 1];
    int32_t lx = INT32_MAX, ly = INT32_MAX, ux = INT32_MIN, uy = INT32_MIN;
    for (int64_t p = b; p < e; p++) {
      int2 q = pin_pos(w, p);
      lx = min(lx, q.x);
      ly = min(ly, q.y);
      ux = max(ux, q.x);
      uy = max(uy, q.y);
    }
    if (ux >= lx) h = ((long long)ux - lx) + ((long long)uy - ly);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) h += __shfl_down_sync(0xffffffffu, h, o);
  if ((threadIdx.x & 31) == 0 && h) atomicAdd(out, (unsigned long long)h);
}

// The HPWL over a tile of consecutive nets: pins' positions loaded by the whole block, a
// thread per net for its box. Integer sums: the order does not matter.
__global__ void __launch_bounds__(kThreads) k_hpwl_tiles(WaArgs w, unsigned long long *__restrict__ out) {
  __shared__ int2 s_pos[kWaTilePins];
  __shared__ int32_t s_nstart[kWaTileNets + 1];
  const int4 t = w.tiles[blockIdx.x];
  const int32_t nn = t.y - t.x, np = t.w;
  const int64_t p0 = t.z;
  for (int j = threadIdx.x; j <= nn; j += blockDim.x) s_nstart[j] = (int32_t)(w.net_start[t.x + j] - p0);
  for (int j = threadIdx.x; j < np; j += blockDim.x) s_pos[j] = pin_pos(w, p0 + j);
  __syncthreads();
  long long h = 0;
  for (int j = threadIdx.x; j < nn; j += blockDim.x) {
    int32_t lx = INT32_MAX, ly = INT32_MAX, ux = INT32_MIN, uy = INT32_MIN;
    for (int32_t k = s_nstart[j]; k < s_nstart[j + 1]; k++) {
      int2 q = s_pos[k];
      lx = min(lx, q.x);
      ly = min(ly, q.y);
      ux = max(ux, q.x);
      uy = max(uy, q.y);
    }
    if (ux >= lx) h += ((long long)ux - lx) + ((long long)uy - ly);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) h += __shfl_down_sync(0xffffffffu, h, o);
  if ((threadIdx.x & 31) == 0 && h) atomicAdd(out, (unsigned long long)h);
}

__global__ void k_pack_centres(int64_t n, const int32_t *__restrict__ x, const int32_t *__restrict__ y, int2 *__restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = make_int2(x[i], y[i]);
}

void wa_tiles(const int64_t *net_start, int32_t lo, int32_t hi, std::vector<int4> &tiles, std::vector<int32_t> &big) {
  int32_t first = lo;
  // a tile: its nets [first, end), its first pin and its pin count (pin numbers below 2^31)
  auto close = [&](int32_t end) {
    if (end > first) tiles.push_back(make_int4(first, end, (int32_t)net_start[first], (int32_t)(net_start[end] - net_start[first])));
  };
  for (int32_t n = lo; n < hi; n++) {
    int64_t deg = net_start[n + 1] - net_start[n];
    if (deg > kWaTilePins) {
      close(n);
      big.push_back(n);
      first = n + 1;
      continue;
    }
    if (n - first + 1 > kWaTileNets || net_start[n + 1] - net_start[first] > kWaTilePins) {
      close(n);
      first = n;
    }
  }
  close(hi);
}

WaSmall wa_small_ranges(const int64_t *net_start, int32_t n_nets) {
  WaSmall s{};
  for (int k = 0; k < 3; k++) {
    const int64_t d = 2 + k;
    int32_t n = 0;
    while (n < n_nets && net_start[n + 1] - net_start[n] < d) n++;
    s.first[k] = n;
    while (n < n_nets && net_start[n + 1] - net_start[n] == d) n++;
    s.count[k] = n - s.first[k];
    s.pin0[k] = net_start[s.first[k]];
  }
  return s;
}

int wa_small_blocks(const WaSmall &s) {
  int b = 0;
  for (int k = 0; k < 3; k++) b += (s.count[k] + kThreads - 1) / kThreads;
  return b;
}

// ---- the locked cells' next state (:2848-2859).
__global__ void k_hold_locked(RegionArgs r, CellArgs c) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r.n_cells || !c.locked || !c.locked[i] || c.kind[i] == CELL_FILLER) return;
  c.next_slp[i] = c.cur_slp[i];
  c.next_slp_sum[i] = c.cur_slp_sum[i];
  c.next[i] = c.cur[i];
}


void load_kernel_modules() {
  cudaFuncAttributes a;
  cudaFuncGetAttributes(&a, k_place_cells);
  load_module_b2b();
  load_module_bicgstab();
  load_module_poisson();
  load_module_poisson_tc();
  load_module_cell_order();
}

}  // namespace gpl
