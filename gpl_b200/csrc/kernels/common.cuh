// Shared device helpers for the placement kernels.
//
// Every kernel file that restates the placer's float arithmetic is compiled with
// --fmad=false, so a*b+c is two rounded operations exactly as the reference evaluates it
// (no fused multiply-add anywhere on the reference-ordered paths).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gpl {

// Chained launches (programmatic dependent launch) for kernels that follow one another on a
// stream: a chained kernel's blocks may become resident while the kernel before it drains;
// each first waits in hardware (griddepcontrol.wait) until that kernel has completed and its
// memory is visible, before it reads anything, then admits the next kernel's blocks. Launched
// unchained, the wait and the release do nothing. No result changes.
__device__ __forceinline__ void chain_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
template <typename... KArgs, typename... Args>
inline cudaError_t launch_chained(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

constexpr int kThreads = 256;

// Rust `as i32` from f32/f64: round toward zero, saturating, NaN to 0 (PTX cvt.rzi clamps).
__device__ __forceinline__ int32_t f2i_rz(float v) { return __float2int_rz(v); }
__device__ __forceinline__ int64_t f2l_rz(float v) { return __float2ll_rz(v); }
__device__ __forceinline__ int32_t d2i_rz(double v) { return __double2int_rz(v); }

// `fastExp` (src/nesterov.rs:308-314): (1 + x/1024)^1024 by ten squarings, in float. x/1024
// is taken as x * 2^-10: both are the one correctly rounded value of the same real number.
__device__ __forceinline__ float fast_exp(float x) {
  float e = __fadd_rn(1.0f, __fmul_rn(x, 0.0009765625f));
#pragma unroll
  for (int i = 0; i < 10; i++) e = __fmul_rn(e, e);
  return e;
}

// Truncation and ceiling of the correctly rounded double quotient num / size. The product
// with the rounded reciprocal `inv` is within 1e-15 (relative) of that quotient, so where no
// integer lies within 1e-9 of the product both have the same truncation and ceiling; near
// an integer the IEEE division itself decides.
__device__ __forceinline__ int32_t quot_trunc(int32_t num, double size, double inv) {
  double a = (double)num, q = __dmul_rn(a, inv);
  if (fabs(q - rint(q)) > 1e-9 * fmax(fabs(q), 1.0)) return d2i_rz(q);
  return d2i_rz(__ddiv_rn(a, size));
}
__device__ __forceinline__ int32_t quot_ceil(int32_t num, double size, double inv) {
  double a = (double)num, q = __dmul_rn(a, inv);
  if (fabs(q - rint(q)) > 1e-9 * fmax(fabs(q), 1.0)) return d2i_rz(ceil(q));
  return d2i_rz(ceil(__ddiv_rn(a, size)));
}

// Bin span of [lo, hi) on an axis whose bins start at g0 and are `size` wide, clamped to
// [0, cnt] (`BinGrid::density_idx_x`, src/nesterov.rs:275-284): the quotient in double.
__device__ __forceinline__ void bin_span(int32_t lo, int32_t hi, int32_t g0, double size, double inv, int32_t cnt, int32_t &a, int32_t &b) {
  a = quot_trunc(lo - g0, size, inv);
  b = quot_ceil(hi - g0, size, inv);
  a = a < 0 ? 0 : a;
  b = b > cnt ? cnt : b;
}

// A block's sum of `v` (double), valid in thread 0. Fixed order for a fixed launch shape.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double s = 0;
  if (threadIdx.x < 32) {
    s = threadIdx.x < NT / 32 ? sh[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  }
  __syncthreads();
  return s;
}

// Whether this block is the last of its nblk (by default the launch's blocks) to finish: its
// partials written and fenced before it counts itself, so the last one sees every block's
// partials. The count is left at zero for the next launch.
__device__ __forceinline__ bool last_block_done(unsigned int *ticket, unsigned int nblk) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    last = atomicAdd(ticket, 1u) == nblk - 1;
    if (last) *ticket = 0;
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}
__device__ __forceinline__ bool last_block_done(unsigned int *ticket) { return last_block_done(ticket, gridDim.x); }

// Sums `nblk` rows of `width` partials into out[0..width): each thread over rows t,
// t + NT, ... then the block's sum, so the order is fixed for a block of NT threads.
template <int NT>
__device__ __forceinline__ void reduce_rows(const double *partials, int nblk, int width, double *out, double *sh) {
  if ((width == 2 || width == 4) && ((uintptr_t)partials & 15) == 0) {
    // a row's columns in 16-byte loads, four rows in flight; each column's terms still add in
    // the same order (rows t, t + NT, ...) and meet in the same block sum
    double s[4] = {0, 0, 0, 0};
    const int h = width / 2;
    const double2 *p = reinterpret_cast<const double2 *>(partials);
    int b = threadIdx.x;
    for (; b + 3 * NT < nblk; b += 4 * NT) {
      double2 v[4][2];
#pragma unroll
      for (int u = 0; u < 4; u++)
        for (int q = 0; q < h; q++) v[u][q] = __ldcg(p + (size_t)(b + u * NT) * h + q);
#pragma unroll
      for (int u = 0; u < 4; u++)
        for (int q = 0; q < h; q++) {
          s[2 * q] += v[u][q].x;
          s[2 * q + 1] += v[u][q].y;
        }
    }
    for (; b < nblk; b += NT)
      for (int q = 0; q < h; q++) {
        const double2 v = __ldcg(p + (size_t)b * h + q);
        s[2 * q] += v.x;
        s[2 * q + 1] += v.y;
      }
    for (int j = 0; j < width; j++) {
      double t = block_sum<NT>(s[j], sh);
      if (threadIdx.x == 0) out[j] = t;
    }
    return;
  }
  for (int j = 0; j < width; j++) {
    double s = 0;
    for (int b = threadIdx.x; b < nblk; b += NT) s += __ldcg(partials + (size_t)b * width + j);
    double t = block_sum<NT>(s, sh);
    if (threadIdx.x == 0) out[j] = t;
  }
}

// A block's sums of four doubles at once (one barrier pass), valid in thread 0. Fixed order
// for a fixed launch shape.
template <int NT>
__device__ __forceinline__ double4 block_sum4(double4 v, double4 *sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, o);
    v.y += __shfl_down_sync(0xffffffffu, v.y, o);
    v.z += __shfl_down_sync(0xffffffffu, v.z, o);
    v.w += __shfl_down_sync(0xffffffffu, v.w, o);
  }
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double4 s = make_double4(0, 0, 0, 0);
  if (threadIdx.x == 0)
    for (int k = 0; k < NT / 32; k++) {
      s.x += sh[k].x;
      s.y += sh[k].y;
      s.z += sh[k].z;
      s.w += sh[k].w;
    }
  return s;
}

}  // namespace gpl
