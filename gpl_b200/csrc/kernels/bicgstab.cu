// The initial placement's solver (`bicgstab`, src/bicgstab.rs:615-669) on the device: CSR
// SpMV with each row summed in column order (the reference's `Csr::mul` order), float vectors,
// and the inner products and residual norms in double (deterministic block partials). The
// scalars (rho, alpha, omega) live on the device, and so do the loop's tests: the last kernel
// of an iteration decides whether the loop goes on, ends (the residual bound, the iteration
// cap) or must restart (rho too small), and every kernel of the next iteration returns at once
// unless it goes on. The host enqueues iterations in batches, reads the loop's state once per
// batch and runs a restart itself when the device asks for one.
#include "bicgstab.h"

#include <algorithm>

#include "common.cuh"
#include "tune.h"

namespace gpl {

namespace {

enum Scal { S_RHO = 0, S_RHO_OLD, S_ALPHA, S_W, S_RR, S_R0R, S_R0SQ, S_BB, S_COUNT };
// The loop's state, after the three sums k_scalar's case 0 writes from S_R0SQ: the iteration
// count, the state (0 iterate, 1 waiting for a restart, 2 ended), and the bounds the tests
// compare with. Small integers, exact in double.
enum Loop { S_I = 10, S_STATE, S_TOL2, S_EPS2, S_MAXIT, S_END };
constexpr int S_TICKET = 16;  // the fused reductions' arrival count (an unsigned int)
constexpr double kIterate = 0.0, kRestart = 1.0, kEnded = 2.0;
// Which launches run: every one (kAlways), or only while the loop iterates (kLive).
enum Gate { kAlways = -1, kLive = 0 };
__device__ __forceinline__ bool gated_off(const double *S, int gate) {
  return gate == kLive && S[S_STATE] != kIterate;
}


// The loop's tests (`while rr > tol2 && i < max_iters`, then the restart test
// |rho| < eps^2 |r0|^2 at the head of the next iteration), in the reference's order.
__device__ __forceinline__ double loop_state(const double *S) {
  if (!(S[S_RR] > S[S_TOL2] && S[S_I] < S[S_MAXIT])) return kEnded;
  return fabs(S[S_RHO]) < S[S_EPS2] * S[S_R0SQ] ? kRestart : kIterate;
}

// y = A x, then `0 + 1 * tmp` as the library writes it, each row's products summed in
// column order (the reference's order). Two forms with the same results (SpmvForm):
//  rows:  a thread per row straight from memory;
//  tiled: a block's rows are contiguous in the CSR arrays, so the block first forms every
//         product vals[k] * x[cols[k]] of its rows with coalesced loads into shared memory
//         (eight entries per thread in flight), then each thread sums its row's products; a
//         block whose rows hold more than kSpmvTile entries sums straight from memory.
constexpr int kSpmvTile = 6144;
constexpr int kSpmvUnroll = 8;

// Each form hands every row it forms to emit(row, value), at most one row per thread, and
// returns nowhere early, so a block-wide step may follow.
template <class Emit>
__device__ __forceinline__ void spmv_rows_rows(int64_t n, const int64_t *__restrict__ rs, const int32_t *__restrict__ cols, const float *__restrict__ vals, const float *__restrict__ x, Emit emit) {
  const int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x;
  if (i < n) {
    float tmp = 0.0f;
    const int64_t b = rs[i], e = rs[i + 1];
    for (int64_t k = b; k < e; k++) tmp = __fadd_rn(tmp, __fmul_rn(vals[k], x[cols[k]]));
    emit(i, __fadd_rn(0.0f, __fmul_rn(1.0f, tmp)));
  }
}
__device__ __forceinline__ void spmv_rows_body(int64_t n, const int64_t *__restrict__ rs, const int32_t *__restrict__ cols, const float *__restrict__ vals, const float *__restrict__ x, float *__restrict__ y, const double *__restrict__ S, int gate) {
  if (gated_off(S, gate)) return;
  spmv_rows_rows(n, rs, cols, vals, x, [&](int64_t r, float v) { y[r] = v; });
}
__global__ void __launch_bounds__(kThreads) k_spmv_rows(int64_t n, const int64_t *__restrict__ rs, const int32_t *__restrict__ cols, const float *__restrict__ vals, const float *__restrict__ x, float *__restrict__ y, const double *__restrict__ S, int gate) { spmv_rows_body(n, rs, cols, vals, x, y, S, gate); }

template <class Emit>
__device__ __forceinline__ void spmv_tiled_rows(int64_t n, const int64_t *__restrict__ rs, const int32_t *__restrict__ cols, const float *__restrict__ vals, const float *__restrict__ x, Emit emit) {
  __shared__ float prod[kSpmvTile];
  const int64_t r0 = blockIdx.x * (int64_t)kThreads;
  const int64_t r1 = min(n, r0 + (int64_t)kThreads);
  const int64_t k0 = rs[r0], k1 = rs[r1];
  const int64_t i = r0 + threadIdx.x;
  int64_t b = 0, e = 0;
  if (i < n) {
    b = rs[i];
    e = rs[i + 1];
  }
  const bool tiled = k1 - k0 <= kSpmvTile;
  if (tiled) {
    const int cnt = (int)(k1 - k0);
    const int32_t *c = cols + k0;
    const float *v = vals + k0;
    for (int j = threadIdx.x; j < cnt; j += kSpmvUnroll * kThreads) {
      int cc[kSpmvUnroll];
      float vv[kSpmvUnroll], xv[kSpmvUnroll];
#pragma unroll
      for (int u = 0; u < kSpmvUnroll; u++) {
        int q = j + u * kThreads;
        cc[u] = q < cnt ? __ldg(c + q) : 0;
        vv[u] = q < cnt ? __ldg(v + q) : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < kSpmvUnroll; u++) xv[u] = j + u * kThreads < cnt ? __ldg(x + cc[u]) : 0.0f;
#pragma unroll
      for (int u = 0; u < kSpmvUnroll; u++) {
        int q = j + u * kThreads;
        if (q < cnt) prod[q] = __fmul_rn(vv[u], xv[u]);
      }
    }
  }
  __syncthreads();
  if (i < n) {
    float tmp = 0.0f;
    if (tiled) {
      const int lb = (int)(b - k0), le = (int)(e - k0);
      for (int k = lb; k < le; k++) tmp = __fadd_rn(tmp, prod[k]);
    } else {
      for (int64_t k = b; k < e; k++) tmp = __fadd_rn(tmp, __fmul_rn(vals[k], x[cols[k]]));
    }
    emit(i, __fadd_rn(0.0f, __fmul_rn(1.0f, tmp)));
  }
}
__device__ __forceinline__ void spmv_tiled_body(int64_t n, const int64_t *__restrict__ rs, const int32_t *__restrict__ cols, const float *__restrict__ vals, const float *__restrict__ x, float *__restrict__ y, const double *__restrict__ S, int gate) {
  if (gated_off(S, gate)) return;
  spmv_tiled_rows(n, rs, cols, vals, x, [&](int64_t r, float v) { y[r] = v; });
}
__global__ void __launch_bounds__(kThreads) k_spmv_tiled(int64_t n, const int64_t *__restrict__ rs, const int32_t *__restrict__ cols, const float *__restrict__ vals, const float *__restrict__ x, float *__restrict__ y, const double *__restrict__ S, int gate) { spmv_tiled_body(n, rs, cols, vals, x, y, S, gate); }

//  sliced: over the sliced copy (rows in order of length). The long rows first, a warp per
//         row: the lanes form 32 products at a time from the CSR arrays (coalesced, several
//         chunks in flight) and every lane adds them in column order through shuffles. Then
//         a thread per short row: at step k a warp's rows read one coalesced run of entries
//         (the slice's column k), each row summed in column order and stopping at its own
//         length. y is written at the row's own index. Blocks [0, long_blocks) take the long
//         rows, kThreads / 32 rows each.
constexpr int kLongChunks = 4;
__host__ __device__ __forceinline__ int64_t sliced_long_blocks(int64_t n_long) { return (n_long + kThreads / 32 - 1) / (kThreads / 32); }
__host__ __device__ __forceinline__ int64_t sliced_blocks(int64_t n, int64_t n_long) { return sliced_long_blocks(n_long) + (n - n_long + kThreads - 1) / kThreads; }
template <class Emit>
__device__ __forceinline__ void spmv_sliced_rows(int64_t n, int64_t n_long, const int64_t *__restrict__ rs, const int32_t *__restrict__ cols, const float *__restrict__ vals, const int32_t *__restrict__ sl_row, const int32_t *__restrict__ sl_len, const int64_t *__restrict__ sl_start, const int2 *__restrict__ sl_ent, const float *__restrict__ x, Emit emit) {
  const int64_t lb = sliced_long_blocks(n_long);
  if (blockIdx.x < lb) {
    const int64_t w = blockIdx.x * (int64_t)(kThreads / 32) + (threadIdx.x >> 5);
    if (w >= n_long) return;  // the whole warp; such a warp forms no row
    const int lane = threadIdx.x & 31;
    const int32_t row = sl_row[w];
    const int64_t b = rs[row], e = rs[row + 1];
    float sum = 0.0f;
    for (int64_t m = b; m < e; m += 32 * kLongChunks) {
      float p[kLongChunks];
#pragma unroll
      for (int u = 0; u < kLongChunks; u++) {
        const int64_t k = m + 32 * u + lane;
        p[u] = k < e ? __fmul_rn(__ldg(vals + k), __ldg(x + __ldg(cols + k))) : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < kLongChunks; u++) {
        const int64_t c0 = m + 32 * u;
        if (c0 >= e) break;  // uniform across the warp
        if (e - c0 >= 32) {
#pragma unroll
          for (int t = 0; t < 32; t++) sum = __fadd_rn(sum, __shfl_sync(0xffffffffu, p[u], t));
        } else {
          const int cnt = (int)(e - c0);
          for (int t = 0; t < cnt; t++) sum = __fadd_rn(sum, __shfl_sync(0xffffffffu, p[u], t));
        }
      }
    }
    if (lane == 0) emit(row, __fadd_rn(0.0f, __fmul_rn(1.0f, sum)));
    return;
  }
  const int64_t i = (blockIdx.x - lb) * (int64_t)kThreads + threadIdx.x;  // short position
  const int64_t j = n_long + i;
  if (j >= n) return;
  const int32_t len = sl_len[j];
  const int32_t row = sl_row[j];
  const int64_t base = sl_start[i / kSliceRows] + (i % kSliceRows);
  const int2 *ent = sl_ent + base;
  // kSpmvUnroll entries at a time, the last group's loads predicated, so every group costs
  // two dependent round trips (its entries, then their x) whatever the row's length; the
  // products still add in column order
  float tmp = 0.0f;
  for (int32_t k = 0; k < len; k += kSpmvUnroll) {
    int2 cv[kSpmvUnroll];
    float xv[kSpmvUnroll];
#pragma unroll
    for (int u = 0; u < kSpmvUnroll; u++) cv[u] = k + u < len ? __ldg(ent + (int64_t)(k + u) * kSliceRows) : make_int2(0, 0);
#pragma unroll
    for (int u = 0; u < kSpmvUnroll; u++) xv[u] = k + u < len ? __ldg(x + cv[u].x) : 0.0f;
#pragma unroll
    for (int u = 0; u < kSpmvUnroll; u++)
      if (k + u < len) tmp = __fadd_rn(tmp, __fmul_rn(__int_as_float(cv[u].y), xv[u]));
  }
  emit(row, __fadd_rn(0.0f, __fmul_rn(1.0f, tmp)));
}
__device__ __forceinline__ void spmv_sliced_body(int64_t n, int64_t n_long, const int64_t *__restrict__ rs, const int32_t *__restrict__ cols, const float *__restrict__ vals, const int32_t *__restrict__ sl_row, const int32_t *__restrict__ sl_len, const int64_t *__restrict__ sl_start, const int2 *__restrict__ sl_ent, const float *__restrict__ x, float *__restrict__ y, const double *__restrict__ S, int gate) {
  if (gated_off(S, gate)) return;
  spmv_sliced_rows(n, n_long, rs, cols, vals, sl_row, sl_len, sl_start, sl_ent, x, [&](int64_t r, float v) { y[r] = v; });
}
__global__ void __launch_bounds__(kThreads) k_spmv_sliced(int64_t n, int64_t n_long, const int64_t *__restrict__ rs, const int32_t *__restrict__ cols, const float *__restrict__ vals, const int32_t *__restrict__ sl_row, const int32_t *__restrict__ sl_len, const int64_t *__restrict__ sl_start, const int2 *__restrict__ sl_ent, const float *__restrict__ x, float *__restrict__ y, const double *__restrict__ S, int gate) { spmv_sliced_body(n, n_long, rs, cols, vals, sl_row, sl_len, sl_start, sl_ent, x, y, S, gate); }

// The order by length: a histogram of the (capped) lengths per block in shared memory, the
// buckets' starts longest first, then each row's position from its bucket's cursor (a warp's
// rows of one bucket take one atomic between them).
__global__ void __launch_bounds__(kThreads) k_len_hist(int64_t n, const int64_t *__restrict__ rs, int32_t *__restrict__ count) {
  __shared__ int32_t h[kSliceLenCap + 1];
  for (int b = threadIdx.x; b <= kSliceLenCap; b += kThreads) h[b] = 0;
  __syncthreads();
  const int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x;
  if (i < n) atomicAdd(&h[(int)min(rs[i + 1] - rs[i], (int64_t)kSliceLenCap)], 1);
  __syncthreads();
  for (int b = threadIdx.x; b <= kSliceLenCap; b += kThreads)
    if (h[b]) atomicAdd(&count[b], h[b]);
}
// The counts to starts, longest first: one warp, each lane a run of classes (its loads in
// flight together), the runs' totals scanned across the warp.
constexpr int kLenPerLane = (kSliceLenCap + 1 + 31) / 32;
__global__ void k_len_starts(int32_t *count) {
  const int lane = threadIdx.x;
  int32_t c[kLenPerLane];
  int32_t sum = 0;
#pragma unroll
  for (int q = 0; q < kLenPerLane; q++) {
    const int b = kSliceLenCap - (lane * kLenPerLane + q);  // descending
    c[q] = b >= 0 ? count[b] : 0;
    sum += c[q];
  }
  int32_t run = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t y = __shfl_up_sync(0xffffffffu, run, o);
    if (lane >= o) run += y;
  }
  run -= sum;  // exclusive
#pragma unroll
  for (int q = 0; q < kLenPerLane; q++) {
    const int b = kSliceLenCap - (lane * kLenPerLane + q);
    if (b >= 0) count[b] = run;
    run += c[q];
  }
}
__global__ void __launch_bounds__(kThreads) k_len_scatter(int64_t n, const int64_t *__restrict__ rs, int32_t *__restrict__ cursor, int32_t *__restrict__ row, int32_t *__restrict__ len) {
  const int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x;
  const bool live = i < n;
  const int64_t l = live ? rs[i + 1] - rs[i] : 0;
  const int b = live ? (int)min(l, (int64_t)kSliceLenCap) : -1;
  const unsigned peers = __match_any_sync(0xffffffffu, b);
  const int leader = __ffs(peers) - 1, lane = threadIdx.x & 31;
  int32_t at = 0;
  if (live && lane == leader) at = atomicAdd(&cursor[b], __popc(peers));
  at = __shfl_sync(0xffffffffu, at, leader);
  if (!live) return;
  at += __popc(peers & ((1u << lane) - 1u));
  row[at] = (int32_t)i;
  len[at] = (int32_t)l;
}
// kSliceRows times each slice's longest row (a warp's short positions are one slice).
__global__ void __launch_bounds__(kThreads) k_slice_widths(int64_t n, int64_t n_long, const int32_t *__restrict__ len, int64_t *__restrict__ widths) {
  static_assert(kSliceRows == 32 && kThreads % 32 == 0, "a slice is a warp's rows");
  const int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x, ns = n - n_long;
  if (i - (threadIdx.x & 31) >= ns) return;  // the warp's slice starts past the end
  const unsigned l = i < ns ? (unsigned)len[n_long + i] : 0u;
  const unsigned m = __reduce_max_sync(0xffffffffu, l);
  if ((threadIdx.x & 31) == 0) widths[i / kSliceRows] = (int64_t)m * kSliceRows;
}
__global__ void __launch_bounds__(kThreads) k_slice_fill(int64_t n, int64_t n_long, const int64_t *__restrict__ rs, const int32_t *__restrict__ cols, const float *__restrict__ vals, const int32_t *__restrict__ sl_row, const int32_t *__restrict__ sl_len, const int64_t *__restrict__ sl_start, int2 *__restrict__ sl_ent) {
  const int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x, j = n_long + i;
  if (j >= n) return;
  const int64_t b = rs[sl_row[j]];
  const int32_t len = sl_len[j];
  const int64_t base = sl_start[i / kSliceRows] + (i % kSliceRows);
  for (int32_t k = 0; k < len; k++) sl_ent[base + (int64_t)k * kSliceRows] = make_int2(cols[b + k], __float_as_int(vals[b + k]));
}

static void spmv_launch(int form, int eb, cudaStream_t st, const CsrDev &A, const float *in, float *o, const double *S, int gate) {
  if (form == kSpmvSliced)
    k_spmv_sliced<<<(unsigned)std::max<int64_t>(sliced_blocks(A.n, A.sl_long), 1), kThreads, 0, st>>>(A.n, A.sl_long, A.rs, A.cols, A.vals, A.sl_row, A.sl_len, A.sl_start, A.sl_ent, in, o, S, gate);
  else if (form == kSpmvTiled)
    k_spmv_tiled<<<eb, kThreads, 0, st>>>(A.n, A.rs, A.cols, A.vals, in, o, S, gate);
  else
    k_spmv_rows<<<eb, kThreads, 0, st>>>(A.n, A.rs, A.cols, A.vals, in, o, S, gate);
}

// Reduce the partials and apply one scalar step (the block's threads over the blocks'
// partials, in a fixed order, so every launch shape gives the same sums):
//  which 0: S[dst0..dst0+2] = sums
//  which 1 (alpha): S_ALPHA = rho / sum0
//  which 2 (omega): S_W = sum0 > 0 ? sum1 / sum0 : 0
//  which 3 (end of iteration): S_RR = sum0; S_RHO_OLD = S_RHO; S_RHO = sum1; one more
//           iteration; the loop's tests for the next one
//  which 4 (restart): S_R0SQ = S_RHO = S_RR = sum0
__device__ void scalar_step(const double *part, int nblk, double *S, int which, int dst0, double *sh) {
  double v[3];
  for (int j = 0; j < 3; j++) {
    double s = 0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += __ldcg(part + 3 * b + j);
    v[j] = block_sum<kThreads>(s, sh);
  }
  if (threadIdx.x != 0) return;
  switch (which) {
    case 0:
      S[dst0] = v[0];
      S[dst0 + 1] = v[1];
      S[dst0 + 2] = v[2];
      break;
    case 1: S[S_ALPHA] = S[S_RHO] / v[0]; break;
    case 2: S[S_W] = v[0] > 0.0 ? v[1] / v[0] : 0.0; break;
    case 3:
      S[S_RR] = v[0];
      S[S_RHO_OLD] = S[S_RHO];
      S[S_RHO] = v[1];
      S[S_I] += 1.0;
      S[S_STATE] = loop_state(S);
      break;
    case 4:
      S[S_R0SQ] = v[0];
      S[S_RHO] = v[0];
      S[S_RR] = v[0];
      break;
  }
}

// Whether this block is the last of its launch to finish (its partial written and fenced
// before it counts itself); the last one then sees every block's partial. The count is left
// at zero for the next launch.
__device__ bool last_block(unsigned int *ticket) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    if (last) *ticket = 0;
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

// Up to three dot products at once; partials[blk * 3 + j]. With which >= 0 the last block to
// finish also takes that scalar step (one launch fewer than a separate k_scalar).
__device__ __forceinline__ void dots_body(int64_t n, const float *__restrict__ a0, const float *__restrict__ b0, const float *__restrict__ a1, const float *__restrict__ b1, const float *__restrict__ a2, const float *__restrict__ b2, double *__restrict__ part, double *__restrict__ S, int gate, int which, unsigned int *ticket) {
  if (gated_off(S, gate)) return;
  __shared__ double sh[kThreads / 32];
  double s0 = 0, s1 = 0, s2 = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    s0 += (double)a0[i] * (double)b0[i];
    if (a1) s1 += (double)a1[i] * (double)b1[i];
    if (a2) s2 += (double)a2[i] * (double)b2[i];
  }
  double t0 = block_sum<kThreads>(s0, sh);
  double t1 = block_sum<kThreads>(s1, sh);
  double t2 = block_sum<kThreads>(s2, sh);
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x] = t0;
    part[3 * blockIdx.x + 1] = t1;
    part[3 * blockIdx.x + 2] = t2;
  }
  if (which >= 0 && last_block(ticket)) scalar_step(part, gridDim.x, S, which, 0, sh);
}

// The loop's two inner-product steps, each thread reading 16-byte runs of four, kVecUnroll
// runs in flight (its terms summed in index order), when the vectors start on a 16-byte
// boundary, else one element at a time: TWO 0 is r0.v (then alpha), TWO 1 is t.t and t.s
// (then omega), t read once for both.
constexpr int kVecUnroll = 2;
__device__ __forceinline__ bool all_aligned16(const void *a, const void *b, const void *c, const void *d, const void *e, const void *f) {
  return (((uintptr_t)a | (uintptr_t)b | (uintptr_t)c | (uintptr_t)d | (uintptr_t)e | (uintptr_t)f) & 15) == 0;
}
__device__ __forceinline__ double dot4(float4 a, float4 b, double s) {
  s += (double)a.x * (double)b.x;
  s += (double)a.y * (double)b.y;
  s += (double)a.z * (double)b.z;
  s += (double)a.w * (double)b.w;
  return s;
}
template <int TWO>
__device__ __forceinline__ void loop_dots_body(int64_t n, const float *__restrict__ a, const float *__restrict__ b, double *__restrict__ part, double *__restrict__ S, unsigned int *ticket) {
  if (gated_off(S, kLive)) return;
  __shared__ double sh[kThreads / 32];
  double s0 = 0, s1 = 0;
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
  int64_t done = 0;
  if (all_aligned16(a, b, a, b, a, b)) {
    const int64_t n4 = n / 4;
    const float4 *A = (const float4 *)a, *B = (const float4 *)b;
    for (int64_t i = tid; i < n4; i += kVecUnroll * stride) {
      float4 x[kVecUnroll], y[kVecUnroll];
#pragma unroll
      for (int u = 0; u < kVecUnroll; u++) {
        const int64_t k = i + u * stride;
        const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
        x[u] = k < n4 ? A[k] : z;
        y[u] = k < n4 ? B[k] : z;
      }
#pragma unroll
      for (int u = 0; u < kVecUnroll; u++) {
        if (i + u * stride >= n4) break;
        if (TWO) {
          s0 = dot4(x[u], x[u], s0);
          s1 = dot4(x[u], y[u], s1);
        } else {
          s0 = dot4(x[u], y[u], s0);
        }
      }
    }
    done = 4 * n4;
  }
  for (int64_t i = done + tid; i < n; i += stride) {
    if (TWO) {
      s0 += (double)a[i] * (double)a[i];
      s1 += (double)a[i] * (double)b[i];
    } else {
      s0 += (double)a[i] * (double)b[i];
    }
  }
  double t0 = block_sum<kThreads>(s0, sh);
  double t1 = TWO ? block_sum<kThreads>(s1, sh) : 0.0;
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x] = t0;
    part[3 * blockIdx.x + 1] = t1;
    part[3 * blockIdx.x + 2] = 0.0;
  }
  if (last_block(ticket)) scalar_step(part, gridDim.x, S, TWO ? 2 : 1, 0, sh);
}
__global__ void __launch_bounds__(kThreads, 4) k_loop_dots_alpha(int64_t n, const float *__restrict__ r0, const float *__restrict__ v, double *__restrict__ part, double *__restrict__ S, unsigned int *ticket) { loop_dots_body<0>(n, r0, v, part, S, ticket); }
__global__ void __launch_bounds__(kThreads, 4) k_loop_dots_omega(int64_t n, const float *__restrict__ t, const float *__restrict__ s, double *__restrict__ part, double *__restrict__ S, unsigned int *ticket) { loop_dots_body<1>(n, t, s, part, S, ticket); }
__global__ void k_dots(int64_t n, const float *__restrict__ a0, const float *__restrict__ b0, const float *__restrict__ a1, const float *__restrict__ b1, const float *__restrict__ a2, const float *__restrict__ b2, double *__restrict__ part, double *__restrict__ S, int gate, int which, unsigned int *ticket) { dots_body(n, a0, b0, a1, b1, a2, b2, part, S, gate, which, ticket); }

__global__ void k_scalar(const double *__restrict__ part, int nblk, double *__restrict__ S, int which, int dst0, int gate) {
  if (gated_off(S, gate)) return;
  __shared__ double sh[kThreads / 32];
  scalar_step(part, nblk, S, which, dst0, sh);
}

// After a restart (which 4 above): the first one sets the iteration count back to zero.
__global__ void k_restart_done(double *S, int first) {
  if (first) S[S_I] = 0.0;
  S[S_STATE] = kIterate;
}

__global__ void k_loop_init(double *S, double tol2, double eps2, int max_iters) {
  S[S_I] = 0.0;
  S[S_TOL2] = tol2;
  S[S_EPS2] = eps2;
  S[S_MAXIT] = (double)max_iters;
  S[S_STATE] = loop_state(S);
}

__global__ void k_residual(int64_t n, const float *__restrict__ b, const float *__restrict__ ax, float *__restrict__ r, float *__restrict__ r0, const double *__restrict__ S, int gate) {
  if (gated_off(S, gate)) return;
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float v = __fsub_rn(b[i], ax[i]);
  r[i] = v;
  r0[i] = v;
}

// The elementwise updates: a thread per run of four elements (one 16-byte load per vector
// when they all start on a 16-byte boundary); vec_blocks(n) blocks.
__host__ __device__ __forceinline__ int64_t vec_blocks(int64_t n) { return std::max<int64_t>((n + 4 * kThreads - 1) / (4 * kThreads), 1); }
// p = r + beta (p - w v), beta = (rho / rho_old) (alpha / w)
__device__ __forceinline__ void update_p_body(int64_t n, const double *__restrict__ S, const float *__restrict__ r, const float *__restrict__ v, float *__restrict__ p) {
  if (gated_off(S, kLive)) return;
  const int64_t i = 4 * (blockIdx.x * (int64_t)blockDim.x + threadIdx.x);
  if (i >= n) return;
  const float beta = (float)((S[S_RHO] / S[S_RHO_OLD]) * (S[S_ALPHA] / S[S_W]));
  const float w = (float)S[S_W];
  auto f = [&](float ri, float pi, float vi) { return __fadd_rn(ri, __fmul_rn(beta, __fsub_rn(pi, __fmul_rn(w, vi)))); };
  if (i + 4 <= n && all_aligned16(r, v, p, r, v, p)) {
    const float4 R = *(const float4 *)(r + i), V = *(const float4 *)(v + i), Pv = *(const float4 *)(p + i);
    *(float4 *)(p + i) = make_float4(f(R.x, Pv.x, V.x), f(R.y, Pv.y, V.y), f(R.z, Pv.z, V.z), f(R.w, Pv.w, V.w));
  } else {
    for (int64_t k = i; k < min(n, i + 4); k++) p[k] = f(r[k], p[k], v[k]);
  }
}
__global__ void k_update_p(int64_t n, const double *__restrict__ S, const float *__restrict__ r, const float *__restrict__ v, float *__restrict__ p) { update_p_body(n, S, r, v, p); }

__device__ __forceinline__ void update_s_body(int64_t n, const double *__restrict__ S, const float *__restrict__ r, const float *__restrict__ v, float *__restrict__ s) {
  if (gated_off(S, kLive)) return;
  const int64_t i = 4 * (blockIdx.x * (int64_t)blockDim.x + threadIdx.x);
  if (i >= n) return;
  const float a = (float)S[S_ALPHA];
  auto f = [&](float ri, float vi) { return __fsub_rn(ri, __fmul_rn(a, vi)); };
  if (i + 4 <= n && all_aligned16(r, v, s, r, v, s)) {
    const float4 R = *(const float4 *)(r + i), V = *(const float4 *)(v + i);
    *(float4 *)(s + i) = make_float4(f(R.x, V.x), f(R.y, V.y), f(R.z, V.z), f(R.w, V.w));
  } else {
    for (int64_t k = i; k < min(n, i + 4); k++) s[k] = f(r[k], v[k]);
  }
}
__global__ void k_update_s(int64_t n, const double *__restrict__ S, const float *__restrict__ r, const float *__restrict__ v, float *__restrict__ s) { update_s_body(n, S, r, v, s); }

// x += alpha p + w s; r = s - w t; partials of |r|^2 and r0.r, the last block taking the
// iteration's end (scalar step 3). Runs of four as in the loop's dot products.
__device__ __forceinline__ void update_xr_body(int64_t n, double *__restrict__ S, const float *__restrict__ p, const float *__restrict__ s, const float *__restrict__ t, const float *__restrict__ r0, float *__restrict__ x, float *__restrict__ r, double *__restrict__ part, unsigned int *ticket) {
  if (gated_off(S, kLive)) return;
  __shared__ double sh[kThreads / 32];
  const float a = (float)S[S_ALPHA], w = (float)S[S_W];
  double rr = 0, r0r = 0;
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
  auto fx = [&](float xi, float pi, float si) { return __fadd_rn(xi, __fadd_rn(__fmul_rn(a, pi), __fmul_rn(w, si))); };
  auto fr = [&](float si, float ti) { return __fsub_rn(si, __fmul_rn(w, ti)); };
  int64_t done = 0;
  if (all_aligned16(p, s, t, r0, x, r)) {
    const int64_t n4 = n / 4;
    constexpr int U = 1;
    for (int64_t i = tid; i < n4; i += U * stride) {
      float4 X[U], Pp[U], Sv[U], T[U], R0[U];
      const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int64_t k = i + u * stride;
        const bool in = k < n4;
        X[u] = in ? ((const float4 *)x)[k] : z;
        Pp[u] = in ? ((const float4 *)p)[k] : z;
        Sv[u] = in ? ((const float4 *)s)[k] : z;
        T[u] = in ? ((const float4 *)t)[k] : z;
        R0[u] = in ? ((const float4 *)r0)[k] : z;
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int64_t k = i + u * stride;
        if (k >= n4) break;
        ((float4 *)x)[k] = make_float4(fx(X[u].x, Pp[u].x, Sv[u].x), fx(X[u].y, Pp[u].y, Sv[u].y), fx(X[u].z, Pp[u].z, Sv[u].z), fx(X[u].w, Pp[u].w, Sv[u].w));
        const float4 R = make_float4(fr(Sv[u].x, T[u].x), fr(Sv[u].y, T[u].y), fr(Sv[u].z, T[u].z), fr(Sv[u].w, T[u].w));
        ((float4 *)r)[k] = R;
        rr = dot4(R, R, rr);
        r0r = dot4(R0[u], R, r0r);
      }
    }
    done = 4 * n4;
  }
  for (int64_t i = done + tid; i < n; i += stride) {
    x[i] = fx(x[i], p[i], s[i]);
    float rv = fr(s[i], t[i]);
    r[i] = rv;
    rr += (double)rv * (double)rv;
    r0r += (double)r0[i] * (double)rv;
  }
  double t0 = block_sum<kThreads>(rr, sh);
  double t1 = block_sum<kThreads>(r0r, sh);
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x] = t0;
    part[3 * blockIdx.x + 1] = t1;
    part[3 * blockIdx.x + 2] = 0.0;
  }
  if (last_block(ticket)) scalar_step(part, gridDim.x, S, 3, 0, sh);  // the iteration's end
}
__global__ void __launch_bounds__(kThreads, 4) k_update_xr(int64_t n, double *__restrict__ S, const float *__restrict__ p, const float *__restrict__ s, const float *__restrict__ t, const float *__restrict__ r0, float *__restrict__ x, float *__restrict__ r, double *__restrict__ part, unsigned int *ticket) { update_xr_body(n, S, p, s, t, r0, x, r, part, ticket); }

// Both axes' systems in one launch (blockIdx.y picks the system): the initial placement solves
// its x and y systems side by side, so each launch carries twice the work and the loop half
// the launches. Each system keeps its own scalars, state and arrival count, so every one
// takes exactly the steps it would take alone.
struct SysDev {
  int64_t n;
  const int64_t *rs;
  const int32_t *cols;
  const float *vals;
  int64_t sl_long;
  const int32_t *sl_row, *sl_len;
  const int64_t *sl_start;
  const int2 *sl_ent;
  float *x, *r, *r0, *v, *p, *s, *t;
  double *part, *S;
  unsigned int *ticket;
};
struct SysPair {
  SysDev a[2];
};
__device__ __forceinline__ SysDev pick(const SysPair &P) { return blockIdx.y ? P.a[1] : P.a[0]; }

// The loop's kernels are launched chained (common.cuh: chain_enter, launch_chained).

__global__ void __launch_bounds__(kThreads) k2_update_p(SysPair P) {
  chain_enter();
  SysDev q = pick(P);
  update_p_body(q.n, q.S, q.r, q.v, q.p);
}
// sel 0: v = A p; sel 1: t = A s (each system's rows in the form's order, gated as a whole).
__global__ void __launch_bounds__(kThreads) k2_spmv_rows(SysPair P, int sel) {
  chain_enter();
  SysDev q = pick(P);
  spmv_rows_body(q.n, q.rs, q.cols, q.vals, sel ? q.s : q.p, sel ? q.t : q.v, q.S, kLive);
}
__global__ void __launch_bounds__(kThreads) k2_spmv_tiled(SysPair P, int sel) {
  chain_enter();
  SysDev q = pick(P);
  spmv_tiled_body(q.n, q.rs, q.cols, q.vals, sel ? q.s : q.p, sel ? q.t : q.v, q.S, kLive);
}
__global__ void __launch_bounds__(kThreads) k2_spmv_sliced(SysPair P, int sel) {
  chain_enter();
  SysDev q = pick(P);
  spmv_sliced_body(q.n, q.sl_long, q.rs, q.cols, q.vals, q.sl_row, q.sl_len, q.sl_start, q.sl_ent, sel ? q.s : q.p, sel ? q.t : q.v, q.S, kLive);
}
// The inner products after each product, in their own launch over the vectors in order
// (sel 0: r0.v, then alpha; sel 1: t.t and t.s, then omega), the last block taking the scalar
// step. (Forming them in the SpMV's own launch was measured 11 % slower over the whole
// initial placement: the sliced form's rows are in length order, so their r0 and s reads
// scatter, and the fused tail's block reductions stall every block.)
__global__ void __launch_bounds__(kThreads, 4) k2_dots(SysPair P, int sel) {
  chain_enter();
  SysDev q = pick(P);
  if (sel == 0)
    loop_dots_body<0>(q.n, q.r0, q.v, q.part, q.S, q.ticket);
  else
    loop_dots_body<1>(q.n, q.t, q.s, q.part, q.S, q.ticket);
}

__global__ void __launch_bounds__(kThreads) k2_update_s(SysPair P) {
  chain_enter();
  SysDev q = pick(P);
  update_s_body(q.n, q.S, q.r, q.v, q.s);
}
__global__ void __launch_bounds__(kThreads, 4) k2_update_xr(SysPair P) {
  chain_enter();
  SysDev q = pick(P);
  update_xr_body(q.n, q.S, q.p, q.s, q.t, q.r0, q.x, q.r, q.part, q.ticket);
}
__global__ void k_set_ended(double *S) { S[S_STATE] = kEnded; }

__global__ void k_fill(int64_t n, float *a, float v) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}
__global__ void k_scal_init(double *S) {
  S[S_RHO] = S[S_COUNT];  // dot(r0, r) of the start point
  S[S_RR] = S[S_R0SQ];
  S[S_RHO_OLD] = 1.0;
  S[S_ALPHA] = 1.0;
  S[S_W] = 1.0;
}

}  // namespace

// Iterations enqueued between two reads of the loop's state.
constexpr int kBicgBatch = 8;

size_t bicgstab_scratch_bytes(int64_t n) {
  size_t vec = (size_t)n * sizeof(float);
  vec = (vec + 255) / 256 * 256;
  return 7 * vec + (size_t)kBicgBlocks * 3 * sizeof(double) + 64 * sizeof(double);
}

size_t bicgstab_pair_scratch_bytes(int64_t n) { return bicgstab_scratch_bytes(n); }

cudaError_t csr_slice_order(const CsrDev &A, int32_t *row, int32_t *len, int32_t *count, cudaStream_t st) {
  if (A.n <= 0) return cudaSuccess;
  const unsigned g = (unsigned)((A.n + kThreads - 1) / kThreads);
  cudaError_t e = cudaMemsetAsync(count, 0, (kSliceLenCap + 1) * sizeof(int32_t), st);
  if (e != cudaSuccess) return e;
  k_len_hist<<<g, kThreads, 0, st>>>(A.n, A.rs, count);
  k_len_starts<<<1, 32, 0, st>>>(count);
  k_len_scatter<<<g, kThreads, 0, st>>>(A.n, A.rs, count, row, len);
  return cudaGetLastError();
}

cudaError_t csr_slice_widths(int64_t n, int64_t n_long, const int32_t *len, int64_t *widths, cudaStream_t st) {
  if (n - n_long <= 0) return cudaSuccess;
  k_slice_widths<<<(unsigned)((n - n_long + kThreads - 1) / kThreads), kThreads, 0, st>>>(n, n_long, len, widths);
  return cudaGetLastError();
}

cudaError_t csr_slice_fill(const CsrDev &A, int2 *sl_ent, cudaStream_t st) {
  if (A.n - A.sl_long <= 0) return cudaSuccess;
  k_slice_fill<<<(unsigned)((A.n - A.sl_long + kThreads - 1) / kThreads), kThreads, 0, st>>>(A.n, A.sl_long, A.rs, A.cols, A.vals, A.sl_row, A.sl_len, A.sl_start, sl_ent);
  return cudaGetLastError();
}

cudaError_t spmv(const CsrDev &A, const float *x, float *y, int form, cudaStream_t st) {
  if (form != kSpmvRows && form != kSpmvTiled && form != kSpmvSliced) return cudaErrorInvalidValue;
  if (form == kSpmvSliced && (!A.sl_start || !A.sl_row || !A.sl_len)) return cudaErrorInvalidValue;
  if (A.n <= 0) return cudaSuccess;
  spmv_launch(form, (int)((A.n + kThreads - 1) / kThreads), st, A, x, y, nullptr, kAlways);
  return cudaGetLastError();
}

cudaError_t bicgstab_solve(const CsrDev &A, const float *b, float *x, int max_iters, void *scratch, cudaStream_t st, BicgResult *out, int form) {
  static_assert(S_END <= S_TICKET && S_TICKET < 64, "the scalars fit the scratch's 64 doubles");
  if (form == kSpmvSliced && (!A.sl_start || !A.sl_row || !A.sl_len)) return cudaErrorInvalidValue;
  int64_t n = A.n;
  size_t vec = ((size_t)n * sizeof(float) + 255) / 256 * 256;
  char *base = (char *)scratch;
  float *r = (float *)(base), *r0 = (float *)(base + vec), *v = (float *)(base + 2 * vec), *p = (float *)(base + 3 * vec);
  float *s = (float *)(base + 4 * vec), *t = (float *)(base + 5 * vec), *ax = (float *)(base + 6 * vec);
  double *part = (double *)(base + 7 * vec);
  double *S = part + (size_t)kBicgBlocks * 3;
  unsigned int *ticket = (unsigned int *)(S + S_TICKET);
  int eb = (int)((n + kThreads - 1) / kThreads);
  if (eb < 1) eb = 1;
  int rb = kBicgBlocks;
  const float tol = 1.1920929e-07f;
  double hs[S_END];
  auto spmv = [&](const float *in, float *o, int gate) { spmv_launch(form, eb, st, A, in, o, S, gate); };
  auto pull = [&]() -> cudaError_t {
    cudaError_t e = cudaMemcpyAsync(hs, S, sizeof hs, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);
  };
  cudaError_t e;
  spmv(x, ax, kAlways);
  k_residual<<<eb, kThreads, 0, st>>>(n, b, ax, r, r0, S, kAlways);
  cudaMemsetAsync(ticket, 0, sizeof(unsigned int), st);
  k_dots<<<rb, kThreads, 0, st>>>(n, r0, r0, b, b, r0, r, part, S, kAlways, -1, ticket);
  k_scalar<<<1, kThreads, 0, st>>>(part, rb, S, 0, S_R0SQ, kAlways);  // S_R0SQ, S_BB, then dot(r0, r) in S[S_COUNT]
  if ((e = pull()) != cudaSuccess) return e;
  double rhs_sqnorm = hs[S_BB];
  if (rhs_sqnorm == 0.0) {
    k_fill<<<eb, kThreads, 0, st>>>(n, x, 0.0f);
    out->iterations = max_iters;
    out->error = tol;
    out->converged = true;
    return cudaGetLastError();
  }
  k_scal_init<<<1, 1, 0, st>>>(S);
  cudaMemsetAsync(v, 0, (size_t)n * sizeof(float), st);
  cudaMemsetAsync(p, 0, (size_t)n * sizeof(float), st);
  double tol2 = (double)tol * (double)tol * rhs_sqnorm;
  double eps2 = (double)tol * (double)tol;
  k_loop_init<<<1, 1, 0, st>>>(S, tol2, eps2, max_iters);
  // Every iteration counts one and only the first restart sets the count back, so the loop
  // ends within 2 max_iters + 1 iterations; a batch that asks for a restart holds until the
  // host has run it, and every batch but the last runs at least one iteration.
  const int64_t max_batches = 2 * (int64_t)max_iters + 3;
  int64_t batches = 0;
  int restarts = 0;
  for (;;) {
    for (int k = 0; k < kBicgBatch; k++) {
      k_update_p<<<(unsigned)vec_blocks(n), kThreads, 0, st>>>(n, S, r, v, p);
      spmv(p, v, kLive);
      k_loop_dots_alpha<<<rb, kThreads, 0, st>>>(n, r0, v, part, S, ticket);
      k_update_s<<<(unsigned)vec_blocks(n), kThreads, 0, st>>>(n, S, r, v, s);
      spmv(s, t, kLive);
      k_loop_dots_omega<<<rb, kThreads, 0, st>>>(n, t, s, part, S, ticket);
      k_update_xr<<<rb, kThreads, 0, st>>>(n, S, p, s, t, r0, x, r, part, ticket);
    }
    if ((e = pull()) != cudaSuccess) return e;
    if (hs[S_STATE] == kEnded) break;
    if (++batches > max_batches) return cudaErrorUnknown;  // cannot happen: the count above
    if (hs[S_STATE] == kRestart) {
      // too orthogonal to r0: restart from the current residual
      spmv(x, ax, kAlways);
      k_residual<<<eb, kThreads, 0, st>>>(n, b, ax, r, r0, S, kAlways);
      k_dots<<<rb, kThreads, 0, st>>>(n, r, r, nullptr, nullptr, nullptr, nullptr, part, S, kAlways, -1, ticket);
      k_scalar<<<1, kThreads, 0, st>>>(part, rb, S, 4, 0, kAlways);
      k_restart_done<<<1, 1, 0, st>>>(S, restarts == 0 ? 1 : 0);
      restarts++;
    }
  }
  double rr = hs[S_RR];
  out->iterations = (int)hs[S_I];
  out->error = (float)std::sqrt(rr / rhs_sqnorm);
  out->converged = out->error <= tol;
  return cudaGetLastError();
}

// One chained launch of a loop kernel (kThreads a block, no dynamic shared memory).
template <typename... KArgs, typename... Args>
static cudaError_t chained(void (*kernel)(KArgs...), dim3 grid, cudaStream_t st, Args... args) {
  return launch_chained(kernel, grid, dim3(kThreads), 0, st, args...);
}
#define CK_LAUNCH(x)                        \
  do {                                      \
    if ((e = (x)) != cudaSuccess) return e; \
  } while (0)

cudaError_t bicgstab_solve_pair(const CsrDev A[2], const float *const b[2], float *const x[2], int max_iters, void *const scratch[2], cudaStream_t st, BicgResult out[2], int form, Tuner *tune) {
  const int64_t n = A[0].n;
  if (A[1].n != n) return cudaErrorInvalidValue;
  for (int a = 0; a < 2; a++)
    if ((form == kSpmvSliced || tune) && (!A[a].sl_start || !A[a].sl_row || !A[a].sl_len)) return cudaErrorInvalidValue;
  const size_t vec = ((size_t)n * sizeof(float) + 255) / 256 * 256;
  SysPair P{};
  for (int a = 0; a < 2; a++) {
    char *base = (char *)scratch[a];
    SysDev &q = P.a[a];
    q.n = n;
    q.rs = A[a].rs;
    q.cols = A[a].cols;
    q.vals = A[a].vals;
    q.sl_long = A[a].sl_long;
    q.sl_row = A[a].sl_row;
    q.sl_len = A[a].sl_len;
    q.sl_start = A[a].sl_start;
    q.sl_ent = A[a].sl_ent;
    q.x = x[a];
    q.r = (float *)base;
    q.r0 = (float *)(base + vec);
    q.v = (float *)(base + 2 * vec);
    q.p = (float *)(base + 3 * vec);
    q.s = (float *)(base + 4 * vec);
    q.t = (float *)(base + 5 * vec);
    q.part = (double *)(base + 7 * vec);
    q.S = q.part + (size_t)kBicgBlocks * 3;
    q.ticket = (unsigned int *)(q.S + S_TICKET);
  }
  auto ax_of = [&](int a) { return (float *)((char *)scratch[a] + 6 * vec); };
  int eb = (int)((n + kThreads - 1) / kThreads);
  if (eb < 1) eb = 1;
  const int rb = kBicgBlocks;
  const float tol = 1.1920929e-07f;
  double hs[2][S_END];
  auto pull = [&]() -> cudaError_t {
    for (int a = 0; a < 2; a++) {
      cudaError_t e = cudaMemcpyAsync(hs[a], P.a[a].S, sizeof hs[a], cudaMemcpyDeviceToHost, st);
      if (e != cudaSuccess) return e;
    }
    return cudaStreamSynchronize(st);
  };
  auto restart = [&](int a, bool first) {
    // too orthogonal to r0: restart from the current residual (that system alone)
    const SysDev &q = P.a[a];
    spmv_launch(form, eb, st, A[a], q.x, ax_of(a), q.S, kAlways);
    k_residual<<<eb, kThreads, 0, st>>>(n, b[a], ax_of(a), q.r, q.r0, q.S, kAlways);
    k_dots<<<rb, kThreads, 0, st>>>(n, q.r, q.r, nullptr, nullptr, nullptr, nullptr, q.part, q.S, kAlways, -1, q.ticket);
    k_scalar<<<1, kThreads, 0, st>>>(q.part, rb, q.S, 4, 0, kAlways);
    k_restart_done<<<1, 1, 0, st>>>(q.S, first ? 1 : 0);
  };
  cudaError_t e;
  // each system's start, as the single solve takes it
  for (int a = 0; a < 2; a++) {
    const SysDev &q = P.a[a];
    spmv_launch(form, eb, st, A[a], q.x, ax_of(a), q.S, kAlways);
    k_residual<<<eb, kThreads, 0, st>>>(n, b[a], ax_of(a), q.r, q.r0, q.S, kAlways);
    cudaMemsetAsync(q.ticket, 0, sizeof(unsigned int), st);
    k_dots<<<rb, kThreads, 0, st>>>(n, q.r0, q.r0, b[a], b[a], q.r0, q.r, q.part, q.S, kAlways, -1, q.ticket);
    k_scalar<<<1, kThreads, 0, st>>>(q.part, rb, q.S, 0, S_R0SQ, kAlways);
  }
  if ((e = pull()) != cudaSuccess) return e;
  double rhs_sqnorm[2];
  bool live[2];
  for (int a = 0; a < 2; a++) {
    const SysDev &q = P.a[a];
    rhs_sqnorm[a] = hs[a][S_BB];
    live[a] = rhs_sqnorm[a] != 0.0;
    if (!live[a]) {
      k_fill<<<eb, kThreads, 0, st>>>(n, q.x, 0.0f);
      k_set_ended<<<1, 1, 0, st>>>(q.S);
      out[a].iterations = max_iters;
      out[a].error = tol;
      out[a].converged = true;
      continue;
    }
    k_scal_init<<<1, 1, 0, st>>>(q.S);
    cudaMemsetAsync(q.v, 0, (size_t)n * sizeof(float), st);
    cudaMemsetAsync(q.p, 0, (size_t)n * sizeof(float), st);
    double tol2 = (double)tol * (double)tol * rhs_sqnorm[a];
    double eps2 = (double)tol * (double)tol;
    k_loop_init<<<1, 1, 0, st>>>(q.S, tol2, eps2, max_iters);
  }
  if (!live[0] && !live[1]) return cudaGetLastError();
  // both systems' iterations in each launch; the bound on batches is the single solve's
  const int64_t max_batches = 2 * (int64_t)max_iters + 3;
  int64_t batches = 0;
  int restarts[2] = {0, 0};
  const dim3 ge(eb, 2), gr(rb, 2), gv((unsigned)vec_blocks(n), 2);
  const dim3 gs((unsigned)std::max<int64_t>({sliced_blocks(n, A[0].sl_long), sliced_blocks(n, A[1].sl_long), 1}), 2);
  for (;;) {
    const int f = tune ? kSpmvTiled + tune->start(st) : form;  // the tuner's candidates: tiled, sliced
    for (int k = 0; k < kBicgBatch; k++) {
      CK_LAUNCH(chained(k2_update_p, gv, st, P));
      for (int sel = 0; sel < 2; sel++) {
        if (f == kSpmvSliced)
          CK_LAUNCH(chained(k2_spmv_sliced, gs, st, P, sel));
        else if (f == kSpmvTiled)
          CK_LAUNCH(chained(k2_spmv_tiled, ge, st, P, sel));
        else
          CK_LAUNCH(chained(k2_spmv_rows, ge, st, P, sel));
        CK_LAUNCH(chained(k2_dots, gr, st, P, sel));
        if (sel == 0) CK_LAUNCH(chained(k2_update_s, gv, st, P));
      }
      CK_LAUNCH(chained(k2_update_xr, gr, st, P));
    }
    if (tune) tune->stop(st);
    if ((e = pull()) != cudaSuccess) return e;
    // a batch counts for the tuner when both systems ran all of it
    if (tune) tune->finish(hs[0][S_STATE] == kIterate && hs[1][S_STATE] == kIterate);
    if (hs[0][S_STATE] == kEnded && hs[1][S_STATE] == kEnded) break;
    if (++batches > max_batches) return cudaErrorUnknown;  // cannot happen: the single solve's count
    for (int a = 0; a < 2; a++)
      if (hs[a][S_STATE] == kRestart) restart(a, restarts[a]++ == 0);
  }
  for (int a = 0; a < 2; a++) {
    if (!live[a]) continue;
    out[a].iterations = (int)hs[a][S_I];
    out[a].error = (float)std::sqrt(hs[a][S_RR] / rhs_sqnorm[a]);
    out[a].converged = out[a].error <= tol;
  }
  return cudaGetLastError();
}


// Loads this file's module (the driver loads a module at its first launch otherwise).
void load_module_bicgstab() {
  cudaFuncAttributes a;
  cudaFuncGetAttributes(&a, k2_update_xr);
}

}  // namespace gpl
