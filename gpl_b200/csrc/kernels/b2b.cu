// The initial placement on the device: bound-to-bound assembly (`createSparseMatrix`,
// src/initial_place.rs:264-355), the triplets' collapse into CSR (`Csr::from_triplets`,
// src/bicgstab.rs:501-541), BiCGSTAB, `updateCoordi` and the report's HPWL.
//
// Bit-exact with the host restatement: every triplet and right-hand-side term is written at
// the position the host's net loop would append it (per-net counts, an exclusive scan, then
// the same loop writing), and each row's duplicates are summed in that order (a row's
// entries sorted by (column, position)), the first occurrence first, as the reference sums
// them into the first.
#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "b2b.h"
#include "common.cuh"
#include "engine_kernels.h"

namespace gpl {
void progress(const char *fmt, ...) __attribute__((format(printf, 1, 2)));

namespace {

constexpr int kScanBlock = 1024;

enum PinFlag : uint8_t { F_MIN_X = 1, F_MAX_X = 2, F_MIN_Y = 4, F_MAX_Y = 8 };

struct IpArgs {
  int32_t n_nets;
  const int64_t *net_start;
  const int32_t *pin_e, *pin_inst;
  const uint8_t *pin_mio;
  const int2 *pin_xy;
  uint8_t *pin_flag;
  const int4 *box;
  const uint8_t *locked;
  int32_t max_fanout, min_diff;
  float weight_scale;
};

// Where one axis's terms go: triplets (row, col, value) and right-hand-side terms (row,
// value), each net's run starting at its scanned offset.
struct AxisOut {
  int32_t *t_row, *t_col;
  float *t_val;
  int32_t *r_row;
  float *r_val;
  const int64_t *t_off, *r_off;  // per net
  int64_t t_base;                // the locked diagonal precedes the nets' triplets
};

// `updatePinInfo` (src/initial_place.rs:203-252): per net, the first strict extreme per side.
__global__ void k_pin_info(IpArgs a) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.n_nets) return;
  int64_t b = a.net_start[n], e = a.net_start[n + 1];
  int32_t lx = INT32_MAX, ly = INT32_MAX, ux = INT32_MIN, uy = INT32_MIN;
  int64_t pminx = -1, pmaxx = -1, pminy = -1, pmaxy = -1;
  for (int64_t k = b; k < e; k++) a.pin_flag[k] = 0;
  for (int64_t k = b; k < e; k++) {
    if (a.pin_mio[k]) continue;
    int2 q = a.pin_xy[k];
    if (lx > q.x) {
      if (pminx >= 0) a.pin_flag[pminx] &= (uint8_t)~F_MIN_X;
      lx = q.x;
      pminx = k;
      a.pin_flag[k] |= F_MIN_X;
    }
    if (ux < q.x) {
      if (pmaxx >= 0) a.pin_flag[pmaxx] &= (uint8_t)~F_MAX_X;
      ux = q.x;
      pmaxx = k;
      a.pin_flag[k] |= F_MAX_X;
    }
    if (ly > q.y) {
      if (pminy >= 0) a.pin_flag[pminy] &= (uint8_t)~F_MIN_Y;
      ly = q.y;
      pminy = k;
      a.pin_flag[k] |= F_MIN_Y;
    }
    if (uy < q.y) {
      if (pmaxy >= 0) a.pin_flag[pmaxy] &= (uint8_t)~F_MAX_Y;
      uy = q.y;
      pmaxy = k;
      a.pin_flag[k] |= F_MAX_Y;
    }
  }
}

__device__ __forceinline__ int32_t centre(const int4 &b, int axis) { return axis == 0 ? (b.x + b.z) / 2 : (b.y + b.w) / 2; }

// One net's pairs in the host's order (the second pin from the second solve pin on, the first
// below it; x then y): counted (EMIT false) or written at the net's offsets (EMIT true).
// A pair counts on an axis only when one of its pins is that axis's extreme, so a second pin
// that is no extreme pairs only with the net's extreme pins: for it the first pin runs over
// the (at most four) extremes below it, in index order, instead of every pin below it; the
// pairs visited, and their order, are the reference's, in O(degree) per net.
template <bool EMIT>
__device__ void net_pairs(const IpArgs &a, int n, int64_t *cnt, int64_t stride, const AxisOut *out) {
  int64_t b = a.net_start[n], e = a.net_start[n + 1];
  int64_t deg = e - b;
  int64_t tpos[2] = {0, 0}, rpos[2] = {0, 0};
  if (EMIT) {
#pragma unroll
    for (int ax = 0; ax < 2; ax++) {
      tpos[ax] = out[ax].t_base + out[ax].t_off[n];
      rpos[ax] = out[ax].r_off[n];
    }
  }
  int64_t tc[2] = {0, 0}, rc[2] = {0, 0};
  if (deg > 1 && deg < a.max_fanout) {
    float net_weight = __fdiv_rn(a.weight_scale, (float)(deg - 1));
    // the net's extreme pins (a pin flagged on any side), in index order; at most four
    int64_t ext[4];
    int n_ext = 0;
    for (int64_t k = b; k < e && n_ext < 4; k++)
      if (a.pin_flag[k]) ext[n_ext++] = k;
    for (int64_t k1 = b; k1 < e; k1++) {
      if (a.pin_mio[k1]) continue;
      const bool k1_ext = a.pin_flag[k1] != 0;
      const int64_t n2 = k1_ext ? k1 - b : (int64_t)n_ext;
      for (int64_t j = 0; j < n2; j++) {
        const int64_t k2 = k1_ext ? b + j : ext[j];
        if (k2 >= k1) break;  // the extremes are in index order
        if (a.pin_mio[k2]) continue;
        if (a.pin_inst[k1] == a.pin_inst[k2]) continue;
        uint8_t f = a.pin_flag[k1] | a.pin_flag[k2];
        int2 q1 = a.pin_xy[k1], q2 = a.pin_xy[k2];
        int32_t ea = a.pin_e[k1], eb = a.pin_e[k2];
#pragma unroll
        for (int axis = 0; axis < 2; axis++) {
          uint8_t mask = axis == 0 ? (F_MIN_X | F_MAX_X) : (F_MIN_Y | F_MAX_Y);
          if (!(f & mask)) continue;
          int32_t c1 = axis == 0 ? q1.x : q1.y, c2 = axis == 0 ? q2.x : q2.y;
          int32_t diff = abs(c1 - c2);
          float weight = diff > a.min_diff ? __fdiv_rn(net_weight, (float)diff) : __fdiv_rn(net_weight, (float)a.min_diff);
          int nt = 0, nr = 0;
          int32_t rows[4], cols[4], rr[2];
          float vals[4], rv[2];
          if (ea >= 0 && eb >= 0) {
            bool la = a.locked[ea], lb = a.locked[eb];
            if (!la && !lb) {
              int32_t ca = centre(a.box[ea], axis), cb = centre(a.box[eb], axis);
              rows[0] = ea, cols[0] = ea, vals[0] = weight;
              rows[1] = eb, cols[1] = eb, vals[1] = weight;
              rows[2] = ea, cols[2] = eb, vals[2] = -weight;
              rows[3] = eb, cols[3] = ea, vals[3] = -weight;
              nt = 4;
              rr[0] = ea, rv[0] = __fmul_rn(-weight, (float)((c1 - ca) - (c2 - cb)));
              rr[1] = eb, rv[1] = __fmul_rn(-weight, (float)((c2 - cb) - (c1 - ca)));
              nr = 2;
            } else if (la && !lb) {
              int32_t cb = centre(a.box[eb], axis);
              rows[0] = eb, cols[0] = eb, vals[0] = weight, nt = 1;
              rr[0] = eb, rv[0] = __fmul_rn(weight, (float)(c1 - (c2 - cb))), nr = 1;
            } else if (!la && lb) {
              int32_t ca = centre(a.box[ea], axis);
              rows[0] = ea, cols[0] = ea, vals[0] = weight, nt = 1;
              rr[0] = ea, rv[0] = __fmul_rn(weight, (float)(c2 - (c1 - ca))), nr = 1;
            }
          } else if (ea < 0 && eb >= 0) {
            int32_t cb = centre(a.box[eb], axis);
            rows[0] = eb, cols[0] = eb, vals[0] = weight, nt = 1;
            rr[0] = eb, rv[0] = __fmul_rn(weight, (float)(c1 - (c2 - cb))), nr = 1;
          } else if (ea >= 0 && eb < 0) {
            int32_t ca = centre(a.box[ea], axis);
            rows[0] = ea, cols[0] = ea, vals[0] = weight, nt = 1;
            rr[0] = ea, rv[0] = __fmul_rn(weight, (float)(c2 - (c1 - ca))), nr = 1;
          }
          if (EMIT) {
            const AxisOut &o = out[axis];
            for (int q = 0; q < nt; q++) {
              int64_t at = tpos[axis]++;
              o.t_row[at] = rows[q];
              o.t_col[at] = cols[q];
              o.t_val[at] = vals[q];
            }
            for (int q = 0; q < nr; q++) {
              int64_t at = rpos[axis]++;
              o.r_row[at] = rr[q];
              o.r_val[at] = rv[q];
            }
          }
          tc[axis] += nt;
          rc[axis] += nr;
        }
      }
    }
  }
  if (!EMIT) {
    cnt[n] = tc[0];
    cnt[stride + n] = tc[1];
    cnt[2 * stride + n] = rc[0];
    cnt[3 * stride + n] = rc[1];
  }
}

__global__ void k_count(IpArgs a, int64_t *cnt, int64_t stride) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n < a.n_nets) net_pairs<false>(a, n, cnt, stride, nullptr);
}

__global__ void k_emit(IpArgs a, AxisOut x, AxisOut y) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  AxisOut out[2] = {x, y};
  if (n < a.n_nets) net_pairs<true>(a, n, nullptr, 0, out);
}

// The locked instances' unit diagonal (first in the triplet list, in instance order), and
// each axis's start vector: the instances' centres.
__global__ void k_locked_and_x0(int64_t n, const int4 *box, const uint8_t *locked, const int32_t *rank, AxisOut x, AxisOut y, float *x0, float *y0) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= n) return;
  int4 b = box[e];
  x0[e] = (float)centre(b, 0);
  y0[e] = (float)centre(b, 1);
  if (locked[e]) {
    int32_t at = rank[e];
    x.t_row[at] = (int32_t)e, x.t_col[at] = (int32_t)e, x.t_val[at] = 1.0f;
    y.t_row[at] = (int32_t)e, y.t_col[at] = (int32_t)e, y.t_val[at] = 1.0f;
  }
}

// ---- the collapse into CSR: rows bucketed, each row's entries ordered by (column, position)
__global__ void k_row_count(int64_t nt, const int32_t *row, unsigned long long *cnt) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < nt) atomicAdd(&cnt[row[t]], 1ull);
}

// Each triplet's key (column << 32 | position) into its row's bucket; the order within a
// bucket is settled by the sort that follows.
__global__ void k_bucket(int64_t nt, const int32_t *row, const int32_t *col, const int64_t *row_off, int32_t *fill, unsigned long long *bucket) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nt) return;
  int32_t r = row[t];
  int64_t at = row_off[r] + atomicAdd(&fill[r], 1);
  uint32_t c = col ? (uint32_t)col[t] : 0u;
  bucket[at] = ((unsigned long long)c << 32) | (unsigned long long)(uint32_t)t;
}

// Per row: keys sorted (column, then position; the keys are distinct), each column's run
// summed in position order (the first value, then the rest added to it), the distinct columns
// compacted. Tiers by the row's length: a warp per row with its keys in registers (R per
// lane, bitonic-sorted across the warp) for rows of up to 32, then 64, then 256 keys; a block
// per row (bitonic sort in shared memory) up to 8192; a block per row merging sorted chunks
// beyond. Every tier gives the same result.
constexpr int kRowTiny = 32, kRowShort = 64, kRowMid = 256;

// One column's run [p, end) of a sorted row summed in position order: the first value, then
// the rest added to it; the values' loads go four at a time ahead of the adds.
__device__ __forceinline__ float run_sum(const unsigned long long *sk, int p, int end, const float *val) {
  float s = val[(uint32_t)sk[p]];
  int q = p + 1;
  for (; q + 4 <= end; q += 4) {
    float t0 = val[(uint32_t)sk[q]], t1 = val[(uint32_t)sk[q + 1]], t2 = val[(uint32_t)sk[q + 2]], t3 = val[(uint32_t)sk[q + 3]];
    s = __fadd_rn(s, t0);
    s = __fadd_rn(s, t1);
    s = __fadd_rn(s, t2);
    s = __fadd_rn(s, t3);
  }
  for (; q < end; q++) s = __fadd_rn(s, val[(uint32_t)sk[q]]);
  return s;
}

// Sums and compacts a sorted row held in shared memory (sk: m keys), a warp's lanes taking
// the run starts; returns the row's distinct columns.
__device__ __forceinline__ int64_t warp_runs(const unsigned long long *sk, int m, int64_t b, const float *val, int32_t *ucol, float *uval) {
  const int lane = threadIdx.x & 31;
  int64_t base = 0;
  for (int p0 = 0; p0 < m; p0 += 32) {
    int p = p0 + lane;
    bool start = p < m && (p == 0 || (uint32_t)(sk[p] >> 32) != (uint32_t)(sk[p - 1] >> 32));
    unsigned mask = __ballot_sync(0xffffffffu, start);
    if (start) {
      unsigned long long key = sk[p];
      uint32_t c = (uint32_t)(key >> 32);
      int end = p + 1;
      while (end < m && (uint32_t)(sk[end] >> 32) == c) end++;
      float s = run_sum(sk, p, end, val);
      int64_t u = base + __popc(mask & ((1u << lane) - 1u));
      ucol[b + u] = (int32_t)c;
      uval[b + u] = s;
    }
    base += __popc(mask);
  }
  return base;
}

// The same for a block's warps at once (rows of the block tiers): the sorted positions cut
// into one contiguous section of whole 32-position steps per warp, each warp counting the runs
// that start in its section, a scan of those counts, then each warp summing and writing its
// runs (a run that starts in a section may end in the next) from its offset. The distinct
// columns come out in position order, as warp_runs writes them. Every thread of the block
// calls it; returns the row's distinct columns.
__device__ __forceinline__ int64_t block_runs(const unsigned long long *sk, int m, int64_t b, const float *val, int32_t *ucol, float *uval) {
  __shared__ int64_t counts[kThreads / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int steps = (m + 31) / 32, per = (steps + nw - 1) / nw;
  const int lo = w * per * 32, hi = min(m, (w + 1) * per * 32);
  auto starts_at = [&](int p) { return p < hi && (p == 0 || (uint32_t)(sk[p] >> 32) != (uint32_t)(sk[p - 1] >> 32)); };
  int64_t cnt = 0;
  for (int p0 = lo; p0 < hi; p0 += 32) cnt += __popc(__ballot_sync(0xffffffffu, starts_at(p0 + lane)));
  if (lane == 0) counts[w] = cnt;
  __syncthreads();
  int64_t base = 0, total = 0;
  for (int k = 0; k < nw; k++) {
    if (k < w) base += counts[k];
    total += counts[k];
  }
  for (int p0 = lo; p0 < hi; p0 += 32) {
    const int p = p0 + lane;
    const bool start = starts_at(p);
    const unsigned mask = __ballot_sync(0xffffffffu, start);
    if (start) {
      const uint32_t c = (uint32_t)(sk[p] >> 32);
      int end = p + 1;
      while (end < m && (uint32_t)(sk[end] >> 32) == c) end++;
      const int64_t u = base + __popc(mask & ((1u << lane) - 1u));
      ucol[b + u] = (int32_t)c;
      uval[b + u] = run_sum(sk, p, end, val);
    }
    base += __popc(mask);
  }
  __syncthreads();  // counts free for the block's next row
  return total;
}

// A warp per row of at most 32 R keys: element i = j * 32 + lane lives in register j.
template <int R>
__device__ __forceinline__ void warp_bitonic(unsigned long long (&v)[R]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 2; k <= 32 * R; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j >= 32) {
        const int jr = j >> 5;
#pragma unroll
        for (int a = 0; a < R; a++) {
          const int bb = a ^ jr;
          if (bb > a) {
            const int i = a * 32 + lane;
            const bool up = (i & k) == 0;
            unsigned long long x = v[a], y = v[bb];
            bool sw = up ? (x > y) : (x < y);
            v[a] = sw ? y : x;
            v[bb] = sw ? x : y;
          }
        }
      } else {
#pragma unroll
        for (int a = 0; a < R; a++) {
          const int i = a * 32 + lane;
          const bool up = (i & k) == 0, lower = (lane & j) == 0;
          unsigned long long o = __shfl_xor_sync(0xffffffffu, v[a], j);
          unsigned long long mn = v[a] < o ? v[a] : o, mx = v[a] < o ? o : v[a];
          v[a] = (lower == up) ? mn : mx;
        }
      }
    }
  }
}

// Rows of up to 32 R keys, a warp each: rows [0, n) when `list` is null, else the `*count`
// rows of `list`; longer rows go to `next` (with `next_count`) for the next tier.
template <int R>
__global__ void __launch_bounds__(kThreads) k_row_collapse_warp(int64_t n, const int32_t *list, const int *count, const int64_t *row_off, const unsigned long long *bucket, const float *val, int32_t *ucol, float *uval, int64_t *ucount, int32_t *next, int *next_count) {
  __shared__ unsigned long long sk[kThreads / 32][32 * R];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t total = list ? (int64_t)*count : n;
  const int64_t warps = (int64_t)gridDim.x * (kThreads / 32);
  for (int64_t w = blockIdx.x * (int64_t)(kThreads / 32) + wib; w < total; w += warps) {
    const int64_t r = list ? (int64_t)list[w] : w;
    const int64_t b = row_off[r], e = row_off[r + 1];
    const int64_t m = e - b;
    if (m > 32 * R) {
      if (lane == 0) next[atomicAdd(next_count, 1)] = (int32_t)r;
      continue;
    }
    if (m <= 1) {  // nothing to sort (most right-hand-side rows): the key as it is
      if (lane == 0) {
        if (m == 1) {
          const unsigned long long k = bucket[b];
          ucol[b] = (int32_t)(uint32_t)(k >> 32);
          uval[b] = val[(uint32_t)k];
        }
        ucount[r] = m;
      }
      continue;
    }
    unsigned long long v[R];
#pragma unroll
    for (int a = 0; a < R; a++) {
      const int i = a * 32 + lane;
      v[a] = i < m ? bucket[b + i] : ~0ull;
    }
    warp_bitonic<R>(v);
#pragma unroll
    for (int a = 0; a < R; a++) sk[wib][a * 32 + lane] = v[a];
    __syncwarp();
    int64_t u = warp_runs(sk[wib], (int)m, b, val, ucol, uval);
    if (lane == 0) ucount[r] = u;
    __syncwarp();
  }
}

// Rows of up to kRowLong keys, a block each: the keys bitonic-sorted in shared memory
// (padded to a power of two), then the block's warps walk the runs. Longer rows go to `next`.
constexpr int kRowLong = 8192;
__global__ void __launch_bounds__(kThreads) k_row_collapse_block(const int32_t *list, const int *count, const int64_t *row_off, const unsigned long long *bucket, const float *val, int32_t *ucol, float *uval, int64_t *ucount, int32_t *next, int *next_count) {
  extern __shared__ unsigned long long skb[];
  const int64_t total = *count;
  for (int64_t w = blockIdx.x; w < total; w += gridDim.x) {
    const int64_t r = list[w];
    const int64_t b = row_off[r], e = row_off[r + 1];
    const int64_t m = e - b;
    if (m > kRowLong) {
      if (threadIdx.x == 0) next[atomicAdd(next_count, 1)] = (int32_t)r;
      continue;
    }
    int N = 1;
    while (N < m) N <<= 1;
    for (int i = threadIdx.x; i < N; i += blockDim.x) skb[i] = i < m ? bucket[b + i] : ~0ull;
    __syncthreads();
    for (int k = 2; k <= N; k <<= 1)
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int i = threadIdx.x; i < N; i += blockDim.x) {
          const int o = i ^ j;
          if (o > i) {
            const bool up = (i & k) == 0;
            unsigned long long x = skb[i], y = skb[o];
            if (up ? (x > y) : (x < y)) {
              skb[i] = y;
              skb[o] = x;
            }
          }
        }
        __syncthreads();
      }
    const int64_t u = block_runs(skb, (int)m, b, val, ucol, uval);
    if (threadIdx.x == 0) ucount[r] = u;
    __syncthreads();
  }
}

// The longest rows, a block each: chunks of kRowLong keys bitonic-sorted in shared memory and
// written back, then runs merged pairwise between the bucket and a scratch of the same span
// (merge path: each thread's share of a merged run starts where a binary search on its
// diagonal puts it, then it merges that share in order) until one run remains, whose column
// runs the block's warps walk as in the block tier.
__device__ __forceinline__ void merge_share(const unsigned long long *A, int64_t la, const unsigned long long *B, int64_t lb, unsigned long long *out) {
  const int64_t total = la + lb, per = (total + blockDim.x - 1) / blockDim.x;
  const int64_t d = (int64_t)threadIdx.x * per;
  if (d >= total) return;
  int64_t lo = d > lb ? d - lb : 0, hi = d < la ? d : la;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (A[mid] < B[d - 1 - mid]) lo = mid + 1; else hi = mid;
  }
  int64_t i = lo, j = d - lo;
  const int64_t end = d + per < total ? d + per : total;
  for (int64_t k = d; k < end; k++) out[k] = (j >= lb || (i < la && A[i] < B[j])) ? A[i++] : B[j++];
}

__global__ void __launch_bounds__(kThreads) k_row_collapse_long(const int32_t *list, const int *count, const int64_t *row_off, unsigned long long *bucket, unsigned long long *scratch, const float *val, int32_t *ucol, float *uval, int64_t *ucount) {
  extern __shared__ unsigned long long skl[];
  const int64_t total = *count;
  for (int64_t w = blockIdx.x; w < total; w += gridDim.x) {
    const int64_t r = list[w];
    const int64_t b = row_off[r], e = row_off[r + 1], m = e - b;
    unsigned long long *keys = bucket + b, *tmp = scratch + b;
    for (int64_t c0 = 0; c0 < m; c0 += kRowLong) {
      const int cm = (int)(m - c0 < kRowLong ? m - c0 : kRowLong);
      int N = 1;
      while (N < cm) N <<= 1;
      for (int i = threadIdx.x; i < N; i += blockDim.x) skl[i] = i < cm ? keys[c0 + i] : ~0ull;
      __syncthreads();
      for (int k = 2; k <= N; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
          for (int i = threadIdx.x; i < N; i += blockDim.x) {
            const int o = i ^ j;
            if (o > i) {
              const bool up = (i & k) == 0;
              unsigned long long x = skl[i], y = skl[o];
              if (up ? (x > y) : (x < y)) {
                skl[i] = y;
                skl[o] = x;
              }
            }
          }
          __syncthreads();
        }
      for (int i = threadIdx.x; i < cm; i += blockDim.x) keys[c0 + i] = skl[i];
      __syncthreads();
    }
    unsigned long long *src = keys, *dst = tmp;
    for (int64_t run = kRowLong; run < m; run <<= 1) {
      for (int64_t a0 = 0; a0 < m; a0 += 2 * run) {
        const int64_t la = run < m - a0 ? run : m - a0;
        const int64_t lb = a0 + run < m ? (a0 + 2 * run < m ? run : m - a0 - run) : 0;
        merge_share(src + a0, la, src + a0 + la, lb, dst + a0);
      }
      __syncthreads();
      unsigned long long *t = src;
      src = dst;
      dst = t;
    }
    if (src != keys) {
      for (int64_t i = threadIdx.x; i < m; i += blockDim.x) keys[i] = src[i];
      __syncthreads();
    }
    const int64_t u = block_runs(keys, (int)m, b, val, ucol, uval);
    if (threadIdx.x == 0) ucount[r] = u;
    __syncthreads();
  }
}

__global__ void k_row_fill(int64_t n, const int64_t *row_off, const int64_t *starts, const int32_t *ucol, const float *uval, int32_t *cols, float *vals) {
  int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  int64_t b = row_off[r], o = starts[r], m = starts[r + 1] - o;
  for (int64_t j = 0; j < m; j++) {
    cols[o + j] = ucol[b + j];
    vals[o + j] = uval[b + j];
  }
}

// The right-hand side: the locked rows' centre, else the row's terms summed in order onto 0.
__global__ void k_rhs(int64_t n, int axis, const int4 *box, const uint8_t *locked, const int64_t *row_off, const int64_t *ucount, const float *uval, float *rhs) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= n) return;
  if (locked[e]) {
    rhs[e] = (float)centre(box[e], axis);
    return;
  }
  // the host adds every term onto 0.0f; the run's sum from its first term differs from that
  // only in the sign of a zero, which one more + 0.0f settles
  rhs[e] = ucount[e] ? __fadd_rn(uval[row_off[e]], 0.0f) : 0.0f;
}

// ---- exclusive scan of int64 counts (in place; data[n] receives the total)
__global__ void k_scan_block(int64_t *data, int64_t n, int64_t *totals) {
  __shared__ int64_t warp_sum[kScanBlock / 32];
  int64_t i = blockIdx.x * (int64_t)kScanBlock + threadIdx.x;
  int64_t v = i < n ? data[i] : 0;
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int64_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int64_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sum[w] = x;
  __syncthreads();
  if (w == 0) {
    int64_t s = warp_sum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int64_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    warp_sum[lane] = s;
  }
  __syncthreads();
  int64_t before = w ? warp_sum[w - 1] : 0;
  if (i < n) data[i] = before + x - v;
  if (threadIdx.x == kScanBlock - 1) totals[blockIdx.x] = before + x;
}

// The block totals' exclusive scan: one block of 1024 threads, a chunk of totals each.
__global__ void k_scan_totals(int64_t *totals, int64_t nb) {
  __shared__ int64_t part[kScanBlock];
  const int64_t per = (nb + kScanBlock - 1) / kScanBlock;
  const int64_t lo = threadIdx.x * per, hi = min(nb, lo + per);
  int64_t s = 0;
  for (int64_t b = lo; b < hi; b++) s += totals[b];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t run = 0;
    for (int t = 0; t < kScanBlock; t++) {
      int64_t q = part[t];
      part[t] = run;
      run += q;
    }
    totals[nb] = run;
  }
  __syncthreads();
  int64_t run = part[threadIdx.x];
  for (int64_t b = lo; b < hi; b++) {
    int64_t q = totals[b];
    totals[b] = run;
    run += q;
  }
}

__global__ void k_scan_add(int64_t *data, int64_t n, const int64_t *totals, int64_t nb) {
  int64_t i = blockIdx.x * (int64_t)kScanBlock + threadIdx.x;
  if (i < n) data[i] += totals[blockIdx.x];
  if (i == 0) data[n] = totals[nb];
}

// ---- the solver's row order
// Row i' of the renumbered system is row perm[i'] with its entries in their own order and each
// column j renumbered inv[j], so each product y'[i'] sums the same terms in the same order as
// y[perm[i']]; only the cross-row sums (the inner products) see their terms in another order.
__global__ void k_perm_len(int64_t n, const int32_t *__restrict__ perm, const int64_t *__restrict__ starts, int64_t *__restrict__ len) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t r = perm[i];
  len[i] = starts[r + 1] - starts[r];
}
__global__ void k_perm_inv(int64_t n, const int32_t *__restrict__ perm, int32_t *__restrict__ inv) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) inv[perm[i]] = (int32_t)i;
}
// A warp per row: the row's entries copied in order, 32 at a time.
__global__ void k_perm_rows(int64_t n, const int32_t *__restrict__ perm, const int32_t *__restrict__ inv, const int64_t *__restrict__ starts, const int32_t *__restrict__ cols, const float *__restrict__ vals,
                            const int64_t *__restrict__ pstarts, int32_t *__restrict__ pcols, float *__restrict__ pvals) {
  const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= n) return;
  const int32_t r = perm[w];
  const int64_t s0 = starts[r], len = starts[r + 1] - s0, d0 = pstarts[w];
  for (int64_t k = lane; k < len; k += 32) {
    pcols[d0 + k] = inv[cols[s0 + k]];
    pvals[d0 + k] = vals[s0 + k];
  }
}
// out[i'] = in[perm[i']] (into the solver's order), and back: out[perm[i']] = in[i'].
__global__ void k_perm_gather(int64_t n, const int32_t *__restrict__ perm, const float *__restrict__ in, float *__restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[perm[i]];
}
__global__ void k_perm_scatter(int64_t n, const int32_t *__restrict__ perm, const float *__restrict__ in, float *__restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[perm[i]] = in[i];
}

// ---- updateCoordi (src/initial_place.rs:391-417) and setCenterLocation (:152-165)
__global__ void k_update(int64_t n, const float *x, const float *y, int4 core, const int4 *region, const uint8_t *grouped, const uint8_t *locked, int4 *box, int4 *db_box, const int2 *db_size) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= n || locked[e]) return;
  int32_t nx = f2i_rz(x[e]), ny = f2i_rz(y[e]);
  nx = min(max(nx, core.x), core.z);
  ny = min(max(ny, core.y), core.w);
  if (grouped[e]) {
    int4 r = region[e];
    nx = min(max(nx, r.x), r.z);
    ny = min(max(ny, r.y), r.w);
  }
  int4 b = box[e];
  int32_t hx = (b.z - b.x) / 2, hy = (b.w - b.y) / 2;
  b = make_int4(nx - hx, ny - hy, nx + hx, ny + hy);
  box[e] = b;
  int2 d = db_size[e];
  db_box[e] = make_int4(b.x, b.y, b.x + d.x, b.y + d.y);
}

__global__ void k_pins(int64_t np, const int32_t *pin_e, const uint8_t *locked, const int4 *box, const int2 *off, int2 *xy) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= np) return;
  int32_t e = pin_e[k];
  if (e < 0 || locked[e]) return;
  int4 b = box[e];
  int2 o = off[k];
  xy[k] = make_int2(centre(b, 0) + o.x, centre(b, 1) + o.y);
}

// The report's HPWL over the database boxes (src/initial_place.rs:359-386).
__global__ void k_db_hpwl(int32_t n_nets, const int64_t *net_start, const int32_t *pin_e, const uint8_t *hp, const int4 *stat, const int4 *db_box, unsigned long long *out) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  long long h = 0;
  if (n < n_nets) {
    int32_t lx = INT32_MAX, ly = INT32_MAX, ux = INT32_MIN, uy = INT32_MIN;
    for (int64_t k = net_start[n]; k < net_start[n + 1]; k++) {
      uint8_t m = hp[k];
      if (m == 2) continue;
      int4 b = m == 0 ? db_box[pin_e[k]] : stat[k];
      lx = min(lx, b.x);
      ly = min(ly, b.y);
      ux = max(ux, b.z);
      uy = max(uy, b.w);
    }
    if (ux >= lx) h = ((long long)ux - lx) + ((long long)uy - ly);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) h += __shfl_down_sync(0xffffffffu, h, o);
  if ((threadIdx.x & 31) == 0 && h) atomicAdd(out, (unsigned long long)h);
}

unsigned grid(int64_t n) { return (unsigned)std::max<int64_t>(1, (n + kThreads - 1) / kThreads); }

// The initial placement's buffers come from the device's stream-ordered pool, which keeps
// what they free (the release threshold is raised once per device): freeing a few GB at the
// end of the initial placement then costs no unmapping, and the next run reuses the memory.
void keep_pool_once() {
  static bool kept[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 || kept[dev]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) return;
  uint64_t keep = UINT64_MAX;
  if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) == cudaSuccess) kept[dev] = true;
}
template <class T>
cudaError_t alloc(T **p, size_t n, cudaStream_t s) {
  *p = nullptr;
  return cudaMallocAsync((void **)p, std::max<size_t>(n, 1) * sizeof(T), s);
}
template <class T, class A>
cudaError_t put(T **p, const std::vector<T, A> &v, cudaStream_t s, int64_t &bytes) {
  cudaError_t e = alloc(p, v.size(), s);
  if (e != cudaSuccess || v.empty()) return e;
  bytes += (int64_t)(v.size() * sizeof(T));
  return cudaMemcpyAsync(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

// Grows a set of buffers to hold n entries each.
template <class... T>
cudaError_t grow(cudaStream_t s, size_t n, size_t &cap, T **...bufs) {
  if (n <= cap) return cudaSuccess;
  size_t c = (size_t)(n * 1.1) + 16;
  cudaError_t e = cudaSuccess;
  auto one = [&](auto **p) {
    if (*p) cudaFreeAsync(*p, s);
    *p = nullptr;
    if (e == cudaSuccess) e = alloc(p, c, s);
  };
  (one(bufs), ...);
  cap = e == cudaSuccess ? c : 0;
  return e;
}

}  // namespace

#define CK(x)                         \
  do {                                \
    cudaError_t _e = (x);             \
    if (_e != cudaSuccess) return _e; \
  } while (0)

IpDevice::~IpDevice() { release(); }

void IpDevice::release() {
  void *ptrs[] = {box_, clamp_, db_box_, pin_static_, db_size_, pin_off_, pin_xy_, locked_, grouped_, pin_mio_, pin_hp_, pin_flag_, pin_e_, pin_inst_, locked_rank_,
                  net_start_, cnt_, scan_tmp_, t_row_, t_col_, t_val_, r_row_, r_val_, bucket_, bucket2_, fill_, row_off_, ucount_, ucol_, uval_, scratch_, hpwl_acc_, tier_rows_, tier_n_};
  for (void *p : ptrs)
    if (p) cudaFreeAsync(p, s_);
  for (void *p : {(void *)perm_, (void *)inv_, (void *)ord_idx_, (void *)ord_hist_, (void *)ord_key0_, (void *)ord_key1_})
    if (p) cudaFreeAsync(p, s_);
  perm_ = inv_ = ord_idx_ = ord_hist_ = nullptr;
  ord_key0_ = ord_key1_ = nullptr;
  solves_ = 0;
  for (auto &a : ax_) {
    void *q[] = {a.starts, a.cols, a.vals, a.rhs, a.x, a.sl_row, a.sl_len, a.sl_count, a.sl_start, a.sl_ent, a.p_starts, a.p_cols, a.p_vals, a.p_rhs, a.p_x};
    for (void *p : q)
      if (p) cudaFreeAsync(p, s_);
    a = Axis{};
  }
  box_ = clamp_ = db_box_ = pin_static_ = nullptr;
  db_size_ = pin_off_ = pin_xy_ = nullptr;
  locked_ = grouped_ = pin_mio_ = pin_hp_ = pin_flag_ = nullptr;
  pin_e_ = pin_inst_ = locked_rank_ = nullptr;
  net_start_ = cnt_ = scan_tmp_ = row_off_ = ucount_ = nullptr;
  t_row_ = t_col_ = r_row_ = fill_ = ucol_ = nullptr;
  t_val_ = r_val_ = uval_ = nullptr;
  bucket_ = bucket2_ = nullptr;
  scratch_ = nullptr;
  hpwl_acc_ = nullptr;
  tier_rows_ = nullptr;
  tier_n_ = nullptr;
  t_cap_ = r_cap_ = w_cap_ = scan_tmp_n_ = 0;
}

cudaError_t IpDevice::upload(const IpSetup &s) {
  release();
  keep_pool_once();
  cfg_.max_fanout = s.max_fanout;
  cfg_.min_diff = s.min_diff;
  cfg_.weight_scale = s.weight_scale;
  cfg_.core = s.core;
  n_ = (int64_t)s.box.size();
  n_pins_ = (int64_t)s.pin_e.size();
  n_nets_ = (int32_t)(s.net_start.size() - 1);
  std::vector<int32_t> rank(n_, -1);
  n_locked_ = 0;
  for (int64_t e = 0; e < n_; e++)
    if (s.locked[e]) rank[e] = (int32_t)n_locked_++;
  int64_t &b = h2d_bytes;
  CK(put(&box_, s.box, s_, b));
  CK(put(&locked_, s.locked, s_, b));
  CK(put(&clamp_, s.clamp, s_, b));
  CK(put(&grouped_, s.grouped, s_, b));
  CK(put(&db_box_, s.db_box, s_, b));
  CK(put(&db_size_, s.db_size, s_, b));
  CK(put(&locked_rank_, rank, s_, b));
  CK(put(&pin_e_, s.pin_e, s_, b));
  CK(put(&pin_inst_, s.pin_inst, s_, b));
  CK(put(&pin_mio_, s.pin_mio, s_, b));
  CK(put(&pin_off_, s.pin_off, s_, b));
  CK(put(&pin_xy_, s.pin_xy, s_, b));
  CK(put(&pin_hp_, s.pin_hp, s_, b));
  CK(put(&pin_static_, s.pin_static, s_, b));
  CK(put(&net_start_, s.net_start, s_, b));
  CK(alloc(&pin_flag_, n_pins_, s_));
  CK(alloc(&cnt_, 4 * ((size_t)n_nets_ + 1), s_));
  CK(alloc(&row_off_, n_ + 1, s_));
  CK(alloc(&ucount_, n_ + 1, s_));
  CK(cudaFuncSetAttribute(k_row_collapse_block, cudaFuncAttributeMaxDynamicSharedMemorySize, kRowLong * (int)sizeof(unsigned long long)));
  CK(cudaFuncSetAttribute(k_row_collapse_long, cudaFuncAttributeMaxDynamicSharedMemorySize, kRowLong * (int)sizeof(unsigned long long)));
  CK(alloc(&tier_rows_, 4 * std::max<int64_t>(n_, 1), s_));
  CK(alloc(&tier_n_, 4, s_));
  CK(alloc(&fill_, n_, s_));
  CK(alloc(&hpwl_acc_, 1, s_));
  for (auto &a : ax_) {
    CK(alloc(&a.starts, n_ + 1, s_));
    CK(alloc(&a.rhs, n_, s_));
    CK(alloc(&a.x, n_, s_));
  }
  // the two axes' solver scratch, side by side (256-byte aligned halves)
  scratch_bytes_ = (bicgstab_pair_scratch_bytes(n_) + 255) / 256 * 256;
  CK(cudaMallocAsync(&scratch_, 2 * scratch_bytes_, s_));
  return cudaStreamSynchronize(s_);
}

size_t scan_i64_tmp(int64_t n) { return (size_t)((n + kScanBlock - 1) / kScanBlock + 1); }

cudaError_t scan_i64(int64_t *data, int64_t n, int64_t *tmp, cudaStream_t s) {
  const int64_t nb = (n + kScanBlock - 1) / kScanBlock;
  if (nb == 0) return cudaMemsetAsync(data, 0, sizeof(int64_t), s);
  k_scan_block<<<(unsigned)nb, kScanBlock, 0, s>>>(data, n, tmp);
  k_scan_totals<<<1, kScanBlock, 0, s>>>(tmp, nb);
  k_scan_add<<<(unsigned)nb, kScanBlock, 0, s>>>(data, n, tmp, nb);
  return cudaGetLastError();
}

cudaError_t IpDevice::scan(int64_t *data, int64_t n) {
  int64_t nb = (n + kScanBlock - 1) / kScanBlock;
  if ((size_t)(nb + 1) > scan_tmp_n_) {
    if (scan_tmp_) cudaFreeAsync(scan_tmp_, s_);
    scan_tmp_n_ = (size_t)(nb + 1);
    CK(alloc(&scan_tmp_, scan_tmp_n_, s_));
  }
  if (nb == 0) return cudaMemsetAsync(data, 0, sizeof(int64_t), s_);
  k_scan_block<<<(unsigned)nb, kScanBlock, 0, s_>>>(data, n, scan_tmp_);
  k_scan_totals<<<1, kScanBlock, 0, s_>>>(scan_tmp_, nb);
  k_scan_add<<<(unsigned)nb, kScanBlock, 0, s_>>>(data, n, scan_tmp_, nb);
  launches += 3;
  return cudaGetLastError();
}

// Collapses triplets (row, col or one column, val) [0, n_trip) into CSR rows; with no
// output arrays it stops at the per-row sums (row_off_, ucount_, uval_).
cudaError_t IpDevice::collapse(int64_t n_trip, const int32_t *row, const int32_t *col, const float *val, int64_t *starts_out, int32_t **cols, float **vals, size_t *cap, int64_t *nnz) {
  CK(cudaMemsetAsync(row_off_, 0, (n_ + 1) * sizeof(int64_t), s_));
  CK(cudaMemsetAsync(fill_, 0, std::max<int64_t>(n_, 1) * sizeof(int32_t), s_));
  if (n_trip) k_row_count<<<grid(n_trip), kThreads, 0, s_>>>(n_trip, row, (unsigned long long *)row_off_);
  CK(scan(row_off_, n_));
  if (n_trip) k_bucket<<<grid(n_trip), kThreads, 0, s_>>>(n_trip, row, col, row_off_, fill_, bucket_);
  if (n_) {
    // tiers: a warp per row up to 32 keys, then up to 64, then up to 256, a block per row up
    // to 8192, then a block per row merging sorted chunks
    CK(cudaMemsetAsync(tier_n_, 0, 4 * sizeof(int), s_));
    const int wblocks = (int)std::min<int64_t>((n_ + kThreads / 32 - 1) / (kThreads / 32), 148 * 64);
    k_row_collapse_warp<kRowTiny / 32><<<wblocks, kThreads, 0, s_>>>(n_, nullptr, nullptr, row_off_, bucket_, val, ucol_, uval_, ucount_, tier_rows_, tier_n_);
    k_row_collapse_warp<kRowShort / 32><<<148 * 16, kThreads, 0, s_>>>(n_, tier_rows_, tier_n_, row_off_, bucket_, val, ucol_, uval_, ucount_, tier_rows_ + n_, tier_n_ + 1);
    k_row_collapse_warp<kRowMid / 32><<<148 * 4, kThreads, 0, s_>>>(n_, tier_rows_ + n_, tier_n_ + 1, row_off_, bucket_, val, ucol_, uval_, ucount_, tier_rows_ + 2 * n_, tier_n_ + 2);
    k_row_collapse_block<<<148 * 2, kThreads, kRowLong * sizeof(unsigned long long), s_>>>(tier_rows_ + 2 * n_, tier_n_ + 2, row_off_, bucket_, val, ucol_, uval_, ucount_, tier_rows_ + 3 * n_, tier_n_ + 3);
    k_row_collapse_long<<<148 * 2, kThreads, kRowLong * sizeof(unsigned long long), s_>>>(tier_rows_ + 3 * n_, tier_n_ + 3, row_off_, bucket_, bucket2_, val, ucol_, uval_, ucount_);
    launches += 5;
  }
  launches += 2;
  if (!cols) return cudaGetLastError();
  CK(cudaMemcpyAsync(starts_out, ucount_, n_ * sizeof(int64_t), cudaMemcpyDeviceToDevice, s_));
  CK(scan(starts_out, n_));
  CK(cudaMemcpyAsync(nnz, starts_out + n_, sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  d2h_bytes += 8;
  if ((size_t)*nnz > *cap) {
    if (*cols) cudaFreeAsync(*cols, s_);
    if (*vals) cudaFreeAsync(*vals, s_);
    *cols = nullptr;
    *vals = nullptr;
    *cap = (size_t)(*nnz * 1.25) + 16;
    CK(alloc(cols, *cap, s_));
    CK(alloc(vals, *cap, s_));
  }
  if (n_) k_row_fill<<<grid(n_), kThreads, 0, s_>>>(n_, row_off_, starts_out, ucol_, uval_, *cols, *vals);
  launches += 1;
  return cudaGetLastError();
}

cudaError_t IpDevice::csr_from_triplets(int64_t n, int64_t nt, const int32_t *row, const int32_t *col, const float *val, int64_t *starts, int32_t *cols, float *vals, int64_t *nnz) {
  release();
  keep_pool_once();
  n_ = n;
  CK(cudaFuncSetAttribute(k_row_collapse_block, cudaFuncAttributeMaxDynamicSharedMemorySize, kRowLong * (int)sizeof(unsigned long long)));
  CK(cudaFuncSetAttribute(k_row_collapse_long, cudaFuncAttributeMaxDynamicSharedMemorySize, kRowLong * (int)sizeof(unsigned long long)));
  CK(alloc(&row_off_, n_ + 1, s_));
  CK(alloc(&ucount_, n_ + 1, s_));
  CK(alloc(&fill_, n_, s_));
  CK(alloc(&tier_rows_, 4 * std::max<int64_t>(n_, 1), s_));
  CK(alloc(&tier_n_, 4, s_));
  CK(grow(s_, (size_t)std::max<int64_t>(nt, 1), w_cap_, &bucket_, &bucket2_, &ucol_, &uval_));
  size_t cap = (size_t)std::max<int64_t>(nt, 1);  // nnz <= nt: the caller's buffers suffice
  int32_t *c = cols;
  float *v = vals;
  CK(collapse(nt, row, col, val, starts, &c, &v, &cap, nnz));
  if (c != cols || v != vals) return cudaErrorUnknown;  // cannot happen: nnz <= nt
  return cudaStreamSynchronize(s_);
}

cudaError_t IpDevice::assemble(IpAxisResult out[2]) {
  IpArgs a{};
  a.n_nets = n_nets_;
  a.net_start = net_start_;
  a.pin_e = pin_e_;
  a.pin_inst = pin_inst_;
  a.pin_mio = pin_mio_;
  a.pin_xy = pin_xy_;
  a.pin_flag = pin_flag_;
  a.box = box_;
  a.locked = locked_;
  a.max_fanout = cfg_.max_fanout;
  a.min_diff = cfg_.min_diff;
  a.weight_scale = cfg_.weight_scale;
  const int64_t stride = (int64_t)n_nets_ + 1;
  if (n_nets_) {
    k_pin_info<<<grid(n_nets_), kThreads, 0, s_>>>(a);
    k_count<<<grid(n_nets_), kThreads, 0, s_>>>(a, cnt_, stride);
    launches += 2;
  }
  for (int q = 0; q < 4; q++) CK(scan(cnt_ + q * stride, n_nets_));
  int64_t tot[4];
  for (int q = 0; q < 4; q++) CK(cudaMemcpyAsync(&tot[q], cnt_ + q * stride + n_nets_, sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  d2h_bytes += 32;
  const bool first = t_cap_ == 0;
  if (first) progress("    round 1: triplets counted");
  // both axes side by side: x's triplets (the locked diagonal first) then y's; the same
  // for the right-hand-side terms
  const int64_t nt[2] = {n_locked_ + tot[0], n_locked_ + tot[1]}, nr[2] = {tot[2], tot[3]};
  CK(grow(s_, (size_t)(nt[0] + nt[1]), t_cap_, &t_row_, &t_col_, &t_val_));
  CK(grow(s_, (size_t)(nr[0] + nr[1]), r_cap_, &r_row_, &r_val_));
  CK(grow(s_, (size_t)std::max({nt[0], nt[1], nr[0], nr[1]}), w_cap_, &bucket_, &bucket2_, &ucol_, &uval_));
  if (first) {
    CK(cudaStreamSynchronize(s_));
    progress("    round 1: triplet buffers allocated");
  }
  AxisOut ox{}, oy{};
  ox.t_row = t_row_, ox.t_col = t_col_, ox.t_val = t_val_;
  oy.t_row = t_row_ + nt[0], oy.t_col = t_col_ + nt[0], oy.t_val = t_val_ + nt[0];
  ox.t_off = cnt_, oy.t_off = cnt_ + stride;
  ox.t_base = oy.t_base = n_locked_;
  ox.r_row = r_row_, ox.r_val = r_val_;
  oy.r_row = r_row_ + nr[0], oy.r_val = r_val_ + nr[0];
  ox.r_off = cnt_ + 2 * stride, oy.r_off = cnt_ + 3 * stride;
  if (n_) k_locked_and_x0<<<grid(n_), kThreads, 0, s_>>>(n_, box_, locked_, locked_rank_, ox, oy, ax_[0].x, ax_[1].x);
  if (n_nets_) k_emit<<<grid(n_nets_), kThreads, 0, s_>>>(a, ox, oy);
  launches += 2;
  CK(cudaGetLastError());
  if (first) {
    CK(cudaStreamSynchronize(s_));
    progress("    round 1: triplets emitted");
  }
  for (int ax = 0; ax < 2; ax++) {
    Axis &A = ax_[ax];
    int64_t o = ax ? nt[0] : 0;
    CK(collapse(nt[ax], t_row_ + o, t_col_ + o, t_val_ + o, A.starts, &A.cols, &A.vals, &A.cap, &A.nnz));
    if (first) {
      CK(cudaStreamSynchronize(s_));
      progress("    round 1: axis %d collapsed", ax);
    }
    out[ax].triplets = nt[ax];
    // the right-hand side: this axis's terms as one-column triplets, summed per row in order
    int64_t r = ax ? nr[0] : 0;
    CK(collapse(nr[ax], r_row_ + r, nullptr, r_val_ + r, nullptr, nullptr, nullptr, nullptr, nullptr));
    if (n_) {
      k_rhs<<<grid(n_), kThreads, 0, s_>>>(n_, ax, box_, locked_, row_off_, ucount_, uval_, A.rhs);
      launches += 1;
    }
    CK(cudaGetLastError());
  }
  return cudaStreamSynchronize(s_);
}

// The sliced copy: the rows in order of length and the count of long rows read back, the
// slice widths of the rest, their scan (the starts), the total read back to size the
// entries, then the entries.
cudaError_t IpDevice::slice(Axis &A, CsrDev m) {
  CK(grow(s_, (size_t)std::max<int64_t>(n_, 1), A.sl_row_cap, &A.sl_row, &A.sl_len));
  CK(grow(s_, (size_t)kSliceLenCap + 1, A.sl_count_cap, &A.sl_count));
  CK(csr_slice_order(m, A.sl_row, A.sl_len, A.sl_count, s_));
  int32_t n_long = 0;
  CK(cudaMemcpyAsync(&n_long, A.sl_count + kSliceLongRow + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  A.sl_long = n_long;
  const int64_t ns = (n_ - n_long + kSliceRows - 1) / kSliceRows;
  CK(grow(s_, (size_t)ns + 1, A.sl_start_cap, &A.sl_start));
  CK(csr_slice_widths(n_, n_long, A.sl_len, A.sl_start, s_));
  CK(scan(A.sl_start, ns));
  int64_t total = 0;
  CK(cudaMemcpyAsync(&total, A.sl_start + ns, sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  d2h_bytes += sizeof(int64_t) + sizeof(int32_t);
  CK(grow(s_, (size_t)std::max<int64_t>(total, 1), A.sl_cap, &A.sl_ent));
  m.sl_long = n_long;
  m.sl_row = A.sl_row;
  m.sl_len = A.sl_len;
  m.sl_start = A.sl_start;
  CK(csr_slice_fill(m, A.sl_ent, s_));
  launches += 8;
  return cudaSuccess;
}

// The rows sorted by the Hilbert index of their centres (the solve's start point) on a
// 1024 x 1024 grid over the core, and each axis's system and vectors renumbered.
cudaError_t IpDevice::solver_order() {
  const int64_t n = n_;
  if (!perm_) {
    const size_t tiles = (size_t)order_tiles((int32_t)n);
    CK(alloc(&perm_, (size_t)n, s_));
    CK(alloc(&inv_, (size_t)n, s_));
    CK(alloc(&ord_idx_, (size_t)n, s_));
    CK(alloc(&ord_hist_, 64 * tiles, s_));
    CK(alloc(&ord_key0_, (size_t)n, s_));
    CK(alloc(&ord_key1_, (size_t)n, s_));
  }
  const int4 c = cfg_.core;
  const double tw = std::max(1.0, (double)(c.z - c.x) / 1024.0), th = std::max(1.0, (double)(c.w - c.y) / 1024.0);
  CK(order_sort_xy((int32_t)n, ax_[0].x, ax_[1].x, (double)c.x, (double)c.y, tw, th, ord_key0_, perm_, ord_key1_, ord_idx_, ord_hist_, s_));
  k_perm_inv<<<grid(n), kThreads, 0, s_>>>(n, perm_, inv_);
  launches += 14;
  for (Axis &A : ax_) {
    CK(grow(s_, (size_t)std::max<int64_t>(A.nnz, 1), A.p_cap, &A.p_cols, &A.p_vals));
    if (!A.p_starts) {
      CK(alloc(&A.p_starts, (size_t)n + 1, s_));
      CK(alloc(&A.p_rhs, (size_t)n, s_));
      CK(alloc(&A.p_x, (size_t)n, s_));
    }
    k_perm_len<<<grid(n), kThreads, 0, s_>>>(n, perm_, A.starts, A.p_starts);
    CK(scan(A.p_starts, n));
    k_perm_rows<<<grid(n * 32), kThreads, 0, s_>>>(n, perm_, inv_, A.starts, A.cols, A.vals, A.p_starts, A.p_cols, A.p_vals);
    k_perm_gather<<<grid(n), kThreads, 0, s_>>>(n, perm_, A.rhs, A.p_rhs);
    k_perm_gather<<<grid(n), kThreads, 0, s_>>>(n, perm_, A.x, A.p_x);
    launches += 7;
  }
  return cudaGetLastError();
}

cudaError_t IpDevice::solve(int max_iters, IpAxisResult out[2]) {
  // the forms give the same products bit for bit, so the choice changes only the speed
  // GPL_SPMV_FORM=0|1|2 fixes the form (a thread per row, tiled, sliced); else the tuner picks
  // between the tiled and the sliced form (a thread per row is never the faster)
  if (!spmv_tune_) {
    spmv_tune_ = std::make_unique<Tuner>("initial placement SpMV", std::vector<std::string>{"tiled", "sliced"}, nullptr, 2, 48);
    if (const char *f = std::getenv("GPL_SPMV_FORM"))
      if (f[0] >= '0' && f[0] <= '2' && f[1] == 0) spmv_fixed_ = f[0] - '0';
  }
  if (ip_order_ < 0) {
    // off by default: measured, the x gathers' locality it buys (under 1 % of a batch) does
    // not pay for the renumbering each round
    const char *f = std::getenv("GPL_IP_ORDER");
    ip_order_ = f && f[0] == '1' ? 1 : 0;
  }
  // the first solve starts every row at one point (the core centre): no order to take yet
  const bool ordered = ip_order_ && solves_ > 0 && n_ > 0;
  solves_++;
  if (ordered) CK(solver_order());
  // the sliced copies whenever the sliced form may run
  const bool sliced = spmv_fixed_ < 0 || spmv_fixed_ == kSpmvSliced;
  CsrDev m[2];
  const float *b[2];
  float *x[2];
  void *scratch[2];
  for (int a = 0; a < 2; a++) {
    Axis &A = ax_[a];
    m[a] = ordered ? CsrDev{n_, A.p_starts, A.p_cols, A.p_vals} : CsrDev{n_, A.starts, A.cols, A.vals};
    if (sliced) {
      CK(slice(A, m[a]));
      m[a].sl_long = A.sl_long;
      m[a].sl_row = A.sl_row;
      m[a].sl_len = A.sl_len;
      m[a].sl_start = A.sl_start;
      m[a].sl_ent = A.sl_ent;
    }
    b[a] = ordered ? A.p_rhs : A.rhs;
    x[a] = ordered ? A.p_x : A.x;
    scratch[a] = (char *)scratch_ + a * scratch_bytes_;
  }
  BicgResult r[2]{};
  Tuner *t = spmv_fixed_ >= 0 ? nullptr : spmv_tune_.get();
  const int form = spmv_fixed_ >= 0 ? spmv_fixed_ : kSpmvTiled + spmv_tune_->best();
  cudaError_t e = bicgstab_solve_pair(m, b, x, max_iters, scratch, s_, r, form, t);
  const int iters = std::max(r[0].iterations, r[1].iterations);
  launches += 10 + (int64_t)iters * 7;
  d2h_bytes += (int64_t)(iters / 8 + 2) * 2 * 120;
  out[0].solve = r[0];
  out[1].solve = r[1];
  if (e == cudaSuccess && ordered) {
    for (Axis &A : ax_) k_perm_scatter<<<grid(n_), kThreads, 0, s_>>>(n_, perm_, A.p_x, A.x);
    launches += 2;
    e = cudaGetLastError();
  }
  return e;
}

cudaError_t IpDevice::hpwl(int64_t *out) {
  CK(cudaMemsetAsync(hpwl_acc_, 0, sizeof(int64_t), s_));
  if (n_nets_) {
    k_db_hpwl<<<grid(n_nets_), kThreads, 0, s_>>>(n_nets_, net_start_, pin_e_, pin_hp_, pin_static_, db_box_, (unsigned long long *)hpwl_acc_);
    launches += 1;
  }
  CK(cudaMemcpyAsync(out, hpwl_acc_, sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
  d2h_bytes += 8;
  return cudaStreamSynchronize(s_);
}

cudaError_t IpDevice::update() {
  if (n_) {
    k_update<<<grid(n_), kThreads, 0, s_>>>(n_, ax_[0].x, ax_[1].x, cfg_.core, clamp_, grouped_, locked_, box_, db_box_, db_size_);
    launches += 1;
  }
  if (n_pins_) {
    k_pins<<<grid(n_pins_), kThreads, 0, s_>>>(n_pins_, pin_e_, locked_, box_, pin_off_, pin_xy_);
    launches += 1;
  }
  return cudaGetLastError();
}

cudaError_t IpDevice::solution(int axis, std::vector<float> &x) {
  x.resize(n_);
  if (n_) CK(cudaMemcpyAsync(x.data(), ax_[axis].x, n_ * sizeof(float), cudaMemcpyDeviceToHost, s_));
  d2h_bytes += n_ * 4;
  return cudaStreamSynchronize(s_);
}

cudaError_t IpDevice::download(std::vector<int4> &box, std::vector<int4> &db_box) {
  box.resize(n_);
  db_box.resize(n_);
  if (n_) {
    CK(cudaMemcpyAsync(box.data(), box_, n_ * sizeof(int4), cudaMemcpyDeviceToHost, s_));
    CK(cudaMemcpyAsync(db_box.data(), db_box_, n_ * sizeof(int4), cudaMemcpyDeviceToHost, s_));
  }
  d2h_bytes += n_ * 32;
  return cudaStreamSynchronize(s_);
}

void keep_device_pool() { keep_pool_once(); }


// Loads this file's module (the driver loads a module at its first launch otherwise).
void load_module_b2b() {
  cudaFuncAttributes a;
  cudaFuncGetAttributes(&a, k_emit);
}

}  // namespace gpl
