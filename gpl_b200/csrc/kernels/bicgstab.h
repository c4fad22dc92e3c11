// The initial placement's BiCGSTAB on the device (src/bicgstab.rs:615-669).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace gpl {

class Tuner;

constexpr int kBicgBlocks = 296;  // two blocks per SM for the reductions

// Rows per slice of the sliced copy of a matrix (below).
constexpr int kSliceRows = 32;
struct CsrDev {
  int64_t n;
  const int64_t *rs;
  const int32_t *cols;
  const float *vals;
  // Optional: the rows in order of length (longest first; the order within a length does
  // not matter): the row at position j is sl_row[j], of sl_len[j] entries. The first sl_long
  // positions (rows over kSliceLongRow entries) are read from the CSR arrays, a warp per row;
  // the rest are cut into slices of kSliceRows positions, each slice stored column-major at
  // its longest row's width: with i = j - sl_long, entry k sits at sl_start[i / kSliceRows] +
  // kSliceRows * k + i % kSliceRows, so a warp's k-th entries are one coalesced run and its
  // rows end together; an entry is one 8-byte word (x: the column, y: the value's bits), so
  // a step is one load. Built by csr_slice_order, csr_slice_widths, a scan, and
  // csr_slice_fill; NULL when not built.
  int64_t sl_long = 0;
  const int32_t *sl_row = nullptr;
  const int32_t *sl_len = nullptr;
  const int64_t *sl_start = nullptr;
  const int2 *sl_ent = nullptr;
};
struct BicgResult {
  int iterations;
  float error;
  bool converged;
};
// The SpMV's forms, bit for bit the same y: a thread per row straight from memory (best
// when a row's columns are scattered: the gathers from x overlap across the block), a
// block's products staged through shared memory with coalesced loads (best when columns lie
// near their rows), or a thread per row over the sliced copy (coalesced without staging;
// needs the copy).
enum SpmvForm { kSpmvRows = 0, kSpmvTiled = 1, kSpmvSliced = 2 };
// The sliced copy's row order: rows by length, longest first (lengths from kSliceLenCap up
// count as one), into row[n] and len[n]; `count` holds kSliceLenCap + 1 ints of scratch, and
// count[kSliceLongRow + 1] ends as the number of rows over kSliceLongRow entries (sl_long).
constexpr int kSliceLenCap = 1024;
constexpr int kSliceLongRow = 64;
cudaError_t csr_slice_order(const CsrDev &A, int32_t *row, int32_t *len, int32_t *count, cudaStream_t s);
// The slice widths: for each of the ceil((n - n_long) / kSliceRows) slices after the first
// n_long positions, kSliceRows times its longest row's length into widths[slice]; an
// exclusive scan of them (total at [slices]) gives sl_start.
cudaError_t csr_slice_widths(int64_t n, int64_t n_long, const int32_t *len, int64_t *widths, cudaStream_t s);
// The sliced copy's entries from A's CSR arrays (A.sl_long, sl_row, sl_len, sl_start set).
cudaError_t csr_slice_fill(const CsrDev &A, int2 *sl_ent, cudaStream_t s);
// Scratch the solve needs (seven vectors of n floats, the partials and the scalars).
size_t bicgstab_scratch_bytes(int64_t n);
// Solve A x = b from the start point in x; `scratch` holds bicgstab_scratch_bytes(n) bytes.
cudaError_t bicgstab_solve(const CsrDev &A, const float *b, float *x, int max_iters, void *scratch, cudaStream_t s, BicgResult *out, int spmv = kSpmvRows);
// y = A x in the given form (SpmvForm).
cudaError_t spmv(const CsrDev &A, const float *x, float *y, int form, cudaStream_t s);
// Two systems of the same size solved side by side (each launch carries both): each takes
// the steps of bicgstab_solve on its own; scratch[a] holds bicgstab_pair_scratch_bytes(n)
// bytes for system a.
size_t bicgstab_pair_scratch_bytes(int64_t n);
// With `tune` (two candidates: the tiled and the sliced form), each batch of iterations runs
// the form the tuner picks (A then needs its sliced copy), timed in place; `spmv` is then the
// form of the start and restarts.
cudaError_t bicgstab_solve_pair(const CsrDev A[2], const float *const b[2], float *const x[2], int max_iters, void *const scratch[2], cudaStream_t s, BicgResult out[2], int spmv = kSpmvRows, Tuner *tune = nullptr);

}  // namespace gpl
