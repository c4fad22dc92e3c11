// The initial placement's BiCGSTAB on the device (src/bicgstab.rs:615-669).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace gpl {

constexpr int kBicgBlocks = 296;  // two blocks per SM for the reductions

struct CsrDev {
  int64_t n;
  const int64_t *rs;
  const int32_t *cols;
  const float *vals;
};
struct BicgResult {
  int iterations;
  float error;
  bool converged;
};
// The SpMV's two forms, bit for bit the same y: a thread per row straight from memory (best
// when a row's columns are scattered: the gathers from x overlap across the block), or a
// block's products staged through shared memory with coalesced loads (best when columns lie
// near their rows).
enum SpmvForm { kSpmvRows = 0, kSpmvTiled = 1 };
// Scratch the solve needs (seven vectors of n floats, the partials and the scalars).
size_t bicgstab_scratch_bytes(int64_t n);
// Solve A x = b from the start point in x; `scratch` holds bicgstab_scratch_bytes(n) bytes.
cudaError_t bicgstab_solve(const CsrDev &A, const float *b, float *x, int max_iters, void *scratch, cudaStream_t s, BicgResult *out, int spmv = kSpmvRows);
// y = A x in the given form (SpmvForm).
cudaError_t spmv(const CsrDev &A, const float *x, float *y, int form, cudaStream_t s);
// Two systems of the same size solved side by side (each launch carries both): each takes
// exactly the steps, and gives exactly the result, of bicgstab_solve on its own; scratch[a]
// holds bicgstab_scratch_bytes(n) bytes for system a.
cudaError_t bicgstab_solve_pair(const CsrDev A[2], const float *const b[2], float *const x[2], int max_iters, void *const scratch[2], cudaStream_t s, BicgResult out[2], int spmv = kSpmvRows);
// The faster SpMV form for A, timed on the device (a few products of x into the scratch).
cudaError_t bicgstab_pick_spmv(const CsrDev &A, const float *x, void *scratch, cudaStream_t s, int *form);

}  // namespace gpl
