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
// Scratch the solve needs (seven vectors of n floats, the partials and the scalars).
size_t bicgstab_scratch_bytes(int64_t n);
// Solve A x = b from the start point in x; `scratch` holds bicgstab_scratch_bytes(n) bytes.
cudaError_t bicgstab_solve(const CsrDev &A, const float *b, float *x, int max_iters, void *scratch, cudaStream_t s, BicgResult *out);

}  // namespace gpl
