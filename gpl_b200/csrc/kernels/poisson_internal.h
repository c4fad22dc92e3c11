// The density solver's internals: GEMM problem descriptors, the plan, the basis matrices.
#pragma once
#include <cstdint>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace gpl {

// D[m][n] = sum_k A[m][k] * B[n][k], row-major, leading dimensions in elements.
template <typename T>
struct GemmProblemT {
  int M, N, K;
  const T *A;
  int lda;
  const T *B;
  int ldb;
  T *D;
  int ldd;
};
template <typename T>
struct GemmBatchT {
  GemmProblemT<T> p[2];
};
using GemmProblem = GemmProblemT<float>;
using GemmBatch = GemmBatchT<float>;
cudaError_t sgemm_tn(const GemmBatch &gb, int count, cudaStream_t s);
cudaError_t dgemm_tn(const GemmBatchT<double> &gb, int count, cudaStream_t s);

// The six basis matrices in double (see poisson.cu): CyTs[v][y], CxTs[u][x] (forward, scaled
// and halved), Cy[y][v], Sy[y][v], Sx[x][u], Cx[x][u] (inverses).
struct BasisHost {
  std::vector<double> CyTs, CxTs, Cy, Sy, Sx, Cx;
};
void build_basis(int nx, int ny, BasisHost &b);

// The plans' device memory comes from the device's stream-ordered pool (kept warm, so a plan
// made after another, or after the initial placement, maps no new memory), ordered on the
// legacy stream: a plan or group is complete once its create has synchronised that stream,
// and its destroy synchronises the device before it returns the memory, as cudaFree would.
inline cudaError_t pool_alloc(void **p, size_t bytes) { return cudaMallocAsync(p, bytes, 0); }
inline cudaError_t pool_upload(void *d, const void *h, size_t bytes) { return cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, 0); }
inline void pool_free(void *p) {
  if (p) cudaFreeAsync(p, 0);
}

struct TcState;  // the split-BF16 tensor-core path's buffers (poisson_tc.cu)

struct PoissonPlan {
  int nx = 0, ny = 0, mode = 0;
  float *wx = nullptr, *wx2 = nullptr, *wy = nullptr, *wy2 = nullptr;
  // FP32 path
  float *CyTs = nullptr, *CxTs = nullptr, *Cy = nullptr, *Sy = nullptr, *Sx = nullptr, *Cx = nullptr;
  float *t1 = nullptr, *ah = nullptr, *exh = nullptr, *eyh = nullptr, *t2 = nullptr, *t3 = nullptr;
  // tensor-core path
  __nv_bfloat16 *tc_dens = nullptr;  // density as [nx][2*ny] bf16 (hi | lo)
  TcState *tc = nullptr;
  // FP64 path (the yardstick): the FP32 path's matrices and sequence in double
  double *d_basis[6] = {};           // CyTs, CxTs, Cy, Sy, Sx, Cx
  double *d_buf[8] = {};             // rho, t1, ah, exh, eyh, t2, t3, and the fields' staging
};

cudaError_t tc_plan_init(PoissonPlan *p, const BasisHost &b);
void tc_plan_free(PoissonPlan *p);
cudaError_t tc_solve(PoissonPlan *p, float *field_x, float *field_y, cudaStream_t s);
int tc_launches(const PoissonPlan *p);

}  // namespace gpl
