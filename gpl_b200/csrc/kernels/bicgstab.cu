// The initial placement's solver (`bicgstab`, src/bicgstab.rs:615-669) on the device: CSR
// SpMV with each row summed in column order (the reference's `Csr::mul` order), float vectors,
// and the inner products and residual norms in double (deterministic block partials). The
// scalars (rho, alpha, omega) live on the device; the host reads two numbers per iteration
// (the residual norm and the next rho) to run the loop's tests, restart included.
#include "bicgstab.h"
#include "common.cuh"

namespace gpl {

namespace {

enum Scal { S_RHO = 0, S_RHO_OLD, S_ALPHA, S_W, S_RR, S_R0R, S_R0SQ, S_BB, S_COUNT };

// y = A x, then `0 + 1 * tmp` as the library writes it. A block's rows are contiguous in
// the CSR arrays: the block first forms every product vals[k] * x[cols[k]] of its rows with
// coalesced loads into shared memory, then each thread sums its row's products in column
// order (the reference's order). A block whose rows hold more than kSpmvTile entries sums
// straight from memory.
constexpr int kSpmvTile = 6144;

__global__ void __launch_bounds__(kThreads) k_spmv(int64_t n, const int64_t *__restrict__ rs, const int32_t *__restrict__ cols, const float *__restrict__ vals, const float *__restrict__ x, float *__restrict__ y) {
  __shared__ float prod[kSpmvTile];
  const int64_t r0 = blockIdx.x * (int64_t)blockDim.x;
  const int64_t r1 = min(n, r0 + (int64_t)blockDim.x);
  const int64_t k0 = rs[r0], k1 = rs[r1];
  const bool tiled = k1 - k0 <= kSpmvTile;
  if (tiled)
    for (int64_t k = k0 + threadIdx.x; k < k1; k += blockDim.x) prod[k - k0] = __fmul_rn(vals[k], x[cols[k]]);
  __syncthreads();
  const int64_t i = r0 + threadIdx.x;
  if (i >= n) return;
  float tmp = 0.0f;
  if (tiled)
    for (int64_t k = rs[i]; k < rs[i + 1]; k++) tmp = __fadd_rn(tmp, prod[k - k0]);
  else
    for (int64_t k = rs[i]; k < rs[i + 1]; k++) tmp = __fadd_rn(tmp, __fmul_rn(vals[k], x[cols[k]]));
  y[i] = __fadd_rn(0.0f, __fmul_rn(1.0f, tmp));
}

// Up to three dot products at once; partials[blk * 3 + j].
__global__ void k_dots(int64_t n, const float *__restrict__ a0, const float *__restrict__ b0, const float *__restrict__ a1, const float *__restrict__ b1, const float *__restrict__ a2, const float *__restrict__ b2, double *__restrict__ part) {
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
}

// Reduce the partials and apply one scalar step:
//  which 0: S[dst0..dst0+2] = sums
//  which 1 (alpha): S_ALPHA = rho / sum0
//  which 2 (omega): S_W = sum0 > 0 ? sum1 / sum0 : 0
//  which 3 (end of iteration): S_RR = sum0; S_RHO_OLD = S_RHO; S_RHO = sum1
//  which 4 (restart): S_R0SQ = S_RHO = S_RR = sum0
__global__ void k_scalar(const double *__restrict__ part, int nblk, double *__restrict__ S, int which, int dst0) {
  __shared__ double sh[kThreads / 32];
  double v[3];
  for (int j = 0; j < 3; j++) {
    double s = 0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += part[3 * b + j];
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
      break;
    case 4:
      S[S_R0SQ] = v[0];
      S[S_RHO] = v[0];
      S[S_RR] = v[0];
      break;
  }
}

__global__ void k_residual(int64_t n, const float *__restrict__ b, const float *__restrict__ ax, float *__restrict__ r, float *__restrict__ r0) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float v = __fsub_rn(b[i], ax[i]);
  r[i] = v;
  r0[i] = v;
}

// p = r + beta (p - w v), beta = (rho / rho_old) (alpha / w)
__global__ void k_update_p(int64_t n, const double *__restrict__ S, const float *__restrict__ r, const float *__restrict__ v, float *__restrict__ p) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float beta = (float)((S[S_RHO] / S[S_RHO_OLD]) * (S[S_ALPHA] / S[S_W]));
  float w = (float)S[S_W];
  p[i] = __fadd_rn(r[i], __fmul_rn(beta, __fsub_rn(p[i], __fmul_rn(w, v[i]))));
}

__global__ void k_update_s(int64_t n, const double *__restrict__ S, const float *__restrict__ r, const float *__restrict__ v, float *__restrict__ s) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float a = (float)S[S_ALPHA];
  s[i] = __fsub_rn(r[i], __fmul_rn(a, v[i]));
}

// x += alpha p + w s; r = s - w t; partials of |r|^2 and r0.r
__global__ void k_update_xr(int64_t n, const double *__restrict__ S, const float *__restrict__ p, const float *__restrict__ s, const float *__restrict__ t, const float *__restrict__ r0, float *__restrict__ x, float *__restrict__ r, double *__restrict__ part) {
  __shared__ double sh[kThreads / 32];
  float a = (float)S[S_ALPHA], w = (float)S[S_W];
  double rr = 0, r0r = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] = __fadd_rn(x[i], __fadd_rn(__fmul_rn(a, p[i]), __fmul_rn(w, s[i])));
    float rv = __fsub_rn(s[i], __fmul_rn(w, t[i]));
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
}

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

size_t bicgstab_scratch_bytes(int64_t n) {
  size_t vec = (size_t)n * sizeof(float);
  vec = (vec + 255) / 256 * 256;
  return 7 * vec + (size_t)kBicgBlocks * 3 * sizeof(double) + 64 * sizeof(double);
}

cudaError_t bicgstab_solve(const CsrDev &A, const float *b, float *x, int max_iters, void *scratch, cudaStream_t st, BicgResult *out) {
  int64_t n = A.n;
  size_t vec = ((size_t)n * sizeof(float) + 255) / 256 * 256;
  char *base = (char *)scratch;
  float *r = (float *)(base), *r0 = (float *)(base + vec), *v = (float *)(base + 2 * vec), *p = (float *)(base + 3 * vec);
  float *s = (float *)(base + 4 * vec), *t = (float *)(base + 5 * vec), *ax = (float *)(base + 6 * vec);
  double *part = (double *)(base + 7 * vec);
  double *S = part + (size_t)kBicgBlocks * 3;
  int eb = (int)((n + kThreads - 1) / kThreads);
  if (eb < 1) eb = 1;
  int rb = kBicgBlocks;
  const float tol = 1.1920929e-07f;
  double hs[S_COUNT];
  auto spmv = [&](const float *in, float *o) { k_spmv<<<eb, kThreads, 0, st>>>(n, A.rs, A.cols, A.vals, in, o); };
  auto pull = [&]() -> cudaError_t {
    cudaError_t e = cudaMemcpyAsync(hs, S, sizeof hs, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);
  };
  cudaError_t e;
  spmv(x, ax);
  k_residual<<<eb, kThreads, 0, st>>>(n, b, ax, r, r0);
  k_dots<<<rb, kThreads, 0, st>>>(n, r0, r0, b, b, r0, r, part);
  k_scalar<<<1, kThreads, 0, st>>>(part, rb, S, 0, S_R0SQ);  // S_R0SQ, S_BB, then dot(r0, r) in S[S_COUNT]
  if ((e = pull()) != cudaSuccess) return e;
  double r0_sqnorm = hs[S_R0SQ], rhs_sqnorm = hs[S_BB];
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
  double rr = r0_sqnorm;       // r == r0 at the start
  double rho_next = r0_sqnorm;  // dot(r0, r)
  int i = 0, restarts = 0;
  while (rr > tol2 && i < max_iters) {
    if (std::fabs(rho_next) < eps2 * r0_sqnorm) {
      // too orthogonal to r0: restart from the current residual
      spmv(x, ax);
      k_residual<<<eb, kThreads, 0, st>>>(n, b, ax, r, r0);
      k_dots<<<rb, kThreads, 0, st>>>(n, r, r, nullptr, nullptr, nullptr, nullptr, part);
      k_scalar<<<1, kThreads, 0, st>>>(part, rb, S, 4, 0);
      if ((e = pull()) != cudaSuccess) return e;
      r0_sqnorm = hs[S_R0SQ];
      if (restarts == 0) i = 0;
      restarts++;
    }
    k_update_p<<<eb, kThreads, 0, st>>>(n, S, r, v, p);
    spmv(p, v);
    k_dots<<<rb, kThreads, 0, st>>>(n, r0, v, nullptr, nullptr, nullptr, nullptr, part);
    k_scalar<<<1, kThreads, 0, st>>>(part, rb, S, 1, 0);
    k_update_s<<<eb, kThreads, 0, st>>>(n, S, r, v, s);
    spmv(s, t);
    k_dots<<<rb, kThreads, 0, st>>>(n, t, t, t, s, nullptr, nullptr, part);
    k_scalar<<<1, kThreads, 0, st>>>(part, rb, S, 2, 0);
    k_update_xr<<<rb, kThreads, 0, st>>>(n, S, p, s, t, r0, x, r, part);
    k_scalar<<<1, kThreads, 0, st>>>(part, rb, S, 3, 0);
    if ((e = pull()) != cudaSuccess) return e;
    rr = hs[S_RR];
    rho_next = hs[S_RHO];
    i++;
  }
  out->iterations = i;
  out->error = (float)std::sqrt(rr / rhs_sqnorm);
  out->converged = out->error <= tol;
  return cudaGetLastError();
}

}  // namespace gpl
