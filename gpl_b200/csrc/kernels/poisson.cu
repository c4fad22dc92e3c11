// The density solver (`Fft::solve`, src/nesterov.rs:412-444) as dense transforms: each 2-D
// cosine/sine transform of Ooura's package (src/ooura.rs:71-98) is a product with basis
// matrices on both sides, B_x^T * A * B_y, so the solve is six GEMMs and one spectral step:
//
//   T1t[v][x] = sum_y CyTs[v][y] rho[x][y]        forward along y (scale and halving folded in)
//   Ah[u][v]  = sum_x CxTs[u][x] T1t[v][x]        forward along x
//   Exh = Ah wx/(wx^2+wy^2), Eyh = Ah wy/(wx^2+wy^2), 0 at (0,0)
//   T2t[y][u] = sum_v Cy[y][v] Exh[u][v]   ;  Ex[x][y] = sum_u Sx[x][u] T2t[y][u]   (ddsct2d)
//   T3t[y][u] = sum_v Sy[y][v] Eyh[u][v]   ;  Ey[x][y] = sum_u Cx[x][u] T3t[y][u]   (ddcst2d)
//
// Every GEMM is D[m][n] = sum_k A[m][k] B[n][k] with both operands K-contiguous. The forward
// halving of row and column 0 and the 4/(nx*ny) scale are separable (h_u h_v (2/nx)(2/ny);
// the (0,0) term they disagree on is zeroed by the solve). Ooura's sine inverse keeps A[n] in
// a[0]; its basis column 0 is therefore (-1)^x. The potential is not computed: nothing but
// the reference's probes reads it.
//
// Mode 0 (this file): FP32 SIMT GEMMs. Mode 1: split-BF16 tcgen05 GEMMs (poisson_tc.cu).
// Mode 2 (this file): the FP32 form's sequence in double, the precision yardstick.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "engine_kernels.h"
#include "poisson_internal.h"
#include "parallel.h"

namespace gpl {
void progress(const char *fmt, ...) __attribute__((format(printf, 1, 2)));

// ---------------------------------------------------------------- FP32 SIMT GEMM
// 128 x 64 output tile per block, K-step 8, 256 threads with 8 x 4 outputs each.
constexpr int SG_BM = 128, SG_BN = 64, SG_BK = 8;

// One 128 x 64 output tile of D = A B^T from (m0, n0).
template <typename T>
__device__ __forceinline__ void gemm_tile(const GemmProblemT<T> &P, const int m0, const int n0) {
  __shared__ __align__(16) T As[SG_BK][SG_BM + 4];
  __shared__ __align__(16) T Bs[SG_BK][SG_BN + 4];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int ar = tid >> 1, ak = (tid & 1) * 4;  // A loader: row, first k
  const int br = tid >> 2, bk = (tid & 3) * 2;  // B loader
  T acc[8][4];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = (T)0;
  T ra[4], rb[2];
  auto load = [&](int k0) {
    int gm = m0 + ar;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      int gk = k0 + ak + q;
      ra[q] = (gm < P.M && gk < P.K) ? P.A[(size_t)gm * P.lda + gk] : (T)0;
    }
    int gn = n0 + br;
#pragma unroll
    for (int q = 0; q < 2; q++) {
      int gk = k0 + bk + q;
      rb[q] = (gn < P.N && gk < P.K) ? P.B[(size_t)gn * P.ldb + gk] : (T)0;
    }
  };
  load(0);
  for (int k0 = 0; k0 < P.K; k0 += SG_BK) {
#pragma unroll
    for (int q = 0; q < 4; q++) As[ak + q][ar] = ra[q];
#pragma unroll
    for (int q = 0; q < 2; q++) Bs[bk + q][br] = rb[q];
    __syncthreads();
    if (k0 + SG_BK < P.K) load(k0 + SG_BK);
#pragma unroll
    for (int kk = 0; kk < SG_BK; kk++) {
      T a[8], b[4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        a[q] = As[kk][ty * 4 + q];
        a[4 + q] = As[kk][64 + ty * 4 + q];
        b[q] = Bs[kk][tx * 4 + q];
      }
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 8; i++) {
    int gm = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
    if (gm >= P.M) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      int gn = n0 + tx * 4 + j;
      if (gn < P.N) P.D[(size_t)gm * P.ldd + gn] = acc[i][j];
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_gemm_tn(GemmBatchT<T> gb) {
  const GemmProblemT<T> P = gb.p[blockIdx.z];
  const int m0 = blockIdx.y * SG_BM, n0 = blockIdx.x * SG_BN;
  if (m0 >= P.M || n0 >= P.N) return;
  gemm_tile<T>(P, m0, n0);
}

// Many problems in one launch: block b takes tile b - first[k] of problem k (the last with
// first[k] <= b), tiles row-major over the problem's (M / 128) x (N / 64) grid.
__global__ void __launch_bounds__(256) k_gemm_grouped(const GemmProblem *__restrict__ probs, const int *__restrict__ first, int n) {
  __shared__ int s_k;
  if (threadIdx.x == 0) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (first[mid] <= (int)blockIdx.x) lo = mid; else hi = mid - 1;
    }
    s_k = lo;
  }
  __syncthreads();
  const GemmProblem P = probs[s_k];
  const int t = (int)blockIdx.x - first[s_k];
  const int tn = (P.N + SG_BN - 1) / SG_BN;
  gemm_tile<float>(P, (t / tn) * SG_BM, (t % tn) * SG_BN);
}

template <typename T>
cudaError_t gemm_tn(const GemmBatchT<T> &gb, int count, cudaStream_t s) {
  int M = 0, N = 0;
  for (int i = 0; i < count; i++) {
    M = M > gb.p[i].M ? M : gb.p[i].M;
    N = N > gb.p[i].N ? N : gb.p[i].N;
  }
  dim3 grid((N + SG_BN - 1) / SG_BN, (M + SG_BM - 1) / SG_BM, count);
  k_gemm_tn<T><<<grid, 256, 0, s>>>(gb);
  return cudaGetLastError();
}
cudaError_t sgemm_tn(const GemmBatch &gb, int count, cudaStream_t s) { return gemm_tn<float>(gb, count, s); }
cudaError_t dgemm_tn(const GemmBatchT<double> &gb, int count, cudaStream_t s) { return gemm_tn<double>(gb, count, s); }

// ---------------------------------------------------------------- the spectral step
// (src/nesterov.rs:425-440) on the scaled forward transform: phi = Ah / (wx2 + wy2),
// Ex = phi wx, Ey = phi wy, in float as the reference; all three zero at (0, 0).
__global__ void k_spectral(int nx, int ny, const float *__restrict__ ah, const float *__restrict__ wx, const float *__restrict__ wx2, const float *__restrict__ wy, const float *__restrict__ wy2, float *__restrict__ exh, float *__restrict__ eyh) {
  int64_t n = (int64_t)nx * ny;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    int u = (int)(k / ny), v = (int)(k % ny);
    float ex = 0.0f, ey = 0.0f;
    if (u != 0 || v != 0) {
      float p = __fdiv_rn(ah[k], __fadd_rn(wx2[u], wy2[v]));
      ex = __fmul_rn(p, wx[u]);
      ey = __fmul_rn(p, wy[v]);
    }
    exh[k] = ex;
    eyh[k] = ey;
  }
}
// The FP64 yardstick's spectral step: the same in double (wavenumbers widened from float).
__global__ void k_spectral_d(int nx, int ny, const double *__restrict__ ah, const float *__restrict__ wx, const float *__restrict__ wy, double *__restrict__ exh, double *__restrict__ eyh) {
  int64_t n = (int64_t)nx * ny;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    int u = (int)(k / ny), v = (int)(k % ny);
    double ex = 0.0, ey = 0.0;
    if (u != 0 || v != 0) {
      const double a = (double)wx[u], b = (double)wy[v];
      const double p = ah[k] / (a * a + b * b);
      ex = p * a;
      ey = p * b;
    }
    exh[k] = ex;
    eyh[k] = ey;
  }
}
template <typename A, typename B>
__global__ void k_convert(int64_t n, const A *__restrict__ in, B *__restrict__ out) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) out[k] = (B)in[k];
}

// ---------------------------------------------------------------- basis matrices (host)
// Built in double from exact arguments, rounded once.
void build_basis(int nx, int ny, BasisHost &b) {
  auto cosv = [](int k, int j, int n) { return std::cos(M_PI * (double)k * ((double)j + 0.5) / (double)n); };
  auto sinv = [](int k, int j, int n) { return k == 0 ? ((j & 1) ? -1.0 : 1.0) : std::sin(M_PI * (double)k * ((double)j + 0.5) / (double)n); };
  b.CyTs.assign((size_t)ny * ny, 0);
  b.Cy.assign((size_t)ny * ny, 0);
  b.Sy.assign((size_t)ny * ny, 0);
  parallel_for((size_t)ny, [&](size_t v0, size_t v1) {
    for (int v = (int)v0; v < (int)v1; v++)
      for (int y = 0; y < ny; y++) {
        double h = (v == 0 ? 0.5 : 1.0) * 2.0 / (double)ny;
        b.CyTs[(size_t)v * ny + y] = h * cosv(v, y, ny);
        b.Cy[(size_t)y * ny + v] = cosv(v, y, ny);
        b.Sy[(size_t)y * ny + v] = sinv(v, y, ny);
      }
  }, 16);
  b.CxTs.assign((size_t)nx * nx, 0);
  b.Cx.assign((size_t)nx * nx, 0);
  b.Sx.assign((size_t)nx * nx, 0);
  parallel_for((size_t)nx, [&](size_t u0, size_t u1) {
    for (int u = (int)u0; u < (int)u1; u++)
      for (int x = 0; x < nx; x++) {
        double h = (u == 0 ? 0.5 : 1.0) * 2.0 / (double)nx;
        b.CxTs[(size_t)u * nx + x] = h * cosv(u, x, nx);
        b.Cx[(size_t)x * nx + u] = cosv(u, x, nx);
        b.Sx[(size_t)x * nx + u] = sinv(u, x, nx);
      }
  }, 16);
}

static cudaError_t upload_f32(const std::vector<double> &h, float **d) {
  std::vector<float> f(h.size());
  for (size_t i = 0; i < h.size(); i++) f[i] = (float)h[i];
  cudaError_t e = pool_alloc((void **)d, f.size() * sizeof(float));
  if (e != cudaSuccess) return e;
  return pool_upload(*d, f.data(), f.size() * sizeof(float));
}

size_t poisson_workspace_bytes(int nx, int ny) {
  size_t n = (size_t)nx * ny;
  size_t basis = 3 * (size_t)nx * nx + 3 * (size_t)ny * ny;
  return (basis + 6 * n) * sizeof(float) + 2 * (size_t)(nx + ny) * sizeof(float);
}

PoissonPlan *poisson_plan_create(int nx, int ny, const float *wx_host, const float *wy_host, int mode, cudaError_t *err) {
  PoissonPlan *p = new PoissonPlan();
  p->nx = nx;
  p->ny = ny;
  // the tensor-core tiles are 128 x 64 with K-blocks of 64: a grid whose sides are not
  // multiples of 128 (small or odd -bin_grid_count grids) is solved with the FP32 GEMMs
  if (mode == 1 && (nx % 128 != 0 || ny % 128 != 0)) mode = 0;
  p->mode = mode;
  *err = cudaSuccess;
  std::vector<float> w2((size_t)nx + ny);
  BasisHost b;
  build_basis(nx, ny, b);
  if (nx >= 512) progress("    plan: bases built");
  size_t n = (size_t)nx * ny;
#define TRY(x)              \
  do {                      \
    cudaError_t e_ = (x);   \
    if (e_ != cudaSuccess) { \
      *err = e_;            \
      poisson_plan_destroy(p); \
      return nullptr;       \
    }                       \
  } while (0)
  TRY(pool_alloc((void **)&p->wx, nx * sizeof(float)));
  TRY(pool_alloc((void **)&p->wx2, nx * sizeof(float)));
  TRY(pool_alloc((void **)&p->wy, ny * sizeof(float)));
  TRY(pool_alloc((void **)&p->wy2, ny * sizeof(float)));
  std::vector<float> sq(std::max(nx, ny));
  for (int i = 0; i < nx; i++) sq[i] = wx_host[i] * wx_host[i];
  TRY(pool_upload(p->wx, wx_host, nx * sizeof(float)));
  TRY(pool_upload(p->wx2, sq.data(), nx * sizeof(float)));
  for (int i = 0; i < ny; i++) sq[i] = wy_host[i] * wy_host[i];
  TRY(pool_upload(p->wy, wy_host, ny * sizeof(float)));
  TRY(pool_upload(p->wy2, sq.data(), ny * sizeof(float)));
  if (mode == 2) {
    const std::vector<double> *mats[6] = {&b.CyTs, &b.CxTs, &b.Cy, &b.Sy, &b.Sx, &b.Cx};
    for (int k = 0; k < 6; k++) {
      TRY(pool_alloc((void **)&p->d_basis[k], mats[k]->size() * sizeof(double)));
      TRY(pool_upload(p->d_basis[k], mats[k]->data(), mats[k]->size() * sizeof(double)));
    }
    for (int k = 0; k < 8; k++) TRY(pool_alloc((void **)&p->d_buf[k], n * sizeof(double)));
  } else if (mode == 0) {
    TRY(upload_f32(b.CyTs, &p->CyTs));
    TRY(upload_f32(b.CxTs, &p->CxTs));
    TRY(upload_f32(b.Cy, &p->Cy));
    TRY(upload_f32(b.Sy, &p->Sy));
    TRY(upload_f32(b.Sx, &p->Sx));
    TRY(upload_f32(b.Cx, &p->Cx));
    TRY(pool_alloc((void **)&p->t1, n * sizeof(float)));
    TRY(pool_alloc((void **)&p->ah, n * sizeof(float)));
    TRY(pool_alloc((void **)&p->exh, n * sizeof(float)));
    TRY(pool_alloc((void **)&p->eyh, n * sizeof(float)));
    TRY(pool_alloc((void **)&p->t2, n * sizeof(float)));
    TRY(pool_alloc((void **)&p->t3, n * sizeof(float)));
  } else {
    if (nx >= 512) progress("    plan: wavenumbers uploaded");
    cudaError_t e = tc_plan_init(p, b);
    if (e != cudaSuccess) {
      *err = e;
      poisson_plan_destroy(p);
      return nullptr;
    }
  }
#undef TRY
  if ((*err = cudaStreamSynchronize(0)) != cudaSuccess) {
    poisson_plan_destroy(p);
    return nullptr;
  }
  return p;
}

void poisson_plan_destroy(PoissonPlan *p) {
  if (!p) return;
  cudaDeviceSynchronize();
  float *bufs[] = {p->wx, p->wx2, p->wy, p->wy2, p->CyTs, p->CxTs, p->Cy, p->Sy, p->Sx, p->Cx, p->t1, p->ah, p->exh, p->eyh, p->t2, p->t3};
  for (float *b : bufs)
    pool_free(b);
  for (double *b : p->d_basis)
    pool_free(b);
  for (double *b : p->d_buf)
    pool_free(b);
  tc_plan_free(p);
  delete p;
}

__nv_bfloat16 *poisson_split_input(PoissonPlan *p, int *ld) {
  if (p->mode != 1) return nullptr;
  *ld = 2 * p->ny;
  return p->tc_dens;
}

__global__ void k_split_density(int nx, int ny, const float *__restrict__ d, __nv_bfloat16 *__restrict__ out, int ld) {
  int64_t n = (int64_t)nx * ny;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    int64_t x = k / ny, y = k % ny;
    float v = d[k];
    __nv_bfloat16 hi = __float2bfloat16_rn(v);
    out[x * ld + y] = hi;
    out[x * ld + ny + y] = __float2bfloat16_rn(v - __bfloat162float(hi));
  }
}

cudaError_t poisson_split_density(PoissonPlan *p, const float *density, cudaStream_t s) {
  if (p->mode != 1) return cudaSuccess;
  int64_t n = (int64_t)p->nx * p->ny;
  int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
  k_split_density<<<blocks, 256, 0, s>>>(p->nx, p->ny, density, p->tc_dens, 2 * p->ny);
  return cudaGetLastError();
}

int poisson_plan_mode(const PoissonPlan *p) { return p->mode; }

int poisson_launches(const PoissonPlan *p) { return p->mode == 0 ? 5 : p->mode == 2 ? 9 : tc_launches(p); }

// The FP64 form: the density widened to double, the FP32 form's six GEMMs and spectral step
// in double throughout, the fields rounded to float once at the end. The yardstick the
// other forms' placements are compared with; not a speed path.
static cudaError_t solve_fp64(PoissonPlan *p, const float *density, float *field_x, float *field_y, cudaStream_t s) {
  const int nx = p->nx, ny = p->ny;
  const int64_t n = (int64_t)nx * ny;
  const int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
  double *const *B = p->d_basis;
  double *rho = p->d_buf[0], *t1 = p->d_buf[1], *ah = p->d_buf[2], *exh = p->d_buf[3], *eyh = p->d_buf[4], *t2 = p->d_buf[5], *t3 = p->d_buf[6], *f = p->d_buf[7];
  k_convert<float, double><<<blocks, 256, 0, s>>>(n, density, rho);
  GemmBatchT<double> g{};
  g.p[0] = GemmProblemT<double>{ny, nx, ny, B[0], ny, rho, ny, t1, nx};
  cudaError_t e = gemm_tn<double>(g, 1, s);
  if (e != cudaSuccess) return e;
  g.p[0] = GemmProblemT<double>{nx, ny, nx, B[1], nx, t1, nx, ah, ny};
  if ((e = gemm_tn<double>(g, 1, s)) != cudaSuccess) return e;
  k_spectral_d<<<blocks, 256, 0, s>>>(nx, ny, ah, p->wx, p->wy, exh, eyh);
  g.p[0] = GemmProblemT<double>{ny, nx, ny, B[2], ny, exh, ny, t2, nx};
  g.p[1] = GemmProblemT<double>{ny, nx, ny, B[3], ny, eyh, ny, t3, nx};
  if ((e = gemm_tn<double>(g, 2, s)) != cudaSuccess) return e;
  g.p[0] = GemmProblemT<double>{nx, ny, nx, B[4], nx, t2, nx, f, ny};
  if ((e = gemm_tn<double>(g, 1, s)) != cudaSuccess) return e;
  k_convert<double, float><<<blocks, 256, 0, s>>>(n, f, field_x);
  g.p[0] = GemmProblemT<double>{nx, ny, nx, B[5], nx, t3, nx, f, ny};
  if ((e = gemm_tn<double>(g, 1, s)) != cudaSuccess) return e;
  k_convert<double, float><<<blocks, 256, 0, s>>>(n, f, field_y);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- many FP32 solves at once
// The FP32 solves of several regions (each its own grid) as five launches: each GEMM stage
// over every region's problems, the spectral step over every region's spectrum. Each
// problem's tiles are those poisson_solve computes, so every field is the same bit for bit.
struct SpectralJob {
  int nx, ny, first, blocks;
  const float *ah, *wx, *wx2, *wy, *wy2;
  float *exh, *eyh;
};
__global__ void k_spectral_grouped(const SpectralJob *__restrict__ jobs, int n) {
  __shared__ int s_k;
  if (threadIdx.x == 0) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (jobs[mid].first <= (int)blockIdx.x) lo = mid; else hi = mid - 1;
    }
    s_k = lo;
  }
  __syncthreads();
  const SpectralJob J = jobs[s_k];
  const int64_t cnt = (int64_t)J.nx * J.ny;
  for (int64_t k = ((int64_t)blockIdx.x - J.first) * blockDim.x + threadIdx.x; k < cnt; k += (int64_t)J.blocks * blockDim.x) {
    int u = (int)(k / J.ny), v = (int)(k % J.ny);
    float ex = 0.0f, ey = 0.0f;
    if (u != 0 || v != 0) {
      float p = __fdiv_rn(J.ah[k], __fadd_rn(J.wx2[u], J.wy2[v]));
      ex = __fmul_rn(p, J.wx[u]);
      ey = __fmul_rn(p, J.wy[v]);
    }
    J.exh[k] = ex;
    J.eyh[k] = ey;
  }
}

struct PoissonGroup {
  // per stage: problems and each one's first tile; the spectral jobs
  GemmProblem *probs[4] = {};
  int *first[4] = {};
  int count[4] = {}, tiles[4] = {};
  SpectralJob *jobs = nullptr;
  int n_jobs = 0, job_blocks = 0;
};

PoissonGroup *poisson_group_create(PoissonPlan *const *plans, const float *const *density, float *const *field_x, float *const *field_y, int n, cudaError_t *err) {
  *err = cudaSuccess;
  PoissonGroup *g = new PoissonGroup();
  std::vector<GemmProblem> st[4];
  std::vector<SpectralJob> jobs;
  int jb = 0;
  for (int k = 0; k < n; k++) {
    PoissonPlan *p = plans[k];
    if (p->mode != 0) {
      *err = cudaErrorInvalidValue;  // the FP32 form's plans only
      poisson_group_destroy(g);
      return nullptr;
    }
    const int nx = p->nx, ny = p->ny;
    st[0].push_back(GemmProblem{ny, nx, ny, p->CyTs, ny, density[k], ny, p->t1, nx});
    st[1].push_back(GemmProblem{nx, ny, nx, p->CxTs, nx, p->t1, nx, p->ah, ny});
    st[2].push_back(GemmProblem{ny, nx, ny, p->Cy, ny, p->exh, ny, p->t2, nx});
    st[2].push_back(GemmProblem{ny, nx, ny, p->Sy, ny, p->eyh, ny, p->t3, nx});
    st[3].push_back(GemmProblem{nx, ny, nx, p->Sx, nx, p->t2, nx, field_x[k], ny});
    st[3].push_back(GemmProblem{nx, ny, nx, p->Cx, nx, p->t3, nx, field_y[k], ny});
    const int64_t cells = (int64_t)nx * ny;
    const int blocks = (int)std::min<int64_t>((cells + 255) / 256, 148 * 8);
    jobs.push_back(SpectralJob{nx, ny, jb, blocks, p->ah, p->wx, p->wx2, p->wy, p->wy2, p->exh, p->eyh});
    jb += blocks;
  }
  auto put = [&](auto **d, const auto &v) {
    if (*err != cudaSuccess || v.empty()) return;
    using E = typename std::remove_reference<decltype(v)>::type::value_type;
    *err = pool_alloc((void **)d, v.size() * sizeof(E));
    if (*err == cudaSuccess) *err = pool_upload(*d, v.data(), v.size() * sizeof(E));
  };
  for (int q = 0; q < 4; q++) {
    std::vector<int> first;
    int t = 0;
    for (const GemmProblem &P : st[q]) {
      first.push_back(t);
      t += ((P.M + SG_BM - 1) / SG_BM) * ((P.N + SG_BN - 1) / SG_BN);
    }
    g->count[q] = (int)st[q].size();
    g->tiles[q] = t;
    put(&g->probs[q], st[q]);
    put(&g->first[q], first);
  }
  g->n_jobs = (int)jobs.size();
  g->job_blocks = jb;
  put(&g->jobs, jobs);
  if (*err == cudaSuccess) *err = cudaStreamSynchronize(0);
  if (*err != cudaSuccess) {
    poisson_group_destroy(g);
    return nullptr;
  }
  return g;
}

void poisson_group_destroy(PoissonGroup *g) {
  if (!g) return;
  cudaDeviceSynchronize();
  for (int q = 0; q < 4; q++) {
    pool_free(g->probs[q]);
    pool_free(g->first[q]);
  }
  pool_free(g->jobs);
  delete g;
}

cudaError_t poisson_group_solve(const PoissonGroup *g, cudaStream_t s) {
  if (!g || g->n_jobs == 0) return cudaSuccess;
  for (int q = 0; q < 4; q++) {
    k_gemm_grouped<<<g->tiles[q], 256, 0, s>>>(g->probs[q], g->first[q], g->count[q]);
    if (q == 1) k_spectral_grouped<<<g->job_blocks, 256, 0, s>>>(g->jobs, g->n_jobs);
  }
  return cudaGetLastError();
}

int poisson_group_launches(const PoissonGroup *g) { return g && g->n_jobs ? 5 : 0; }

cudaError_t poisson_solve(PoissonPlan *p, const float *density, float *field_x, float *field_y, cudaStream_t s) {
  if (p->mode == 2) return solve_fp64(p, density, field_x, field_y, s);
  if (p->mode != 0) return tc_solve(p, field_x, field_y, s);
  int nx = p->nx, ny = p->ny;
  GemmBatch g{};
  g.p[0] = GemmProblem{ny, nx, ny, p->CyTs, ny, density, ny, p->t1, nx};
  cudaError_t e = sgemm_tn(g, 1, s);
  if (e != cudaSuccess) return e;
  g.p[0] = GemmProblem{nx, ny, nx, p->CxTs, nx, p->t1, nx, p->ah, ny};
  if ((e = sgemm_tn(g, 1, s)) != cudaSuccess) return e;
  int64_t n = (int64_t)nx * ny;
  int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
  k_spectral<<<blocks, 256, 0, s>>>(nx, ny, p->ah, p->wx, p->wx2, p->wy, p->wy2, p->exh, p->eyh);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  g.p[0] = GemmProblem{ny, nx, ny, p->Cy, ny, p->exh, ny, p->t2, nx};
  g.p[1] = GemmProblem{ny, nx, ny, p->Sy, ny, p->eyh, ny, p->t3, nx};
  if ((e = sgemm_tn(g, 2, s)) != cudaSuccess) return e;
  g.p[0] = GemmProblem{nx, ny, nx, p->Sx, nx, p->t2, nx, field_x, ny};
  g.p[1] = GemmProblem{nx, ny, nx, p->Cx, nx, p->t3, nx, field_y, ny};
  return sgemm_tn(g, 2, s);
}


// Loads this file's module (the driver loads a module at its first launch otherwise).
void load_module_poisson() {
  cudaFuncAttributes a;
  cudaFuncGetAttributes(&a, k_gemm_grouped);
}

}  // namespace gpl
