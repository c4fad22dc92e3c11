// The two objectives of the Nesterov placer and their hand-written adjoints, in double, for
// gradient checks and for callers that differentiate through the placer's objective.
//
// The reference takes only gradients (forces) of these objectives and never their values:
//  * WA wirelength: `update_wirelength_force_wa` + `wl_gradient_pin` (src/nesterov.rs:2325-2430)
//    differentiate, per net and axis, W = sum x e^{c x} / sum e^{c x} - sum x e^{-c x} / sum
//    e^{-c x} (the smooth max minus the smooth min), each exponential shifted by the net's
//    box edge; they use (1 + e/1024)^1024 for e^e. Here W itself and dW/dx are taken with
//    exact exponentials (exp in double), so a central difference of W checks dW/dx.
//  * Electrostatic energy: the density force of `density_gradient` (:2434-2449) is the
//    overlap-weighted field of the bin density's Poisson solution (`Fft::solve`, :412-444).
//    Here E = 1/2 rho^T G rho over uniform bins, rho the cells' continuous overlap areas times
//    their density scales, G the reference's DCT solve (forward DCT-II with the index-0
//    halving and 4/(nx ny), division by wx^2 + wy^2 with wy scaled by the bin aspect, inverse
//    DCT-III): G is symmetric, so dE/drho = G rho = phi and dE/dx_i = sum_b drho_b/dx_i phi_b,
//    the overlap's derivative being the cell's other-axis overlap where its moving edges sit.
#include <algorithm>
#include <cmath>
#include <vector>

#include "../../../include/gpl.h"
#include "common.cuh"
#include "poisson_internal.h"

namespace gpl {

namespace {

// ---- WA
struct NetSums {
  double smax, sxmax, smin, sxmin;
};

// One axis of one net: the shifted exponential sums (shift by the box edges, as the
// reference does), into s.
__device__ void wa_axis_sums(const double *xy, int64_t b, int64_t e, int axis, double c, NetSums &s, double &lo, double &hi) {
  lo = INFINITY, hi = -INFINITY;
  for (int64_t p = b; p < e; p++) {
    double v = xy[2 * p + axis];
    lo = fmin(lo, v);
    hi = fmax(hi, v);
  }
  s = NetSums{0, 0, 0, 0};
  for (int64_t p = b; p < e; p++) {
    double v = xy[2 * p + axis];
    double ep = exp(c * (v - hi)), em = exp(c * (lo - v));
    s.smax += ep;
    s.sxmax += v * ep;
    s.smin += em;
    s.sxmin += v * em;
  }
}

__global__ void k_wa_value(int64_t n_nets, const int64_t *net_start, const double *xy, const float *w, double cx, double cy, double *net_value) {
  int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= n_nets) return;
  int64_t b = net_start[n], e = net_start[n + 1];
  double v = 0;
  if (e > b) {
    for (int axis = 0; axis < 2; axis++) {
      NetSums s;
      double lo, hi;
      wa_axis_sums(xy, b, e, axis, axis ? cy : cx, s, lo, hi);
      v += s.sxmax / s.smax - s.sxmin / s.smin;
    }
  }
  net_value[n] = v * (w ? (double)w[n] : 1.0);
}

// dW/dx_p = w [ e+_p ((1 + c x_p) S+ - c A+) / S+^2 - e-_p ((1 - c x_p) S- + c A-) / S-^2 ]
__global__ void k_wa_grad(int64_t n_nets, const int64_t *net_start, const double *xy, const float *w, double cx, double cy, double seed, double *grad) {
  int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= n_nets) return;
  int64_t b = net_start[n], e = net_start[n + 1];
  if (e <= b) return;
  double wt = (w ? (double)w[n] : 1.0) * seed;
  for (int axis = 0; axis < 2; axis++) {
    double c = axis ? cy : cx;
    NetSums s;
    double lo, hi;
    wa_axis_sums(xy, b, e, axis, c, s, lo, hi);
    for (int64_t p = b; p < e; p++) {
      double v = xy[2 * p + axis];
      double ep = exp(c * (v - hi)), em = exp(c * (lo - v));
      double dmax = ep * ((1.0 + c * v) * s.smax - c * s.sxmax) / (s.smax * s.smax);
      double dmin = em * ((1.0 - c * v) * s.smin + c * s.sxmin) / (s.smin * s.smin);
      grad[2 * p + axis] = wt * (dmax - dmin);
    }
  }
}

// ---- electrostatic energy over uniform bins
struct Grid {
  int32_t nx, ny;
  double lx, ly, bw, bh;
};

__device__ __forceinline__ double overlap1(double a0, double a1, double b0, double b1) { return fmax(0.0, fmin(a1, b1) - fmax(a0, b0)); }

// rho[x*ny + y] += scale * overlap area (double atomics: the order is free at this precision)
__global__ void k_rho(int64_t n, const double *xy, const double *half, const double *scale, Grid g, double *rho) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double x0 = xy[2 * i] - half[2 * i], x1 = xy[2 * i] + half[2 * i];
  double y0 = xy[2 * i + 1] - half[2 * i + 1], y1 = xy[2 * i + 1] + half[2 * i + 1];
  int bx0 = max(0, (int)floor((x0 - g.lx) / g.bw)), bx1 = min(g.nx - 1, (int)floor((x1 - g.lx) / g.bw));
  int by0 = max(0, (int)floor((y0 - g.ly) / g.bh)), by1 = min(g.ny - 1, (int)floor((y1 - g.ly) / g.bh));
  for (int bx = bx0; bx <= bx1; bx++) {
    double ox = overlap1(x0, x1, g.lx + bx * g.bw, g.lx + (bx + 1) * g.bw);
    if (ox <= 0) continue;
    for (int by = by0; by <= by1; by++) {
      double oy = overlap1(y0, y1, g.ly + by * g.bh, g.ly + (by + 1) * g.bh);
      if (oy > 0) atomicAdd(&rho[(size_t)bx * g.ny + by], scale[i] * ox * oy);
    }
  }
}

// dE/dx_i = scale * sum_bins d(ox)/dx * oy * phi: d(ox)/dx is +1 in the bin holding the right
// edge and -1 in the bin holding the left edge (where the edge is inside the grid)
__global__ void k_rho_adjoint(int64_t n, const double *xy, const double *half, const double *scale, Grid g, const double *phi, double seed, double *grad) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double c[2] = {xy[2 * i], xy[2 * i + 1]}, h[2] = {half[2 * i], half[2 * i + 1]};
  for (int axis = 0; axis < 2; axis++) {
    // the moving axis's edges, the other axis's overlaps
    double lo = (axis ? g.ly : g.lx), sz = (axis ? g.bh : g.bw);
    int cnt = axis ? g.ny : g.nx, ocnt = axis ? g.nx : g.ny;
    double olo = (axis ? g.lx : g.ly), osz = (axis ? g.bw : g.bh);
    double o0 = c[1 - axis] - h[1 - axis], o1 = c[1 - axis] + h[1 - axis];
    int ob0 = max(0, (int)floor((o0 - olo) / osz)), ob1 = min(ocnt - 1, (int)floor((o1 - olo) / osz));
    double d = 0;
    for (int side = 0; side < 2; side++) {
      double edge = side ? c[axis] + h[axis] : c[axis] - h[axis];
      double f = (edge - lo) / sz;
      if (f <= 0.0 || f >= (double)cnt) continue;
      int b = (int)floor(f);
      double sgn = side ? 1.0 : -1.0;
      for (int ob = ob0; ob <= ob1; ob++) {
        double oo = overlap1(o0, o1, olo + ob * osz, olo + (ob + 1) * osz);
        if (oo <= 0) continue;
        size_t k = axis ? (size_t)ob * g.ny + b : (size_t)b * g.ny + ob;
        d += sgn * oo * phi[k];
      }
    }
    grad[2 * i + axis] = seed * scale[i] * d;
  }
}

// C = A B (row-major, doubles), or with B transposed: a plain tiled SIMT kernel (the check
// path, not the placer's loop).
template <bool BT>
__global__ void k_dgemm(int M, int N, int K, const double *A, const double *B, double *C) {
  __shared__ double sa[16][17], sb[16][17];
  int row = blockIdx.y * 16 + threadIdx.y, col = blockIdx.x * 16 + threadIdx.x;
  double acc = 0;
  for (int k0 = 0; k0 < K; k0 += 16) {
    int ka = k0 + threadIdx.x, kb = k0 + threadIdx.y;
    sa[threadIdx.y][threadIdx.x] = (row < M && ka < K) ? A[(size_t)row * K + ka] : 0.0;
    sb[threadIdx.y][threadIdx.x] = (col < N && kb < K) ? (BT ? B[(size_t)col * K + kb] : B[(size_t)kb * N + col]) : 0.0;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 16; k++) acc += sa[threadIdx.y][k] * sb[k][threadIdx.x];
    __syncthreads();
  }
  if (row < M && col < N) C[(size_t)row * N + col] = acc;
}

__global__ void k_spectral_scale(int nx, int ny, double aspect, double *a) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= (int64_t)nx * ny) return;
  int u = (int)(k / ny), v = (int)(k % ny);
  double wx = M_PI * u / nx, wy = M_PI * v / ny * aspect;
  double h = (u == 0 ? 0.5 : 1.0) * (v == 0 ? 0.5 : 1.0) * 4.0 / ((double)nx * ny);
  a[k] = (u == 0 && v == 0) ? 0.0 : a[k] * h / (wx * wx + wy * wy);
}

__global__ void k_dot_partial(int64_t n, const double *a, const double *b, double *part) {
  __shared__ double sh[kThreads / 32];
  double s = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) s += a[i] * b[i];
  double t = block_sum<kThreads>(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

unsigned blocks(int64_t n) { return (unsigned)std::max<int64_t>(1, (n + kThreads - 1) / kThreads); }

// The DCT bases C[u][x] = cos(pi u (x + 1/2) / n), row-major (n x n).
std::vector<double> cos_basis(int n) {
  std::vector<double> c((size_t)n * n);
  for (int u = 0; u < n; u++)
    for (int x = 0; x < n; x++) c[(size_t)u * n + x] = std::cos(M_PI * u * (x + 0.5) / n);
  return c;
}

}  // namespace

// The density objective's plan: the grid, the DCT bases on the device (Cy, Cx and their
// transposes) and the solve's buffers, made once for many evaluations.
struct DensityPlan {
  Grid g{};
  double *cx = nullptr, *cxt = nullptr, *cy = nullptr, *cyt = nullptr;
  double *rho = nullptr, *phi = nullptr, *t1 = nullptr, *t2 = nullptr;
  cudaStream_t s = nullptr;
};

namespace {

void plan_free(DensityPlan *p) {
  for (double *b : {p->cx, p->cxt, p->cy, p->cyt, p->rho, p->phi, p->t1, p->t2})
    if (b) cudaFreeAsync(b, p->s);
  cudaStreamSynchronize(p->s);
  delete p;
}

DensityPlan *plan_make(const Grid &g, cudaStream_t s, cudaError_t *err) {
  DensityPlan *p = new DensityPlan();
  p->g = g;
  p->s = s;
  const size_t nb = (size_t)g.nx * g.ny;
  std::vector<double> hx = cos_basis(g.nx), hy = g.ny == g.nx ? hx : cos_basis(g.ny);
  std::vector<double> hxt((size_t)g.nx * g.nx), hyt((size_t)g.ny * g.ny);
  for (int a = 0; a < g.nx; a++)
    for (int b = 0; b < g.nx; b++) hxt[(size_t)a * g.nx + b] = hx[(size_t)b * g.nx + a];
  for (int a = 0; a < g.ny; a++)
    for (int b = 0; b < g.ny; b++) hyt[(size_t)a * g.ny + b] = hy[(size_t)b * g.ny + a];
  cudaError_t e = cudaSuccess;
  auto put = [&](double **d, const std::vector<double> &h) {
    if (e == cudaSuccess) e = cudaMallocAsync((void **)d, h.size() * sizeof(double), s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, s);
  };
  put(&p->cx, hx);
  put(&p->cxt, hxt);
  put(&p->cy, hy);
  put(&p->cyt, hyt);
  for (double **b : {&p->rho, &p->phi, &p->t1, &p->t2})
    if (e == cudaSuccess) e = cudaMallocAsync((void **)b, nb * sizeof(double), s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the host bases outlive their copies
  *err = e;
  if (e != cudaSuccess) {
    plan_free(p);
    return nullptr;
  }
  return p;
}

// phi = G rho: A^ = Cx rho Cy^T (two GEMMs), scaled, then phi = Cx^T A^ Cy (two more), each
// a D = A B^T product of the tiled double GEMM.
cudaError_t potential(DensityPlan *p, cudaStream_t s) {
  const int nx = p->g.nx, ny = p->g.ny;
  GemmBatchT<double> b{};
  b.p[0] = GemmProblemT<double>{ny, nx, ny, p->cy, ny, p->rho, ny, p->t1, nx};   // t1[v][x] = sum_y Cy[v][y] rho[x][y]
  cudaError_t e = dgemm_tn(b, 1, s);
  b.p[0] = GemmProblemT<double>{nx, ny, nx, p->cx, nx, p->t1, nx, p->t2, ny};    // A^[u][v] = sum_x Cx[u][x] t1[v][x]
  if (e == cudaSuccess) e = dgemm_tn(b, 1, s);
  if (e == cudaSuccess) {
    k_spectral_scale<<<blocks((int64_t)nx * ny), kThreads, 0, s>>>(nx, ny, p->g.bh / p->g.bw, p->t2);
    e = cudaGetLastError();
  }
  b.p[0] = GemmProblemT<double>{ny, nx, ny, p->cyt, ny, p->t2, ny, p->t1, nx};   // t1[y][u] = sum_v Cy[v][y] A^[u][v]
  if (e == cudaSuccess) e = dgemm_tn(b, 1, s);
  b.p[0] = GemmProblemT<double>{nx, ny, nx, p->cxt, nx, p->t1, nx, p->phi, ny};  // phi[x][y] = sum_u Cx[u][x] t1[y][u]
  if (e == cudaSuccess) e = dgemm_tn(b, 1, s);
  return e;
}

// The cells' density rho and its potential phi on the plan's buffers.
cudaError_t density_phi(DensityPlan *p, int64_t n, const double *xy, const double *half, const double *scale, cudaStream_t s) {
  const size_t nb = (size_t)p->g.nx * p->g.ny;
  cudaError_t e = cudaMemsetAsync(p->rho, 0, nb * sizeof(double), s);
  if (e == cudaSuccess && n > 0) k_rho<<<blocks(n), kThreads, 0, s>>>(n, xy, half, scale, p->g, p->rho);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = potential(p, s);
  return e;
}

cudaError_t dot(int64_t n, const double *a, const double *b, double *out, cudaStream_t s) {
  const int nblk = 148;
  double *part = nullptr;
  cudaError_t e = cudaMallocAsync((void **)&part, nblk * sizeof(double), s);
  if (e != cudaSuccess) return e;
  k_dot_partial<<<nblk, kThreads, 0, s>>>(n, a, b, part);
  std::vector<double> h(nblk);
  e = cudaMemcpyAsync(h.data(), part, nblk * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFreeAsync(part, s);
  double t = 0;
  for (double v : h) t += v;
  *out = t;
  return e;
}

// The field solve in double: A^ = Cx rho Cy^T scaled (the index-0 halving, 4/(nx ny)),
// phi^ = A^ / (wx^2 + wy^2), Ex = Sx^T (phi^ wx) Cy, Ey = Cx^T (phi^ wy) Sy, with the
// caller's wavenumbers (`Fft::solve`, src/nesterov.rs:412-444; the field's sine sums skip
// index 0, where the wavenumber is 0).
__global__ void k_spectral_fields(int nx, int ny, const double *wx, const double *wy, const double *a, double *ex, double *ey) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= (int64_t)nx * ny) return;
  int u = (int)(k / ny), v = (int)(k % ny);
  double h = (u == 0 ? 0.5 : 1.0) * (v == 0 ? 0.5 : 1.0) * 4.0 / ((double)nx * ny);
  double d = wx[u] * wx[u] + wy[v] * wy[v];
  double p = (u == 0 && v == 0) ? 0.0 : a[k] * h / d;
  ex[k] = p * wx[u];
  ey[k] = p * wy[v];
}

std::vector<double> sin_basis(int n) {
  std::vector<double> c((size_t)n * n);
  for (int u = 0; u < n; u++)
    for (int x = 0; x < n; x++) c[(size_t)u * n + x] = u == 0 ? 0.0 : std::sin(M_PI * u * (x + 0.5) / n);
  return c;
}

std::vector<double> transpose(const std::vector<double> &m, int n) {
  std::vector<double> t(m.size());
  for (int a = 0; a < n; a++)
    for (int b = 0; b < n; b++) t[(size_t)a * n + b] = m[(size_t)b * n + a];
  return t;
}

}  // namespace

}  // namespace gpl

using namespace gpl;

extern "C" {

int gpl_kernel_poisson_fp64(int32_t nx, int32_t ny, const float *wx_host, const float *wy_host, const float *density, double *field_x, double *field_y, void *stream) {
  cudaStream_t s = (cudaStream_t)stream;
  size_t nb = (size_t)nx * ny;
  std::vector<double> cx = cos_basis(nx), cy = cos_basis(ny), sx = sin_basis(nx), sy = sin_basis(ny);
  std::vector<double> cxt = transpose(cx, nx), sxt = transpose(sx, nx);
  std::vector<double> hwx(wx_host, wx_host + nx), hwy(wy_host, wy_host + ny);
  std::vector<float> hd(nb);
  double *d_cx, *d_cy, *d_sy, *d_cxt, *d_sxt, *d_wx, *d_wy, *rho, *t1, *t2, *ex, *ey;
  double **bufs[] = {&d_cx, &d_cy, &d_sy, &d_cxt, &d_sxt, &d_wx, &d_wy, &rho, &t1, &t2, &ex, &ey};
  size_t sizes[] = {cx.size(), cy.size(), sy.size(), cxt.size(), sxt.size(), (size_t)nx, (size_t)ny, nb, nb, nb, nb, nb};
  cudaError_t e = cudaSuccess;
  for (int k = 0; k < 12; k++) {
    *bufs[k] = nullptr;
    if (e == cudaSuccess) e = cudaMalloc((void **)bufs[k], sizes[k] * sizeof(double));
  }
  auto put = [&](double *d, const std::vector<double> &h) {
    if (e == cudaSuccess) e = cudaMemcpy(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice);
  };
  put(d_cx, cx);
  put(d_cy, cy);
  put(d_sy, sy);
  put(d_cxt, cxt);
  put(d_sxt, sxt);
  put(d_wx, hwx);
  put(d_wy, hwy);
  if (e == cudaSuccess) e = cudaMemcpy(hd.data(), density, nb * sizeof(float), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) put(rho, std::vector<double>(hd.begin(), hd.end()));
  if (e == cudaSuccess) {
    dim3 th(16, 16);
    auto g2 = [&](int M, int N) { return dim3((N + 15) / 16, (M + 15) / 16); };
    k_dgemm<false><<<g2(nx, ny), th, 0, s>>>(nx, ny, nx, d_cx, rho, t1);   // Cx rho
    k_dgemm<true><<<g2(nx, ny), th, 0, s>>>(nx, ny, ny, t1, d_cy, t2);     // (Cx rho) Cy^T
    k_spectral_fields<<<blocks((int64_t)nb), kThreads, 0, s>>>(nx, ny, d_wx, d_wy, t2, ex, ey);
    k_dgemm<false><<<g2(nx, ny), th, 0, s>>>(nx, ny, nx, d_sxt, ex, t1);   // Sx^T Ex^
    k_dgemm<false><<<g2(nx, ny), th, 0, s>>>(nx, ny, ny, t1, d_cy, field_x);  // ... Cy
    k_dgemm<false><<<g2(nx, ny), th, 0, s>>>(nx, ny, nx, d_cxt, ey, t1);   // Cx^T Ey^
    k_dgemm<false><<<g2(nx, ny), th, 0, s>>>(nx, ny, ny, t1, d_sy, field_y);  // ... Sy
    e = cudaGetLastError();
  }
  cudaError_t e2 = cudaStreamSynchronize(s);
  for (int k = 0; k < 12; k++)
    if (*bufs[k]) cudaFree(*bufs[k]);
  return (int)(e != cudaSuccess ? e : e2);
}

int gpl_fn_wa_forward(int64_t n_nets, const int64_t *net_start, const double *pin_xy, const float *net_weight, double coef_x, double coef_y, double *value, void *stream) {
  cudaStream_t s = (cudaStream_t)stream;
  *value = 0;
  if (n_nets <= 0) return 0;
  double *nv = nullptr;
  cudaError_t e = cudaMallocAsync((void **)&nv, (size_t)n_nets * sizeof(double), s);
  if (e != cudaSuccess) return (int)e;
  k_wa_value<<<blocks(n_nets), kThreads, 0, s>>>(n_nets, net_start, pin_xy, net_weight, coef_x, coef_y, nv);
  std::vector<double> h(n_nets);
  e = cudaMemcpyAsync(h.data(), nv, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFreeAsync(nv, s);
  double t = 0;
  for (double v : h) t += v;  // in net order
  *value = t;
  return (int)e;
}

int gpl_fn_wa_backward(int64_t n_nets, const int64_t *net_start, const double *pin_xy, const float *net_weight, double coef_x, double coef_y, double seed, double *grad, void *stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (n_nets <= 0) return 0;
  k_wa_grad<<<blocks(n_nets), kThreads, 0, s>>>(n_nets, net_start, pin_xy, net_weight, coef_x, coef_y, seed, grad);
  cudaError_t e = cudaGetLastError();
  cudaError_t e2 = cudaStreamSynchronize(s);
  return (int)(e != cudaSuccess ? e : e2);
}

gpl_fn_density *gpl_fn_density_create(int32_t nx, int32_t ny, double grid_lx, double grid_ly, double bin_w, double bin_h, void *stream) {
  if (nx <= 0 || ny <= 0 || !(bin_w > 0) || !(bin_h > 0)) return nullptr;
  cudaError_t e = cudaSuccess;
  DensityPlan *p = plan_make(Grid{nx, ny, grid_lx, grid_ly, bin_w, bin_h}, (cudaStream_t)stream, &e);
  return reinterpret_cast<gpl_fn_density *>(p);
}

void gpl_fn_density_destroy(gpl_fn_density *f) {
  if (f) plan_free(reinterpret_cast<DensityPlan *>(f));
}

int gpl_fn_density_eval(gpl_fn_density *f, int64_t n_cells, const double *cell_xy, const double *half, const double *scale, double *energy, double seed, double *grad) {
  DensityPlan *p = reinterpret_cast<DensityPlan *>(f);
  if (!p) return (int)cudaErrorInvalidValue;
  cudaStream_t s = p->s;
  cudaError_t e = density_phi(p, n_cells, cell_xy, half, scale, s);
  if (energy) {
    double d = 0;
    if (e == cudaSuccess) e = dot((int64_t)p->g.nx * p->g.ny, p->rho, p->phi, &d, s);
    *energy = 0.5 * d;
  }
  if (grad && e == cudaSuccess && n_cells > 0) {
    k_rho_adjoint<<<blocks(n_cells), kThreads, 0, s>>>(n_cells, cell_xy, half, scale, p->g, p->phi, seed, grad);
    e = cudaGetLastError();
  }
  cudaError_t e2 = cudaStreamSynchronize(s);
  return (int)(e != cudaSuccess ? e : e2);
}

int gpl_fn_density_forward(int64_t n_cells, const double *cell_xy, const double *half, const double *scale, int32_t nx, int32_t ny, double grid_lx, double grid_ly, double bin_w, double bin_h, double *energy, void *stream) {
  gpl_fn_density *f = gpl_fn_density_create(nx, ny, grid_lx, grid_ly, bin_w, bin_h, stream);
  if (!f) return (int)cudaErrorInvalidValue;
  const int r = gpl_fn_density_eval(f, n_cells, cell_xy, half, scale, energy, 0.0, nullptr);
  gpl_fn_density_destroy(f);
  return r;
}

int gpl_fn_density_backward(int64_t n_cells, const double *cell_xy, const double *half, const double *scale, int32_t nx, int32_t ny, double grid_lx, double grid_ly, double bin_w, double bin_h, double seed, double *grad, void *stream) {
  gpl_fn_density *f = gpl_fn_density_create(nx, ny, grid_lx, grid_ly, bin_w, bin_h, stream);
  if (!f) return (int)cudaErrorInvalidValue;
  const int r = gpl_fn_density_eval(f, n_cells, cell_xy, half, scale, nullptr, seed, grad);
  gpl_fn_density_destroy(f);
  return r;
}

}  // extern "C"
