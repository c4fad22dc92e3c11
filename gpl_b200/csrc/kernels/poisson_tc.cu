// The density solver's transforms as split-BF16 GEMMs on the 5th-generation tensor cores.
//
// Every operand X (a basis matrix, the density, an intermediate) is stored as two bfloat16
// halves side by side along K: [X_hi | X_lo] with X_hi = bf16(X) and X_lo = bf16(X - X_hi).
// One GEMM D = A B^T takes, per K step, the compensated product A_hi B_hi + A_hi B_lo +
// A_lo B_hi (A_lo B_lo is below FP32 accumulation noise), accumulated in FP32 in tensor
// memory. The epilogue reads the accumulator back (tcgen05.ld) and writes the next GEMM's
// split operand directly, or the spectral step's two operands, or the FP32 field.
//
// Kernel: one 128 x BN output tile per CTA of 128 threads. Thread 0 issues the TMA loads of
// each K-block (128B-swizzled 64-wide bf16 tiles: A_hi, A_lo, B_hi, B_lo) into a ring of
// stages; thread 32 issues tcgen05.mma (M=128, N=BN, K=16, kind::f16, bf16 in, f32
// accumulate), three per K step, as the stages land, committing each stage back to the
// producer; after the last K-block all four warps read their 32 TMEM lanes, 32 columns at a
// time. The single GEMMs use BN = 64 (a 1024-point grid gives 128 tiles for the 148 SMs), the
// batched pairs BN = 128 (the same 128 tiles over both). Every wait is bounded by the GPU's
// global timer (1 s): a wait that runs out records an error word, and the CTA drains and
// returns.
//
// The four launches of a solve (see poisson.cu for the algebra):
//   1  T1t = CyTs rho^T                      split out
//   2  Ah  = CxTs T1t^T  -> Exh, Eyh         spectral epilogue, two split outs
//   3  T2t = Cy Exh^T ; T3t = Sy Eyh^T       batched, split outs
//   4  Ex  = Sx T2t^T ; Ey  = Cx T3t^T       batched, FP32 outs
// Grid sides must be multiples of 128 (the engine runs the FP32 solver otherwise).
#include <cuda.h>
#include <cuda_bf16.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "engine_kernels.h"
#include "poisson_internal.h"
#include "parallel.h"

namespace gpl {

namespace {

// A stage holds one K-block of both halves of both operands: A_hi, A_lo (BM x BK each) and
// B_hi, B_lo (BN x BK each); its three products hi*hi, hi*lo, lo*hi all accumulate into the
// one TMEM tile, so each operand byte crosses from L2 once per output tile.
constexpr int BM = 128, BK = 64;
constexpr int A_TILE = BM * BK * 2;                    // 16 KB
template <int BN>
struct Tile {
  static constexpr int B_TILE = BN * BK * 2;                   // 8 or 16 KB
  static constexpr int STAGE_BYTES = 2 * A_TILE + 2 * B_TILE;  // 48 or 64 KB, multiples of 1 KB
  static constexpr int STAGES = BN == 64 ? 4 : 3;
  static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
  static constexpr uint32_t TMEM_COLS = BN;                    // fp32 accumulator columns
  // kind::f16 instruction descriptor: D f32, A and B bf16, both K-major, M=BM, N=BN.
  static constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
  static_assert(BN % 16 == 0 && BN >= 32 && BN <= 256 && (BN & (BN - 1)) == 0, "an M=128 MMA shape with a power-of-two TMEM allocation");
  static_assert(SMEM_BYTES <= 227 * 1024, "shared memory per CTA");
};
constexpr int EPI_COLS = 32;                           // accumulator columns per epilogue step
constexpr uint64_t WAIT_NS = 1000000000ull;    // a wait that lasts a second is an error

enum Epi { EPI_SPLIT = 0, EPI_SPECTRAL = 1, EPI_F32 = 2 };

struct TcOut {
  void *out0, *out1;  // split: [M][2*ldk] bf16; f32: [M][N] float
  int ld;             // split: the next GEMM's K (= this N); f32: N
};
struct TcArgs {
  int M, N, K;        // multiples of 128, 64, 64
  TcOut o[2];         // per batch entry (blockIdx.z)
  const float *wx, *wx2, *wy, *wy2;
  int *err;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait on a phase; false (and the error word set) when it runs out or another role
// already failed.
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity, volatile int *fail, int *err, int code) {
  uint64_t t0 = gtimer();
  while (!mbar_try(b, parity)) {
    if (*fail) return false;
    if (gtimer() - t0 > WAIT_NS) {
      *fail = 1;
      atomicExch(err, code);
      return false;
    }
  }
  return true;
}
__device__ __forceinline__ void tma_load(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}
// K-major, 128-byte swizzle, 8-row groups 1 KB apart, Blackwell descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]),
        "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void split_store(__nv_bfloat16 *row_hi, __nv_bfloat16 *row_lo, const float *v) {
  // EPI_COLS values: hi and lo halves, 16-byte stores
#pragma unroll
  for (int c = 0; c < EPI_COLS; c += 8) {
    __align__(16) __nv_bfloat16 h[8], l[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      h[q] = __float2bfloat16_rn(v[c + q]);
      l[q] = __float2bfloat16_rn(v[c + q] - __bfloat162float(h[q]));
    }
    *reinterpret_cast<uint4 *>(row_hi + c) = *reinterpret_cast<const uint4 *>(h);
    *reinterpret_cast<uint4 *>(row_lo + c) = *reinterpret_cast<const uint4 *>(l);
  }
}

template <int EPI, int BN>
__global__ void __launch_bounds__(128, 1) k_tc_gemm(const __grid_constant__ CUtensorMap tA0, const __grid_constant__ CUtensorMap tB0,
                                                   const __grid_constant__ CUtensorMap tA1, const __grid_constant__ CUtensorMap tB1, TcArgs args) {
  chain_enter();
  using T = Tile<BN>;
  constexpr int STAGES = T::STAGES, STAGE_BYTES = T::STAGE_BYTES, B_TILE = T::B_TILE;
  constexpr uint32_t TMEM_COLS = T::TMEM_COLS, IDESC = T::IDESC;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t *full = (uint64_t *)(smem + STAGES * STAGE_BYTES);
  uint64_t *empty = full + STAGES;
  uint64_t *done = empty + STAGES;
  uint32_t *tmem_slot = (uint32_t *)(done + 1);
  volatile int *fail = (volatile int *)(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int z = blockIdx.z;
  const CUtensorMap *mA = z ? &tA1 : &tA0;
  const CUtensorMap *mB = z ? &tB1 : &tB0;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int nkb = args.K / BK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    *fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {  // the whole warp allocates the accumulator columns
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)), "r"(TMEM_COLS) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (threadIdx.x == 0) {
    // producer: K-block kb brings A_hi, A_lo (columns k0 and K + k0 of A) and B_hi, B_lo
    for (int kb = 0; kb < nkb; kb++) {
      int s = kb % STAGES, round = kb / STAGES;
      if (round > 0 && !mbar_wait(&empty[s], (round - 1) & 1, fail, args.err, 1)) break;
      int k0 = kb * BK;
      uint8_t *st = smem + s * STAGE_BYTES;
      mbar_expect_tx(&full[s], STAGE_BYTES);
      tma_load(st, mA, &full[s], k0, m0);
      tma_load(st + A_TILE, mA, &full[s], args.K + k0, m0);
      tma_load(st + 2 * A_TILE, mB, &full[s], k0, n0);
      tma_load(st + 2 * A_TILE + B_TILE, mB, &full[s], args.K + k0, n0);
    }
  } else if (threadIdx.x == 32) {
    // MMA issuer: per 16-wide K step, hi*hi, hi*lo, lo*hi
    for (int kb = 0; kb < nkb; kb++) {
      int s = kb % STAGES, round = kb / STAGES;
      if (!mbar_wait(&full[s], round & 1, fail, args.err, 2)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      uint32_t ahi = smem_u32(smem + s * STAGE_BYTES), alo = ahi + A_TILE, bhi = ahi + 2 * A_TILE, blo = bhi + B_TILE;
#pragma unroll
      for (int kk = 0; kk < BK / 16; kk++) {
        uint32_t o = kk * 32;
        umma(tmem, smem_desc(ahi + o), smem_desc(bhi + o), IDESC, (kb > 0 || kk > 0) ? 1u : 0u);
        umma(tmem, smem_desc(ahi + o), smem_desc(blo + o), IDESC, 1u);
        umma(tmem, smem_desc(alo + o), smem_desc(bhi + o), IDESC, 1u);
      }
      umma_commit(&empty[s]);
    }
    umma_commit(done);
  }
  __syncwarp();
  // epilogue: every warp reads its 32 lanes (rows) of the BM x BN accumulator, EPI_COLS
  // columns at a time; lane 0 waits for the last commit, so the warp stays converged for the
  // aligned TMEM loads
  int okw = 0;
  if (lane == 0) okw = mbar_wait(done, 0, fail, args.err, 3) && !*fail;
  okw = __shfl_sync(0xffffffffu, okw, 0);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (okw) {
    const uint32_t base = tmem + ((uint32_t)(warp * 32) << 16);
    const int m = m0 + warp * 32 + lane;
    const TcOut &o = args.o[z];
    const bool in = m < args.M;
    float wxu = 0.0f, wx2u = 0.0f;
    if (EPI == EPI_SPECTRAL && in) {
      wxu = args.wx[m];
      wx2u = args.wx2[m];
    }
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += EPI_COLS) {
      float v[EPI_COLS];
#pragma unroll
      for (int c = 0; c < EPI_COLS; c += 16) tmem_ld16(base + c0 + c, v + c);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (!in) continue;
      const int nb = n0 + c0;
      if (EPI == EPI_F32) {
        float *row = (float *)o.out0 + (size_t)m * o.ld + nb;
#pragma unroll
        for (int c = 0; c < EPI_COLS; c += 4) *reinterpret_cast<float4 *>(row + c) = make_float4(v[c], v[c + 1], v[c + 2], v[c + 3]);
      } else if (EPI == EPI_SPLIT) {
        __nv_bfloat16 *row = (__nv_bfloat16 *)o.out0 + (size_t)m * 2 * o.ld;
        split_store(row + nb, row + o.ld + nb, v);
      } else {
        // the spectral step (src/nesterov.rs:425-440) on the scaled forward transform
        float ex[EPI_COLS], ey[EPI_COLS];
#pragma unroll
        for (int c = 0; c < EPI_COLS; c++) {
          int n = nb + c;
          // a fast division (within 2 ulp): far below the split-BF16 products' own error
          float p = (m == 0 && n == 0) ? 0.0f : __fdividef(v[c], __fadd_rn(wx2u, args.wy2[n]));
          ex[c] = __fmul_rn(p, wxu);
          ey[c] = __fmul_rn(p, args.wy[n]);
        }
        __nv_bfloat16 *rx = (__nv_bfloat16 *)o.out0 + (size_t)m * 2 * o.ld;
        __nv_bfloat16 *ry = (__nv_bfloat16 *)o.out1 + (size_t)m * 2 * o.ld;
        split_store(rx + nb, rx + o.ld + nb, ex);
        split_store(ry + nb, ry + o.ld + nb, ey);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

// ---------------------------------------------------------------- host side
typedef CUresult (*EncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static EncodeTiled fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess) fn = (EncodeTiled)p;
  }
  return fn;
}

// A split operand [rows][2*k] bf16 as a TMA map with a (box_rows x 64) box, 128B swizzle.
cudaError_t make_map(CUtensorMap *m, const __nv_bfloat16 *base, int rows, int k, int box_rows) {
  EncodeTiled enc = encode_fn();
  if (!enc) return cudaErrorNotSupported;
  if (((uintptr_t)base & 15) != 0 || (k * 2 * 2) % 16 != 0) return cudaErrorInvalidValue;
  cuuint64_t dims[2] = {(cuuint64_t)(2 * k), (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(2 * k) * 2};
  cuuint32_t box[2] = {BK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void *)base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

}  // namespace

struct TcState {
  __nv_bfloat16 *CyTs = nullptr, *CxTs = nullptr, *Cy = nullptr, *Sy = nullptr, *Sx = nullptr, *Cx = nullptr;
  __nv_bfloat16 *t1 = nullptr, *exh = nullptr, *eyh = nullptr, *t2 = nullptr, *t3 = nullptr;
  int *err = nullptr;
  CUtensorMap mCyTs, mCxTs, mCy, mSy, mSx, mCx;  // A operands (BM-row boxes)
  CUtensorMap mDens, mT1;                        // B operands of the single GEMMs (64-row boxes)
  CUtensorMap mExh, mEyh, mT2, mT3;              // B operands of the batched pairs (128-row boxes)
};

static cudaError_t upload_split(const std::vector<double> &h, int rows, int k, __nv_bfloat16 **d) {
  std::vector<__nv_bfloat16> v((size_t)rows * 2 * k);
  parallel_for((size_t)rows, [&](size_t r0, size_t r1) {
    for (size_t r = r0; r < r1; r++)
      for (int c = 0; c < k; c++) {
        float x = (float)h[r * k + c];
        __nv_bfloat16 hi = __float2bfloat16_rn(x);
        v[r * 2 * k + c] = hi;
        v[r * 2 * k + k + c] = __float2bfloat16_rn(x - __bfloat162float(hi));
      }
  }, 16);
  cudaError_t e = pool_alloc((void **)d, v.size() * sizeof(__nv_bfloat16));
  if (e != cudaSuccess) return e;
  return pool_upload(*d, v.data(), v.size() * sizeof(__nv_bfloat16));
}

cudaError_t tc_plan_init(PoissonPlan *p, const BasisHost &b) {
  int nx = p->nx, ny = p->ny;
  if (nx % 128 != 0 || ny % 128 != 0) return cudaErrorNotSupported;
  TcState *t = new TcState();
  p->tc = t;
  cudaError_t e;
#define TRY(x)                            \
  do {                                    \
    if ((e = (x)) != cudaSuccess) return e; \
  } while (0)
  TRY(upload_split(b.CyTs, ny, ny, &t->CyTs));
  TRY(upload_split(b.CxTs, nx, nx, &t->CxTs));
  TRY(upload_split(b.Cy, ny, ny, &t->Cy));
  TRY(upload_split(b.Sy, ny, ny, &t->Sy));
  TRY(upload_split(b.Sx, nx, nx, &t->Sx));
  TRY(upload_split(b.Cx, nx, nx, &t->Cx));
  size_t n = (size_t)nx * ny * 2;
  TRY(pool_alloc((void **)&p->tc_dens, n * sizeof(__nv_bfloat16)));
  TRY(pool_alloc((void **)&t->t1, n * sizeof(__nv_bfloat16)));
  TRY(pool_alloc((void **)&t->exh, n * sizeof(__nv_bfloat16)));
  TRY(pool_alloc((void **)&t->eyh, n * sizeof(__nv_bfloat16)));
  TRY(pool_alloc((void **)&t->t2, n * sizeof(__nv_bfloat16)));
  TRY(pool_alloc((void **)&t->t3, n * sizeof(__nv_bfloat16)));
  TRY(cudaMemsetAsync(p->tc_dens, 0, n * sizeof(__nv_bfloat16), 0));
  TRY(pool_alloc((void **)&t->err, sizeof(int)));
  TRY(cudaMemsetAsync(t->err, 0, sizeof(int), 0));
  // A operands [M][2K]: 128-row boxes
  TRY(make_map(&t->mCyTs, t->CyTs, ny, ny, BM));
  TRY(make_map(&t->mCxTs, t->CxTs, nx, nx, BM));
  TRY(make_map(&t->mCy, t->Cy, ny, ny, BM));
  TRY(make_map(&t->mSy, t->Sy, ny, ny, BM));
  TRY(make_map(&t->mSx, t->Sx, nx, nx, BM));
  TRY(make_map(&t->mCx, t->Cx, nx, nx, BM));
  // B operands [N][2K]: BN-row boxes
  TRY(make_map(&t->mDens, p->tc_dens, nx, ny, 64));  // rows x, K = y
  TRY(make_map(&t->mT1, t->t1, ny, nx, 64));         // rows v, K = x
  TRY(make_map(&t->mExh, t->exh, nx, ny, 128));      // rows u, K = v
  TRY(make_map(&t->mEyh, t->eyh, nx, ny, 128));
  TRY(make_map(&t->mT2, t->t2, ny, nx, 128));        // rows y, K = u
  TRY(make_map(&t->mT3, t->t3, ny, nx, 128));
#undef TRY
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_tc_gemm<EPI_SPLIT, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, Tile<64>::SMEM_BYTES);
    cudaFuncSetAttribute(k_tc_gemm<EPI_SPECTRAL, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, Tile<64>::SMEM_BYTES);
    cudaFuncSetAttribute(k_tc_gemm<EPI_SPLIT, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, Tile<128>::SMEM_BYTES);
    cudaFuncSetAttribute(k_tc_gemm<EPI_F32, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, Tile<128>::SMEM_BYTES);
    attr = true;
  }
  return cudaGetLastError();
}

void tc_plan_free(PoissonPlan *p) {
  pool_free(p->tc_dens);
  p->tc_dens = nullptr;
  TcState *t = p->tc;
  if (!t) return;
  void *bufs[] = {t->CyTs, t->CxTs, t->Cy, t->Sy, t->Sx, t->Cx, t->t1, t->exh, t->eyh, t->t2, t->t3, t->err};
  for (void *b : bufs)
    pool_free(b);
  delete t;
  p->tc = nullptr;
}

int tc_launches(const PoissonPlan *) { return 4; }

cudaError_t tc_solve(PoissonPlan *p, float *field_x, float *field_y, cudaStream_t s) {
  TcState *t = p->tc;
  int nx = p->nx, ny = p->ny;
  TcArgs a{};
  a.wx = p->wx;
  a.wx2 = p->wx2;
  a.wy = p->wy;
  a.wy2 = p->wy2;
  a.err = t->err;
  // 1: T1t[v][x] = sum_y CyTs[v][y] rho[x][y]      M = ny, N = nx, K = ny
  a.M = ny, a.N = nx, a.K = ny;
  a.o[0] = TcOut{t->t1, nullptr, nx};
  cudaError_t le = launch_chained(k_tc_gemm<EPI_SPLIT, 64>, dim3(nx / 64, ny / BM, 1), dim3(128), Tile<64>::SMEM_BYTES, s, t->mCyTs, t->mDens, t->mCyTs, t->mDens, a);
  if (le != cudaSuccess) return le;
  // 2: Ah[u][v] = sum_x CxTs[u][x] T1t[v][x]; spectral  M = nx, N = ny, K = nx
  a.M = nx, a.N = ny, a.K = nx;
  a.o[0] = TcOut{t->exh, t->eyh, ny};
  if ((le = launch_chained(k_tc_gemm<EPI_SPECTRAL, 64>, dim3(ny / 64, nx / BM, 1), dim3(128), Tile<64>::SMEM_BYTES, s, t->mCxTs, t->mT1, t->mCxTs, t->mT1, a)) != cudaSuccess) return le;
  // 3: T2t[y][u] = sum_v Cy[y][v] Exh[u][v]; T3t = Sy Eyh^T   M = ny, N = nx, K = ny
  a.M = ny, a.N = nx, a.K = ny;
  a.o[0] = TcOut{t->t2, nullptr, nx};
  a.o[1] = TcOut{t->t3, nullptr, nx};
  if ((le = launch_chained(k_tc_gemm<EPI_SPLIT, 128>, dim3(nx / 128, ny / BM, 2), dim3(128), Tile<128>::SMEM_BYTES, s, t->mCy, t->mExh, t->mSy, t->mEyh, a)) != cudaSuccess) return le;
  // 4: Ex[x][y] = sum_u Sx[x][u] T2t[y][u]; Ey = Cx T3t^T     M = nx, N = ny, K = nx
  a.M = nx, a.N = ny, a.K = nx;
  a.o[0] = TcOut{field_x, nullptr, ny};
  a.o[1] = TcOut{field_y, nullptr, ny};
  if ((le = launch_chained(k_tc_gemm<EPI_F32, 128>, dim3(ny / 128, nx / BM, 2), dim3(128), Tile<128>::SMEM_BYTES, s, t->mSx, t->mT2, t->mCx, t->mT3, a)) != cudaSuccess) return le;
  return cudaGetLastError();
}

int tc_error(const PoissonPlan *p) {
  int h = 0;
  if (p->tc && p->tc->err) cudaMemcpy(&h, p->tc->err, sizeof h, cudaMemcpyDeviceToHost);
  return h;
}


// Loads this file's module (the driver loads a module at its first launch otherwise).
void load_module_poisson_tc() {
  cudaFuncAttributes a;
  cudaFuncGetAttributes(&a, k_tc_gemm<EPI_SPLIT, 64>);
}

}  // namespace gpl
