// esr_mlp.cu -- BF16 training and inference kernels of the warm-start MLP.
//
// The network corrects an IDW interpolation of the coarse solution cell by
// cell: 32 input features (13 used) -> 256 -> 3 residual blocks of 256 ->
// 4 outputs. Its 256-wide layers are GEMMs of rows (cells) x 256 x 256 run
// on the tensor cores by one kernel template:
//   C[M x N] = A[M x K] * B[K x N], BF16 operands, FP32 accumulation
//   (mma.sync m16n8k16), 128 x 128 x 32 CTA tiles, 8 warps of 64 x 32,
//   3-stage cp.async pipeline, ldmatrix (.trans for the transposed operands)
// with fused epilogues:
//   EPI_F32   store the FP32 tile (split-K partials of the weight gradients)
//   EPI_FWD   z = acc + bias; out = residual + relu(z)   (z kept for backward)
//   EPI_BWD   dh = acc + dh_next; dz_prev = dh * (z_prev > 0)
// The 4-wide head, the loss, AdamW and the fixed-order reductions are plain
// SIMT kernels. Every reduction is deterministic (no atomics).
#include <cuda_bf16.h>
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include <string>

#include "esr_internal.h"

namespace {

using bf16 = __nv_bfloat16;

constexpr int BM = 128, BN = 128, BK = 32, STAGES = 3, THREADS = 256;
constexpr int PAD = 8;
constexpr int LD_K = BK + PAD;     // row stride of K-contiguous tiles (elements)
constexpr int LD_MN = BM + PAD;    // row stride of M/N-contiguous tiles

enum { EPI_F32 = 0, EPI_FWD = 1, EPI_BWD = 2 };

struct Epi {
  const float* bias;     // FWD: per-column bias
  const bf16* res;       // FWD: residual input; BWD: dh of the next layer
  const bf16* aux;       // BWD: z of the previous layer (relu mask)
  void* out0;            // F32: float partials; FWD: activation out; BWD: dh
  bf16* out1;            // FWD: z; BWD: dz_prev
  int ldo;               // leading dimension of res/aux/out0/out1
  long long split_stride;// F32: elements between split-K partial tiles
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void ldsm_x4(unsigned r[4], const void* p) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(s));
}
__device__ __forceinline__ void ldsm_x4_t(unsigned r[4], const void* p) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(s));
}
__device__ __forceinline__ void mma_bf16(float c[4], const unsigned a[4], unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// A(m,k): A_T ? A[k*lda + m] : A[m*lda + k];  B(k,n): B_T ? B[k*ldb + n] : B[n*ldb + k]
template <bool A_T, bool B_T, int EPI>
__global__ void __launch_bounds__(THREADS) k_gemm(int M, int N, int K_split, const bf16* __restrict__ A, int lda,
                                                  const bf16* __restrict__ B, int ldb, Epi e) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int A_ELEMS = A_T ? BK * LD_MN : BM * LD_K;
  constexpr int B_ELEMS = B_T ? BK * LD_MN : BN * LD_K;
  bf16* sA = reinterpret_cast<bf16*>(smem_raw);
  bf16* sB = sA + STAGES * A_ELEMS;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wm = warp >> 2, wn = warp & 3;
  const int m_blk = blockIdx.y * BM, n_blk = blockIdx.x * BN;
  const int k_begin = blockIdx.z * K_split;
  const int KT = K_split / BK;

  auto load_tile = [&](int stage, int kt) {
    const int k0 = k_begin + kt * BK;
    bf16* a = sA + stage * A_ELEMS;
    bf16* b = sB + stage * B_ELEMS;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int c = tid + i * THREADS;   // 512 chunks of 8 elements per operand tile
      if (!A_T) {
        const int r = c >> 2, kc = (c & 3) * 8;
        cp_async16(a + r * LD_K + kc, A + (size_t)(m_blk + r) * lda + k0 + kc);
      } else {
        const int r = c >> 4, mc = (c & 15) * 8;
        cp_async16(a + r * LD_MN + mc, A + (size_t)(k0 + r) * lda + m_blk + mc);
      }
      if (!B_T) {
        const int r = c >> 2, kc = (c & 3) * 8;
        cp_async16(b + r * LD_K + kc, B + (size_t)(n_blk + r) * ldb + k0 + kc);
      } else {
        const int r = c >> 4, nc = (c & 15) * 8;
        cp_async16(b + r * LD_MN + nc, B + (size_t)(k0 + r) * ldb + n_blk + nc);
      }
    }
  };

  float acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < KT) load_tile(s, s);
    cp_async_commit();
  }
  for (int kt = 0; kt < KT; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    const int pf = kt + STAGES - 1;
    if (pf < KT) load_tile(pf % STAGES, pf);
    cp_async_commit();
    const bf16* a = sA + (kt % STAGES) * A_ELEMS;
    const bf16* b = sB + (kt % STAGES) * B_ELEMS;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 16) {
      unsigned af[4][4], bfr[2][4];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) {
        const int m0 = wm * 64 + mi * 16;
        if (!A_T) ldsm_x4(af[mi], a + (m0 + (lane & 15)) * LD_K + kk + (lane >> 4) * 8);
        else ldsm_x4_t(af[mi], a + (kk + (lane & 7) + (lane >> 4) * 8) * LD_MN + m0 + ((lane >> 3) & 1) * 8);
      }
#pragma unroll
      for (int nj = 0; nj < 2; ++nj) {
        const int n0 = wn * 32 + nj * 16;
        if (!B_T) ldsm_x4(bfr[nj], b + (n0 + (lane & 7) + (lane >> 4) * 8) * LD_K + kk + ((lane >> 3) & 1) * 8);
        else ldsm_x4_t(bfr[nj], b + (kk + (lane & 7) + ((lane >> 3) & 1) * 8) * LD_MN + n0 + (lane >> 4) * 8);
      }
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
          mma_bf16(acc[mi][ni], af[mi], bfr[ni >> 1][(ni & 1) * 2], bfr[ni >> 1][(ni & 1) * 2 + 1]);
    }
  }
  cp_async_wait<0>();

  const int g = lane >> 2, tig = lane & 3;
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int m = m_blk + wm * 64 + mi * 16 + g + h * 8;
        const int n = n_blk + wn * 32 + ni * 8 + tig * 2;
        const float v0 = acc[mi][ni][2 * h], v1 = acc[mi][ni][2 * h + 1];
        const size_t o = (size_t)m * e.ldo + n;
        if (EPI == EPI_F32) {
          float* out = static_cast<float*>(e.out0) + (size_t)blockIdx.z * e.split_stride;
          *reinterpret_cast<float2*>(out + o) = make_float2(v0, v1);
        } else if (EPI == EPI_FWD) {
          const float z0 = v0 + e.bias[n], z1 = v1 + e.bias[n + 1];
          float r0 = 0.f, r1 = 0.f;
          if (e.res) {
            const __nv_bfloat162 r = *reinterpret_cast<const __nv_bfloat162*>(e.res + o);
            r0 = __bfloat162float(r.x);
            r1 = __bfloat162float(r.y);
          }
          *reinterpret_cast<__nv_bfloat162*>(e.out1 + o) = __floats2bfloat162_rn(z0, z1);
          *reinterpret_cast<__nv_bfloat162*>(static_cast<bf16*>(e.out0) + o) =
              __floats2bfloat162_rn(r0 + fmaxf(z0, 0.f), r1 + fmaxf(z1, 0.f));
        } else {
          float d0 = v0, d1 = v1;
          if (e.res) {
            const __nv_bfloat162 r = *reinterpret_cast<const __nv_bfloat162*>(e.res + o);
            d0 += __bfloat162float(r.x);
            d1 += __bfloat162float(r.y);
          }
          *reinterpret_cast<__nv_bfloat162*>(static_cast<bf16*>(e.out0) + o) = __floats2bfloat162_rn(d0, d1);
          if (e.aux) {
            const __nv_bfloat162 z = *reinterpret_cast<const __nv_bfloat162*>(e.aux + o);
            *reinterpret_cast<__nv_bfloat162*>(e.out1 + o) = __floats2bfloat162_rn(
                __bfloat162float(z.x) > 0.f ? d0 : 0.f, __bfloat162float(z.y) > 0.f ? d1 : 0.f);
          }
        }
      }
}

// ------------------------------------------------------------- SIMT kernels
// y[r][j] = sum_k H[r][k] W[j][k] + b[j], 4 outputs, FP32 accumulation
__global__ void k_head_fwd(const bf16* __restrict__ H, int rows, int K, const float* __restrict__ W,
                           const float* __restrict__ b, const float* __restrict__ base, float* __restrict__ y) {
  const int r = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (r >= rows) return;
  float s[4] = {0.f, 0.f, 0.f, 0.f};
  for (int k = lane; k < K; k += 32) {
    const float h = __bfloat162float(H[(size_t)r * K + k]);
#pragma unroll
    for (int j = 0; j < 4; ++j) s[j] += h * W[j * K + k];
  }
#pragma unroll
  for (int j = 0; j < 4; ++j)
    for (int o = 16; o > 0; o >>= 1) s[j] += __shfl_xor_sync(0xffffffffu, s[j], o);
  if (lane < 4) y[(size_t)r * 4 + lane] = s[lane] + b[lane] + (base ? base[(size_t)r * 4 + lane] : 0.f);
}

// dH[r][k] = sum_j dY[r][j] W[j][k] as BF16, and dz = dH * (z > 0) of the
// last hidden pre-activation
__global__ void k_head_bwd_dx(const float* __restrict__ dY, int rows, int K, const float* __restrict__ W,
                              const bf16* __restrict__ z, bf16* __restrict__ dH, bf16* __restrict__ dZ) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)rows * K) return;
  const int r = (int)(i / K), k = (int)(i % K);
  float s = 0.f;
#pragma unroll
  for (int j = 0; j < 4; ++j) s += dY[(size_t)r * 4 + j] * W[j * K + k];
  dH[i] = __float2bfloat16(s);
  dZ[i] = __float2bfloat16(__bfloat162float(z[i]) > 0.f ? s : 0.f);
}

// Per-cell inputs of one case (BF16 rows of `ld` columns, zero padded):
// [x, y, wall distance, wall normal x, y (5 static), IDW primitives
// normalised (4), asinh(IDW dp/dx / s_p), asinh(dp/dy / s_p) (2), M_n, alpha_n]
__global__ void k_features(const float* __restrict__ stat5, const float* __restrict__ idw_prim,
                           const float* __restrict__ idw_gradp, int rows, float mach_n, float aoa_n,
                           const float* __restrict__ mu, const float* __restrict__ sig, int ld, bf16* __restrict__ X,
                           float* __restrict__ base) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  bf16* x = X + (size_t)r * ld;
  for (int j = 0; j < 5; ++j) x[j] = __float2bfloat16(stat5[(size_t)r * 5 + j]);
  for (int v = 0; v < 4; ++v) {
    const float q = (idw_prim[(size_t)r * 4 + v] - mu[v]) / sig[v];
    x[5 + v] = __float2bfloat16(q);
    if (base) base[(size_t)r * 4 + v] = q;   // the IDW prediction the MLP corrects
  }
  const float sp = sig[3] + 1e-8f;
  x[9] = __float2bfloat16(asinhf(idw_gradp[(size_t)r * 2] / sp));
  x[10] = __float2bfloat16(asinhf(idw_gradp[(size_t)r * 2 + 1] / sp));
  x[11] = __float2bfloat16(mach_n);
  x[12] = __float2bfloat16(aoa_n);
  for (int j = 13; j < ld; ++j) x[j] = __float2bfloat16(0.f);
}

// normalised primitive prediction -> conserved state (float64 rows), with
// density and pressure kept above `floor_frac` of their freestream values
__global__ void k_decode(const float* __restrict__ pred_n, int rows, const float* __restrict__ mu,
                         const float* __restrict__ sig, float gamma, float rho_floor, float p_floor,
                         double* __restrict__ W) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const float rho = fmaxf(pred_n[(size_t)r * 4] * sig[0] + mu[0], rho_floor);
  const float u = pred_n[(size_t)r * 4 + 1] * sig[1] + mu[1];
  const float v = pred_n[(size_t)r * 4 + 2] * sig[2] + mu[2];
  const float p = fmaxf(pred_n[(size_t)r * 4 + 3] * sig[3] + mu[3], p_floor);
  W[(size_t)r * 4] = rho;
  W[(size_t)r * 4 + 1] = (double)rho * u;
  W[(size_t)r * 4 + 2] = (double)rho * v;
  W[(size_t)r * 4 + 3] = (double)p / (gamma - 1.0) + 0.5 * (double)rho * ((double)u * u + (double)v * v);
}

// per-block partials of dW_head[j][k] = sum_r dY[r][j] H[r][k] and db[j] = sum_r dY[r][j]
__global__ void k_head_bwd_dw(const float* __restrict__ dY, const bf16* __restrict__ H, int rows, int K,
                              int rows_per_block, float* __restrict__ part) {
  const int k = threadIdx.x;            // blockDim.x == K (256)
  const int r0 = blockIdx.x * rows_per_block, r1 = min(rows, r0 + rows_per_block);
  float s[4] = {0.f, 0.f, 0.f, 0.f}, sb[4] = {0.f, 0.f, 0.f, 0.f};
  for (int r = r0; r < r1; ++r) {
    const float h = __bfloat162float(H[(size_t)r * K + k]);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float d = dY[(size_t)r * 4 + j];
      s[j] += d * h;
      sb[j] += d;
    }
  }
  float* p = part + (size_t)blockIdx.x * (4 * K + 4);
#pragma unroll
  for (int j = 0; j < 4; ++j) p[j * K + k] = s[j];
  if (k < 4) p[4 * K + k] = sb[k];
}

// out[i] = sum_s part[s * stride + i] in split order
__global__ void k_reduce_splits(const float* __restrict__ part, int splits, long long stride, long long n,
                                float* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = 0.f;
  for (int z = 0; z < splits; ++z) s += part[(size_t)z * stride + i];
  out[i] = s;
}

// column sums of a BF16 [rows x C] matrix in fixed row blocks (bias gradients)
__global__ void k_colsum_part(const bf16* __restrict__ X, int rows, int C, int rows_per_block, float* __restrict__ part) {
  const int c = blockIdx.y * blockDim.x + threadIdx.x;
  if (c >= C) return;
  const int r0 = blockIdx.x * rows_per_block, r1 = min(rows, r0 + rows_per_block);
  float s = 0.f;
  for (int r = r0; r < r1; ++r) s += __bfloat162float(X[(size_t)r * C + c]);
  part[(size_t)blockIdx.x * C + c] = s;
}

// shock-weighted relative MSE (loss.py:20-23) on pred = base + head:
// L = mean_v [ sum_r w_r (p - t)^2 / R / (mean_r t^2 + 1e-8) ]; dpred written;
// per-block partial sums of the loss numerators
__global__ void k_loss(const float* __restrict__ pred, const float* __restrict__ tgt, const float* __restrict__ w,
                       int rows, const float* __restrict__ inv_den, float* __restrict__ dpred,
                       float* __restrict__ part) {
  __shared__ float sh[256];
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (r < rows) {
    const float wr = w ? w[r] : 1.f;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const float d = pred[(size_t)r * 4 + v] - tgt[(size_t)r * 4 + v];
      l += wr * d * d * inv_den[v];
      dpred[(size_t)r * 4 + v] = 2.f * wr * d * inv_den[v] / (4.f * rows);
    }
  }
  sh[threadIdx.x] = l;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0] / (4.f * rows);
}

// AdamW on FP32 master weights with a BF16 (or FP32) working copy
__global__ void k_adamw(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                        float* __restrict__ v, long long n, float lr, float b1, float b2, float eps, float wd,
                        float bc1, float bc2, bf16* __restrict__ p_bf16) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float mh = mi / bc1, vh = vi / bc2;
  const float pi = p[i] * (1.f - lr * wd) - lr * mh / (sqrtf(vh) + eps);
  p[i] = pi;
  if (p_bf16) p_bf16[i] = __float2bfloat16(pi);
}

// ------------------------------------------------------ tcgen05 GEMM path
// The same C = A B with the fifth-generation tensor cores: TMA boxes bring
// the operands into shared memory in the 128-byte swizzled canonical layouts
// the UMMA descriptors describe, one thread issues the loads and
// tcgen05.mma (128 x N x 16, BF16 in, FP32 accumulators in tensor memory),
// mbarriers track each stage (tiles landed / MMAs done reading), and the
// epilogue reads the accumulators back with tcgen05.ld, stages them in shared
// memory and applies the epilogue in row-contiguous order.
namespace tc {

constexpr int BM = 128, BK = 64, THREADS = 256;
constexpr int A_BYTES = BM * BK * 2;                    // 16 KB of A per stage
constexpr int SLD = 128 + 4;                            // row stride (floats) of a staged 128-column accumulator half
constexpr long long kSpinLimit = 1LL << 20;             // bounded mbarrier polls

// Tile width 128 (3 stages) or 256 (2 stages): a 256-wide tile reads each
// 128-row block of A once for the whole 256-column output; both use 96 KB of
// pipeline buffers, so two CTAs fit on an SM.
template <int TBN>
struct Cfg {
  static constexpr int BN = TBN;
  static constexpr int STAGES = TBN == 256 ? 2 : 3;
  static constexpr int B_BYTES = TBN * BK * 2;
  static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  static constexpr int SMEM = 1024 + STAGES * STAGE_BYTES + (2 * STAGES + 1) * 8 + 16;
  static_assert(BM * SLD * 4 <= STAGES * STAGE_BYTES, "accumulator staging must fit the pipeline buffers");
};

__device__ int g_tc_error = 0;                          // set when a wait gave up

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count));
}
// true once the barrier's phase with this parity has completed; false after the spin limit
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (long long i = 0; i < kSpinLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done) : "r"(bar), "r"(parity) : "memory");
    if (done) return true;
  }
  atomicExch(&g_tc_error, 1);
  return false;
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// Shared-memory matrix descriptor, 128-byte swizzle. K-major: rows of 64
// elements (128 B), 8-row groups 1024 B apart (SBO), LBO unused (1).
// MN-major: 64-element MN groups `lbo` bytes apart, 8-row K groups 1024 B apart.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;                // descriptor version of sm_100
  d |= (uint64_t)2 << 61;                // SWIZZLE_128B
  return d;
}

// kind::f16 instruction descriptor: FP32 accumulate, BF16 A and B, majors, N, M
template <bool A_MN, bool B_MN, int N>
__host__ __device__ constexpr uint32_t instr_desc() {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((A_MN ? 1u : 0u) << 15) | ((B_MN ? 1u : 0u) << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
      ::"r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar) : "memory");
}
// TMA: one 2-D box of a tensor map into shared memory, completion counted in
// bytes on an mbarrier (no multicast)
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
      ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t v[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// Shared-memory tile layouts (what the TMA boxes with the 128-byte swizzle
// produce and the UMMA descriptors describe). K-major tile (rows x 64 K):
// row r at r * 128 B, its 16-byte chunk c at ((c ^ (r & 7)) * 16). MN-major
// tile (64 K-rows x MN): groups of 64 MN elements 8 KB apart, K-row k of a
// group at (k >> 3) * 1024 + (k & 7) * 128 B, chunk c at ((c ^ (k & 7)) * 16).

template <bool A_T, bool B_T, int EPI, int TBN>
__global__ void __launch_bounds__(THREADS) k_gemm_tc(int M, int N, int K_split, const __grid_constant__ CUtensorMap tmA,
                                                     const __grid_constant__ CUtensorMap tmB, Epi e) {
  using C = Cfg<TBN>;
  constexpr int BN = C::BN, STAGES = C::STAGES, STAGE_BYTES = C::STAGE_BYTES;
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = saddr(smem_raw);
  const uint32_t tiles = (raw + 1023u) & ~1023u;                   // swizzle atoms need 1 KB alignment
  unsigned char* gtiles = smem_raw + (tiles - raw);
  const uint32_t empty = tiles + STAGES * STAGE_BYTES;             // per stage: MMAs done reading it
  const uint32_t full = empty + STAGES * 8;                        // per stage: its tiles have landed
  const uint32_t done = full + STAGES * 8;                         // all MMAs of the tile are done
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gtiles + STAGES * STAGE_BYTES + (2 * STAGES + 1) * 8);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m_blk = blockIdx.y * BM, n_blk = blockIdx.x * BN;
  const int k_begin = blockIdx.z * K_split;
  const int KT = K_split / BK;

  __shared__ int s_abort;   // set when a pipeline wait gave up: the tile is not written
  if (tid == 0) {
    s_abort = 0;
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(empty + 8 * s, 1);
      mbar_init(full + 8 * s, 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {   // BN TMEM columns: the 128 x BN FP32 accumulator
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(saddr(tmem_slot)), "n"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  // One thread is both the TMA producer and the MMA issuer; the other warps
  // wait for the last MMA and then run the epilogue.
  if (warp == 0) {
    if (lane == 0) {
      // the tiles of K-block kt into stage s: K-major boxes are 64 K x rows,
      // MN-major boxes 64 MN x 64 K, one per 64-element MN group (8 KB apart)
      auto produce = [&](int kt, int s) {
        const int k0 = k_begin + kt * BK;
        const uint32_t a = tiles + s * STAGE_BYTES, b = a + A_BYTES, bar = full + 8 * s;
        mbar_expect_tx(bar, STAGE_BYTES);
        if (!A_T) tma_load_2d(a, &tmA, k0, m_blk, bar);
        else for (int g = 0; g < BM / 64; ++g) tma_load_2d(a + g * 8192, &tmA, m_blk + 64 * g, k0, bar);
        if (!B_T) tma_load_2d(b, &tmB, k0, n_blk, bar);
        else for (int g = 0; g < BN / 64; ++g) tma_load_2d(b + g * 8192, &tmB, n_blk + 64 * g, k0, bar);
      };
      constexpr uint32_t idesc = instr_desc<A_T, B_T, BN>();
      int issued = 0;      // K-blocks whose loads have been issued
      int landed = 0;      // K-blocks whose loads are known to have landed
      bool ok = true;
      for (int p = 0; p < STAGES && p < KT; ++p) { produce(p, p); issued = p + 1; }
      for (int kt = 0; kt < KT && ok; ++kt) {
        const int s = kt % STAGES;
        if (!mbar_wait(full + 8 * s, (kt / STAGES) & 1)) { ok = false; break; }
        landed = kt + 1;
        tc_fence_after();
        const uint32_t a = tiles + s * STAGE_BYTES, b = a + A_BYTES;
#pragma unroll
        for (int j = 0; j < BK / 16; ++j) {   // K = 16 per instruction
          const uint64_t ad = A_T ? smem_desc(a + j * 2048, 8192, 1024) : smem_desc(a + j * 32, 16, 1024);
          const uint64_t bd = B_T ? smem_desc(b + j * 2048, 8192, 1024) : smem_desc(b + j * 32, 16, 1024);
          umma(tmem, ad, bd, idesc, (kt | j) != 0);
        }
        umma_commit(empty + 8 * s);   // arrives when these MMAs (and all earlier ones) are done
        // refill the stage the MMAs of the previous K-block read, once they are done
        const int nxt = kt - 1 + STAGES;
        if (kt >= 1 && nxt < KT) {
          const int ps = (kt - 1) % STAGES;
          if (!mbar_wait(empty + 8 * ps, ((kt - 1) / STAGES) & 1)) { ok = false; break; }
          produce(nxt, ps);
          issued = nxt + 1;
        }
      }
      if (!ok) {
        // A wait gave up: nothing more is issued. Loads already issued may
        // still be landing in shared memory; give each a bounded wait before
        // the block can exit (each stage has at most one load outstanding).
        for (int j = landed; j < issued; ++j) mbar_wait(full + 8 * (j % STAGES), (j / STAGES) & 1);
        s_abort = 1;
      }
      umma_commit(done);   // its one phase completes when every MMA issued so far has
    }
    __syncwarp();
  }
  // The other warps reach this wait while the mainloop is still running. A
  // stage barrier cannot serve here: waiting on parity 1 of a barrier still in
  // its first phase returns at once. `done` completes exactly once.
  const bool done_ok = mbar_wait(done, 0);
  if (!done_ok) atomicOr(&s_abort, 1);
  __syncthreads();
  if (s_abort) {
    // The tile is not complete: write nothing. The accumulator is released
    // once the MMAs issued have finished (one more bounded wait), so the
    // block holds no tensor memory when it returns; the host sees the flag.
    if (warp == 0) {
      if (!done_ok) mbar_wait(done, 0);
      __syncwarp();
      tc_fence_after();
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "n"(BN));
    }
    return;
  }
  tc_fence_after();

  // Accumulators -> shared memory (the pipeline buffers are free now), 128
  // columns at a time: warp w reads TMEM lanes 32 (w % 4) .. +31 (rows) and
  // columns 64 (w / 4) .. +63 of the half.
  float* stile = reinterpret_cast<float*>(gtiles);
#pragma unroll 1
  for (int h = 0; h < BN / 128; ++h) {
    if (h > 0) __syncthreads();   // the previous half has been stored
    {
      const int wq = warp & 3, col0 = (warp >> 2) * 64;
      const int r = wq * 32 + lane;
#pragma unroll
      for (int cc = 0; cc < 64; cc += 16) {
        uint32_t v[16];
        tmem_ld16(tmem + ((uint32_t)(wq * 32) << 16) + (uint32_t)(h * 128 + col0 + cc), v);
        float4* dst = reinterpret_cast<float4*>(stile + r * SLD + col0 + cc);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          dst[q] = make_float4(__uint_as_float(v[4 * q]), __uint_as_float(v[4 * q + 1]), __uint_as_float(v[4 * q + 2]),
                               __uint_as_float(v[4 * q + 3]));
      }
    }
    tc_fence_before();
    __syncthreads();
    if (h == BN / 128 - 1 && warp == 0) {   // every tcgen05.ld has completed: release the accumulator
      tc_fence_after();
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "n"(BN));
    }
    // epilogue in row-contiguous order: a warp covers 32 column pairs of one row
#pragma unroll 4
    for (int it = 0; it < (BM * 128 / 2) / THREADS; ++it) {
      const int q = it * THREADS + tid;
      const int r = q / 64, cp = q % 64;
      const int m = m_blk + r, n = n_blk + h * 128 + 2 * cp;
      const float2 acc = *reinterpret_cast<const float2*>(stile + r * SLD + 2 * cp);
      const float v0 = acc.x, v1 = acc.y;
      const size_t o = (size_t)m * e.ldo + n;
      if (EPI == EPI_F32) {
        float* out = static_cast<float*>(e.out0) + (size_t)blockIdx.z * e.split_stride;
        *reinterpret_cast<float2*>(out + o) = make_float2(v0, v1);
      } else if (EPI == EPI_FWD) {
        const float z0 = v0 + e.bias[n], z1 = v1 + e.bias[n + 1];
        float r0 = 0.f, r1 = 0.f;
        if (e.res) {
          const __nv_bfloat162 rr = *reinterpret_cast<const __nv_bfloat162*>(e.res + o);
          r0 = __bfloat162float(rr.x);
          r1 = __bfloat162float(rr.y);
        }
        *reinterpret_cast<__nv_bfloat162*>(e.out1 + o) = __floats2bfloat162_rn(z0, z1);
        *reinterpret_cast<__nv_bfloat162*>(static_cast<bf16*>(e.out0) + o) =
            __floats2bfloat162_rn(r0 + fmaxf(z0, 0.f), r1 + fmaxf(z1, 0.f));
      } else {
        float d0 = v0, d1 = v1;
        if (e.res) {
          const __nv_bfloat162 rr = *reinterpret_cast<const __nv_bfloat162*>(e.res + o);
          d0 += __bfloat162float(rr.x);
          d1 += __bfloat162float(rr.y);
        }
        *reinterpret_cast<__nv_bfloat162*>(static_cast<bf16*>(e.out0) + o) = __floats2bfloat162_rn(d0, d1);
        if (e.aux) {
          const __nv_bfloat162 zz = *reinterpret_cast<const __nv_bfloat162*>(e.aux + o);
          *reinterpret_cast<__nv_bfloat162*>(e.out1 + o) = __floats2bfloat162_rn(
              __bfloat162float(zz.x) > 0.f ? d0 : 0.f, __bfloat162float(zz.y) > 0.f ? d1 : 0.f);
        }
      }
    }
  }
}

}  // namespace tc

int mfail(int code, const std::string& msg) { return esr::report_error(code, msg); }

template <bool AT, bool BT, int EPI>
int launch_gemm(int M, int N, int K, int splits, const bf16* A, int lda, const bf16* B, int ldb, const Epi& e,
                cudaStream_t st) {
  constexpr int A_ELEMS = AT ? BK * LD_MN : BM * LD_K;
  constexpr int B_ELEMS = BT ? BK * LD_MN : BN * LD_K;
  const int smem = STAGES * (A_ELEMS + B_ELEMS) * (int)sizeof(bf16);
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_gemm<AT, BT, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    attr_set = true;
  }
  dim3 grid(N / BN, M / BM, splits);
  k_gemm<AT, BT, EPI><<<grid, THREADS, smem, st>>>(M, N, K / splits, A, lda, B, ldb, e);
  return ESR_OK;
}

// 2-D BF16 tensor map: `inner` contiguous elements per row, `outer` rows,
// rows `ld` elements apart; boxes of box_in x box_out with the 128-byte swizzle
// the UMMA descriptors expect
int make_map(CUtensorMap* map, const bf16* base, uint64_t inner, uint64_t outer, uint64_t ld, uint32_t box_in,
             uint32_t box_out) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult q{};
    void* fn = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return mfail(ESR_ERR_CUDA, "gemm: cuTensorMapEncodeTiled is not available");
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  const cuuint64_t dims[2] = {inner, outer};
  const cuuint64_t strides[1] = {ld * sizeof(bf16)};
  const cuuint32_t box[2] = {box_in, box_out};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16*>(base), dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return mfail(ESR_ERR_ARG, "gemm: tensor map rejected (error " + std::to_string((int)r) + ")");
  return ESR_OK;
}

template <bool AT, bool BT, int EPI>
int launch_gemm_tc(int M, int N, int K, int splits, const bf16* A, int lda, const bf16* B, int ldb, const Epi& e,
                   cudaStream_t st) {
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(tc::k_gemm_tc<AT, BT, EPI, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         tc::Cfg<128>::SMEM);
    cudaFuncSetAttribute(tc::k_gemm_tc<AT, BT, EPI, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         tc::Cfg<256>::SMEM);
    attr_set = true;
  }
  // 256-wide tiles (A read once per row block) when there are still enough
  // of them to give every SM one; otherwise 128-wide tiles for parallelism
  const int tbn = (N % 256 == 0 && (long long)(M / tc::BM) * (N / 256) * splits >= 148) ? 256 : 128;
  CUtensorMap ma, mb;
  int rc = AT ? make_map(&ma, A, M, K, lda, 64, 64) : make_map(&ma, A, K, M, lda, 64, tc::BM);
  if (rc != ESR_OK) return rc;
  rc = BT ? make_map(&mb, B, N, K, ldb, 64, 64) : make_map(&mb, B, K, N, ldb, 64, tbn);
  if (rc != ESR_OK) return rc;
  if (tbn == 256) {
    dim3 grid(N / 256, M / tc::BM, splits);
    tc::k_gemm_tc<AT, BT, EPI, 256><<<grid, tc::THREADS, tc::Cfg<256>::SMEM, st>>>(M, N, K / splits, ma, mb, e);
  } else {
    dim3 grid(N / 128, M / tc::BM, splits);
    tc::k_gemm_tc<AT, BT, EPI, 128><<<grid, tc::THREADS, tc::Cfg<128>::SMEM, st>>>(M, N, K / splits, ma, mb, e);
  }
  return ESR_OK;
}

}  // namespace

extern "C" {

// C = A * B with the epilogue `epi` (0 F32 split-K partials, 1 forward, 2 backward).
// trans_a: A stored [K][M] (lda >= M); else [M][K] (lda >= K).
// trans_b: B stored [K][N] (ldb >= N); else [N][K] (ldb >= K).
// M, N multiples of 128; K a multiple of 32 * splits; rows 16-byte aligned.
namespace {
// argument checks shared by both GEMM paths; bk = K granularity of the kernel
int gemm_check(int32_t trans_a, int32_t trans_b, int32_t M, int32_t N, int32_t K, const void* A, int32_t lda,
               const void* B, int32_t ldb, int32_t epi, const float* bias, const void* aux, void* out0, void* out1,
               int32_t ldo, int32_t splits, int bk) {
  if (!A || !B || !out0) return mfail(ESR_ERR_ARG, "gemm: null operand");
  if (M <= 0 || N <= 0 || K <= 0 || M % BM || N % BN) return mfail(ESR_ERR_ARG, "gemm: M and N must be multiples of 128");
  if (splits < 1 || K % (bk * splits))
    return mfail(ESR_ERR_ARG, "gemm: K must be a multiple of " + std::to_string(bk) + " x splits");
  if (lda % 8 || ldb % 8 || ldo % 2) return mfail(ESR_ERR_ARG, "gemm: leading dimensions must keep 16-byte rows");
  if ((trans_a ? lda < M : lda < K) || (trans_b ? ldb < N : ldb < K) || ldo < N)
    return mfail(ESR_ERR_ARG, "gemm: leading dimension too small");
  if (((uintptr_t)A | (uintptr_t)B) & 15) return mfail(ESR_ERR_ARG, "gemm: operands must be 16-byte aligned");
  if (epi == EPI_FWD && (!bias || !out1)) return mfail(ESR_ERR_ARG, "gemm: forward epilogue needs bias and z output");
  if (epi == EPI_BWD && aux && !out1) return mfail(ESR_ERR_ARG, "gemm: backward epilogue with z needs dz output");
  if (epi != EPI_F32 && splits != 1) return mfail(ESR_ERR_ARG, "gemm: split-K only with the F32 epilogue");
  return ESR_OK;
}
}  // namespace

int esr_gemm_bf16(int32_t trans_a, int32_t trans_b, int32_t M, int32_t N, int32_t K, const void* A, int32_t lda,
                  const void* B, int32_t ldb, int32_t epi, const float* bias, const void* res, const void* aux,
                  void* out0, void* out1, int32_t ldo, int32_t splits, void* stream) {
  const int rc = gemm_check(trans_a, trans_b, M, N, K, A, lda, B, ldb, epi, bias, aux, out0, out1, ldo, splits, tc::BK);
  if (rc != ESR_OK) return rc;
  Epi e{bias, (const bf16*)res, (const bf16*)aux, out0, (bf16*)out1, ldo, (long long)M * ldo};
  cudaStream_t st = (cudaStream_t)stream;
  const bf16* a = (const bf16*)A;
  const bf16* b = (const bf16*)B;
#define ESR_GEMM_CASE(TA, TB, E) \
  if (!!trans_a == TA && !!trans_b == TB && epi == E) launch_gemm_tc<TA, TB, E>(M, N, K, splits, a, lda, b, ldb, e, st); else
  ESR_GEMM_CASE(false, false, EPI_FWD)
  ESR_GEMM_CASE(false, true, EPI_BWD)
  ESR_GEMM_CASE(true, true, EPI_F32)
  ESR_GEMM_CASE(false, false, EPI_F32)
  ESR_GEMM_CASE(false, true, EPI_F32)
  ESR_GEMM_CASE(false, false, EPI_BWD)
  return mfail(ESR_ERR_ARG, "gemm: unsupported layout/epilogue combination");
#undef ESR_GEMM_CASE
  cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? ESR_OK : mfail(ESR_ERR_CUDA, std::string("gemm: ") + cudaGetErrorString(err));
}

int esr_gemm_bf16_mma_sync(int32_t trans_a, int32_t trans_b, int32_t M, int32_t N, int32_t K, const void* A,
                           int32_t lda, const void* B, int32_t ldb, int32_t epi, const float* bias, const void* res,
                           const void* aux, void* out0, void* out1, int32_t ldo, int32_t splits, void* stream) {
  const int rc = gemm_check(trans_a, trans_b, M, N, K, A, lda, B, ldb, epi, bias, aux, out0, out1, ldo, splits, BK);
  if (rc != ESR_OK) return rc;
  Epi e{bias, (const bf16*)res, (const bf16*)aux, out0, (bf16*)out1, ldo, (long long)M * ldo};
  cudaStream_t st = (cudaStream_t)stream;
  const bf16* a = (const bf16*)A;
  const bf16* b = (const bf16*)B;
#define ESR_GEMM_CASE(TA, TB, E) \
  if (!!trans_a == TA && !!trans_b == TB && epi == E) launch_gemm<TA, TB, E>(M, N, K, splits, a, lda, b, ldb, e, st); else
  ESR_GEMM_CASE(false, false, EPI_FWD)
  ESR_GEMM_CASE(false, true, EPI_BWD)
  ESR_GEMM_CASE(true, true, EPI_F32)
  ESR_GEMM_CASE(false, false, EPI_F32)
  ESR_GEMM_CASE(false, true, EPI_F32)
  ESR_GEMM_CASE(false, false, EPI_BWD)
  return mfail(ESR_ERR_ARG, "gemm: unsupported layout/epilogue combination");
#undef ESR_GEMM_CASE
  cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? ESR_OK : mfail(ESR_ERR_CUDA, std::string("gemm: ") + cudaGetErrorString(err));
}

int esr_gemm_tc_status(int32_t* gave_up) {
  if (!gave_up) return mfail(ESR_ERR_ARG, "gemm_tc_status: null output");
  int v = 0;
  const int zero = 0;
  cudaError_t err = cudaMemcpyFromSymbol(&v, tc::g_tc_error, sizeof(int));
  if (err == cudaSuccess) err = cudaMemcpyToSymbol(tc::g_tc_error, &zero, sizeof(int));
  if (err != cudaSuccess) return mfail(ESR_ERR_CUDA, std::string("gemm_tc_status: ") + cudaGetErrorString(err));
  *gave_up = v;
  return ESR_OK;
}

// 4-wide head: y = H W^T + b (+ base); H [rows x K] BF16, W [4 x K] FP32
int esr_mlp_head_fwd(const void* H, int32_t rows, int32_t K, const float* W, const float* b, const float* base,
                     float* y, void* stream) {
  if (!H || !W || !b || !y || rows <= 0 || K <= 0) return mfail(ESR_ERR_ARG, "head_fwd: bad argument");
  const int wpb = 8;
  k_head_fwd<<<(rows + wpb - 1) / wpb, wpb * 32, 0, (cudaStream_t)stream>>>((const bf16*)H, rows, K, W, b, base, y);
  cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? ESR_OK : mfail(ESR_ERR_CUDA, cudaGetErrorString(err));
}

// head backward: dH = dY W and dZ = dH * (z > 0) (BF16), dW/db partials per
// block of `rpb` rows (4*K + 4 floats per block)
int esr_mlp_head_bwd(const float* dY, const void* H, const void* Z, int32_t rows, int32_t K, const float* W, void* dH,
                     void* dZ, float* part, int32_t rpb, void* stream) {
  if (!dY || !H || !Z || !W || !dH || !dZ || !part || rows <= 0 || K != 256 || rpb <= 0)
    return mfail(ESR_ERR_ARG, "head_bwd: bad argument");
  cudaStream_t st = (cudaStream_t)stream;
  const long long n = (long long)rows * K;
  k_head_bwd_dx<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(dY, rows, K, W, (const bf16*)Z, (bf16*)dH, (bf16*)dZ);
  k_head_bwd_dw<<<(rows + rpb - 1) / rpb, K, 0, st>>>(dY, (const bf16*)H, rows, K, rpb, part);
  cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? ESR_OK : mfail(ESR_ERR_CUDA, cudaGetErrorString(err));
}

int esr_mlp_features(const float* stat5, const float* idw_prim, const float* idw_gradp, int32_t rows, float mach_n,
                     float aoa_n, const float* mu, const float* sig, int32_t ld, void* X, float* base, void* stream) {
  if (!stat5 || !idw_prim || !idw_gradp || !mu || !sig || !X || rows <= 0 || ld < 13)
    return mfail(ESR_ERR_ARG, "features: bad argument");
  k_features<<<(rows + 127) / 128, 128, 0, (cudaStream_t)stream>>>(stat5, idw_prim, idw_gradp, rows, mach_n, aoa_n,
                                                                   mu, sig, ld, (bf16*)X, base);
  cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? ESR_OK : mfail(ESR_ERR_CUDA, cudaGetErrorString(err));
}

int esr_mlp_decode(const float* pred_n, int32_t rows, const float* mu, const float* sig, float gamma, float rho_floor,
                   float p_floor, double* W, void* stream) {
  if (!pred_n || !mu || !sig || !W || rows <= 0) return mfail(ESR_ERR_ARG, "decode: bad argument");
  k_decode<<<(rows + 127) / 128, 128, 0, (cudaStream_t)stream>>>(pred_n, rows, mu, sig, gamma, rho_floor, p_floor, W);
  cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? ESR_OK : mfail(ESR_ERR_CUDA, cudaGetErrorString(err));
}

int esr_reduce_splits(const float* part, int32_t splits, int64_t stride, int64_t n, float* out, void* stream) {
  if (!part || !out || splits <= 0 || n <= 0 || stride < n) return mfail(ESR_ERR_ARG, "reduce_splits: bad argument");
  k_reduce_splits<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(part, splits, stride, n, out);
  cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? ESR_OK : mfail(ESR_ERR_CUDA, cudaGetErrorString(err));
}

int esr_colsum_bf16(const void* X, int32_t rows, int32_t C, int32_t rpb, float* part, void* stream) {
  if (!X || !part || rows <= 0 || C <= 0 || rpb <= 0) return mfail(ESR_ERR_ARG, "colsum: bad argument");
  dim3 grid((rows + rpb - 1) / rpb, (C + 127) / 128);
  k_colsum_part<<<grid, 128, 0, (cudaStream_t)stream>>>((const bf16*)X, rows, C, rpb, part);
  cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? ESR_OK : mfail(ESR_ERR_CUDA, cudaGetErrorString(err));
}

int esr_mlp_loss(const float* pred, const float* tgt, const float* w, int32_t rows, const float* inv_den,
                 float* dpred, float* part, void* stream) {
  if (!pred || !tgt || !inv_den || !dpred || !part || rows <= 0) return mfail(ESR_ERR_ARG, "loss: bad argument");
  k_loss<<<(rows + 255) / 256, 256, 0, (cudaStream_t)stream>>>(pred, tgt, w, rows, inv_den, dpred, part);
  cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? ESR_OK : mfail(ESR_ERR_CUDA, cudaGetErrorString(err));
}

int esr_adamw(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2, float eps,
              float wd, int32_t step, void* p_bf16, void* stream) {
  if (!p || !g || !m || !v || n <= 0 || step < 1) return mfail(ESR_ERR_ARG, "adamw: bad argument");
  const float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
  k_adamw<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(p, g, m, v, n, lr, b1, b2, eps, wd, bc1, bc2,
                                                                         (bf16*)p_bf16);
  cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? ESR_OK : mfail(ESR_ERR_CUDA, cudaGetErrorString(err));
}

}  // extern "C"
