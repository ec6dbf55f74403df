// Learned value surrogate: BF16 tensor-core GEMMs with FP32 accumulation and
// the fused element-wise kernels of an MLP's forward pass, backward pass and
// Adam update.  The reference's precedent is a SiLU MLP trained by Adam on
// MSE against DP labels (local_game/learning.py:32-38, training.py:185-186,
// :352); here every kernel is hand-written.
//
// GEMM: C[M x N] = A[M x K] * B[K x N] with A stored either K-major
// ([M][K]) or M-major ([K][M]) and B stored either K-major ([N][K]) or
// N-major ([K][N]), bf16 operands, fp32 accumulation through
// mma.sync.m16n8k16, 128 x 128 x 32 CTA tiles of 8 warps (64 x 32 each),
// cp.async double buffering and ldmatrix(.trans) fragment loads.  Epilogues:
// store fp32, bias + SiLU (fp32 pre-activation and bf16 activation out),
// split-K atomic accumulation, and "times SiLU'(z)" for back-propagation.
#include <cuda_bf16.h>

#include <cstdint>

#include "pe_internal.h"

namespace pe {
namespace {

constexpr int BM = 128, BN = 128, BK = 32;
constexpr int THREADS = 256;
constexpr int PAD = 8;  // bf16 elements of row padding against bank conflicts

enum Epilogue { EPI_F32 = 0, EPI_BIAS_SILU = 1, EPI_ATOMIC = 2, EPI_DSILU = 3 };

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem)),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void ldsm_x4(uint32_t &r0, uint32_t &r1, uint32_t &r2,
                                        uint32_t &r3, const void *p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t &r0, uint32_t &r1, uint32_t &r2,
                                          uint32_t &r3, const void *p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(smem_u32(p)));
}

__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4],
                                         const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ float silu(float z) { return z / (1.f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = 1.f / (1.f + __expf(-z));
  return s * (1.f + z * (1.f - s));
}

struct GemmArgs {
  const __nv_bfloat16 *A, *B;
  int M, N, K;        // K: this launch's full reduction length
  int lda, ldb;       // leading dimensions (elements) of the stored arrays
  int k_split;        // reduction length per CTA (split-K), multiple of BK
  float *C32;         // EPI_F32 / EPI_ATOMIC / EPI_BIAS_SILU (pre-activation)
  __nv_bfloat16 *C16; // EPI_BIAS_SILU (activation) / EPI_DSILU (gradient)
  int ldc;
  const float *bias;  // EPI_BIAS_SILU
  const float *zpre;  // EPI_DSILU: pre-activation of the layer, [M][ldc]
};

// Shared tile of A: K-major [BM][BK+PAD] or M-major [BK][BM+PAD]; of B:
// K-major [BN][BK+PAD] or N-major [BK][BN+PAD].
template <bool A_MMAJOR>
__device__ __forceinline__ int a_tile_elems() {
  return A_MMAJOR ? BK * (BM + PAD) : BM * (BK + PAD);
}
template <bool B_NMAJOR>
__device__ __forceinline__ int b_tile_elems() {
  return B_NMAJOR ? BK * (BN + PAD) : BN * (BK + PAD);
}

template <bool A_MMAJOR, bool B_NMAJOR>
__device__ __forceinline__ void load_tiles(const GemmArgs &g, __nv_bfloat16 *As,
                                           __nv_bfloat16 *Bs, int m0, int n0,
                                           int k0) {
  const int tid = threadIdx.x;
  // 512 16-byte chunks per tile, two per thread.
#pragma unroll
  for (int i = 0; i < 2; i++) {
    const int c = tid + i * THREADS;
    if (A_MMAJOR) {  // rows k (BK), 16 chunks of 8 m per row
      const int r = c / 16, col = (c % 16) * 8;
      cp_async16(As + r * (BM + PAD) + col, g.A + (int64_t)(k0 + r) * g.lda + m0 + col);
    } else {  // rows m (BM), 4 chunks of 8 k per row
      const int r = c / 4, col = (c % 4) * 8;
      cp_async16(As + r * (BK + PAD) + col, g.A + (int64_t)(m0 + r) * g.lda + k0 + col);
    }
    if (B_NMAJOR) {
      const int r = c / 16, col = (c % 16) * 8;
      cp_async16(Bs + r * (BN + PAD) + col, g.B + (int64_t)(k0 + r) * g.ldb + n0 + col);
    } else {
      const int r = c / 4, col = (c % 4) * 8;
      cp_async16(Bs + r * (BK + PAD) + col, g.B + (int64_t)(n0 + r) * g.ldb + k0 + col);
    }
  }
}

template <bool A_MMAJOR, bool B_NMAJOR, int EPI>
__global__ void __launch_bounds__(THREADS) gemm_kernel(const GemmArgs g) {
  extern __shared__ __align__(128) __nv_bfloat16 smem[];
  const int a_elems = a_tile_elems<A_MMAJOR>(), b_elems = b_tile_elems<B_NMAJOR>();
  __nv_bfloat16 *As[2] = {smem, smem + a_elems};
  __nv_bfloat16 *Bs[2] = {smem + 2 * a_elems, smem + 2 * a_elems + b_elems};
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int kbeg = blockIdx.z * g.k_split;
  const int kend = min(g.K, kbeg + g.k_split);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = (warp >> 2) * 64, wn = (warp & 3) * 32;  // warp tile origin
  float acc[4][4][4] = {};

  int stage = 0;
  if (kbeg < kend) load_tiles<A_MMAJOR, B_NMAJOR>(g, As[0], Bs[0], m0, n0, kbeg);
  cp_async_commit();
  for (int k0 = kbeg; k0 < kend; k0 += BK) {
    if (k0 + BK < kend) load_tiles<A_MMAJOR, B_NMAJOR>(g, As[stage ^ 1], Bs[stage ^ 1], m0, n0, k0 + BK);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const __nv_bfloat16 *as = As[stage], *bs = Bs[stage];
#pragma unroll
    for (int kk = 0; kk < BK; kk += 16) {
      uint32_t af[4][4], bf[4][2];
      const int j = lane >> 3, r = lane & 7;
#pragma unroll
      for (int mi = 0; mi < 4; mi++) {
        const int mrow = wm + mi * 16;
        if (A_MMAJOR)  // stored [k][m]: matrix j covers k half j/2, m half j%2
          ldsm_x4_t(af[mi][0], af[mi][1], af[mi][2], af[mi][3],
                    as + (kk + (j >> 1) * 8 + r) * (BM + PAD) + mrow + (j & 1) * 8);
        else           // stored [m][k]: matrix j covers m half j%2, k half j/2
          ldsm_x4(af[mi][0], af[mi][1], af[mi][2], af[mi][3],
                  as + (mrow + (j & 1) * 8 + r) * (BK + PAD) + kk + (j >> 1) * 8);
      }
#pragma unroll
      for (int ni = 0; ni < 4; ni += 2) {
        const int ncol = wn + ni * 8;
        uint32_t r0, r1, r2, r3;
        if (B_NMAJOR) {  // stored [k][n]: matrix j: k half j%2, n tile j/2
          ldsm_x4_t(r0, r1, r2, r3,
                    bs + (kk + (j & 1) * 8 + r) * (BN + PAD) + ncol + (j >> 1) * 8);
        } else {         // stored [n][k]: matrix j: k half j%2, n tile j/2
          ldsm_x4(r0, r1, r2, r3,
                  bs + (ncol + (j >> 1) * 8 + r) * (BK + PAD) + kk + (j & 1) * 8);
        }
        bf[ni][0] = r0;
        bf[ni][1] = r1;
        bf[ni + 1][0] = r2;
        bf[ni + 1][1] = r3;
      }
#pragma unroll
      for (int mi = 0; mi < 4; mi++)
#pragma unroll
        for (int ni = 0; ni < 4; ni++) mma_bf16(acc[mi][ni], af[mi], bf[ni]);
    }
    __syncthreads();
    stage ^= 1;
  }

  // Epilogue.  acc[mi][ni] = rows {g, g+8}, cols {2t, 2t+1} of the 16x8 tile.
  const int gid = lane >> 2, tig = lane & 3;
#pragma unroll
  for (int mi = 0; mi < 4; mi++)
#pragma unroll
    for (int ni = 0; ni < 4; ni++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int row = m0 + wm + mi * 16 + gid + h * 8;
        const int col = n0 + wn + ni * 8 + tig * 2;
        float v0 = acc[mi][ni][2 * h], v1 = acc[mi][ni][2 * h + 1];
        const int64_t o = (int64_t)row * g.ldc + col;
        if (EPI == EPI_F32) {
          *reinterpret_cast<float2 *>(g.C32 + o) = make_float2(v0, v1);
        } else if (EPI == EPI_ATOMIC) {
          atomicAdd(g.C32 + o, v0);
          atomicAdd(g.C32 + o + 1, v1);
        } else if (EPI == EPI_BIAS_SILU) {
          v0 += g.bias[col];
          v1 += g.bias[col + 1];
          if (g.C32) *reinterpret_cast<float2 *>(g.C32 + o) = make_float2(v0, v1);
          *reinterpret_cast<__nv_bfloat162 *>(g.C16 + o) =
              __floats2bfloat162_rn(silu(v0), silu(v1));
        } else {  // EPI_DSILU: gradient w.r.t. the pre-activation
          const float2 z = *reinterpret_cast<const float2 *>(g.zpre + o);
          *reinterpret_cast<__nv_bfloat162 *>(g.C16 + o) =
              __floats2bfloat162_rn(v0 * silu_grad(z.x), v1 * silu_grad(z.y));
        }
      }
}

template <bool AM, bool BN_, int EPI>
cudaError_t launch_gemm(const GemmArgs &g, int splits, cudaStream_t stream) {
  const size_t smem = sizeof(__nv_bfloat16) *
                      (2 * (AM ? BK * (BM + PAD) : BM * (BK + PAD)) +
                       2 * (BN_ ? BK * (BN + PAD) : BN * (BK + PAD)));
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(gemm_kernel<AM, BN_, EPI>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  const dim3 grid(g.N / BN, g.M / BM, splits);
  gemm_kernel<AM, BN_, EPI><<<grid, THREADS, smem, stream>>>(g);
  return cudaGetLastError();
}

// -------------------------------------------------------- element-wise kernels
__global__ void adam_kernel(float *w, __nv_bfloat16 *w16, const float *grad,
                            float *m, float *v, int64_t n, float lr, float b1,
                            float b2, float eps, const float *corr, float scale) {
  const float c1 = corr[0], c2 = corr[1];  // 1 - beta^step, read on the device
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float gr = grad[i] * scale;
    const float mi = b1 * m[i] + (1.f - b1) * gr;
    const float vi = b2 * v[i] + (1.f - b2) * gr * gr;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (w16) w16[i] = __float2bfloat16_rn(wi);
  }
}

// Output layer: y = h . w + b (fp32), and the MSE gradient dy = 2 (y - t)/B.
__global__ void head_forward_kernel(const __nv_bfloat16 *h, const float *w,
                                    const float *b, const float *target, float *y,
                                    float *dy, float *loss, int rows, int width,
                                    float inv_rows) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= rows) return;
  float s = 0.f;
  for (int k = lane; k < width; k += 32)
    s = fmaf(__bfloat162float(h[(int64_t)warp * width + k]), w[k], s);
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) {
    const float out = s + b[0];
    y[warp] = out;
    if (target) {
      const float r = out - target[warp];
      dy[warp] = 2.f * r * inv_rows;
      atomicAdd(loss, r * r * inv_rows);
    }
  }
}

// Output layer backward: dw += sum_r dy_r h_r; db += sum_r dy_r;
// dz_prev = dy_r * w * silu'(z_prev) (bf16).
__global__ void head_backward_kernel(const __nv_bfloat16 *h, const float *zprev,
                                     const float *w, const float *dy, float *dw,
                                     float *db, __nv_bfloat16 *dz, int rows,
                                     int width) {
  const int col = threadIdx.x;  // one thread per hidden unit, width <= 1024
  float accw = 0.f, accb = 0.f;
  for (int r = blockIdx.x; r < rows; r += gridDim.x) {
    const float d = dy[r];
    const int64_t o = (int64_t)r * width + col;
    if (col < width) {
      accw = fmaf(d, __bfloat162float(h[o]), accw);
      dz[o] = __float2bfloat16_rn(d * w[col] * silu_grad(zprev[o]));
    }
    accb += d;
  }
  if (col < width) atomicAdd(dw + col, accw);
  if (col == 0) atomicAdd(db, accb);
}

// dst[c][r] = src[r][c] (bf16, rows x cols), through a 32 x 33 shared tile.
__global__ void transpose_kernel(const __nv_bfloat16 *src, __nv_bfloat16 *dst, int rows,
                                 int cols) {
  __shared__ __nv_bfloat16 tile[32][33];
  const int c = blockIdx.x * 32 + threadIdx.x;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = blockIdx.y * 32 + k;
    if (r < rows && c < cols) tile[k][threadIdx.x] = src[(int64_t)r * cols + c];
  }
  __syncthreads();
  const int r = blockIdx.y * 32 + threadIdx.x;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int cc = blockIdx.x * 32 + k;
    if (r < rows && cc < cols) dst[(int64_t)cc * rows + r] = tile[threadIdx.x][k];
  }
}

// Column sums of a bf16 matrix (bias gradients): out[c] += sum_r x[r][c].
__global__ void colsum_kernel(const __nv_bfloat16 *x, float *out, int rows, int cols) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.f;
  const int chunk = (rows + gridDim.y - 1) / gridDim.y;
  const int r0 = blockIdx.y * chunk, r1 = min(rows, r0 + chunk);
  for (int r = r0; r < r1; r++) s += __bfloat162float(x[(int64_t)r * cols + c]);
  atomicAdd(out + c, s);
}

// Relative 5D state [x, y, psi, vP, vE] -> features
// [x/e, y/e, cos psi, sin psi, vP~, vE~, 0...] (speeds mapped to [-1, 1]),
// bf16 rows of `ld` elements.
struct RelFeatureScale {
  float inv_extent, vp_mid, vp_inv_half, ve_mid, ve_inv_half;
};

__device__ __forceinline__ void write_rel_features(__nv_bfloat16 *row, int ld,
                                                   const RelFeatureScale &f, float x,
                                                   float y, float psi, float vp,
                                                   float ve) {
  float s, c;
  sincosf(psi, &s, &c);
  const float vals[6] = {x * f.inv_extent, y * f.inv_extent, c, s,
                         (vp - f.vp_mid) * f.vp_inv_half, (ve - f.ve_mid) * f.ve_inv_half};
  for (int k = 0; k < ld; k++) row[k] = __float2bfloat16_rn(k < 6 ? vals[k] : 0.f);
}

// Grid-node samples of a dense [vP, vE, psi, y, x] table.
__global__ void encode_relative_nodes_kernel(const float *table, const int64_t *idx,
                                             int n, int nx, int nh, int nve,
                                             float extent, float dx, float dphi,
                                             float vp_lo, float dvp, float ve_lo,
                                             float dve, RelFeatureScale f,
                                             __nv_bfloat16 *feat, int ld, float *target) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t j = idx[i];
  const int ix = (int)(j % nx);
  j /= nx;
  const int iy = (int)(j % nx);
  j /= nx;
  const int ip = (int)(j % nh);
  j /= nh;
  const int ie = (int)(j % nve);
  const int iv = (int)(j / nve);
  write_rel_features(feat + (int64_t)i * ld, ld, f, fmaf((float)ix, dx, -extent),
                     fmaf((float)iy, dx, -extent), fmaf((float)ip, dphi, -3.14159265358979f),
                     fmaf((float)iv, dvp, vp_lo), fmaf((float)ie, dve, ve_lo));
  if (target) target[i] = table[idx[i]];
}

// Arbitrary relative states [n][5].
__global__ void encode_relative_states_kernel(const float *states, int n,
                                              RelFeatureScale f, __nv_bfloat16 *feat,
                                              int ld) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float *s = states + (int64_t)i * 5;
  write_rel_features(feat + (int64_t)i * ld, ld, f, s[0], s[1], s[2], s[3], s[4]);
}

// 8D world nodes [xP, yP, thP, vP, xE, yE, thE, vE] -> 10 features.
__global__ void encode_world_nodes_kernel(const float *table, const int64_t *idx, int n,
                                          int npos, int nh, int np, int ne, float extent,
                                          float dx, float dh, float vp_lo, float dvp,
                                          float ve_lo, float dve, RelFeatureScale f,
                                          __nv_bfloat16 *feat, int ld, float *target) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t j = idx[i];
  const int q7 = (int)(j % ne);
  j /= ne;
  const int q6 = (int)(j % nh);
  j /= nh;
  const int q5 = (int)(j % npos);
  j /= npos;
  const int q4 = (int)(j % npos);
  j /= npos;
  const int q3 = (int)(j % np);
  j /= np;
  const int q2 = (int)(j % nh);
  j /= nh;
  const int q1 = (int)(j % npos);
  const int q0 = (int)(j / npos);
  float sp, cp, se, ce;
  sincosf(fmaf((float)q2, dh, -3.14159265358979f), &sp, &cp);
  sincosf(fmaf((float)q6, dh, -3.14159265358979f), &se, &ce);
  const float vals[10] = {fmaf((float)q0, dx, -extent) * f.inv_extent,
                          fmaf((float)q1, dx, -extent) * f.inv_extent, cp, sp,
                          (fmaf((float)q3, dvp, vp_lo) - f.vp_mid) * f.vp_inv_half,
                          fmaf((float)q4, dx, -extent) * f.inv_extent,
                          fmaf((float)q5, dx, -extent) * f.inv_extent, ce, se,
                          (fmaf((float)q7, dve, ve_lo) - f.ve_mid) * f.ve_inv_half};
  __nv_bfloat16 *row = feat + (int64_t)i * ld;
  for (int k = 0; k < ld; k++) row[k] = __float2bfloat16_rn(k < 10 ? vals[k] : 0.f);
  if (target) target[i] = table[idx[i]];
}

}  // namespace
}  // namespace pe

using pe::GemmArgs;

extern "C" {

// C = A x B; layouts: a_mmajor (A stored [K][M]) else [M][K]; b_nmajor (B
// stored [K][N]) else [N][K].  epilogue 0: C32 = acc; 1: C32 = acc + bias
// (may be NULL), C16 = bf16(silu(acc + bias)); 2: C32 += acc (split-K over
// `splits` CTAs, C32 must be pre-zeroed); 3: C16 = bf16(acc * silu'(zpre)).
// M, N multiples of 128; K multiple of 32 * splits.
int pe_mlp_gemm(const void *A, const void *B, int M, int N, int K, int lda, int ldb,
                int a_mmajor, int b_nmajor, int epilogue, int splits, float *C32,
                void *C16, int ldc, const float *bias, const float *zpre,
                void *cuda_stream) {
  if (!A || !B || M <= 0 || N <= 0 || K <= 0 || M % pe::BM || N % pe::BN || splits < 1 ||
      K % (pe::BK * splits))
    return pe::fail(PE_EINVAL, "gemm: M, N multiples of 128, K multiple of 32*splits");
  if ((epilogue == 0 || epilogue == 2) && !C32)
    return pe::fail(PE_EINVAL, "gemm: C32 required");
  if ((epilogue == 1 || epilogue == 3) && !C16)
    return pe::fail(PE_EINVAL, "gemm: C16 required");
  if (epilogue == 1 && !bias) return pe::fail(PE_EINVAL, "gemm: bias required");
  if (epilogue == 3 && !zpre) return pe::fail(PE_EINVAL, "gemm: zpre required");
  if (epilogue != 2 && splits != 1)
    return pe::fail(PE_EINVAL, "gemm: split-K needs the accumulate epilogue");
  GemmArgs g{};
  g.A = static_cast<const __nv_bfloat16 *>(A);
  g.B = static_cast<const __nv_bfloat16 *>(B);
  g.M = M;
  g.N = N;
  g.K = K;
  g.lda = lda;
  g.ldb = ldb;
  g.k_split = K / splits;
  g.C32 = C32;
  g.C16 = static_cast<__nv_bfloat16 *>(C16);
  g.ldc = ldc;
  g.bias = bias;
  g.zpre = zpre;
  cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
  cudaError_t e = cudaErrorInvalidValue;
  const int sel = (a_mmajor ? 8 : 0) | (b_nmajor ? 4 : 0) | (epilogue & 3);
  switch (sel) {
#define PE_GEMM_CASE(AM, BNM, EP)                                     \
  case ((AM) ? 8 : 0) | ((BNM) ? 4 : 0) | (EP):                       \
    e = pe::launch_gemm<(AM) != 0, (BNM) != 0, EP>(g, splits, s);     \
    break;
    PE_GEMM_CASE(0, 0, 0) PE_GEMM_CASE(0, 0, 1) PE_GEMM_CASE(0, 0, 2) PE_GEMM_CASE(0, 0, 3)
    PE_GEMM_CASE(0, 1, 0) PE_GEMM_CASE(0, 1, 1) PE_GEMM_CASE(0, 1, 2) PE_GEMM_CASE(0, 1, 3)
    PE_GEMM_CASE(1, 0, 0) PE_GEMM_CASE(1, 0, 1) PE_GEMM_CASE(1, 0, 2) PE_GEMM_CASE(1, 0, 3)
    PE_GEMM_CASE(1, 1, 0) PE_GEMM_CASE(1, 1, 1) PE_GEMM_CASE(1, 1, 2) PE_GEMM_CASE(1, 1, 3)
#undef PE_GEMM_CASE
  }
  if (e != cudaSuccess) return pe::cuda_fail(e, "pe_mlp_gemm");
  pe::count_launches(1);
  return PE_OK;
}

// Adam update of n fp32 weights (and their bf16 copy when w16 != NULL).
// corr: device pointer to {1 - beta1^step, 1 - beta2^step}, read by the
// kernel so that a captured CUDA graph can be replayed across steps.
int pe_mlp_adam(float *w, void *w16, const float *grad, float *m, float *v, int64_t n,
                float lr, float beta1, float beta2, float eps, const float *corr,
                float grad_scale, void *cuda_stream) {
  if (!w || !grad || !m || !v || !corr || n <= 0)
    return pe::fail(PE_EINVAL, "adam: invalid arguments");
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  pe::adam_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(cuda_stream)>>>(
      w, static_cast<__nv_bfloat16 *>(w16), grad, m, v, n, lr, beta1, beta2, eps, corr,
      grad_scale);
  PE_CUDA_TRY(cudaGetLastError());
  pe::count_launches(1);
  return PE_OK;
}

int pe_mlp_head_forward(const void *h, const float *w, const float *b,
                        const float *target, float *y, float *dy, float *loss,
                        int rows, int width, void *cuda_stream) {
  if (!h || !w || !b || !y || rows <= 0 || width <= 0 || (target && (!dy || !loss)))
    return pe::fail(PE_EINVAL, "head_forward: invalid arguments");
  const int blocks = (rows * 32 + 255) / 256;
  pe::head_forward_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(cuda_stream)>>>(
      static_cast<const __nv_bfloat16 *>(h), w, b, target, y, dy, loss, rows, width,
      1.f / rows);
  PE_CUDA_TRY(cudaGetLastError());
  pe::count_launches(1);
  return PE_OK;
}

int pe_mlp_head_backward(const void *h, const float *zprev, const float *w,
                         const float *dy, float *dw, float *db, void *dz, int rows,
                         int width, void *cuda_stream) {
  if (!h || !zprev || !w || !dy || !dw || !db || !dz || rows <= 0 || width <= 0 ||
      width > 1024)
    return pe::fail(PE_EINVAL, "head_backward: invalid arguments");
  pe::head_backward_kernel<<<148 * 4, width, 0, static_cast<cudaStream_t>(cuda_stream)>>>(
      static_cast<const __nv_bfloat16 *>(h), zprev, w, dy, dw, db,
      static_cast<__nv_bfloat16 *>(dz), rows, width);
  PE_CUDA_TRY(cudaGetLastError());
  pe::count_launches(1);
  return PE_OK;
}

static pe::RelFeatureScale feature_scale(float extent, float vp_lo, float vp_hi,
                                         float ve_lo, float ve_hi) {
  pe::RelFeatureScale f;
  f.inv_extent = 1.f / extent;
  f.vp_mid = 0.5f * (vp_lo + vp_hi);
  f.vp_inv_half = 2.f / (vp_hi - vp_lo);
  f.ve_mid = 0.5f * (ve_lo + ve_hi);
  f.ve_inv_half = 2.f / (ve_hi - ve_lo);
  return f;
}

// Features (and table targets when table != NULL) of relative 5D grid nodes
// given by flat indices into a dense [vP, vE, psi, y, x] table.
int pe_mlp_encode_relative_nodes(const float *table, const int64_t *idx, int n,
                                 int positions, int headings, int p_speeds,
                                 int e_speeds, double extent, double p_min,
                                 double p_max, double e_min, double e_max, void *feat,
                                 int ld, float *target, void *cuda_stream) {
  if (!idx || !feat || n <= 0 || ld < 6 || (target && !table))
    return pe::fail(PE_EINVAL, "encode_relative_nodes: invalid arguments");
  const double pi = 3.14159265358979323846;
  pe::encode_relative_nodes_kernel<<<(n + 255) / 256, 256, 0,
                                     static_cast<cudaStream_t>(cuda_stream)>>>(
      table, idx, n, positions, headings, e_speeds, (float)extent,
      (float)(2 * extent / (positions - 1)), (float)(2 * pi / headings), (float)p_min,
      (float)((p_max - p_min) / (p_speeds - 1)), (float)e_min,
      (float)((e_max - e_min) / (e_speeds - 1)),
      feature_scale((float)extent, (float)p_min, (float)p_max, (float)e_min, (float)e_max),
      static_cast<__nv_bfloat16 *>(feat), ld, target);
  PE_CUDA_TRY(cudaGetLastError());
  pe::count_launches(1);
  return PE_OK;
}

// Features of arbitrary relative states [n][5] (x, y, psi, vP, vE).
int pe_mlp_encode_relative_states(const float *states, int n, double extent,
                                  double p_min, double p_max, double e_min,
                                  double e_max, void *feat, int ld, void *cuda_stream) {
  if (!states || !feat || n <= 0 || ld < 6)
    return pe::fail(PE_EINVAL, "encode_relative_states: invalid arguments");
  pe::encode_relative_states_kernel<<<(n + 255) / 256, 256, 0,
                                      static_cast<cudaStream_t>(cuda_stream)>>>(
      states, n,
      feature_scale((float)extent, (float)p_min, (float)p_max, (float)e_min, (float)e_max),
      static_cast<__nv_bfloat16 *>(feat), ld);
  PE_CUDA_TRY(cudaGetLastError());
  pe::count_launches(1);
  return PE_OK;
}

// Features (and targets) of 8D world grid nodes, dense table order
// [xP, yP, thP, vP, xE, yE, thE, vE].
int pe_mlp_encode_world_nodes(const float *table, const int64_t *idx, int n,
                              int positions, int headings, int p_speeds, int e_speeds,
                              double extent, double p_min, double p_max, double e_min,
                              double e_max, void *feat, int ld, float *target,
                              void *cuda_stream) {
  if (!idx || !feat || n <= 0 || ld < 10 || (target && !table))
    return pe::fail(PE_EINVAL, "encode_world_nodes: invalid arguments");
  const double pi = 3.14159265358979323846;
  pe::encode_world_nodes_kernel<<<(n + 255) / 256, 256, 0,
                                  static_cast<cudaStream_t>(cuda_stream)>>>(
      table, idx, n, positions, headings, p_speeds, e_speeds, (float)extent,
      (float)(2 * extent / (positions - 1)), (float)(2 * pi / headings), (float)p_min,
      (float)((p_max - p_min) / (p_speeds - 1)), (float)e_min,
      (float)((e_max - e_min) / (e_speeds - 1)),
      feature_scale((float)extent, (float)p_min, (float)p_max, (float)e_min, (float)e_max),
      static_cast<__nv_bfloat16 *>(feat), ld, target);
  PE_CUDA_TRY(cudaGetLastError());
  pe::count_launches(1);
  return PE_OK;
}

int pe_mlp_transpose(const void *src, void *dst, int rows, int cols, void *cuda_stream) {
  if (!src || !dst || rows <= 0 || cols <= 0)
    return pe::fail(PE_EINVAL, "transpose: invalid arguments");
  const dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
  pe::transpose_kernel<<<grid, block, 0, static_cast<cudaStream_t>(cuda_stream)>>>(
      static_cast<const __nv_bfloat16 *>(src), static_cast<__nv_bfloat16 *>(dst), rows, cols);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return pe::cuda_fail(e, "pe_mlp_transpose");
  pe::count_launches(1);
  return PE_OK;
}

int pe_mlp_colsum(const void *x, float *out, int rows, int cols, void *cuda_stream) {
  if (!x || !out || rows <= 0 || cols <= 0)
    return pe::fail(PE_EINVAL, "colsum: invalid arguments");
  const dim3 grid((cols + 255) / 256, 64);
  pe::colsum_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(cuda_stream)>>>(
      static_cast<const __nv_bfloat16 *>(x), out, rows, cols);
  PE_CUDA_TRY(cudaGetLastError());
  pe::count_launches(1);
  return PE_OK;
}

}  // extern "C"
