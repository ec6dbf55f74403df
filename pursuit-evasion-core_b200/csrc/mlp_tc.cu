// BF16 GEMM of the value surrogate on the 5th-generation tensor cores:
// TMA (cp.async.bulk.tensor) loads 128B-swizzled tiles into a shared-memory
// ring, one elected thread issues tcgen05.mma with the FP32 accumulator in
// tensor memory (TMEM), and four warps read the accumulator back with
// tcgen05.ld for the epilogue.
//
// C[M][N] = A[M][K] * B[N][K]^T with both operands K-major (row-major A,
// and B stored as [N][K], the layout of a Linear layer's weight), the case
// of the forward layers and, with a transposed weight copy, of the
// activation gradients.  Epilogues as pe_mlp_gemm: 0 FP32 store, 1 bias +
// SiLU (FP32 pre-activation optional, BF16 activation), 2 FP32 accumulate
// (split-K: grid z splits the K range, each CTA adds its partial tile with
// 16-byte vector atomics; the weight gradients, from transposed activation
// copies), 3 product with SiLU'(pre-activation) to BF16.
//
// CTA tile 128 x TN x 64 (TN = 256 where N allows, else 128), 2 pipeline
// stages (the surrogate's K is 128 or 256; 97 KB of shared memory and 256
// tensor-memory columns let two CTAs share an SM, so one's epilogue
// overlaps the other's loads and MMAs), 128 threads: warp 0 lane 0 issues
// the TMA loads, warp 1 lane 0 the MMAs (4 of K=16 per stage); all four
// warps run the epilogue, warp w on accumulator lanes 32w..32w+31 (= tile
// rows).  Every mbarrier wait is bounded; a timed-out wait sets the
// error flag and the CTA still releases its tensor memory.
#include <cuda.h>
#include <cuda_bf16.h>

#include "pe_internal.h"

namespace pe {
namespace {

constexpr int TM = 128, TK = 64, STAGES = 2, THREADS = 128;
constexpr int A_BYTES = TM * TK * 2;  // 16 KB
constexpr uint32_t WAIT_LIMIT = 1u << 24;

__device__ __forceinline__ float silu(float z) { return z / (1.f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = 1.f / (1.f + __expf(-z));
  return s * (1.f + z * (1.f - s));
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile(
      "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait on a phase; false (and the error flag set) on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, unsigned *error) {
  for (uint32_t i = 0; i < WAIT_LIMIT; i++)
    if (mbar_try_wait(bar, parity)) return true;
  atomicOr(error, 1u);
  return false;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// Shared-memory matrix descriptor of a K-major, 128B-swizzled operand tile
// (rows of 128 bytes, 8-row groups 1024 bytes apart): start address and
// offsets in 16-byte units, descriptor version 1, swizzle mode 128B.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr & 0x3FFFF) >> 4);  // start address
  d |= (uint64_t)1 << 16;                  // leading byte offset (unused when swizzled)
  d |= (uint64_t)(1024 >> 4) << 32;        // stride byte offset: next 8-row group
  d |= (uint64_t)1 << 46;                  // descriptor version
  d |= (uint64_t)2 << 61;                  // 128-byte swizzle
  return d;
}

// Instruction descriptor: BF16 x BF16 -> FP32, both K-major, M = 128, N = TN.
template <int TN>
__host__ __device__ constexpr uint32_t idesc() {
  return (1u << 4)      // D format FP32
         | (1u << 7)    // A format BF16
         | (1u << 10)   // B format BF16
         | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
}

template <int TN>
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n"
      " setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc<TN>()), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

struct TcArgs {
  int M, N, K, ldc;
  int ksteps;  // k-steps of TK per CTA (K / TK without split-K)
  float *C32;
  __nv_bfloat16 *C16;
  const float *bias, *zpre;
  unsigned *error;
};

template <int EPI, int TN>
__global__ void __launch_bounds__(THREADS, 1)
    gemm_tc_kernel(const __grid_constant__ CUtensorMap tma_a,
                   const __grid_constant__ CUtensorMap tma_b, const TcArgs g) {
  constexpr int B_BYTES = TN * TK * 2;
  constexpr uint32_t TMEM_COLS = TN;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // 1024-byte alignment of every tile (the swizzle atom)
  uint8_t *base = reinterpret_cast<uint8_t *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t *sA = base, *sB = base + STAGES * A_BYTES;
  uint64_t *full = reinterpret_cast<uint64_t *>(sB + STAGES * B_BYTES);
  uint64_t *empty = full + STAGES;
  uint64_t *done = empty + STAGES;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
  const int kt = g.ksteps, kbase = blockIdx.z * g.ksteps;  // this CTA's K range

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {  // tensor memory for the 128 x 128 FP32 accumulator
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  bool ok = true;
  if (warp == 0 && lane == 0) {
    // producer: stage s of k-step k is free once the MMAs of k - STAGES finished
    int issued = 0;
    for (int k = 0; k < kt && ok; k++) {
      const int s = k % STAGES;
      if (k >= STAGES) ok = mbar_wait(&empty[s], ((k / STAGES) - 1) & 1, g.error);
      if (!ok) break;
      mbar_expect_tx(&full[s], A_BYTES + B_BYTES);
      tma_load_2d(sA + s * A_BYTES, &tma_a, (kbase + k) * TK, m0, &full[s]);
      tma_load_2d(sB + s * B_BYTES, &tma_b, (kbase + k) * TK, n0, &full[s]);
      issued = k + 1;
    }
    // no copy may still be landing when the CTA leaves: wait (bounded) for
    // the last use of every stage (already complete on the normal path)
    for (int k = issued > STAGES ? issued - STAGES : 0; k < issued; k++)
      mbar_wait(&full[k % STAGES], (k / STAGES) & 1, g.error);
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    for (int k = 0; k < kt && ok; k++) {
      const int s = k % STAGES;
      ok = mbar_wait(&full[s], (k / STAGES) & 1, g.error);
      if (!ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = smem_u32(sA + s * A_BYTES), b0 = smem_u32(sB + s * B_BYTES);
#pragma unroll
      for (int kk = 0; kk < TK / 16; kk++)  // K = 16 per instruction: 32 bytes along a row
        mma_bf16<TN>(tmem, smem_desc_sw128(a0 + kk * 32), smem_desc_sw128(b0 + kk * 32),
                     (k | kk) != 0);
      mma_commit(&empty[s]);  // frees the stage when these MMAs complete
    }
    mma_commit(done);  // the accumulator is complete (or the loop stopped early)
  }
  __syncwarp();

  // epilogue: warp w reads accumulator lanes (tile rows) 32w..32w+31, 32
  // columns at a time (thread l holds row 32w + l), turns the 32 x 32 block
  // around in shared memory (the operand ring is idle once `done` fired)
  // and stores it row by row, lane l on column l: coalesced loads of the
  // pre-activation and coalesced stores
  const bool have = mbar_wait(done, 0, g.error);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  float *stage = reinterpret_cast<float *>(sA) + warp * 32 * 33;
#pragma unroll 1
  for (int c0 = 0; c0 < TN; c0 += 32) {
    uint32_t r[32];
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
        "%10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, "
        "%27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; j++) stage[lane * 33 + j] = __uint_as_float(r[j]);
    __syncwarp();
    if (have && EPI == 2) {
      // lane l adds columns 4(l%8) .. 4(l%8)+3 of row l/8 of each group of
      // four rows: one 16-byte atomic per lane, 128 contiguous bytes per row
      const int rs = lane >> 3, cq = (lane & 7) * 4;
#pragma unroll 4
      for (int rr = 0; rr < 32; rr += 4) {
        const int rl = rr + rs;
        const float *src = stage + rl * 33 + cq;
        float *dst = g.C32 + (size_t)(m0 + warp * 32 + rl) * g.ldc + n0 + c0 + cq;
        atomicAdd(reinterpret_cast<float4 *>(dst), make_float4(src[0], src[1], src[2], src[3]));
      }
    } else if (have) {
      const int n = n0 + c0 + lane;
      const float bn = EPI == 1 ? g.bias[n] : 0.f;
#pragma unroll 4
      for (int rr = 0; rr < 32; rr++) {
        const int row = m0 + warp * 32 + rr;
        const size_t o = (size_t)row * g.ldc + n;
        const float acc = stage[rr * 33 + lane];
        if (EPI == 0) {
          g.C32[o] = acc;
        } else if (EPI == 1) {
          const float z = acc + bn;
          if (g.C32) g.C32[o] = z;
          g.C16[o] = __float2bfloat16_rn(silu(z));
        } else {
          g.C16[o] = __float2bfloat16_rn(acc * silu_grad(g.zpre[o]));
        }
      }
    }
    __syncwarp();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TMEM_COLS)
                 : "memory");
}

template <int TN>
__host__ __device__ constexpr size_t smem_bytes() {
  return 1024 + STAGES * (A_BYTES + TN * TK * 2) + (2 * STAGES + 1) * 8 + 16;
}

// 2D tensor map of a K-major bf16 matrix [rows][K] with row pitch ld
// elements, box 64 (K) x box_rows, 128-byte swizzle.
// The driver's tensor-map encoder, fetched through the runtime so that the
// library does not link libcuda (it loads on machines without a driver).
using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                 const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                 const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
  static EncodeTiled fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  }
  return fn;
}

CUresult make_map(CUtensorMap *map, const void *ptr, int rows, int K, int ld, int box_rows) {
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {TK, (cuuint32_t)box_rows};
  const cuuint32_t elem[2] = {1, 1};
  EncodeTiled encode = encoder();
  if (!encode) return CUDA_ERROR_NOT_FOUND;
  return encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                                const_cast<void *>(ptr), dims, strides, box, elem,
                                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}

unsigned *error_word() {
  static unsigned *word = nullptr;  // one per process (first device used)
  if (!word && cudaMalloc(&word, sizeof(unsigned)) == cudaSuccess)
    cudaMemset(word, 0, sizeof(unsigned));
  return word;
}

template <int EPI, int TN>
cudaError_t launch(const CUtensorMap &a, const CUtensorMap &b, const TcArgs &g,
                   cudaStream_t stream) {
  auto kernel = gemm_tc_kernel<EPI, TN>;
  constexpr size_t smem = smem_bytes<TN>();
  cudaError_t e =
      cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kernel<<<dim3(g.N / TN, g.M / TM, g.K / (g.ksteps * TK)), THREADS, smem, stream>>>(a, b, g);
  return cudaGetLastError();
}

template <int TN>
cudaError_t launch_epi(int epilogue, const CUtensorMap &a, const CUtensorMap &b,
                       const TcArgs &g, cudaStream_t s) {
  return epilogue == 0   ? launch<0, TN>(a, b, g, s)
         : epilogue == 1 ? launch<1, TN>(a, b, g, s)
                         : launch<3, TN>(a, b, g, s);
}

}  // namespace
}  // namespace pe

extern "C" {

int pe_mlp_gemm_tc(const void *A, const void *B, int M, int N, int K, int lda, int ldb,
                   int epilogue, float *C32, void *C16, int ldc, const float *bias,
                   const float *zpre, void *cuda_stream) {
  using namespace pe;
  if (!A || !B || M <= 0 || N <= 0 || K <= 0 || M % TM || N % 128 || K % TK)
    return fail(PE_EINVAL, "gemm_tc: M, N multiples of 128, K a multiple of 64");
  if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) % 16 || lda % 8 ||
      ldb % 8 || lda < K || ldb < K)
    return fail(PE_EINVAL, "gemm_tc: 16-byte aligned operands, lda and ldb >= K, multiples of 8");
  if (epilogue != 0 && epilogue != 1 && epilogue != 3)
    return fail(PE_EINVAL, "gemm_tc: epilogue 0, 1 or 3");
  if (epilogue == 0 && !C32) return fail(PE_EINVAL, "gemm_tc: C32 required");
  if (epilogue != 0 && !C16) return fail(PE_EINVAL, "gemm_tc: C16 required");
  if (epilogue == 1 && !bias) return fail(PE_EINVAL, "gemm_tc: bias required");
  if (epilogue == 3 && !zpre) return fail(PE_EINVAL, "gemm_tc: zpre required");
  if (ldc % 4) return fail(PE_EINVAL, "gemm_tc: ldc must be a multiple of 4");
  // a CTA covers 128 x 256 of C where N allows and that still gives two
  // CTAs per SM of the device (148 SMs: 296), else 128 x 128
  const int tn = N % 256 == 0 && (int64_t)(M / TM) * (N / 256) >= 296 ? 256 : 128;
  CUtensorMap ma, mb;
  if (make_map(&ma, A, M, K, lda, TM) != CUDA_SUCCESS ||
      make_map(&mb, B, N, K, ldb, tn) != CUDA_SUCCESS)
    return fail(PE_EINVAL, "gemm_tc: tensor map encoding failed");
  TcArgs g{M, N, K, ldc, K / TK, C32, static_cast<__nv_bfloat16 *>(C16), bias, zpre,
           error_word()};
  if (!g.error) return fail(PE_ENOMEM, "gemm_tc: error word");
  cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
  cudaError_t e = tn == 256 ? launch_epi<256>(epilogue, ma, mb, g, s)
                            : launch_epi<128>(epilogue, ma, mb, g, s);
  if (e != cudaSuccess) return cuda_fail(e, "pe_mlp_gemm_tc");
  count_launches(1);
  return PE_OK;
}

int pe_mlp_gemm_tc_splitk(const void *A, const void *B, int M, int N, int K, int lda, int ldb,
                          int splits, float *C32, int ldc, void *cuda_stream) {
  using namespace pe;
  if (!A || !B || !C32 || M <= 0 || N <= 0 || K <= 0 || splits < 1 || M % TM || N % 128 ||
      K % (TK * splits))
    return fail(PE_EINVAL,
                "gemm_tc_splitk: M, N multiples of 128, K a multiple of 64 * splits");
  if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B) |
       reinterpret_cast<uintptr_t>(C32)) % 16 ||
      lda % 8 || ldb % 8 || lda < K || ldb < K || ldc % 4 || ldc < N)
    return fail(PE_EINVAL,
                "gemm_tc_splitk: 16-byte aligned operands and C, lda, ldb >= K multiples "
                "of 8, ldc >= N a multiple of 4");
  CUtensorMap ma, mb;
  if (make_map(&ma, A, M, K, lda, TM) != CUDA_SUCCESS ||
      make_map(&mb, B, N, K, ldb, 128) != CUDA_SUCCESS)
    return fail(PE_EINVAL, "gemm_tc_splitk: tensor map encoding failed");
  TcArgs g{M, N, K, ldc, K / (TK * splits), C32, nullptr, nullptr, nullptr, error_word()};
  if (!g.error) return fail(PE_ENOMEM, "gemm_tc_splitk: error word");
  cudaError_t e = launch<2, 128>(ma, mb, g, static_cast<cudaStream_t>(cuda_stream));
  if (e != cudaSuccess) return cuda_fail(e, "pe_mlp_gemm_tc_splitk");
  count_launches(1);
  return PE_OK;
}

// Timeouts of bounded waits seen by pe_mlp_gemm_tc launches so far (and
// clear the flag).  Synchronises the device.
int pe_mlp_gemm_tc_timeouts(int32_t *count) {
  using namespace pe;
  if (!count) return fail(PE_EINVAL, "count is NULL");
  unsigned *w = error_word(), h = 0;
  if (!w) return fail(PE_ENOMEM, "gemm_tc: error word");
  PE_CUDA_TRY(cudaMemcpy(&h, w, sizeof h, cudaMemcpyDeviceToHost));
  PE_CUDA_TRY(cudaMemset(w, 0, sizeof h));
  *count = (int32_t)h;
  return PE_OK;
}

}  // extern "C"
