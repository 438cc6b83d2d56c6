// BF16 tensor-core kernels of the loss-prediction surrogate (sm_100a tcgen05).
//
// One GEMM kernel serves every layer of the forward and backward pass:
//     C[M x N] = A[M x K] * B[N x K]^T        (A, B bf16, K contiguous)
// accumulated in FP32 in tensor memory.  Each CTA owns a 128-row block of C and
// the full N (<= 256 columns of TMEM).  K is consumed in chunks: the threads
// copy a chunk of A and B from global memory into shared memory in the
// no-swizzle K-major core-matrix layout (8 rows x 16 bytes per core matrix,
// LBO = 128 B between the two K-halves of an MMA step, SBO = 1 KiB between
// 8-row groups), one elected thread issues tcgen05.mma (kind::f16, M = 128,
// N, K = 16) for every 16-wide K step, and tcgen05.commit signals an mbarrier
// when the chunk's MMAs have completed.  The epilogue reads the accumulator
// back with tcgen05.ld (32x32b: one row per thread) and applies the layer's
// fused operation (bias + GELU with a transposed bf16 copy for the backward
// pass, GELU derivative, or a plain FP32 store).
//
// Descriptor bit layouts (shared-memory matrix descriptor and instruction
// descriptor for kind::f16) follow the sm_100 UMMA descriptor definitions in
// CUTLASS's cute/arch/mma_sm100_desc.hpp.  Every wait is bounded: a timeout
// sets the status word and the CTA still releases its tensor memory.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "stb_mlp.hpp"

namespace stb {

namespace {

constexpr int kM = 128;          // rows per CTA (one MMA M)
constexpr int kKC = 64;          // K elements per shared-memory chunk
constexpr int kThreads = 128;    // one thread per accumulator row
constexpr uint32_t kCoreBytes = 128;            // 8 rows x 16 bytes
constexpr uint32_t kSBO = (kKC / 8) * kCoreBytes;  // 1024: next 8-row group
constexpr uint32_t kLBO = kCoreBytes;              // 128: next 8 elements of K

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: start address, LBO and SBO in 16-byte
// units, version 1 (sm_100), no swizzle.
__device__ __forceinline__ uint64_t make_smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, lbo mode 0, layout type 0 (no swizzle)
}

// Instruction descriptor: D = F32, A = B = BF16, both K-major, M and N.
__device__ __forceinline__ uint32_t make_idesc(int M, int N) {
  uint32_t d = 0;
  d |= 1u << 4;                       // C format F32
  d |= 1u << 7;                       // A format BF16
  d |= 1u << 10;                      // B format BF16
  d |= ((uint32_t)(N >> 3) & 0x3Fu) << 17;
  d |= ((uint32_t)(M >> 4) & 0x1Fu) << 24;
  return d;
}

__device__ __forceinline__ float gelu_f(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float dgelu_f(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// Copies rows [row0, row0 + nrows) x K-chunk [k0, k0 + kn) of a K-contiguous
// bf16 matrix into the core-matrix layout at `dst` (kn a multiple of 16,
// missing rows filled with zeros).
__device__ __forceinline__ void load_chunk(const __nv_bfloat16 *src, int ld, int row0, int nrows, int rows_valid,
                                           int k0, int kn, unsigned char *dst) {
  const int vec_per_row = kn / 8;  // 16-byte vectors
  const int total = nrows * vec_per_row;
  for (int v = threadIdx.x; v < total; v += kThreads) {
    const int r = v / vec_per_row, c8 = v % vec_per_row;
    uint4 val = make_uint4(0, 0, 0, 0);
    if (r < rows_valid) val = *reinterpret_cast<const uint4 *>(src + (size_t)(row0 + r) * ld + k0 + c8 * 8);
    const uint32_t off = (uint32_t)((r >> 3) * (kKC / 8) + c8) * kCoreBytes + (uint32_t)(r & 7) * 16u;
    *reinterpret_cast<uint4 *>(dst + off) = val;
  }
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  uint32_t done = 0;
  for (int i = 0; i < (1 << 24) && !done; i++) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
  }
  return done != 0;
}

__global__ void __launch_bounds__(kThreads, 1) mlp_gemm_kernel(const __grid_constant__ GemmArgs g) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base_s;
  unsigned char *sA = smem;
  unsigned char *sB = smem + kM * kKC * 2;
  const int m0 = blockIdx.x * kM;
  const int warp = threadIdx.x >> 5;
  const uint32_t ncols = g.N <= 32 ? 32u : (g.N <= 64 ? 64u : (g.N <= 128 ? 128u : 256u));

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_base_s)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_base_s;
  const uint32_t idesc = make_idesc(kM, g.N);
  uint32_t phase = 0;
  bool ok = true;

  for (int k0 = 0; k0 < g.K && ok; k0 += kKC) {
    const int kn = (g.K - k0) < kKC ? (g.K - k0) : kKC;
    load_chunk(g.A, g.lda, m0, kM, g.M - m0, k0, kn, sA);
    load_chunk(g.B, g.ldb, 0, g.N, g.N, k0, kn, sB);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      for (int ks = 0; ks < kn / 16; ks++) {
        const uint64_t ad = make_smem_desc(smem_u32(sA) + (uint32_t)ks * 2u * kCoreBytes, kLBO, kSBO);
        const uint64_t bd = make_smem_desc(smem_u32(sB) + (uint32_t)ks * 2u * kCoreBytes, kLBO, kSBO);
        const uint32_t acc = (k0 > 0 || ks > 0) ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                       smem_u32(&mbar))
                   : "memory");
    }
    ok = mbar_wait(smem_u32(&mbar), phase);
    ok = __syncthreads_and(ok ? 1 : 0) != 0;
    phase ^= 1u;
  }
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");

  if (ok) {
    const int row = m0 + threadIdx.x;
    const bool row_ok = row < g.M;
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < g.N; c0 += 16) {
      uint32_t r[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr + (uint32_t)c0)
          : "memory");
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      if (!row_ok) continue;
      const int nv = g.n_valid > 0 ? g.n_valid : g.N;
      for (int j = 0; j < 16; j++) {
        const int col = c0 + j;
        const float acc = __uint_as_float(r[j]);
        switch (g.mode) {
          case EPI_F32:
            if (col >= nv) break;
            if (g.transpose_out) g.C[(size_t)col * g.ldc + row] = acc;
            else g.C[(size_t)row * g.ldc + col] = acc;
            break;
          case EPI_BIAS_F32:
            g.C[(size_t)row * g.ldc + col] = acc + ((g.bias && col < nv) ? g.bias[col] : 0.0f);
            break;
          case EPI_BIAS_GELU: {
            const float z = acc + g.bias[col];
            g.C[(size_t)row * g.ldc + col] = z;  // pre-activation, kept for the backward pass
            const __nv_bfloat16 h = __float2bfloat16_rn(gelu_f(z));
            g.H[(size_t)row * g.ldh + col] = h;
            g.HT[(size_t)col * g.ldht + row] = h;
            break;
          }
          case EPI_DGELU: {
            const float dz = acc * dgelu_f(g.Z[(size_t)row * g.ldz + col]);
            const __nv_bfloat16 h = __float2bfloat16_rn(dz);
            g.H[(size_t)row * g.ldh + col] = h;
            g.HT[(size_t)col * g.ldht + row] = h;
            if (g.C) g.C[(size_t)row * g.ldc + col] = dz;
            break;
          }
          default:
            break;
        }
      }
    }
  } else if (threadIdx.x == 0) {
    atomicExch(g.status, STB_ETIMEOUT);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(ncols) : "memory");
  }
}

}  // namespace

size_t mlp_gemm_smem_bytes() {
  // The A and B chunks need 48 KiB; asking for 120 KiB keeps at most one CTA
  // (one tensor-memory allocation of <= 256 columns) resident per SM, so an
  // allocation never waits for another CTA's release.
  return 120 * 1024;
}

cudaError_t mlp_gemm_launch(const GemmArgs &g, cudaStream_t st) {
  if (g.M <= 0 || g.N < 16 || g.N > 256 || (g.N % 16) || g.K <= 0 || (g.K % 16) || (g.lda % 8) || (g.ldb % 8))
    return cudaErrorInvalidValue;
  const size_t sm = mlp_gemm_smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(mlp_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  mlp_gemm_kernel<<<(g.M + kM - 1) / kM, kThreads, sm, st>>>(g);
  return cudaGetLastError();
}

}  // namespace stb
