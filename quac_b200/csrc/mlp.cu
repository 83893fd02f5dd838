// Dense layers of the steady-state warm-start network on the 5th-generation
// tensor cores (tcgen05, TF32 inputs, FP32 accumulation in tensor memory).
//
//   C[M x N] = act(A[M x K] . B[N x K]^T + bias[N])     (both operands K-major)
//
// One CTA of 128 threads computes a 128 x 128 output tile; two CTAs share an
// SM.  Warp 0 (one thread) streams 128 x 32 tiles of A and B into shared
// memory by TMA, 128-byte swizzled (each tile row of 32 floats is one
// 128-byte swizzle row; zero fill past the matrix edge), NST stages deep;
// warp 1 (one thread) waits for each stage, issues four tcgen05.mma
// (K = 8 each, the descriptor's start address advanced 32 bytes inside the
// swizzle atom) and commits them to the stage's empty barrier, which hands
// the stage back to the producer.  After the last stage the MMAs are
// committed to a done barrier; the four warps then read the accumulator
// (128 lanes x 128 columns of FP32) back with tcgen05.ld and apply bias and
// activation on the way out.
//
// Every mbarrier wait is bounded in time; a wait that runs out sets the
// error word, the thread stops issuing work, the CTA waits (again bounded)
// for the copies and MMAs it started, frees its tensor memory and returns.
#include <cstdint>
#include <cstring>

#include <cuda.h>

#include "runtime.h"

namespace quac {
namespace {

constexpr int BM = 128, BN = 128, BK = 32;
constexpr int A_BYTES = BM * BK * 4, B_BYTES = BN * BK * 4;  // 16 KB each per stage
constexpr int ST_BYTES = A_BYTES + B_BYTES;
constexpr int NST = 3;  // 96 KB of stages (+1 KB for alignment): two CTAs per SM
constexpr unsigned long long WAIT_NS = 2000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait; false (and *err set) if the phase did not complete in time.
__device__ bool mbar_wait(uint32_t bar, uint32_t parity, int *err) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = gtimer();
  while (!mbar_try(bar, parity)) {
    if (gtimer() - t0 > WAIT_NS) {
      atomicExch(err, 1);
      return false;
    }
  }
  return true;
}

// Shared-memory matrix descriptor of a K-major operand tile in the 128-byte
// swizzled layout: 8-row x 128-byte swizzle atoms, consecutive 8-row groups
// 1024 bytes apart (stride byte offset), leading byte offset unused (16),
// descriptor version 1 (sm_100), base offset 0 (atoms 1024-byte aligned),
// layout type 2 = 128-byte swizzle.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

// Instruction descriptor: kind::tf32, FP32 accumulator, A and B K-major.
__host__ __device__ constexpr uint32_t instr_desc_tf32(int m, int n) {
  return (1u << 4)                   // accumulator format F32
         | (2u << 7)                 // A format TF32
         | (2u << 10)                // B format TF32
         | ((uint32_t)(n >> 3) << 17)
         | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// 2-D TMA tile load (x = k, y = row) into shared memory, completing on bar
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, uint32_t bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__global__ void __launch_bounds__(128) k_gemm_tf32(const __grid_constant__ CUtensorMap ta,
                                                   const __grid_constant__ CUtensorMap tb, float *__restrict__ C,
                                                   const float *__restrict__ bias, int M, int N, int K, int act,
                                                   int *err) {
  extern __shared__ unsigned char sm_raw[];
  __shared__ __align__(8) uint64_t full[NST], empty[NST], done;
  __shared__ uint32_t tmem_slot;
  __shared__ int n_issued, n_consumed;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  // stages on 1024-byte boundaries (the swizzle atoms' alignment)
  const uint32_t base = (smem_u32(sm_raw) + 1023u) & ~1023u;
  auto As = [&](int st) { return base + (uint32_t)(st * ST_BYTES); };
  auto Bs = [&](int st) { return base + (uint32_t)(st * ST_BYTES + A_BYTES); };

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 32) {
    for (int st = 0; st < NST; st++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[st])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[st])));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&done)));
    asm volatile("fence.mbarrier_init.release.cluster;");
    n_issued = 0;
    n_consumed = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_slot;
  const int nk = K / BK;

  if (threadIdx.x == 0) {
    // producer: stage kb waits for the MMAs of step kb - NST to release it
    int kb = 0;
    for (; kb < nk; kb++) {
      const int st = kb % NST;
      if (kb >= NST && !mbar_wait(smem_u32(&empty[st]), ((kb / NST) - 1) & 1, err)) break;
      mbar_expect_tx(smem_u32(&full[st]), ST_BYTES);
      tma_load_2d(As(st), &ta, smem_u32(&full[st]), kb * BK, m0);
      tma_load_2d(Bs(st), &tb, smem_u32(&full[st]), kb * BK, n0);
    }
    n_issued = kb;
  } else if (threadIdx.x == 32) {
    // MMA issuer
    const uint32_t idesc = instr_desc_tf32(BM, BN);
    int kb = 0;
    for (; kb < nk; kb++) {
      const int st = kb % NST;
      if (!mbar_wait(smem_u32(&full[st]), (kb / NST) & 1, err)) break;
      asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
      for (int k8 = 0; k8 < BK / 8; k8++) {
        const uint64_t ad = smem_desc_sw128(As(st) + k8 * 32);
        const uint64_t bd = smem_desc_sw128(Bs(st) + k8 * 32);
        const uint32_t acc = (kb > 0 || k8 > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(&empty[st])));
    }
    n_consumed = kb;
    // arrives once every MMA issued above has completed
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
        smem_u32(&done)));
  }
  bool ok = mbar_wait(smem_u32(&done), 0, err);
  ok = __syncthreads_and(ok) && n_consumed == nk;
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (threadIdx.x == 0) {
    // copies issued but never consumed (only after a time-out) land before exit
    for (int kb = n_consumed; kb < n_issued; kb++) mbar_wait(smem_u32(&full[kb % NST]), (kb / NST) & 1, err);
  }
  if (ok) {
    // epilogue: warp w owns accumulator lanes (rows) 32w .. 32w + 31
    const int row = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < BN; c0 += 16) {
      uint32_t v[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      // load and wait in one statement: the destination registers are
      // written asynchronously and must not be read before the wait
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
          "tcgen05.wait::ld.sync.aligned;"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(taddr)
          : "memory");
      if (row < M) {
        float x[16];
#pragma unroll
        for (int j = 0; j < 16; j++) {
          const int col = n0 + c0 + j;
          x[j] = __uint_as_float(v[j]);
          if (bias && col < N) x[j] += bias[col];
          if (act == 1) x[j] = tanhf(x[j]);
        }
        float *crow = C + (size_t)row * N + n0 + c0;
        if ((N & 3) == 0 && n0 + c0 + 16 <= N) {
#pragma unroll
          for (int j = 0; j < 16; j += 4) *reinterpret_cast<float4 *>(crow + j) = make_float4(x[j], x[j + 1], x[j + 2], x[j + 3]);
        } else {
#pragma unroll
          for (int j = 0; j < 16; j++)
            if (n0 + c0 + j < N) crow[j] = x[j];
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
}

typedef CUresult (*EncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_tiled() {
  static EncodeTiled fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    QCUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !p) fail(9, "ERROR! cuTensorMapEncodeTiled unavailable\n");
    fn = (EncodeTiled)p;
  }
  return fn;
}

// rows x K row-major FP32 matrix as 128 x 32 tiles, 128-byte swizzle
bool encode_operand(const float *p, int rows, int K, CUtensorMap *map) {
  memset(map, 0, sizeof(*map));
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)K * 4};
  const cuuint32_t box[2] = {BK, 128}, estr[2] = {1, 1};
  EncodeTiled f = encode_tiled();
  if (!f) return false;
  return f(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)p, dims, strides, box, estr,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

// C = act(A B^T + bias) on device buffers; K must be a multiple of 32.
void launch_gemm_tf32(const float *A, const float *B, float *C, const float *bias, int M, int N, int K, int act,
                      int *err, cudaStream_t s) {
  // TMA needs 16-byte aligned operands (row pitch K * 4 is, K being a
  // multiple of 32)
  if ((reinterpret_cast<uintptr_t>(A) & 15) || (reinterpret_cast<uintptr_t>(B) & 15)) {
    fail(0, "ERROR! quac_gemm_tf32: operands must be 16-byte aligned\n");
    return;
  }
  CUtensorMap ta, tb;
  if (!encode_operand(A, M, K, &ta) || !encode_operand(B, N, K, &tb)) {
    fail(9, "ERROR! quac_gemm_tf32: tensor map encoding failed\n");
    return;
  }
  const int smem = NST * ST_BYTES + 1024;
  ensure_smem((const void *)k_gemm_tf32, smem);
  dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
  k_gemm_tf32<<<grid, 128, smem, s>>>(ta, tb, C, bias, M, N, K, act, err);
  count_launch();
  QCUDA(cudaGetLastError());
}

}  // namespace quac

using namespace quac;

// Device-pointer GEMM for tests: returns 0, or 1 on invalid sizes or a
// timed-out wait inside the kernel.
extern "C" int quac_gemm_tf32(const float *A, const float *B, float *C, const float *bias, int M, int N, int K,
                              int act) {
  if (M <= 0 || N <= 0 || K <= 0 || K % 32 != 0 || (act != 0 && act != 1)) {
    fail(0, "ERROR! quac_gemm_tf32: invalid sizes (K must be a positive multiple of 32)\n");
    return 1;
  }
  int *err = nullptr;
  QCUDA(cudaMalloc(&err, sizeof(int)));
  QCUDA(cudaMemset(err, 0, sizeof(int)));
  launch_gemm_tf32(A, B, C, bias, M, N, K, act, err, 0);
  int h = 0;
  QCUDA(cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost));
  QCUDA(cudaFree(err));
  if (h) fail(9, "ERROR! quac_gemm_tf32: a tensor-core wait ran out of time\n");
  return has_error() ? 1 : 0;
}
